// gft_fast_kernels.cu -- throughput forms of the leapfrog step, one thread per
// site with neighbours read through L1/L2 (any lattice size), and the Gauss
// residual kernel.  The per-site arithmetic is gft_step_body.cuh.
//
//   GFT_FORM_FP64  : S = double.
//   GFT_FORM_MIXED : S = float (see gft_step_body.cuh for where precision is kept).
#include "gft_device.cuh"
#include "gft_launch.h"
#include "gft_math.cuh"
#include "gft_step_body.cuh"

namespace gft {
namespace {

// Neighbour offsets: the site index is linear in (x, y, z), so the wrap of
// each axis contributes an independent offset.
struct Offs {
    int c, m[3], p[3];
};

__device__ __forceinline__ Offs offsets(const StepParams& P, int x, int y, int z)
{
    Offs o;
    const int plane = P.ny * P.nz;
    o.c = (x * P.ny + y) * P.nz + z;
    o.m[0] = (x == 0) ? (P.nx - 1) * plane : -plane;
    o.p[0] = (x + 1 == P.nx) ? -(P.nx - 1) * plane : plane;
    o.m[1] = (y == 0) ? (P.ny - 1) * P.nz : -P.nz;
    o.p[1] = (y + 1 == P.ny) ? -(P.ny - 1) * P.nz : P.nz;
    o.m[2] = (z == 0) ? P.nz - 1 : -1;
    o.p[2] = (z + 1 == P.nz) ? -(P.nz - 1) : 1;
    return o;
}

// Field access through L1/L2 (read-only path) for the "now" level.
template <class S>
struct GlobalAcc {
    LevelPtrs<S> L;
    __device__ __forceinline__ Q<S> q(int d, int s) const { return ld4<S>(L.q[d], s); }
    __device__ __forceinline__ S th(int d, int s) const { return ld1<S>(L.th[d], s); }
    __device__ __forceinline__ Q<S> ph(int k, int s) const { return ld4<S>(L.ph[k], s); }
    __device__ __forceinline__ S hth(int d, int s) const { return ld1<S>(L.hth[d], s); }
    __device__ __forceinline__ Q<S> hq(int d, int s) const { return ld4<S>(L.hq[d], s); }
};

// One thread per site; the kernel below instantiates it with its launch bounds.
template <class S, int MODEL, int HF, bool ENERGY>
__device__ __forceinline__ void fast_step_body(StepParams P, FConst F, LevelPtrs<S> now, LevelPtrs<S> past,
                                               unsigned* status, double* partials)
{
    const int z = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    const int x = blockIdx.z;
    double obs[kObsCount];
#pragma unroll
    for (int k = 0; k < kObsCount; k++) obs[k] = 0.0;
    unsigned warn = 0;
    if ((z < P.nz) && (y < P.ny) && !frozen(P, x, y, z)) {  // Fixed faces: not evolved
        const Offs o = offsets(P, x, y, z);
        Stencil<int> n;
        n.c = o.c;
#pragma unroll
        for (int a = 0; a < 3; a++) {
            n.m[a] = o.c + o.m[a];
            n.p[a] = o.c + o.p[a];
        }
        n.d01 = o.c + o.p[0] + o.m[1];
        n.d02 = o.c + o.p[0] + o.m[2];
        n.d10 = o.c + o.p[1] + o.m[0];
        n.d12 = o.c + o.p[1] + o.m[2];
        n.d20 = o.c + o.p[2] + o.m[0];
        n.d21 = o.c + o.p[2] + o.m[1];
        XCarry<S, (MODEL == kModelSM) ? 1 : 2> carry;
        carry.valid = false;
        site_step<S, MODEL, ENERGY, HF>(P, F, GlobalAcc<S>{now}, n, PastSite<S>{past, o.c}, carry, obs, warn,
                                        counts(P, x));
    }
    if (ENERGY) {
        energy_total(obs);
        const int b = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z);
        block_reduce_store<kObsCount>(obs, partials + (size_t)b * kObsCount, kObsCount);
    }
    if (warn) atomicOr(status, warn);
}

template <class S, int MODEL, int HF, bool ENERGY>
__global__ void __launch_bounds__(128) fast_step_kernel(StepParams P, FConst F, LevelPtrs<S> now, LevelPtrs<S> past,
                                                        unsigned* status, double* partials)
{
    fast_step_body<S, MODEL, HF, ENERGY>(P, F, now, past, status, partials);
}

// The FP64 SM step: left to itself the compiler takes 176 registers (two blocks,
// 8 warps per SM); capped at three blocks it fits 168 with no spills in the plain
// step, and the extra warps hide more of its load latency (2.68 against 3.41 ms
// per step at 256^3).  The other instances run fastest unbounded, a minimum of one
// block included.
template <>
__global__ void __launch_bounds__(128, 3) fast_step_kernel<double, kModelSM, kHfNone, false>(
    StepParams P, FConst F, LevelPtrs<double> now, LevelPtrs<double> past, unsigned* status, double* partials)
{
    fast_step_body<double, kModelSM, kHfNone, false>(P, F, now, past, status, partials);
}
template <>
__global__ void __launch_bounds__(128, 3) fast_step_kernel<double, kModelSM, kHfNone, true>(
    StepParams P, FConst F, LevelPtrs<double> now, LevelPtrs<double> past, unsigned* status, double* partials)
{
    fast_step_body<double, kModelSM, kHfNone, true>(P, F, now, past, status, partials);
}

// Gauss-law residual after a step (gauss_site in gft_step_body.cuh), one
// thread per site: every load of a site is independent of the others, which
// keeps the most loads in flight (a march along x that carries the x - 1 links
// in registers serialises them and measured slower).
template <class S, int MODEL, int HF>
__global__ void __launch_bounds__(256) fast_gauss_kernel(StepParams P, LevelPtrs<S> now, LevelPtrs<S> fut,
                                                         double* partials)
{
    constexpr int NG = 2 * hf_neq(HF);
    const int z = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    const int x = blockIdx.z;
    double v[NG];
#pragma unroll
    for (int k = 0; k < NG; k++) v[k] = 0.0;
    if (z < P.nz && y < P.ny && counts(P, x) && !frozen(P, x, y, z)) {
        const Offs o = offsets(P, x, y, z);
        gauss_site<S, MODEL, HF>(P, now, fut, o.c, o.c + o.m[0], o.c + o.m[1], o.c + o.m[2], v);
    }
    const int blk = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z);
    block_reduce_store<NG>(v, partials + (size_t)blk * NG, NG / 2);
}

template <class S, int MODEL, int HF>
void fast_step_launch(const StepParams& P, const LevelPtrs<S>& now, const LevelPtrs<S>& past, unsigned* status,
                      double* partials, bool energy, cudaStream_t stream)
{
    const dim3 block(32, 4, 1);
    const dim3 grid((P.nz + 31) / 32, (P.ny + 3) / 4, P.nx);
    if (energy)
        fast_step_kernel<S, MODEL, HF, true><<<grid, block, 0, stream>>>(P, make_fconst(P), now, past, status, partials);
    else
        fast_step_kernel<S, MODEL, HF, false><<<grid, block, 0, stream>>>(P, make_fconst(P), now, past, status, partials);
}

template <class S, int MODEL, int HF>
void fast_gauss_launch(const StepParams& P, const LevelPtrs<S>& now, const LevelPtrs<S>& fut, double* partials,
                       cudaStream_t stream)
{
    const dim3 block(32, 8, 1);  // 32 x 8: 2 % faster than 32 x 4 at 256^3 (624 against 638 us)
    const dim3 grid((P.nz + 31) / 32, (P.ny + 7) / 8, P.nx);
    fast_gauss_kernel<S, MODEL, HF><<<grid, block, 0, stream>>>(P, now, fut, partials);
}

}  // namespace

int fast_launch_blocks(const StepParams& P, int /*variant*/) { return ((P.nz + 31) / 32) * ((P.ny + 3) / 4) * P.nx; }
int fast_gauss_blocks(const StepParams& P) { return ((P.nz + 31) / 32) * ((P.ny + 7) / 8) * P.nx; }

// P.hf selects the Higgs-family variant (2HDM only); the Gauss kernel writes
// 2 * gaugeNum partial slots per block.
template <class S, int MODEL>
cudaError_t launch_fast_step(const StepParams& P, const LevelPtrs<S>& now, const LevelPtrs<S>& past, unsigned* status,
                             double* partials, bool energy, int /*variant*/, cudaStream_t stream)
{
    if constexpr (MODEL == kModel2HDM) {
        if (P.hf == kHfU1)
            fast_step_launch<S, MODEL, kHfU1>(P, now, past, status, partials, energy, stream);
        else if (P.hf == kHfSU2)
            fast_step_launch<S, MODEL, kHfSU2>(P, now, past, status, partials, energy, stream);
        else
            fast_step_launch<S, MODEL, kHfNone>(P, now, past, status, partials, energy, stream);
    } else {
        fast_step_launch<S, MODEL, kHfNone>(P, now, past, status, partials, energy, stream);
    }
    return cudaGetLastError();
}

template <class S, int MODEL>
cudaError_t launch_fast_gauss(const StepParams& P, const LevelPtrs<S>& now, const LevelPtrs<S>& fut, double* partials,
                              cudaStream_t stream)
{
    if constexpr (MODEL == kModel2HDM) {
        if (P.hf == kHfU1)
            fast_gauss_launch<S, MODEL, kHfU1>(P, now, fut, partials, stream);
        else if (P.hf == kHfSU2)
            fast_gauss_launch<S, MODEL, kHfSU2>(P, now, fut, partials, stream);
        else
            fast_gauss_launch<S, MODEL, kHfNone>(P, now, fut, partials, stream);
    } else {
        fast_gauss_launch<S, MODEL, kHfNone>(P, now, fut, partials, stream);
    }
    return cudaGetLastError();
}

#define GFT_INSTANTIATE_FAST(S, M)                                                                                   \
    template cudaError_t launch_fast_step<S, M>(const StepParams&, const LevelPtrs<S>&, const LevelPtrs<S>&,         \
                                                unsigned*, double*, bool, int, cudaStream_t);                         \
    template cudaError_t launch_fast_gauss<S, M>(const StepParams&, const LevelPtrs<S>&, const LevelPtrs<S>&,        \
                                                 double*, cudaStream_t);
GFT_INSTANTIATE_FAST(float, kModelSM)
GFT_INSTANTIATE_FAST(float, kModel2HDM)
GFT_INSTANTIATE_FAST(double, kModelSM)
GFT_INSTANTIATE_FAST(double, kModel2HDM)

}  // namespace gft
