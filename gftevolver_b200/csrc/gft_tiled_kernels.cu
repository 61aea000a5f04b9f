// gft_tiled_kernels.cu -- the throughput step kernel with TMA-staged planes:
// one CTA per tile of (y, z) columns and x-chunk, the per-tile pipeline of
// gft_tiled_tile.cuh.  Host side: tensor-map encoding and launch.
#include <cuda.h>

#include "gft_device.cuh"
#include "gft_launch.h"
#include "gft_pair_body.cuh"
#include "gft_split_body.cuh"
#include "gft_tiled_tile.cuh"

namespace gft {

namespace {

using namespace tiled;

// CTAs per SM the launch bounds ask for: as many as shared memory admits, at
// most 512 threads per SM.  For the SM model in float with 8 x 32 or 16 x 16
// tiles that is two, which caps registers at 128 per thread (the logging-step
// variant would otherwise exceed it); where the staged planes admit one CTA
// (FP64, the 2HDM model's two doublets) the registers are left uncapped.
template <class S, int MODEL, int TY, int TZ>
constexpr int tiled_min_blocks()
{
    using G = Geom<S, TY, TZ, (MODEL == kModelSM) ? 1 : 2>;
    constexpr int by_smem = (228 * 1024) / (G::SMEM + 16 + 1024);
    constexpr int by_threads = 512 / (TY * TZ);
    constexpr int b = by_smem < by_threads ? by_smem : by_threads;
    return b < 1 ? 1 : b;
}

template <class S, int MODEL, int TY, int TZ, bool ENERGY>
__global__ void __launch_bounds__(TY * TZ, tiled_min_blocks<S, MODEL, TY, TZ>()) tiled_step_kernel(const __grid_constant__ TMaps maps,
                                                             const __grid_constant__ TMaps pmaps, StepParams P,
                                                             FConst F, LevelPtrs<S> now, LevelPtrs<S> past, int lx,
                                                             int xa, int xn, unsigned* status, double* partials)
{
    constexpr int ND = (MODEL == kModelSM) ? 1 : 2;
    using G = Geom<S, TY, TZ, ND>;
    extern __shared__ unsigned char smem_raw[];
    unsigned char* smem =
        reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 127) & ~(uintptr_t)127);
    unsigned long long* bars = reinterpret_cast<unsigned long long*>(smem + G::NBUF * G::BUF);
    const int tid = threadIdx.y * TZ + threadIdx.x;

    __shared__ int s_abort;
    if (tid == 0) {
        s_abort = 0;
        for (int b = 0; b < G::NBUF; b++) mbar_init(&bars[b], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();

    double obs[kObsCount];
#pragma unroll
    for (int k = 0; k < kObsCount; k++) obs[k] = 0.0;
    unsigned warn = 0;
    RingPhase ring = {0u};
    const int x0 = xa + blockIdx.z * lx;  // planes [xa, xa + xn) in chunks of lx
    constexpr bool STAGE = !ENERGY && HaloStage<S, TY, TZ, ND>::kUse;
    const bool ok = run_tile<S, MODEL, TY, TZ, ENERGY, LevelPtrs<S>, STAGE>(
        maps, pmaps, P, F, now, past, blockIdx.y * TY, blockIdx.x * TZ, x0, min(lx, xa + xn - x0), smem, bars, ring,
        &s_abort, obs, warn, smem + HaloStage<S, TY, TZ, ND>::OFFSET);
    if (!ok && tid == 0) atomicOr(status, kErrTimeout);

    if (ENERGY) {
        energy_total(obs);
        const int b = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z);
        block_reduce_store<kObsCount>(obs, partials + (size_t)b * kObsCount, kObsCount);
    }
    if (warn) atomicOr(status, warn);
}

// Both sites of a thread from a staged plane: the cell of site A (row ty) and
// the cell TY/2 rows further (site B), as (A, B) pairs.
template <int TY, int TZ>
struct PairAcc {
    using G = Geom<float, TY, TZ, 1>;
    static constexpr int DQ = (TY / 2) * G::QP, DH = (TY / 2) * G::HP;
    __device__ __forceinline__ static pair::Q2 ld2(const unsigned char* base, int cell)
    {
        const float4 a = reinterpret_cast<const float4*>(base)[cell];
        const float4 b = reinterpret_cast<const float4*>(base)[cell + DQ];
        return {make_float2(a.x, b.x), make_float2(a.y, b.y), make_float2(a.z, b.z), make_float2(a.w, b.w)};
    }
    __device__ __forceinline__ pair::Q2 q(int d, TRef r) const { return ld2(r.b + d * G::QB, r.cq); }
    __device__ __forceinline__ pair::V th(int d, TRef r) const
    {
        const float* h = reinterpret_cast<const float*>(r.b + G::OFF_TH + d * G::HB);
        return make_float2(h[r.ch], h[r.ch + DH]);
    }
    __device__ __forceinline__ pair::Q2 ph(TRef r) const { return ld2(r.b + G::OFF_PH, r.cq); }
};

// Plain steps of the SM mixed form with two sites per thread: the CTA's
// TZ x TY/2 threads cover the TY x TZ tile, thread (tz, ty) rows ty and ty + TY/2,
// with the plane ring, halo staging and bounded waits of the one-site kernel
// (run_ring).  Two CTAs per SM: up to 255 registers per thread.
template <int TY, int TZ>
__global__ void __launch_bounds__(TY * TZ / 2, 2) tiled_pair_kernel(const __grid_constant__ TMaps maps,
                                                                   const __grid_constant__ TMaps pmaps, StepParams P,
                                                                   FConst F, LevelPtrs<float> now,
                                                                   LevelPtrs<float> past, int lx, int xa, int xn,
                                                                   unsigned* status)
{
    using G = Geom<float, TY, TZ, 1>;
    using H = HaloStage<float, TY, TZ, 1>;
    extern __shared__ unsigned char smem_raw[];
    unsigned char* smem =
        reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 127) & ~(uintptr_t)127);
    unsigned long long* bars = reinterpret_cast<unsigned long long*>(smem + G::NBUF * G::BUF);
    const int tz = threadIdx.x, ty = threadIdx.y;
    const int tid = ty * TZ + tz;

    __shared__ int s_abort;
    if (tid == 0) {
        s_abort = 0;
        for (int b = 0; b < G::NBUF; b++) mbar_init(&bars[b], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();

    const int y0 = blockIdx.y * TY, z0 = blockIdx.x * TZ, x0 = xa + blockIdx.z * lx;
    const int cq0 = (ty + 1) * G::QP + (tz + 1);
    const int ch0 = (ty + 1) * G::HP + (tz + 1) + G::TP - 1;
    const int y = y0 + ty, z = z0 + tz;
    const int sb_off = (TY / 2) * P.nz;
    pair::Carry2 carry;
    carry.valid = false;
    unsigned warn = 0;
    RingPhase ring = {0u};
    const bool ok = run_ring<float, TY, TZ, 1, LevelPtrs<float>, H::kUse>(
        maps, pmaps, P, now, y0, z0, x0, min(lx, xa + xn - x0), smem, bars, ring, &s_abort, smem + H::OFFSET, tid,
        [&](int i, const unsigned char* bm, const unsigned char* bc, const unsigned char* bp) {
            const Stencil<TRef> n = plane_stencil<G::QP, G::HP>(bm, bc, bp, cq0, ch0);
            const int x = x0 + i;
            const int sa = (x * P.ny + y) * P.nz + z;
            pair::site_step2(F, PairAcc<TY, TZ>{}, n, past, sa, sa + sb_off, carry, warn, counts(P, x));
        });
    if (!ok && tid == 0) atomicOr(status, kErrTimeout);
    if (warn) atomicOr(status, warn);
}

// Shared memory of the split-site kernel: the ring, its barriers, the halo
// staging (when it fits) and the scalars-to-links handoff.
template <int TY, int TZ>
struct SplitLayout {
    using G = Geom<float, TY, TZ, 1>;
    using H = HaloStage<float, TY, TZ, 1>;
    using HO = split::Handoff<TY * TZ>;
    static constexpr bool kStage = H::kUse;
    static constexpr int OFF_HO = kStage ? (H::OFFSET + H::BYTES + 15) / 16 * 16 : G::NBUF * G::BUF + 64;
    static constexpr int SMEM = OFF_HO + HO::kBytes + 128;  // + alignment slack of the dynamic base
};

__device__ __forceinline__ void named_arrive(int id, int count)
{
    asm volatile("bar.arrive %0, %1;" ::"r"(id), "r"(count) : "memory");
}
__device__ __forceinline__ void named_sync(int id, int count)
{
    asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(count) : "memory");
}

// Plain steps of the SM mixed form with each site's update divided between two
// threads (gft_split_body.cuh): warps 0 .. NT/32 - 1 take the links of the
// tile's sites, the next NT/32 warps the scalars of the same sites; warp w of
// the scalars hands E and J to warp w of the links through shared memory,
// ordered by named barrier 1 + w (bar.arrive / bar.sync over the 64 threads of
// the pair).  The plane ring, halo staging and bounded waits are run_ring's.
// Three CTAs per SM: up to 85 registers per thread, 24 warps.
template <int TY, int TZ>
__global__ void __launch_bounds__(2 * TY * TZ, 3) tiled_split_kernel(const __grid_constant__ TMaps maps,
                                                                    const __grid_constant__ TMaps pmaps, StepParams P,
                                                                    FConst F, LevelPtrs<float> now,
                                                                    LevelPtrs<float> past, int lx, int xa, int xn,
                                                                    unsigned* status)
{
    using G = Geom<float, TY, TZ, 1>;
    using L = SplitLayout<TY, TZ>;
    constexpr int NT = TY * TZ;  // sites of the tile = threads per role
    static_assert(NT % 32 == 0, "each role is whole warps");
    extern __shared__ unsigned char smem_raw[];
    unsigned char* smem =
        reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 127) & ~(uintptr_t)127);
    unsigned long long* bars = reinterpret_cast<unsigned long long*>(smem + G::NBUF * G::BUF);
    const int tid = threadIdx.x;
    const bool scalars = tid >= NT;  // warp-uniform
    const int t = scalars ? tid - NT : tid;
    const int ty = t / TZ, tz = t % TZ;
    const int pair_bar = 1 + t / 32;

    __shared__ int s_abort;
    if (tid == 0) {
        s_abort = 0;
        for (int b = 0; b < G::NBUF; b++) mbar_init(&bars[b], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();

    const int y0 = blockIdx.y * TY, z0 = blockIdx.x * TZ, x0 = xa + blockIdx.z * lx;
    const int cq0 = (ty + 1) * G::QP + (tz + 1);
    const int ch0 = (ty + 1) * G::HP + (tz + 1) + G::TP - 1;
    const int y = y0 + ty, z = z0 + tz;
    const split::Handoff<NT> ho{reinterpret_cast<float*>(smem + L::OFF_HO), t};
    split::ScalarCarry carry;
    carry.valid = false;
    unsigned warn = 0;
    RingPhase ring = {0u};
    const bool ok = run_ring<float, TY, TZ, 1, LevelPtrs<float>, L::kStage>(
        maps, pmaps, P, now, y0, z0, x0, min(lx, xa + xn - x0), smem, bars, ring, &s_abort,
        smem + HaloStage<float, TY, TZ, 1>::OFFSET, tid,
        [&](int i, const unsigned char* bm, const unsigned char* bc, const unsigned char* bp) {
            const Stencil<TRef> n = plane_stencil<G::QP, G::HP>(bm, bc, bp, cq0, ch0);
            const int x = x0 + i;
            const int s = (x * P.ny + y) * P.nz + z;
            const unsigned warn_in = warn;
            if (scalars) {
                split::site_scalars(F, TileAcc<float, TY, TZ, 1>{}, n, past, s, carry, ho, warn);
                named_arrive(pair_bar, 64);
            } else {
                split::site_links(F, TileAcc<float, TY, TZ, 1>{}, n, past, s, ho,
                                  [&] { named_sync(pair_bar, 64); }, warn);
            }
            if (!counts(P, x)) warn = warn_in;  // ghost planes of an x-slab
        });
    if (!ok && tid == 0) atomicOr(status, kErrTimeout);
    if (warn) atomicOr(status, warn);
}

// ---- host side ---------------------------------------------------------------
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn()
{
    static EncodeTiledFn fn = nullptr;
    static bool tried = false;
    if (!tried) {
        tried = true;
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiledFn>(p);
    }
    return fn;
}

}  // namespace

template <class S>
bool tiled_encode_maps(const StepParams& P, const LevelPtrs<S>& L, int nd, int ty, int tz, bool halo, TMaps* out)
{
    EncodeTiledFn enc = encode_fn();
    if (!enc) return false;
    const CUtensorMapDataType dt = (sizeof(S) == 4) ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64;
    const cuuint64_t es = sizeof(S);
    const int tp = 16 / (int)sizeof(S);
    const cuuint32_t estr[4] = {1, 1, 1, 1};
    // quaternion / doublet arrays: dims {4, nz, ny, nx}
    const cuuint64_t qdim[4] = {4, (cuuint64_t)P.nz, (cuuint64_t)P.ny, (cuuint64_t)P.nx};
    const cuuint64_t qstr[3] = {4 * es, 4 * es * P.nz, 4 * es * P.nz * P.ny};
    const int hz = halo ? 2 : 0, hy = halo ? 2 : 0, hp = halo ? 2 * tp : 0;
    const cuuint32_t qbox[4] = {4, (cuuint32_t)(tz + hz), (cuuint32_t)(ty + hy), 1};
    // theta arrays: dims {nz, ny, nx}
    const cuuint64_t hdim[3] = {(cuuint64_t)P.nz, (cuuint64_t)P.ny, (cuuint64_t)P.nx};
    const cuuint64_t hstr[2] = {es * P.nz, es * P.nz * P.ny};
    const cuuint32_t hbox[3] = {(cuuint32_t)(tz + hp), (cuuint32_t)(ty + hy), 1};
    for (int d = 0; d < 3; d++) {
        if (enc(&out->q[d], dt, 4, L.q[d], qdim, qstr, qbox, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) !=
            CUDA_SUCCESS)
            return false;
        if (enc(&out->th[d], dt, 3, L.th[d], hdim, hstr, hbox, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) !=
            CUDA_SUCCESS)
            return false;
    }
    for (int k = 0; k < 2; k++) {
        if (k >= nd) {
            out->ph[k] = out->ph[0];
            continue;
        }
        if (enc(&out->ph[k], dt, 4, L.ph[k], qdim, qstr, qbox, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) !=
            CUDA_SUCCESS)
            return false;
    }
    return true;
}


bool tiled_supported(const StepParams& P, int variant)
{
    int ty, tz;
    tiled_tile(variant, ty, tz);
    return encode_fn() != nullptr && P.nz % tz == 0 && P.ny % ty == 0 && P.nx >= 1;
}

int tiled_ctas_per_sm(int variant, bool fp64)
{
    switch (variant) {
    case 0: return fp64 ? tiled_min_blocks<double, kModelSM, 8, 32>() : tiled_min_blocks<float, kModelSM, 8, 32>();
    case 1: return fp64 ? tiled_min_blocks<double, kModelSM, 4, 32>() : tiled_min_blocks<float, kModelSM, 4, 32>();
    case 2: return fp64 ? tiled_min_blocks<double, kModelSM, 4, 16>() : tiled_min_blocks<float, kModelSM, 4, 16>();
    default: return fp64 ? tiled_min_blocks<double, kModelSM, 16, 16>() : tiled_min_blocks<float, kModelSM, 16, 16>();
    }
}

int tiled_blocks(const StepParams& P, int variant, int lx)
{
    int ty, tz;
    tiled_tile(variant, ty, tz);
    return (P.nz / tz) * (P.ny / ty) * ((P.nx + lx - 1) / lx);  // a launch over all planes
}

template <class S, int MODEL, int TY, int TZ>
static cudaError_t launch_tiled_t(const TMaps& maps, const TMaps& pmaps, const StepParams& P, const LevelPtrs<S>& now,
                                  const LevelPtrs<S>& past, int lx, int xa, int xn, unsigned* status, double* partials,
                                  bool energy, cudaStream_t stream)
{
    constexpr int ND = (MODEL == kModelSM) ? 1 : 2;
    using G = Geom<S, TY, TZ, ND>;
    const dim3 block(TZ, TY, 1);
    const dim3 grid(P.nz / TZ, P.ny / TY, (xn + lx - 1) / lx);
    if (energy) {
        auto k = tiled_step_kernel<S, MODEL, TY, TZ, true>;
        cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, G::SMEM);
        k<<<grid, block, G::SMEM, stream>>>(maps, pmaps, P, make_fconst(P), now, past, lx, xa, xn, status, partials);
    } else {
        using H = HaloStage<S, TY, TZ, ND>;
        constexpr int SMEM = H::kUse ? H::SMEM : G::SMEM;  // plain steps stage their wrapped halo cells
        auto k = tiled_step_kernel<S, MODEL, TY, TZ, false>;
        cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM);
        k<<<grid, block, SMEM, stream>>>(maps, pmaps, P, make_fconst(P), now, past, lx, xa, xn, status, partials);
    }
    return cudaGetLastError();
}

template <class S, int MODEL>
cudaError_t launch_tiled_step(const TMaps& maps, const TMaps& pmaps, const StepParams& P, const LevelPtrs<S>& now,
                              const LevelPtrs<S>& past, int variant, int lx, unsigned* status, double* partials,
                              bool energy, cudaStream_t stream, int xa, int xn)
{
    if (xn < 0) xn = P.nx - xa;  // default: every plane from xa on
    switch (variant) {
    case 0: return launch_tiled_t<S, MODEL, 8, 32>(maps, pmaps, P, now, past, lx, xa, xn, status, partials, energy, stream);
    case 1: return launch_tiled_t<S, MODEL, 4, 32>(maps, pmaps, P, now, past, lx, xa, xn, status, partials, energy, stream);
    case 2: return launch_tiled_t<S, MODEL, 4, 16>(maps, pmaps, P, now, past, lx, xa, xn, status, partials, energy, stream);
    default: return launch_tiled_t<S, MODEL, 16, 16>(maps, pmaps, P, now, past, lx, xa, xn, status, partials, energy, stream);
    }
}

template <int TY, int TZ>
static cudaError_t launch_pair_t(const TMaps& maps, const TMaps& pmaps, const StepParams& P,
                                 const LevelPtrs<float>& now, const LevelPtrs<float>& past, int lx, int xa, int xn,
                                 unsigned* status, cudaStream_t stream)
{
    using G = Geom<float, TY, TZ, 1>;
    using H = HaloStage<float, TY, TZ, 1>;
    constexpr int SMEM = H::kUse ? H::SMEM : G::SMEM;
    const dim3 block(TZ, TY / 2, 1);
    const dim3 grid(P.nz / TZ, P.ny / TY, (xn + lx - 1) / lx);
    auto k = tiled_pair_kernel<TY, TZ>;
    cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM);
    k<<<grid, block, SMEM, stream>>>(maps, pmaps, P, make_fconst(P), now, past, lx, xa, xn, status);
    return cudaGetLastError();
}

cudaError_t launch_tiled_pair_step(const TMaps& maps, const TMaps& pmaps, const StepParams& P,
                                   const LevelPtrs<float>& now, const LevelPtrs<float>& past, int variant, int lx,
                                   unsigned* status, cudaStream_t stream, int xa, int xn)
{
    if (xn < 0) xn = P.nx - xa;
    // the 8 x 32 and 16 x 16 tiles (128 threads per CTA); tiled_pair_tile says which
    if (variant == 3) return launch_pair_t<16, 16>(maps, pmaps, P, now, past, lx, xa, xn, status, stream);
    return launch_pair_t<8, 32>(maps, pmaps, P, now, past, lx, xa, xn, status, stream);
}

cudaError_t launch_tiled_split_step(const TMaps& maps, const TMaps& pmaps, const StepParams& P,
                                    const LevelPtrs<float>& now, const LevelPtrs<float>& past, int lx,
                                    unsigned* status, cudaStream_t stream, int xa, int xn)
{
    constexpr int TY = kSplitTileY, TZ = kSplitTileZ;
    using L = SplitLayout<TY, TZ>;
    if (xn < 0) xn = P.nx - xa;
    const dim3 block(2 * TY * TZ, 1, 1);
    const dim3 grid(P.nz / TZ, P.ny / TY, (xn + lx - 1) / lx);
    auto k = tiled_split_kernel<TY, TZ>;
    cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, L::SMEM);
    k<<<grid, block, L::SMEM, stream>>>(maps, pmaps, P, make_fconst(P), now, past, lx, xa, xn, status);
    return cudaGetLastError();
}

template bool tiled_encode_maps<float>(const StepParams&, const LevelPtrs<float>&, int, int, int, bool, TMaps*);
template bool tiled_encode_maps<double>(const StepParams&, const LevelPtrs<double>&, int, int, int, bool, TMaps*);
template cudaError_t launch_tiled_step<float, kModelSM>(const TMaps&, const TMaps&, const StepParams&,
                                                        const LevelPtrs<float>&, const LevelPtrs<float>&, int, int,
                                                        unsigned*, double*, bool, cudaStream_t, int, int);
template cudaError_t launch_tiled_step<double, kModelSM>(const TMaps&, const TMaps&, const StepParams&,
                                                         const LevelPtrs<double>&, const LevelPtrs<double>&, int, int,
                                                         unsigned*, double*, bool, cudaStream_t, int, int);
template cudaError_t launch_tiled_step<float, kModel2HDM>(const TMaps&, const TMaps&, const StepParams&,
                                                          const LevelPtrs<float>&, const LevelPtrs<float>&, int, int,
                                                          unsigned*, double*, bool, cudaStream_t, int, int);

}  // namespace gft
