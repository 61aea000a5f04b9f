// gft_aux_kernels.cu -- layout conversion, initial data and reduction finalisation.
#include <cstring>

#include "gft_device.cuh"
#include "gft_launch.h"
#include "gft_reduce.cuh"
#include "gft_math.cuh"

namespace gft {
namespace {

// Generator w -> quaternion as the reference's getSU2Representation does it
// (WilsonLoops/Source/StandardModel.cpp:76-112, conj = false).
template <class H>
__device__ __forceinline__ void gen_to_quat(const H* w, double tol, double (&c)[4])
{
    double wm = 0.0;
    for (int k = 0; k < 3; k++) wm += (double)w[k] * (double)w[k];
    wm = sqrt(wm);
    c[0] = cos(wm);
    c[1] = c[2] = c[3] = 0.0;
    if (wm > tol) {
        for (int k = 1; k < 4; k++) c[k] = sin(wm) * (double)w[k - 1] / wm;
    } else {
        c[1] = sin(wm);
    }
}

// Quaternion -> generator as invertSU2Representation does it (:114-158).
__device__ __forceinline__ void quat_to_gen(const double (&c)[4], double tol, double (&w)[3])
{
    double cm = sqrt(c[1] * c[1] + c[2] * c[2] + c[3] * c[3]);
    double phase = (cm > 1) ? 1.5707963267948966 : asin(cm);
    if (c[0] < 0) phase = 3.141592653589793 - phase;
    if (cm > tol) {
        for (int k = 0; k < 3; k++) w[k] = phase * c[k + 1] / cm;
    } else {
        w[0] = phase;
        w[1] = w[2] = 0.0;
    }
}

// One SU(2) link of the host record (4 words, or 3 generators) -> a device record.
template <class S, class H>
__device__ __forceinline__ void put_link(S* arr, int s, const H* w, const LinkCodec& cc)
{
    if (!cc.gen) {
        st4(arr, s, (S)w[0], (S)w[1], (S)w[2], (S)w[3]);
    } else if (cc.convert) {
        double c[4];
        gen_to_quat(w, cc.tol, c);
        st4(arr, s, (S)c[0], (S)c[1], (S)c[2], (S)c[3]);
    } else {
        st4(arr, s, (S)w[0], (S)w[1], (S)w[2], (S)0);
    }
}

template <class S, class H>
__device__ __forceinline__ void get_link(const S* arr, int s, H* w, const LinkCodec& cc)
{
    const S* q = arr + 4 * (size_t)s;
    if (!cc.gen) {
        for (int k = 0; k < 4; k++) w[k] = (H)q[k];
    } else if (cc.convert) {
        const double c[4] = {(double)q[0], (double)q[1], (double)q[2], (double)q[3]};
        double g[3];
        quat_to_gen(c, cc.tol, g);
        for (int k = 0; k < 3; k++) w[k] = (H)g[k];
    } else {
        for (int k = 0; k < 3; k++) w[k] = (H)q[k];
    }
}

// Reference AoS record -> structure-of-arrays level (one thread per site).
template <class S, class H>
__global__ void aos_to_soa_kernel(const H* __restrict__ sc, const H* __restrict__ ve, int nsite, int nsc,
                                  LevelPtrs<S> lv, LinkCodec cc)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nsite) return;
    const int lw = cc.gen ? 3 : 4;                                  // words of one SU(2) link
    const int dw = 1 + lw + (lv.hq[0] ? lw : (lv.hth[0] ? 1 : 0));  // link words per direction
    const H* v = ve + (size_t)s * 3 * dw;
#pragma unroll
    for (int d = 0; d < 3; d++) {
        const H* w = v + dw * d;
        lv.th[d][s] = (S)w[0];
        put_link(lv.q[d], s, w + 1, cc);
        if (lv.hth[0]) lv.hth[d][s] = (S)w[1 + lw];
        if (lv.hq[0]) put_link(lv.hq[d], s, w + 1 + lw, cc);
    }
    const H* f = sc + (size_t)s * nsc;
    for (int db = 0; db < nsc / 4; db++)
        st4(lv.ph[db], s, (S)f[4 * db], (S)f[4 * db + 1], (S)f[4 * db + 2], (S)f[4 * db + 3]);
}

template <class S, class H>
__global__ void soa_to_aos_kernel(LevelPtrs<S> lv, int nsite, int nsc, H* __restrict__ sc, H* __restrict__ ve,
                                  LinkCodec cc)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nsite) return;
    const int lw = cc.gen ? 3 : 4;
    const int dw = 1 + lw + (lv.hq[0] ? lw : (lv.hth[0] ? 1 : 0));
    H* v = ve + (size_t)s * 3 * dw;
#pragma unroll
    for (int d = 0; d < 3; d++) {
        H* w = v + dw * d;
        w[0] = (H)lv.th[d][s];
        get_link(lv.q[d], s, w + 1, cc);
        if (lv.hth[0]) w[1 + lw] = (H)lv.hth[d][s];
        if (lv.hq[0]) get_link(lv.hq[d], s, w + 1 + lw, cc);
    }
    H* f = sc + (size_t)s * nsc;
    for (int db = 0; db < nsc / 4; db++) {
        const S* p = lv.ph[db] + 4 * (size_t)s;
#pragma unroll
        for (int k = 0; k < 4; k++) f[4 * db + k] = (H)p[k];
    }
}

// Counter-based generator: SplitMix64 finaliser (Steele, Lea, Flood 2014) keyed by
// (seed, stream, index); uniforms from the top 53 bits; normals by the cosine
// branch of Box-Muller.  Stream ids: scalar component c -> c, theta_Y of
// direction d -> 16 + d, SU(2) angle -> 32 + d, axis cos(polar) -> 48 + d,
// axis azimuth -> 64 + d; Higgs-family phase -> 80 + d, Higgs-family SU(2)
// angle / cos(polar) / azimuth -> 96 / 112 / 128 + d.
__device__ __forceinline__ unsigned long long mix64(unsigned long long z)
{
    z += 0x9E3779B97F4A7C15ULL;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

__device__ __forceinline__ double uniform01(unsigned long long seed, unsigned long long stream, unsigned long long i)
{
    const unsigned long long h = mix64(mix64(seed ^ (stream * 0xD1B54A32D192ED03ULL)) + i);
    return ((double)(h >> 11) + 0.5) * (1.0 / 9007199254740992.0);
}

__device__ __forceinline__ double gaussian(unsigned long long seed, unsigned long long stream, unsigned long long i)
{
    const double two_pi = 6.283185307179586476925286766559;
    const double u1 = uniform01(seed, stream, 2 * i), u2 = uniform01(seed, stream, 2 * i + 1);
    return sqrt(-2.0 * log(u1)) * cos(two_pi * u2);
}

// Unit quaternion (cos eps, sin eps n): eps ~ N(0, eps_sigma^2) from stream s0,
// n uniform on S^2 from streams s0 + 16 (cos polar) and s0 + 32 (azimuth).
// With ic.store_generators the record is (w1, w2, w3, 0), w = eps n: the same
// group element in the generator representation.
__device__ __forceinline__ void random_link(const ICParams& ic, unsigned long long s0, unsigned long long key,
                                            double (&q)[4])
{
    const double two_pi = 6.283185307179586476925286766559;
    q[0] = ic.store_generators ? 0.0 : 1.0;
    q[1] = q[2] = q[3] = 0.0;
    if (ic.eps_sigma > 0.0) {
        const double eps = ic.eps_sigma * gaussian(ic.seed, s0, key);
        const double ct = 2.0 * uniform01(ic.seed, s0 + 16ULL, key) - 1.0;
        const double st = sqrt(1.0 - ct * ct);
        const double ph = two_pi * uniform01(ic.seed, s0 + 32ULL, key);
        if (ic.store_generators) {
            q[0] = eps * st * cos(ph);
            q[1] = eps * st * sin(ph);
            q[2] = eps * ct;
            return;
        }
        const double se = sin(eps);
        q[0] = cos(eps);
        q[1] = se * st * cos(ph);
        q[2] = se * st * sin(ph);
        q[3] = se * ct;
    }
}

template <class S>
__global__ void init_fields_kernel(StepParams P, int nsc, ICParams ic, LevelPtrs<S> a, LevelPtrs<S> b)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= P.nsite) return;
    const int zc = s % P.nz;
    // random-number key: the site's index in the whole lattice (differs from s only on an x-slab)
    const int plane = P.ny * P.nz;
    const int ng = ic.nx_global > 0 ? ic.nx_global : P.nx;
    const int xg = ((s / plane + ic.x_offset) % ng + ng) % ng;
    const unsigned long long key = (unsigned long long)xg * plane + (unsigned long long)(s % plane);
    double f[8];
    for (int c = 0; c < nsc; c++) {
        double v = ic.mean[c] + ic.sigma[c] * gaussian(ic.seed, (unsigned long long)c, key);
        if (c == 0 && ic.wall_width > 0.0) {
            const double zz = (double)zc;
            v += ic.wall_value * 0.5 *
                 (tanh((zz - 0.25 * P.nz) / ic.wall_width) - tanh((zz - 0.75 * P.nz) / ic.wall_width));
        }
        f[c] = v;
    }
    for (int db = 0; db < nsc / 4; db++) {
        st4(a.ph[db], s, (S)f[4 * db], (S)f[4 * db + 1], (S)f[4 * db + 2], (S)f[4 * db + 3]);
        st4(b.ph[db], s, (S)f[4 * db], (S)f[4 * db + 1], (S)f[4 * db + 2], (S)f[4 * db + 3]);
    }
    for (int d = 0; d < 3; d++) {
        const double th = ic.theta_sigma * gaussian(ic.seed, 16ULL + d, key);
        double q[4];
        random_link(ic, 32ULL + d, key, q);
        a.th[d][s] = (S)th;
        b.th[d][s] = (S)th;
        st4(a.q[d], s, (S)q[0], (S)q[1], (S)q[2], (S)q[3]);
        st4(b.q[d], s, (S)q[0], (S)q[1], (S)q[2], (S)q[3]);
        if (a.hth[0]) {
            const double h = ic.theta_sigma * gaussian(ic.seed, 80ULL + d, key);
            a.hth[d][s] = (S)h;
            b.hth[d][s] = (S)h;
        }
        if (a.hq[0]) {
            random_link(ic, 96ULL + d, key, q);
            st4(a.hq[d], s, (S)q[0], (S)q[1], (S)q[2], (S)q[3]);
            st4(b.hq[d], s, (S)q[0], (S)q[1], (S)q[2], (S)q[3]);
        }
    }
}

// Reduces the per-block partials [nblocks][nslots] of a logging step (the
// block reduction is reduce_rows_block, gft_reduce.cuh).  With a grid of G > 1
// blocks, block g reduces rows [g * rows_per_cta, (g + 1) * rows_per_cta) and
// writes one unscaled row out[g][nslots] (stage one of two); with G = 1 it
// reduces all rows and writes out[k] = total * scale[k].
constexpr int kFinMidRows = 512;  // most stage-one rows (the caller's mid buffer holds kFinMidRows x kMaxSlots)
__global__ void __launch_bounds__(kFinThreads) finalize_kernel(const double* __restrict__ partials, int nblocks,
                                                               int nslots, int max_from, const double* scale,
                                                               double* out, int rows_per_cta)
{
    const int b0 = (int)blockIdx.x * rows_per_cta;
    const int b1 = min(nblocks, b0 + rows_per_cta);
    const double total = reduce_rows_block(partials, b0, b1, nslots, max_from);
    if (threadIdx.x < (unsigned)nslots) {
        const int k = threadIdx.x;
        if (gridDim.x > 1)
            out[(size_t)blockIdx.x * nslots + k] = total;
        else
            out[k] = total * scale[k];
    }
}

// Self-test of gft_math.cuh against CUDA's functions: max abs error of
// sin/cos and max relative error of asin, float and double, over n points.
__global__ void math_selftest_kernel(int n, unsigned long long* err_bits)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    // arguments: a dense sweep of [-40, 40], then small magnitudes down to 1e-8
    double x;
    if (i < n / 2) {
        x = -40.0 + 80.0 * ((double)i + 0.5) / (double)(n / 2);
    } else {
        const double t = ((double)(i - n / 2) + 0.5) / (double)(n - n / 2);
        x = ((i & 1) ? -1.0 : 1.0) * exp(log(1e-8) * (1.0 - t) + log(0.5) * t);
    }
    float sf, cf;
    gsincos((float)x, sf, cf);
    const double xf = (double)(float)x;
    const double e0 = fabs((double)sf - sin(xf)), e1 = fabs((double)cf - cos(xf));
    const double e2 = fabs((double)gsin((float)x) - sin(xf));
    double sd, cd;
    gsincos(x, sd, cd);
    const double e3 = fabs(sd - sin(x)), e4 = fabs(cd - cos(x)), e5 = fabs(gsin(x) - sin(x));
    double e6 = 0.0, e7 = 0.0;
    const double ax = fabs(x);
    if (ax <= 0.999) {
        e6 = fabs((double)gasin((float)x) - asin(xf)) / fmax(fabs(asin(xf)), 1e-300);
        e7 = fabs(gasin(x) - asin(x)) / fmax(fabs(asin(x)), 1e-300);
    }
    // one_minus_cos_nr on the quaternion (cos x, sin x n) with |n|^2 = 1 + 2^-20 (not exactly
    // unit, as stored links are not), against the same expression in FP64 from the same floats
    const float w = (float)cos(x), sn = (float)sin(x);
    const float v1 = sn * 0.6f, v3 = sn * 0.8f * 1.0000005f;
    const float v2f = v1 * v1 + v3 * v3;
    const double v2 = (double)v1 * v1 + (double)v3 * v3, nrm = sqrt((double)w * w + v2);
    const double ex = (w >= 0.0f) ? v2 / (nrm * (nrm + w)) : 1.0 - w / nrm;
    const double e8 = (ex > 0.0) ? fabs((double)one_minus_cos_nr(w, v2f) - ex) / ex : 0.0;
    const double e[9] = {e0, e1, e2, e3, e4, e5, e6, e7, e8};
    for (int k = 0; k < 9; k++) atomicMax(err_bits + k, (unsigned long long)__double_as_longlong(e[k]));
}

}  // namespace

cudaError_t run_math_selftest(int n, double* out9)
{
    unsigned long long* d = nullptr;
    cudaError_t e = cudaMalloc(&d, 9 * sizeof(unsigned long long));
    if (e != cudaSuccess) return e;
    cudaMemset(d, 0, 9 * sizeof(unsigned long long));
    math_selftest_kernel<<<(n + 255) / 256, 256>>>(n, d);
    e = cudaGetLastError();
    unsigned long long h[9] = {0};
    if (e == cudaSuccess) e = cudaMemcpy(h, d, sizeof(h), cudaMemcpyDeviceToHost);
    cudaFree(d);
    for (int k = 0; k < 9; k++) {
        double v;
        memcpy(&v, &h[k], sizeof(double));
        out9[k] = v;
    }
    return e;
}

template <class S, class H>
cudaError_t launch_aos_to_soa(const H* aos_sc, const H* aos_ve, int nsite, int nsc, LevelPtrs<S> lv, cudaStream_t s,
                              LinkCodec codec)
{
    aos_to_soa_kernel<S, H><<<(nsite + 255) / 256, 256, 0, s>>>(aos_sc, aos_ve, nsite, nsc, lv, codec);
    return cudaGetLastError();
}

template <class S, class H>
cudaError_t launch_soa_to_aos(LevelPtrs<S> lv, int nsite, int nsc, H* aos_sc, H* aos_ve, cudaStream_t s,
                              LinkCodec codec)
{
    soa_to_aos_kernel<S, H><<<(nsite + 255) / 256, 256, 0, s>>>(lv, nsite, nsc, aos_sc, aos_ve, codec);
    return cudaGetLastError();
}

template <class S>
cudaError_t launch_init_fields(const StepParams& P, int nsc, const ICParams& ic, LevelPtrs<S> a, LevelPtrs<S> b,
                               cudaStream_t s)
{
    init_fields_kernel<S><<<(P.nsite + 255) / 256, 256, 0, s>>>(P, nsc, ic, a, b);
    return cudaGetLastError();
}

cudaError_t launch_finalize(const double* partials, int nblocks, int nslots, int max_from, const double* scale_dev,
                            double* out, double* mid, cudaStream_t s)
{
    if (nslots > kMaxSlots) return cudaErrorInvalidValue;
    if (mid != nullptr && nblocks > 2 * kFinThreads) {
        // two stages: at most kFinMidRows blocks of >= kFinThreads rows each, then one block
        int rpc = (nblocks + kFinMidRows - 1) / kFinMidRows;
        rpc = rpc < kFinThreads ? kFinThreads : rpc;
        const int g = (nblocks + rpc - 1) / rpc;
        finalize_kernel<<<g, kFinThreads, 0, s>>>(partials, nblocks, nslots, max_from, nullptr, mid, rpc);
        finalize_kernel<<<1, kFinThreads, 0, s>>>(mid, g, nslots, max_from, scale_dev, out, g);
        return cudaGetLastError();
    }
    finalize_kernel<<<1, kFinThreads, 0, s>>>(partials, nblocks, nslots, max_from, scale_dev, out, nblocks);
    return cudaGetLastError();
}

int finalize_launches(int nblocks, bool have_mid) { return (have_mid && nblocks > 2 * kFinThreads) ? 2 : 1; }

template cudaError_t launch_aos_to_soa<float, float>(const float*, const float*, int, int, LevelPtrs<float>,
                                                     cudaStream_t, LinkCodec);
template cudaError_t launch_aos_to_soa<float, double>(const double*, const double*, int, int, LevelPtrs<float>,
                                                      cudaStream_t, LinkCodec);
template cudaError_t launch_aos_to_soa<double, float>(const float*, const float*, int, int, LevelPtrs<double>,
                                                      cudaStream_t, LinkCodec);
template cudaError_t launch_aos_to_soa<double, double>(const double*, const double*, int, int, LevelPtrs<double>,
                                                       cudaStream_t, LinkCodec);
template cudaError_t launch_soa_to_aos<float, float>(LevelPtrs<float>, int, int, float*, float*, cudaStream_t, LinkCodec);
template cudaError_t launch_soa_to_aos<float, double>(LevelPtrs<float>, int, int, double*, double*, cudaStream_t, LinkCodec);
template cudaError_t launch_soa_to_aos<double, float>(LevelPtrs<double>, int, int, float*, float*, cudaStream_t, LinkCodec);
template cudaError_t launch_soa_to_aos<double, double>(LevelPtrs<double>, int, int, double*, double*, cudaStream_t, LinkCodec);
template cudaError_t launch_init_fields<float>(const StepParams&, int, const ICParams&, LevelPtrs<float>,
                                               LevelPtrs<float>, cudaStream_t);
template cudaError_t launch_init_fields<double>(const StepParams&, int, const ICParams&, LevelPtrs<double>,
                                                LevelPtrs<double>, cudaStream_t);

}  // namespace gft
