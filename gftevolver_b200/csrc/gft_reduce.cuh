// gft_reduce.cuh -- deterministic FP64 reduction of per-block partial rows.
#pragma once

#include <cuda_runtime.h>

namespace gft {

constexpr int kFinThreads = 1024;
constexpr int kMaxSlots = 16;

// Reduces rows [b0, b1) of partials[*][nslots] over the whole block (blockDim.x
// = kFinThreads, 1-D): each thread accumulates whole rows (coalesced), slot k
// with Neumaier compensation (k < max_from) or as a maximum (k >= max_from;
// values are >= 0); then the per-thread results are combined by a fixed
// shuffle tree and in warp order.  The order is fixed, so the result is
// deterministic.  Thread k < nslots returns the total of slot k.
__device__ __forceinline__ double reduce_rows_block(const double* __restrict__ partials, int b0, int b1, int nslots,
                                                    int max_from)
{
    __shared__ double s_sum[kMaxSlots][kFinThreads / 32];
    __shared__ double s_cmp[kMaxSlots][kFinThreads / 32];
    double sum[kMaxSlots], comp[kMaxSlots];
#pragma unroll
    for (int k = 0; k < kMaxSlots; k++) {
        sum[k] = 0.0;
        comp[k] = 0.0;
    }
    for (int b = b0 + (int)threadIdx.x; b < b1; b += blockDim.x) {
        const double* row = partials + (size_t)b * nslots;
#pragma unroll
        for (int k = 0; k < kMaxSlots; k++) {
            if (k >= nslots) break;
            const double v = row[k];
            if (k >= max_from) {
                sum[k] = fmax(sum[k], v);
            } else {
                const double t = sum[k] + v;
                comp[k] += (fabs(sum[k]) >= fabs(v)) ? (sum[k] - t) + v : (v - t) + sum[k];
                sum[k] = t;
            }
        }
    }
    // warp level: fold compensation in, then a fixed shuffle tree
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < kMaxSlots; k++) {
        if (k >= nslots) break;
        double v = (k >= max_from) ? sum[k] : sum[k] + comp[k];
        double c = 0.0;
        for (int o = 16; o > 0; o >>= 1) {
            // xor partners compute identical sums (addition is commutative)
            const double w = __shfl_xor_sync(0xffffffffu, v, o);
            const double cw = __shfl_xor_sync(0xffffffffu, c, o);
            if (k >= max_from) {
                v = fmax(v, w);
            } else {
                const double t = v + w;
                c = c + cw + ((fabs(v) >= fabs(w)) ? (v - t) + w : (w - t) + v);
                v = t;
            }
        }
        if (lane == 0) {
            s_sum[k][warp] = v;
            s_cmp[k][warp] = c;
        }
    }
    __syncthreads();
    double total = 0.0;
    if (threadIdx.x < (unsigned)nslots) {
        const int k = threadIdx.x;
        const bool is_max = k >= max_from;
        double tsum = 0.0, tcomp = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) {
            const double v = s_sum[k][w];
            if (is_max) {
                tsum = fmax(tsum, v);
            } else {
                const double u = tsum + v;
                tcomp += (fabs(tsum) >= fabs(v)) ? (tsum - u) + v : (v - u) + tsum;
                tsum = u;
                tcomp += s_cmp[k][w];
            }
        }
        total = is_max ? tsum : tsum + tcomp;
    }
    __syncthreads();  // s_sum / s_cmp may be reused by a following call
    return total;
}

}  // namespace gft
