// gft_tiled_tile.cuh -- one tile of the TMA-staged step kernel, shared by the
// single-lattice kernel (gft_tiled_kernels.cu) and the persistent ensemble
// kernel (gft_ensemble.cu).
//
// A tile is a (TY x TZ) set of (y, z) columns of one lattice marching along x
// (the slowest-varying axis) over nloc planes.  The "now" level of every plane
// the stencil touches is brought into shared memory once, by the Tensor Memory
// Accelerator: one cp.async.bulk.tensor per field array per plane, a
// (TY+2) x (TZ+2) box including the one-site halo, completing on an mbarrier.
// Four plane buffers form a ring: while plane x is computed from planes x-1, x
// and x+1, the copy of plane x+2 is in flight.  Halo cells that wrap around
// the periodic boundary (tiles on the lattice faces) are outside the tensor
// and arrive zero-filled; the CTA overwrites them with plain loads of the
// wrapped sites.  The own-site past level is read and written directly
// (coalesced: consecutive threads are consecutive z).
//
// Bounded waits: every mbarrier wait gives up after 2 s of %globaltimer (or the
// shorter diagnostic limit StepParams::wait_limit_ns); the tile then waits, with
// the 2 s bound, for its copies still in flight, reports failure and the caller
// records kErrTimeout in the status word.
#pragma once

#include <cuda.h>

#include "gft_device.cuh"
#include "gft_launch.h"
#include "gft_step_body.cuh"

namespace gft {
namespace tiled {

constexpr unsigned kErrTimeout = 8u;

__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(unsigned long long* bar, unsigned bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(unsigned long long* bar, unsigned parity)
{
    unsigned ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

__device__ __forceinline__ unsigned long long globaltimer_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Non-blocking test of phase `parity` of `bar`.
__device__ __forceinline__ bool mbar_test_wait(unsigned long long* bar, unsigned parity)
{
    unsigned ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Shared-memory counter add with acquire-release semantics at CTA scope:
// returns the previous value.
__device__ __forceinline__ unsigned atom_add_acq_rel(unsigned* p, unsigned v)
{
    unsigned old;
    asm volatile("atom.acq_rel.cta.shared::cta.add.u32 %0, [%1], %2;" : "=r"(old) : "r"(smem_u32(p)), "r"(v) : "memory");
    return old;
}

constexpr unsigned long long kWaitLimitNs = 2000000000ull;  // 2 s

// Wait for phase `parity` of `bar`; false after `limit_ns` (0: 2 s).  A limit
// below 1 us is one non-blocking test (the diagnostic of gft_set_wait_limit:
// it fails whenever the copy has not landed yet).
__device__ __forceinline__ bool mbar_wait_bounded(unsigned long long* bar, unsigned parity, unsigned limit_ns = 0)
{
    if (limit_ns - 1u < 999u) return mbar_test_wait(bar, parity);  // 1 <= limit < 1 us
    if (mbar_try_wait(bar, parity)) return true;
    const unsigned long long t0 = globaltimer_ns();
    for (;;) {
        if (mbar_try_wait(bar, parity)) return true;
        if (globaltimer_ns() - t0 > (limit_ns ? (unsigned long long)limit_ns : kWaitLimitNs)) return false;
    }
}

__device__ __forceinline__ void tma_load_4d(void* dst, const CUtensorMap* map, int c0, int c1, int c2, int c3,
                                            unsigned long long* bar)
{
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, "
        "%5}], [%6];" ::"r"(smem_u32(dst)),
        "l"(map), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int c0, int c1, int c2,
                                            unsigned long long* bar)
{
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
        "[%5];" ::"r"(smem_u32(dst)),
        "l"(map), "r"(c0), "r"(c1), "r"(c2), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ void tma_prefetch_l2_4d(const CUtensorMap* map, int c0, int c1, int c2, int c3)
{
    asm volatile("cp.async.bulk.prefetch.tensor.4d.L2.global.tile [%0, {%1, %2, %3, %4}];" ::"l"(map), "r"(c0),
                 "r"(c1), "r"(c2), "r"(c3)
                 : "memory");
}

__device__ __forceinline__ void tma_prefetch_l2_3d(const CUtensorMap* map, int c0, int c1, int c2)
{
    asm volatile("cp.async.bulk.prefetch.tensor.3d.L2.global.tile [%0, {%1, %2, %3}];" ::"l"(map), "r"(c0), "r"(c1),
                 "r"(c2)
                 : "memory");
}

// Warm L2 with the own-site past-level tile of plane X (boxes without halo).
template <int ND>
__device__ __forceinline__ void prefetch_past(const TMaps& pm, int X, int y0, int z0)
{
#pragma unroll
    for (int d = 0; d < 3; d++) tma_prefetch_l2_4d(&pm.q[d], 0, z0, y0, X);
#pragma unroll
    for (int d = 0; d < 3; d++) tma_prefetch_l2_3d(&pm.th[d], z0, y0, X);
#pragma unroll
    for (int k = 0; k < ND; k++) tma_prefetch_l2_4d(&pm.ph[k], 0, z0, y0, X);
}

// Shared-memory plane geometry.
template <class S, int TY, int TZ, int ND>
struct Geom {
    static constexpr int TP = 16 / (int)sizeof(S);  // theta box starts TP columns left (16-byte aligned)
    static constexpr int ROWS = TY + 2;
    static constexpr int QP = TZ + 2;           // pitch of q / phi tiles (records of 4 S)
    static constexpr int HP = TZ + 2 * TP;      // pitch of theta tiles
    static constexpr int QBOX = ROWS * QP * 4 * (int)sizeof(S);
    static constexpr int HBOX = ROWS * HP * (int)sizeof(S);
    static constexpr int QB = (QBOX + 127) / 128 * 128;
    static constexpr int HB = (HBOX + 127) / 128 * 128;
    static constexpr int OFF_TH = 3 * QB;
    static constexpr int OFF_PH = 3 * QB + 3 * HB;
    static constexpr int BUF = 3 * QB + 3 * HB + ND * QB;
    static constexpr int NBUF = 4;
    static constexpr unsigned TX = 3 * QBOX + 3 * HBOX + ND * QBOX;  // bytes per plane copy
    static constexpr int SMEM = NBUF * BUF + 128 + 64;             // + alignment slack + barriers
};

// Staging area for the wrapped halo cells of one plane (plain steps of the
// tiled kernel): one slot per halo cell (the halo_cell numbering), quaternion
// records [3 + ND][NH] then phases [3][NH], placed after the plane barriers.
// FP32 only (the tiled kernel serves the mixed form).
template <class S, int TY, int TZ, int ND>
struct HaloStage {
    using G = Geom<S, TY, TZ, ND>;
    static constexpr int NH = 2 * G::QP + 2 * TY;
    static constexpr int OFF_H = (3 + ND) * NH * 16;
    static constexpr int BYTES = OFF_H + 3 * NH * 4;
    static constexpr int OFFSET = G::NBUF * G::BUF + 64;  // 16-byte aligned (BUF is a multiple of 128)
    static constexpr int SMEM = OFFSET + BYTES + 128;      // + alignment slack of the dynamic base
    // Used only when it leaves the resident CTAs per SM unchanged: 228 KB of
    // shared memory per SM, 1 KB reserved and 16 bytes static per CTA.
    static constexpr int per_sm(int dyn) { return (228 * 1024) / (dyn + 16 + 1024); }
    static constexpr bool kUse = sizeof(S) == 4 && SMEM <= 227 * 1024 && per_sm(SMEM) >= per_sm(G::SMEM);
};

// Reference to a site in a staged plane: buffer base, q/phi cell, theta cell.
struct TRef {
    const unsigned char* b;
    int cq, ch;
};

template <class S, int TY, int TZ, int ND>
struct TileAcc {
    using G = Geom<S, TY, TZ, ND>;
    __device__ __forceinline__ Q<S> q(int d, TRef r) const { return lds4(r.b + d * G::QB, r.cq); }
    __device__ __forceinline__ S th(int d, TRef r) const
    {
        return reinterpret_cast<const S*>(r.b + G::OFF_TH + d * G::HB)[r.ch];
    }
    __device__ __forceinline__ Q<S> ph(int k, TRef r) const { return lds4(r.b + G::OFF_PH + k * G::QB, r.cq); }

    __device__ __forceinline__ static Q<S> lds4(const unsigned char* base, int cell)
    {
        if constexpr (sizeof(S) == 4) {
            const float4 v = reinterpret_cast<const float4*>(base)[cell];
            return {(S)v.x, (S)v.y, (S)v.z, (S)v.w};
        } else {
            const double2* p = reinterpret_cast<const double2*>(base) + 2 * cell;
            const double2 a = p[0], c = p[1];
            return {(S)a.x, (S)a.y, (S)c.x, (S)c.y};
        }
    }
};

template <class S, int TY, int TZ, int ND>
__device__ __forceinline__ void issue_plane(const TMaps& maps, unsigned char* buf, unsigned long long* bar, int X,
                                            int y0, int z0)
{
    using G = Geom<S, TY, TZ, ND>;
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    mbar_expect_tx(bar, G::TX);
#pragma unroll
    for (int d = 0; d < 3; d++) tma_load_4d(buf + d * G::QB, &maps.q[d], 0, z0 - 1, y0 - 1, X, bar);
#pragma unroll
    for (int d = 0; d < 3; d++) tma_load_3d(buf + G::OFF_TH + d * G::HB, &maps.th[d], z0 - G::TP, y0 - 1, X, bar);
#pragma unroll
    for (int k = 0; k < ND; k++) tma_load_4d(buf + G::OFF_PH + k * G::QB, &maps.ph[k], 0, z0 - 1, y0 - 1, X, bar);
}

// Halo cell handled by thread `tid` (2*QP + 2*TY cells: rows 0 and TY+1, then
// columns 0 and TZ+1); false if tid has none.
template <int TY, int QP>
__device__ __forceinline__ bool halo_cell(int tid, int& ly, int& lz)
{
    if (tid >= 2 * QP + 2 * TY) return false;
    if (tid < QP) {
        ly = 0;
        lz = tid;
    } else if (tid < 2 * QP) {
        ly = TY + 1;
        lz = tid - QP;
    } else if (tid < 2 * QP + TY) {
        ly = 1 + (tid - 2 * QP);
        lz = 0;
    } else {
        ly = 1 + (tid - 2 * QP - TY);
        lz = QP - 1;
    }
    return true;
}

// Warm L2 with the wrapped halo sites of plane X (one plane before they are
// patched), so the patch loads do not wait on DRAM.
template <class S, int TY, int TZ, int ND, class LV>
__device__ __forceinline__ void prefetch_wrapped_halo(const StepParams& P, const LV& now, int X, int y0,
                                                      int z0, int tid)
{
    using G = Geom<S, TY, TZ, ND>;
    int ly, lz;
    if (!halo_cell<TY, G::QP>(tid, ly, lz)) return;
    int y = y0 - 1 + ly, z = z0 - 1 + lz;
    if (y >= 0 && y < P.ny && z >= 0 && z < P.nz) return;
    y = (y < 0) ? y + P.ny : (y >= P.ny ? y - P.ny : y);
    z = (z < 0) ? z + P.nz : (z >= P.nz ? z - P.nz : z);
    const size_t s = ((size_t)X * P.ny + y) * P.nz + z;
#pragma unroll
    for (int d = 0; d < 3; d++) {
        asm volatile("prefetch.global.L2 [%0];" ::"l"(now.q[d] + 4 * s));
        asm volatile("prefetch.global.L2 [%0];" ::"l"(now.th[d] + s));
    }
#pragma unroll
    for (int k = 0; k < ND; k++) asm volatile("prefetch.global.L2 [%0];" ::"l"(now.ph[k] + 4 * s));
}

// Halo cells of plane X whose (y, z) leaves the lattice: load the wrapped
// site from global memory into the staged plane.
template <class S, int TY, int TZ, int ND, class LV>
__device__ __forceinline__ void patch_wrapped_halo(const StepParams& P, const LV& now, unsigned char* buf,
                                                   int X, int y0, int z0, int tid)
{
    using G = Geom<S, TY, TZ, ND>;
    int ly, lz;
    if (!halo_cell<TY, G::QP>(tid, ly, lz)) return;
    int y = y0 - 1 + ly, z = z0 - 1 + lz;
    if (y >= 0 && y < P.ny && z >= 0 && z < P.nz) return;  // delivered by the tensor copy
    y = (y < 0) ? y + P.ny : (y >= P.ny ? y - P.ny : y);
    z = (z < 0) ? z + P.nz : (z >= P.nz ? z - P.nz : z);
    const int s = (X * P.ny + y) * P.nz + z;
    const int cq = ly * G::QP + lz, ch = ly * G::HP + lz + G::TP - 1;
#pragma unroll
    for (int d = 0; d < 3; d++) {
        const Q<S> v = ld4<S>(now.q[d], s);
        st4(reinterpret_cast<S*>(buf + d * G::QB), cq, v.w, v.x, v.y, v.z);
        reinterpret_cast<S*>(buf + G::OFF_TH + d * G::HB)[ch] = ld1<S>(now.th[d], s);
    }
#pragma unroll
    for (int k = 0; k < ND; k++) {
        const Q<S> v = ld4<S>(now.ph[k], s);
        st4(reinterpret_cast<S*>(buf + G::OFF_PH + k * G::QB), cq, v.w, v.x, v.y, v.z);
    }
}

// As prefetch_wrapped_halo, but the wrapped sites of plane X go by cp.async
// into this thread's slots of the staging area, one plane before they are
// patched (patch_from_stage).
template <class S, int TY, int TZ, int ND, class LV>
__device__ __forceinline__ void stage_wrapped_halo(const StepParams& P, const LV& now, int X, int y0, int z0, int tid,
                                                   unsigned char* stage)
{
    using G = Geom<S, TY, TZ, ND>;
    using H = HaloStage<S, TY, TZ, ND>;
    static_assert(sizeof(S) == 4, "the halo stage holds FP32 records");
    int ly, lz;
    if (!halo_cell<TY, G::QP>(tid, ly, lz)) return;
    int y = y0 - 1 + ly, z = z0 - 1 + lz;
    if (y >= 0 && y < P.ny && z >= 0 && z < P.nz) return;
    y = (y < 0) ? y + P.ny : (y >= P.ny ? y - P.ny : y);
    z = (z < 0) ? z + P.nz : (z >= P.nz ? z - P.nz : z);
    const size_t s = ((size_t)X * P.ny + y) * P.nz + z;
#pragma unroll
    for (int d = 0; d < 3; d++) {
        cp_async16(stage + (d * H::NH + tid) * 16, now.q[d] + 4 * s);
        cp_async4(stage + H::OFF_H + (d * H::NH + tid) * 4, now.th[d] + s);
    }
#pragma unroll
    for (int k = 0; k < ND; k++) cp_async16(stage + ((3 + k) * H::NH + tid) * 16, now.ph[k] + 4 * s);
    cp_async_commit();
}

// The wrapped halo cells of the plane in `buf` from this thread's staging
// slots (filled by stage_wrapped_halo for that plane).
template <class S, int TY, int TZ, int ND>
__device__ __forceinline__ void patch_from_stage(const StepParams& P, unsigned char* buf, int y0, int z0, int tid,
                                                 const unsigned char* stage)
{
    using G = Geom<S, TY, TZ, ND>;
    using H = HaloStage<S, TY, TZ, ND>;
    int ly, lz;
    if (!halo_cell<TY, G::QP>(tid, ly, lz)) return;
    const int y = y0 - 1 + ly, z = z0 - 1 + lz;
    if (y >= 0 && y < P.ny && z >= 0 && z < P.nz) return;
    cp_async_wait_all();
    const int cq = ly * G::QP + lz, ch = ly * G::HP + lz + G::TP - 1;
    const float4* sq = reinterpret_cast<const float4*>(stage);
    const float* sh = reinterpret_cast<const float*>(stage + H::OFF_H);
#pragma unroll
    for (int d = 0; d < 3; d++) {
        reinterpret_cast<float4*>(buf + d * G::QB)[cq] = sq[d * H::NH + tid];
        reinterpret_cast<float*>(buf + G::OFF_TH + d * G::HB)[ch] = sh[d * H::NH + tid];
    }
#pragma unroll
    for (int k = 0; k < ND; k++) reinterpret_cast<float4*>(buf + G::OFF_PH + k * G::QB)[cq] = sq[(3 + k) * H::NH + tid];
}

// Parity of the completed phases of the NBUF plane barriers (bit b for
// barrier b), carried from tile to tile by a persistent CTA (every thread
// holds the same value).
struct RingPhase {
    unsigned bits;
};

// The plane ring of one tile (planes x0 .. x0+nloc-1 of columns y0.., z0..):
// TMA copies, waits, wrapped-halo patches and one CTA barrier per plane.
// body(i, bm, bc, bp) evolves the tile's sites of plane x0 + i from the staged
// planes bm (x - 1), bc (x) and bp (x + 1).  tid: the thread's index in the CTA
// (the halo cells and the copy issue are divided by it).  smem: NBUF plane
// buffers followed by NBUF initialised mbarriers; s_abort: a shared flag that
// is 0 on entry.  Returns false (on every thread) if a wait gave up; the ring
// is then drained and must not be reused.  LV: the level pointer struct (its
// q / th / ph members are read).
// STAGE: the wrapped halo cells of plane i+4 are copied by cp.async into
// `stage` (HaloStage) while plane i+1 is computed, instead of prefetched into L2
// and loaded after the plane's wait.
template <class S, int TY, int TZ, int ND, class LV, bool STAGE, class Body>
__device__ __forceinline__ bool run_ring(const TMaps& maps, const TMaps& pmaps, const StepParams& P, const LV& now,
                                         int y0, int z0, int x0, int nloc, unsigned char* smem,
                                         unsigned long long* bars, RingPhase& ring, int* s_abort,
                                         unsigned char* stage, int tid, Body&& body)
{
    using G = Geom<S, TY, TZ, ND>;
    const int nplanes = nloc + 2;  // planes x0-1 .. x0+nloc
    const bool wraps = (y0 == 0) || (y0 + TY == P.ny) || (z0 == 0) || (z0 + TZ == P.nz);
    auto plane_x = [&](int p) {  // global x of relative plane p (p = 0 is x0 - 1)
        int X = x0 - 1 + p;
        return (X < 0) ? X + P.nx : (X >= P.nx ? X - P.nx : X);
    };
    auto parity = [&](int p) { return ((ring.bits >> (p % G::NBUF)) ^ (unsigned)(p / G::NBUF)) & 1u; };
    // Tiles without wrapped halo cells in the FP64 form march without a CTA
    // barrier per plane (below): its warps wait on long FP64 latencies, and the
    // FP64 step (one CTA of 8 warps per SM) measured 2 % faster at 256^3.  The
    // FP32 steps keep the barrier: without it the SM step (two CTAs per SM) was
    // 3 % slower at 256^3 and the 2HDM step (one CTA per SM) 4 % slower at
    // 192^3, their warps waiting on copies and past-level loads instead.
    constexpr bool kFree = sizeof(S) == 8;
    // After the barriers: per buffer, the warps that have computed the plane in
    // it (tiles without wrapped halo); then the number of planes issued.
    unsigned* ctr = reinterpret_cast<unsigned*>(bars + G::NBUF);
    const unsigned nwarps = (blockDim.x * blockDim.y * blockDim.z) >> 5;

    if (tid == 0) {
        for (int p = 0; p < min(G::NBUF, nplanes); p++)
            issue_plane<S, TY, TZ, ND>(maps, smem + p * G::BUF, &bars[p], plane_x(p), y0, z0);
        if constexpr (kFree) {
            for (int b = 0; b < G::NBUF; b++) ctr[b] = 0u;
            ctr[G::NBUF] = (unsigned)min(G::NBUF, nplanes);
        }
    }
    if (tid == 32 % (TY * TZ)) {
        // past level of the first two planes computed (relative planes 1 and 2)
        for (int p = 1; p <= 2 && p <= nloc; p++) prefetch_past<ND>(pmaps, plane_x(p), y0, z0);
    }
    if (wraps && nplanes > 3) {
        if constexpr (STAGE)
            stage_wrapped_halo<S, TY, TZ, ND>(P, now, plane_x(3), y0, z0, tid, stage);
        else
            prefetch_wrapped_halo<S, TY, TZ, ND>(P, now, plane_x(3), y0, z0, tid);
    }

    // planes 0, 1, 2 (x0-1, x0, x0+1) resident and patched before the first site
    bool ok = true;
    for (int p = 0; p < 3; p++) {  // nplanes >= 3
        ok = ok && mbar_wait_bounded(&bars[p], parity(p), P.wait_limit_ns);
        if (ok && wraps) patch_wrapped_halo<S, TY, TZ, ND>(P, now, smem + p * G::BUF, plane_x(p), y0, z0, tid);
    }
    if (!ok) *s_abort = 1;
    __syncthreads();
    // on a failed wait: the copies of planes [drain0, drain1) may still be in flight
    int drain0 = 0, drain1 = min(G::NBUF, nplanes);
    bool aborted = *s_abort != 0;

    // Tiles with wrapped halo cells: one CTA barrier per plane: after computing
    // plane i the threads wait for (and patch) plane i+3, which the next site
    // needs, then synchronise once; that barrier both publishes the patches and
    // frees plane i's buffer for the copy of plane i+4.
    for (int i = 0; i < nloc && !aborted; i++) {
        body(i, smem + (i % G::NBUF) * G::BUF, smem + ((i + 1) % G::NBUF) * G::BUF,
             smem + ((i + 2) % G::NBUF) * G::BUF);

        if (kFree && !wraps) {
            // No patches to publish: plane i's buffer is free once every warp has
            // computed plane i, and the last warp to finish it issues the copy of
            // plane i+4 there (release by each warp's count, acquire by the last),
            // so a warp waits only for the copy of the plane it needs next and may
            // run up to a plane ahead of the slowest.
            __syncwarp();
            if ((tid & 31) == 0 && i + G::NBUF < nplanes &&
                atom_add_acq_rel(&ctr[i % G::NBUF], 1u) % nwarps == nwarps - 1) {
                issue_plane<S, TY, TZ, ND>(maps, smem + (i % G::NBUF) * G::BUF, &bars[i % G::NBUF],
                                           plane_x(i + G::NBUF), y0, z0);
                *reinterpret_cast<volatile unsigned*>(&ctr[G::NBUF]) = (unsigned)(i + G::NBUF + 1);
            }
            if (tid == 32 % (TY * TZ) && i + 3 <= nloc) prefetch_past<ND>(pmaps, plane_x(i + 3), y0, z0);
            if (i + 3 < nplanes && !mbar_wait_bounded(&bars[(i + 3) % G::NBUF], parity(i + 3), P.wait_limit_ns))
                *reinterpret_cast<volatile int*>(s_abort) = 1;
            // leave the march warp by warp (the next __syncwarp needs every lane)
            if (__any_sync(0xffffffffu, *reinterpret_cast<volatile int*>(s_abort) != 0)) break;
            continue;
        }

        // plane i+3 (x+2) for the next site; its copy was issued one plane ago
        bool okn = true;
        if (i + 3 < nplanes) {
            okn = mbar_wait_bounded(&bars[(i + 3) % G::NBUF], parity(i + 3), P.wait_limit_ns);
            if (okn && wraps) {
                if constexpr (STAGE)
                    patch_from_stage<S, TY, TZ, ND>(P, smem + ((i + 3) % G::NBUF) * G::BUF, y0, z0, tid, stage);
                else
                    patch_wrapped_halo<S, TY, TZ, ND>(P, now, smem + ((i + 3) % G::NBUF) * G::BUF, plane_x(i + 3), y0,
                                                      z0, tid);
            }
        }
        if (!okn) *s_abort = 1;
        __syncthreads();
        if (*s_abort) {  // planes 0 .. i+2 were waited; the last copy issued was plane i+3
            aborted = true;
            drain0 = i + 3;
            drain1 = min(nplanes, i + 4);
            break;
        }
        if (tid == 32 % (TY * TZ) && i + 3 <= nloc) prefetch_past<ND>(pmaps, plane_x(i + 3), y0, z0);
        if (wraps && i + 4 < nplanes) {
            if constexpr (STAGE)
                stage_wrapped_halo<S, TY, TZ, ND>(P, now, plane_x(i + 4), y0, z0, tid, stage);
            else
                prefetch_wrapped_halo<S, TY, TZ, ND>(P, now, plane_x(i + 4), y0, z0, tid);
        }
        if (tid == 0 && i + G::NBUF < nplanes)
            issue_plane<S, TY, TZ, ND>(maps, smem + (i % G::NBUF) * G::BUF, &bars[i % G::NBUF],
                                       plane_x(i + G::NBUF), y0, z0);
    }
    if constexpr (STAGE) cp_async_wait_all();  // a staged plane not patched (abort) is still in flight
    if (kFree && !wraps) {
        // every warp is done with the ring (the next tile refills it); on a failed
        // wait, the copies of the last NBUF planes issued may still be in flight
        __syncthreads();
        aborted = *reinterpret_cast<volatile int*>(s_abort) != 0;
        if (aborted) {  // no next tile then
            drain1 = (int)*reinterpret_cast<volatile unsigned*>(&ctr[G::NBUF]);
            drain0 = max(0, drain1 - G::NBUF);
        }
    }
    if (aborted) {
        // drain: wait (bounded) for the copies still in flight into this CTA's buffers
        if (tid == 0)
            for (int p = drain0; p < drain1; p++) mbar_wait_bounded(&bars[p % G::NBUF], parity(p));
        __syncthreads();
        return false;
    }
#pragma unroll
    for (int b = 0; b < G::NBUF; b++)
        if (b < nplanes) ring.bits ^= (((unsigned)((nplanes - b + G::NBUF - 1) / G::NBUF)) & 1u) << b;
    return true;
}

// Stencil references of the site in cell (cq0, ch0) of the staged planes bm, bc, bp.
template <int QP, int HP>
__device__ __forceinline__ Stencil<TRef> plane_stencil(const unsigned char* bm, const unsigned char* bc,
                                                       const unsigned char* bp, int cq0, int ch0)
{
    Stencil<TRef> n;
    n.c = {bc, cq0, ch0};
    n.m[0] = {bm, cq0, ch0};
    n.p[0] = {bp, cq0, ch0};
    n.m[1] = {bc, cq0 - QP, ch0 - HP};
    n.p[1] = {bc, cq0 + QP, ch0 + HP};
    n.m[2] = {bc, cq0 - 1, ch0 - 1};
    n.p[2] = {bc, cq0 + 1, ch0 + 1};
    n.d01 = {bp, cq0 - QP, ch0 - HP};
    n.d02 = {bp, cq0 - 1, ch0 - 1};
    n.d10 = {bm, cq0 + QP, ch0 + HP};
    n.d12 = {bc, cq0 + QP - 1, ch0 + HP - 1};
    n.d20 = {bm, cq0 + 1, ch0 + 1};
    n.d21 = {bc, cq0 - QP + 1, ch0 - HP + 1};
    return n;
}

// Evolves one tile by one step, one site per thread (threads TZ x TY).
template <class S, int MODEL, int TY, int TZ, bool ENERGY, class LV, bool STAGE = false>
__device__ __forceinline__ bool run_tile(const TMaps& maps, const TMaps& pmaps, const StepParams& P, const FConst& F,
                                         const LV& now, const LV& past, int y0, int z0, int x0,
                                         int nloc, unsigned char* smem, unsigned long long* bars, RingPhase& ring,
                                         int* s_abort, double (&obs)[kObsCount], unsigned& warn,
                                         unsigned char* stage = nullptr)
{
    constexpr int ND = (MODEL == kModelSM) ? 1 : 2;
    using G = Geom<S, TY, TZ, ND>;
    const int tz = threadIdx.x, ty = threadIdx.y;
    const int tid = ty * TZ + tz;
    // own cells
    const int cq0 = (ty + 1) * G::QP + (tz + 1);
    const int ch0 = (ty + 1) * G::HP + (tz + 1) + G::TP - 1;
    const int y = y0 + ty, z = z0 + tz;
    XCarry<S, ND> carry;
    carry.valid = false;
    return run_ring<S, TY, TZ, ND, LV, STAGE>(
        maps, pmaps, P, now, y0, z0, x0, nloc, smem, bars, ring, s_abort, stage, tid,
        [&](int i, const unsigned char* bm, const unsigned char* bc, const unsigned char* bp) {
            const Stencil<TRef> n = plane_stencil<G::QP, G::HP>(bm, bc, bp, cq0, ch0);
            const int x = x0 + i;
            const int s = (x * P.ny + y) * P.nz + z;
            if (frozen(P, x, y, z))  // Fixed faces: not evolved, and the next site recomputes what it carries
                carry.valid = false;
            else if (carry.valid)  // every site of the march after the first (uniform without Fixed faces)
                site_step<S, MODEL, ENERGY, kHfNone, true>(P, F, TileAcc<S, TY, TZ, ND>{}, n,
                                                           PastSite<S, LV>{past, s}, carry, obs, warn, counts(P, x));
            else
                site_step<S, MODEL, ENERGY>(P, F, TileAcc<S, TY, TZ, ND>{}, n, PastSite<S, LV>{past, s}, carry, obs,
                                            warn, counts(P, x));
        });
}

}  // namespace tiled
}  // namespace gft
