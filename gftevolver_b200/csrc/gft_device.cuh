// gft_device.cuh -- device-side layout, parameters and algebra shared by the
// step kernels.
//
// HBM layout (structure of arrays, one block per time level):
//   q[d]  : [N][4] storage words, SU(2) quaternion (c0, c1, c2, c3) of the link in direction d
//   th[d] : [N]    storage words, U(1) hypercharge phase theta_Y of the link in direction d
//   ph[k] : [N][4] storage words, Higgs doublet k (k = 0 for SM, 0..1 for 2HDM)
//   hth[d]: [N]    2HDM Higgs-family U(1) phase theta_H (gaugeNum 5 only)
//   hq[d] : [N][4] 2HDM Higgs-family SU(2) quaternion (gaugeNum 7 only)
// Site index s = (x*ny + y)*nz + z as in the reference (Core/Source/Lattice.cpp:658-671).
// The reference's AoS record per site ([theta, c0..c3] x 3 directions, then the
// scalar components) is split so that a warp reads 16- or 32-byte vectors of
// consecutive sites.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace gft {

constexpr int kModelSM = 1;
constexpr int kModel2HDM = 2;

// Observable slots reduced per block on logging steps.
enum ObsSlot : int {
    kObsEnergy = 0,
    kObsPotential,
    kObsGradient,
    kObsKinetic,
    kObsMagnetic,
    kObsElectric,
    kObsPlaqSU2,
    kObsPlaqU1,
    kObsPhiSq,
    kObsCount
};
constexpr int kGaussSlots = 8;  // integrated |viol| (4) then max |viol| (4)

// 2HDM Higgs-family gauge field (WilsonLoops/Source/TwoHDM.cpp:210-242): none
// (gaugeNum 4), a U(1) phase (gaugeNum 5) or an SU(2) quaternion (gaugeNum 7).
constexpr int kHfNone = 0;
constexpr int kHfU1 = 1;
constexpr int kHfSU2 = 2;
constexpr int kEqMax = 7;                     // gauge equations per direction (gaugeNum) at most
constexpr int kGaussSlotsMax = 2 * kEqMax;    // integrated then max |viol| per constraint
__host__ __device__ constexpr int hf_neq(int hf) { return hf == kHfU1 ? 5 : (hf == kHfSU2 ? 7 : 4); }

template <class S>
struct LevelPtrs {
    S* q[3];
    S* th[3];
    S* ph[2];
    S* hth[3];   // Higgs-family U(1) phase (null unless gaugeNum 5)
    S* hq[3];    // Higgs-family SU(2) quaternion (null unless gaugeNum 7)
};

// Per-launch parameters (POD, passed by value).
struct StepParams {
    int nx, ny, nz;
    int nsite;
    double dt, dt2;
    double lap[3];          // 1/dx_a^2 (covariant Laplacian and Wilson-loop weights)
    double inv_dx[3];       // 1/dx_a (forward-difference gradient energy)
    double inv_sqr_dt;      // 1/dt^2
    double gsq[4];          // coupling^2 per equation k % 4 (as the reference's getSqrCouplings returns it)
    double inv_g_sqr, inv_gp_sqr;
    int hf;                 // 2HDM Higgs-family gauge field (kHf*)
    int gen;                // reference-arithmetic form: links stored as generators (WilsonLoops/Source/StandardModel.cpp:76-160)
    double gsq_hf;          // g''^2 of the Higgs-family equations (TwoHDM.cpp:258-267)
    double inv_gpp_sqr;     // 1/g''^2 (0 below the division tolerance)
    double div_tol;         // divisionByZeroTolerance of the generator conversions
    float* loc_energy;      // non-null on a local-output step: per-site densities [N][6] (energy, potential,
                            // gradient, kinetic, magnetic, electric; Analysers/Source/Energy.cpp:117-163)
    float* loc_gauss;       // non-null on a local-output step: per-site signed violations [N][gaugeNum]
                            // (Analysers/Source/GaugeCondition.cpp:117-140)
    double damping_step;    // 0.5 * damping * dt for this step
    // SO_N
    double lambda, eta_sqr;
    // Double_SO_N
    double m1, m2, l1, l2, l3, m12r, l4p5, l6r, l7r, m12i, l4m5, l5i, l6i, l7i;
    int break_son, break_uhalfn, apply_norm;
    unsigned wait_limit_ns;  // limit of the tiled kernels' plane waits (0: 2 s); the drain after a
                             // failed wait keeps the 2 s bound (placed in what was padding)
    double energy_offset;
    int store_energy;       // logging step: renormalise as the reference does and accumulate energies
    int obs_x0, obs_x1;     // planes whose sites count in observables, Gauss residuals and warnings
                            // (all planes, except on an x-slab with ghost planes)
    int fixed_axes;         // bit a: the two faces of axis a are Fixed (frozen, not evolved)
};

// The mixed form's per-site constants in float, precomputed on the host and
// passed by value, so the step's FP32 arithmetic takes them as constant
// operands (no double-to-float conversion or FP64 arithmetic per site, no
// registers held for them; measured 2-3 % on the SM step).
struct FConst {
    float lap[3];      // 1/dx_a^2
    float diag;        // -2 (1/dx^2 + 1/dy^2 + 1/dz^2)
    float dt2, keep;   // dt^2, 1 - damping_step
    float gY, gI;      // g'^2, g^2 as the couplings of the link equations
    float lambda, eta_sqr;
    // Double_SO_N dV/dphi coefficients (Potentials/Source/Double_SO_N.cpp:244-341)
    float m1x2n, l1x4, l3x2, m2x2n, l2x4;        // -2 m1, 4 l1, 2 l3, -2 m2, 4 l2
    float m12rn, l4p5x2, l6r, l7r, l6rx2, l7rx2;  // -m12r, 2 l4p5, l6r, l7r, 2 l6r, 2 l7r
    float m12i, l4m5x2, l5ix2, l6i, l7i, l6ix2, l7ix2;
    // logging-step energy weights (the float values of the FP64 products they replace)
    float e_plaq[3];   // 4 lap_i lap_j for the planes (0,1), (0,2), (1,2)
    float e_grad[3];   // 0.5 / dx_a^2
    float e_elec[3];   // 4 lap_d / dt^2
    float inv_g_sqr, inv_gp_sqr, inv_gpp_sqr;
};

__host__ __device__ inline FConst make_fconst(const StepParams& P)
{
    FConst F;
    for (int a = 0; a < 3; a++) F.lap[a] = (float)P.lap[a];
    F.diag = (float)(-2.0 * (P.lap[0] + P.lap[1] + P.lap[2]));
    F.dt2 = (float)P.dt2;
    F.keep = (float)(1.0 - P.damping_step);
    F.gY = (float)P.gsq[0];
    F.gI = (float)P.gsq[1];
    F.lambda = (float)P.lambda;
    F.eta_sqr = (float)P.eta_sqr;
    F.m1x2n = (float)(-2.0 * P.m1);
    F.l1x4 = (float)(4.0 * P.l1);
    F.l3x2 = (float)(2.0 * P.l3);
    F.m2x2n = (float)(-2.0 * P.m2);
    F.l2x4 = (float)(4.0 * P.l2);
    F.m12rn = (float)(-P.m12r);
    F.l4p5x2 = (float)(2.0 * P.l4p5);
    F.l6r = (float)P.l6r;
    F.l7r = (float)P.l7r;
    F.l6rx2 = (float)(2.0 * P.l6r);
    F.l7rx2 = (float)(2.0 * P.l7r);
    F.m12i = (float)P.m12i;
    F.l4m5x2 = (float)(2.0 * P.l4m5);
    F.l5ix2 = (float)(2.0 * P.l5i);
    F.l6i = (float)P.l6i;
    F.l7i = (float)P.l7i;
    F.l6ix2 = (float)(2.0 * P.l6i);
    F.l7ix2 = (float)(2.0 * P.l7i);
    const int pi[3] = {0, 0, 1}, pj[3] = {1, 2, 2};
    for (int pl = 0; pl < 3; pl++) F.e_plaq[pl] = (float)(4.0 * P.lap[pi[pl]] * P.lap[pj[pl]]);
    for (int a = 0; a < 3; a++) {
        F.e_grad[a] = (float)(0.5 * P.inv_dx[a] * P.inv_dx[a]);
        F.e_elec[a] = (float)(4.0 * P.lap[a] * P.inv_sqr_dt);
    }
    F.inv_g_sqr = (float)P.inv_g_sqr;
    F.inv_gp_sqr = (float)P.inv_gp_sqr;
    F.inv_gpp_sqr = (float)P.inv_gpp_sqr;
    return F;
}

// Per-thread asynchronous copies global -> shared (cp.async): they complete on
// their own (no wait of another thread is involved) and the issuing thread
// sees the data after cp.async.wait_all.  Both addresses aligned to the size.
__device__ __forceinline__ void cp_async16(void* dst, const void* src)
{
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"((unsigned)__cvta_generic_to_shared(dst)),
                 "l"(__cvta_generic_to_global(src))
                 : "memory");
}
__device__ __forceinline__ void cp_async4(void* dst, const void* src)
{
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"((unsigned)__cvta_generic_to_shared(dst)),
                 "l"(__cvta_generic_to_global(src))
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// A site on a Fixed face (BoundaryConditions/Source/Fixed.cpp:159-251): not
// evolved, not part of the analysers' domain.
__device__ __forceinline__ bool frozen(const StepParams& P, int x, int y, int z)
{
    const int f = P.fixed_axes;
    return ((f & 1) && (x == 0 || x == P.nx - 1)) || ((f & 2) && (y == 0 || y == P.ny - 1)) ||
           ((f & 4) && (z == 0 || z == P.nz - 1));
}

__device__ __forceinline__ bool counts(const StepParams& P, int x) { return x >= P.obs_x0 && x < P.obs_x1; }

// ---------------------------------------------------------------------------
// Quaternions: U = c0 + i c.sigma, product (a0 b0 - a.b, a0 b + b0 a - a x b)
// (the convention of WilsonLoops/Source/StandardModel.cpp:160-191).
// ---------------------------------------------------------------------------
template <class C>
struct Q {
    C w, x, y, z;
};

template <class C>
__device__ __forceinline__ Q<C> qconj(Q<C> a) { return {a.w, -a.x, -a.y, -a.z}; }

template <class C>
__device__ __forceinline__ Q<C> qmul(Q<C> a, Q<C> b)
{
    Q<C> r;
    r.w = a.w * b.w - a.x * b.x - a.y * b.y - a.z * b.z;
    r.x = a.w * b.x + a.x * b.w - a.y * b.z + a.z * b.y;
    r.y = a.w * b.y + a.y * b.w - a.z * b.x + a.x * b.z;
    r.z = a.w * b.z + a.z * b.w - a.x * b.y + a.y * b.x;
    return r;
}

// vector part of a * b only
template <class C>
__device__ __forceinline__ void qmul_vec(Q<C> a, Q<C> b, C& rx, C& ry, C& rz)
{
    rx = a.w * b.x + a.x * b.w - a.y * b.z + a.z * b.y;
    ry = a.w * b.y + a.y * b.w - a.z * b.x + a.x * b.z;
    rz = a.w * b.z + a.z * b.w - a.x * b.y + a.y * b.x;
}

// scalar part of a * b only
template <class C>
__device__ __forceinline__ C qmul_w(Q<C> a, Q<C> b)
{
    return a.w * b.w - a.x * b.x - a.y * b.y - a.z * b.z;
}

template <class C>
__device__ __forceinline__ Q<C> qadd_scaled(Q<C> acc, C s, Q<C> a)
{
    acc.w += s * a.w;
    acc.x += s * a.x;
    acc.y += s * a.y;
    acc.z += s * a.z;
    return acc;
}

template <class To, class From>
__device__ __forceinline__ Q<To> qcast(Q<From> a)
{
    return {(To)a.w, (To)a.x, (To)a.y, (To)a.z};
}

// ---------------------------------------------------------------------------
// Vector loads / stores of 4-word records.
// ---------------------------------------------------------------------------
template <class C>
__device__ __forceinline__ Q<C> ld4(const float* p, int s)
{
    float4 v = __ldg(reinterpret_cast<const float4*>(p) + s);
    return {(C)v.x, (C)v.y, (C)v.z, (C)v.w};
}

template <class C>
__device__ __forceinline__ Q<C> ld4(const double* p, int s)
{
    const double2* b = reinterpret_cast<const double2*>(p) + 2 * (size_t)s;
    double2 a0 = __ldg(b), a1 = __ldg(b + 1);
    return {(C)a0.x, (C)a0.y, (C)a1.x, (C)a1.y};
}

template <class C>
__device__ __forceinline__ C ld1(const float* p, int s) { return (C)__ldg(p + s); }
template <class C>
__device__ __forceinline__ C ld1(const double* p, int s) { return (C)__ldg(p + s); }

__device__ __forceinline__ void st4(float* p, int s, float a, float b, float c, float d)
{
    reinterpret_cast<float4*>(p)[s] = make_float4(a, b, c, d);
}
__device__ __forceinline__ void st4(double* p, int s, double a, double b, double c, double d)
{
    double2* o = reinterpret_cast<double2*>(p) + 2 * (size_t)s;
    o[0] = make_double2(a, b);
    o[1] = make_double2(c, d);
}

// ---------------------------------------------------------------------------
// Neighbourhood of a site with periodic wrap (BoundaryConditions/Source/Periodic.cpp:18-57, 125-170):
//   c = x, m[a] = x - e_a, p[a] = x + e_a, dg[a][j] = x + e_a - e_j.
// ---------------------------------------------------------------------------
struct Nbr {
    int c;
    int m[3];
    int p[3];
    int dg[3][3];
};

__device__ __forceinline__ int site_of(const StepParams& P, int x, int y, int z)
{
    return (x * P.ny + y) * P.nz + z;
}

__device__ __forceinline__ Nbr neighbours(const StepParams& P, int x, int y, int z)
{
    const int xm = (x == 0) ? P.nx - 1 : x - 1, xp = (x + 1 == P.nx) ? 0 : x + 1;
    const int ym = (y == 0) ? P.ny - 1 : y - 1, yp = (y + 1 == P.ny) ? 0 : y + 1;
    const int zm = (z == 0) ? P.nz - 1 : z - 1, zp = (z + 1 == P.nz) ? 0 : z + 1;
    Nbr n;
    n.c = site_of(P, x, y, z);
    n.m[0] = site_of(P, xm, y, z);
    n.m[1] = site_of(P, x, ym, z);
    n.m[2] = site_of(P, x, y, zm);
    n.p[0] = site_of(P, xp, y, z);
    n.p[1] = site_of(P, x, yp, z);
    n.p[2] = site_of(P, x, y, zp);
    n.dg[0][0] = n.dg[1][1] = n.dg[2][2] = n.c;
    n.dg[0][1] = site_of(P, xp, ym, z);
    n.dg[0][2] = site_of(P, xp, y, zm);
    n.dg[1][0] = site_of(P, xm, yp, z);
    n.dg[1][2] = site_of(P, x, yp, zm);
    n.dg[2][0] = site_of(P, xm, y, zp);
    n.dg[2][1] = site_of(P, x, ym, zp);
    return n;
}

// ---------------------------------------------------------------------------
// Block reductions (double) into a per-block partials array.
// ---------------------------------------------------------------------------
__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ double warp_max(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// Reduce NV values per thread over the block; thread 0 writes them to out[0..NV).
// `is_max` selects max for slots >= max_from.  Requires blockDim.x*y multiple of 32, <= 1024.
template <int NV>
__device__ __forceinline__ void block_reduce_store(double (&v)[NV], double* out, int max_from)
{
    __shared__ double red[32][NV];
    const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
    const int nthreads = blockDim.x * blockDim.y * blockDim.z;
    const int lane = tid & 31, warp = tid >> 5, nwarps = nthreads >> 5;
#pragma unroll
    for (int k = 0; k < NV; k++) v[k] = (k >= max_from) ? warp_max(v[k]) : warp_sum(v[k]);
    if (lane == 0) {
#pragma unroll
        for (int k = 0; k < NV; k++) red[warp][k] = v[k];
    }
    __syncthreads();
    if (warp == 0) {
#pragma unroll
        for (int k = 0; k < NV; k++) {
            double t = (lane < nwarps) ? red[lane][k] : 0.0;
            t = (k >= max_from) ? warp_max(t) : warp_sum(t);
            if (lane == 0) out[k] = t;
        }
    }
}

// Device status word bits (mirror GFT_W_*).
constexpr unsigned kWarnAsin = 1u;
constexpr unsigned kWarnSqrt = 2u;
constexpr unsigned kWarnNonFinite = 4u;
constexpr unsigned kWarnRange = 16u;  // a link phase beyond the elementary functions' reduction range

}  // namespace gft
