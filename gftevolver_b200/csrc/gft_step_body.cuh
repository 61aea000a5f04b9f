// gft_step_body.cuh -- the per-site leapfrog update of the throughput forms,
// written once against a field accessor so that the same arithmetic serves the
// global-memory kernel (neighbours read through L1/L2) and the tiled kernel
// (neighbours read from TMA-staged shared-memory planes).
//
// Physics: the reference's per-site update (Core/Source/Model.cpp:339-373,
// WilsonLoops/Source/StandardModel.cpp:324-514, Gradients/Source/StandardModel.cpp:72-100,
// 272-363, Potentials/Source/SO_N.cpp:57-75, Potentials/Source/Double_SO_N.cpp:244-341),
// reassociated:
//   * the reference builds, for every link i and plane j, the loops
//       P1 = U_j(x+i)^dag U_i(x+j) U_j(x) U_i(x)^dag,
//       P2 = U_i(x) U_j(x-j) U_i(x-j)^dag U_j(x+i-j)^dag,
//     renormalising intermediate products.  Here the staples are summed first,
//       SA_i = sum_j w_j U_j(x+i)^dag U_i(x+j) U_j(x),   SB_i = sum_j w_j U_j(x-j) U_i(x-j)^dag U_j(x+i-j)^dag,
//     and vec(P1) - vec(P2) summed over j becomes vec(SA_i U_i^dag) - vec(U_i SB_i)
//     (the vector part is linear).  C_ij = U_j(x+i)^dag U_i(x+j) is shared by
//     the staples of links i and j.  Intermediate renormalisation is dropped:
//     it changes products of unit quaternions only at the rounding level.
//   * the U(1) plaquette angle of plane (i,j) is computed once for both links.
//   * sin, cos and asin are the range-reduced series of gft_math.cuh.
// Precision of the mixed form (C = float): operations that would lose
// precision in float are rearranged rather than widened -- the link momentum
// is vec((U_now - U_past) U_past^dag) (exactly vec(U_now U_past^dag) without
// the O(1) terms that cancel), leapfrog sums add a small increment to the
// current value with one rounding, and the renormalisation evaluates
// |U|^2 - 1 with fused multiply-adds.  Energies accumulate in FP64.
#pragma once

#include "gft_device.cuh"
#include "gft_math.cuh"

namespace gft {

__device__ __forceinline__ float sqrt_(float x) { return sqrtf(x); }
// A parameter in the compute type: the precomputed float copy, or the double.
template <class C>
__device__ __forceinline__ C pf(float f, double d)
{
    if constexpr (sizeof(C) == 4)
        return f;
    else
        return d;
}
__device__ __forceinline__ double sqrt_(double x) { return sqrt(x); }

// Doublet phi rotated by the hypercharge phase (cos, sin) then acted on by the
// SU(2) quaternion u as the real 4x4 of Gradients/Source/StandardModel.cpp:94-97.
template <class C>
__device__ __forceinline__ Q<C> transport(Q<C> u, C cs, C sn, Q<C> f)
{
    const C h0 = cs * f.w - sn * f.x;
    const C h1 = cs * f.x + sn * f.w;
    const C h2 = cs * f.y - sn * f.z;
    const C h3 = cs * f.z + sn * f.y;
    Q<C> t;
    t.w = u.w * h0 - u.z * h1 + u.y * h2 - u.x * h3;
    t.x = u.z * h0 + u.w * h1 + u.x * h2 + u.y * h3;
    t.y = -u.y * h0 - u.x * h1 + u.w * h2 + u.z * h3;
    t.z = u.x * h0 - u.y * h1 - u.z * h2 + u.w * h3;
    return t;
}

// The isospin action alone (the 4x4 above on an already phase-rotated h); the
// Higgs-family SU(2) acts with the same matrix on (doublet-1, doublet-2)
// component pairs (Gradients/Source/TwoHDM.cpp:134-146).
template <class C>
__device__ __forceinline__ Q<C> su2_act(Q<C> u, Q<C> h)
{
    Q<C> t;
    t.w = u.w * h.w - u.z * h.x + u.y * h.y - u.x * h.z;
    t.x = u.z * h.w + u.w * h.x + u.x * h.y + u.y * h.z;
    t.y = -u.y * h.w - u.x * h.x + u.w * h.y + u.z * h.z;
    t.z = u.x * h.w - u.y * h.x - u.z * h.y + u.w * h.z;
    return t;
}

// Phase rotation of both complex pairs of a doublet by (cos, sin).
template <class C>
__device__ __forceinline__ Q<C> rot2(Q<C> f, C cs, C sn)
{
    return {cs * f.w - sn * f.x, cs * f.x + sn * f.w, cs * f.y - sn * f.z, cs * f.z + sn * f.y};
}

// Higgs-family part of the 2HDM transport (Gradients/Source/TwoHDM.cpp:118-146),
// applied to the two SM-transported doublets: U(1) = phase +theta_H on doublet 1
// and -theta_H on doublet 2 ((hc, hs) = cos, sin of theta_H, hs negated for the
// conjugate link); SU(2) = hu acting on (doublet 1, doublet 2) pairs.
template <int HF, class C>
__device__ __forceinline__ void hf_act(Q<C>& t1, Q<C>& t2, C hc, C hs, Q<C> hu)
{
    if constexpr (HF == kHfU1) {
        t1 = rot2(t1, hc, hs);
        t2 = rot2(t2, hc, -hs);
    } else if constexpr (HF == kHfSU2) {
        const Q<C> lo = su2_act(hu, Q<C>{t1.w, t1.x, t2.w, t2.x});
        const Q<C> hi = su2_act(hu, Q<C>{t1.y, t1.z, t2.y, t2.z});
        t1 = {lo.w, lo.x, hi.w, hi.x};
        t2 = {lo.y, lo.z, hi.y, hi.z};
    }
}

// Leapfrog update of one SU(2) link from the vector part (R1, R2, R3) of
// u = U(t+dt) U(t)^dag (WilsonLoops/Source/StandardModel.cpp:478-504), written as
// U + correction (see site_step); returns the new link, adds to `check`.
template <class C>
__device__ __forceinline__ Q<C> su2_advance(Q<C> Un, C R1, C R2, C R3, unsigned& warn, C& check)
{
    const C cm = R1 * R1 + R2 * R2 + R3 * R3;
    if (cm > (C)1) warn |= kWarnSqrt;
    const C u0m1 = sqrt1m_minus1(cm);
    const Q<C> dU = qmul(Q<C>{u0m1, R1, R2, R3}, Un);
    C e = fma(Un.w, Un.w, (C)-1);
    e = fma(Un.x, Un.x, e);
    e = fma(Un.y, Un.y, e);
    e = fma(Un.z, Un.z, e);
    const C udu = Un.w * dU.w + Un.x * dU.x + Un.y * dU.y + Un.z * dU.z;
    const C dd = dU.w * dU.w + dU.x * dU.x + dU.y * dU.y + dU.z * dU.z;
    e += (C)2 * udu + dd;
    const C fm1 = e * ((C)0.375 * e - (C)0.5);
    check += e;
    return {Un.w + (dU.w + fm1 * (Un.w + dU.w)), Un.x + (dU.x + fm1 * (Un.x + dU.x)),
            Un.y + (dU.y + fm1 * (Un.y + dU.y)), Un.z + (dU.z + fm1 * (Un.z + dU.z))};
}

// 1 - a0/|a| in the compute type without cancellation: |vec a|^2 / (|a| (|a| + a0))
// when a0 >= 0, else 1 - a0/|a| directly (no cancellation there either).
template <class C>
__device__ __forceinline__ C one_minus_trace(Q<C> a)
{
    const C v2 = a.x * a.x + a.y * a.y + a.z * a.z;
    const C nrm = sqrt_(a.w * a.w + v2);
    return (a.w >= (C)0) ? v2 / (nrm * (nrm + a.w)) : (C)1 - a.w / nrm;
}
// The mixed form's energy terms: the same expression with the square root and the
// division by Newton-refined hardware approximations (one_minus_cos_nr), a fifth
// of the instructions of the IEEE operations; the FP64 forms keep those.
template <>
__device__ __forceinline__ float one_minus_trace<float>(Q<float> a)
{
    return one_minus_cos_nr(a.w, a.x * a.x + a.y * a.y + a.z * a.z);
}

// Neighbour references of one site, in the accessor's own reference type:
//   c = x, m[a] = x - e_a, p[a] = x + e_a, dg(i, j) = x + e_i - e_j (i != j).
template <class R>
struct Stencil {
    R c, m[3], p[3];
    R d01, d02, d10, d12, d20, d21;
    __device__ __forceinline__ R dg(int i, int j) const
    {
        return (i == 0) ? (j == 1 ? d01 : d02) : (i == 1) ? (j == 0 ? d10 : d12) : (j == 0 ? d20 : d21);
    }
};

// Values a site computes that its +x neighbour needs, carried along an x-march:
// the sines of the (0,1) and (0,2) plaquette angles, which are the x+e_0
// site's lower U(1) loop angles, and the doublet transported along the x link,
// U_0(x) R(theta_0(x)) phi(x), which is the x+e_0 site's D- term.
template <class C, int ND>
struct XCarry {
    bool valid;
    C s01, s02;
    Q<C> t0[ND];
};

// Own-site access to the past level (read, then overwritten with t + dt).  LV is
// LevelPtrs<S>, or any struct with its q / th / ph members when no Higgs-family
// field is evolved.
template <class S, class LV = LevelPtrs<S>>
struct PastSite {
    LV L;
    int s;
};

// A thread's total energy from its component sums, set once after its last site
// (no per-site accumulator held through the update).
__device__ __forceinline__ void energy_total(double (&obs)[kObsCount])
{
    obs[kObsEnergy] = obs[kObsPotential] + obs[kObsGradient] + obs[kObsKinetic] + obs[kObsMagnetic] + obs[kObsElectric];
}

// The per-site update.  A provides q(d, R) -> Q<C>, th(d, R) -> C, ph(k, R) -> Q<C>
// for the "now" level (and hth / hq for a 2HDM Higgs-family field, HF != 0).
// obs receives the energy-step observables except the total (energy_total after
// the last site) and warn the warning bits, both only when `count` (the site is
// not on a ghost plane).  With HF != 0 the x-carry is not used (the caller passes
// an invalid one).  STEADY: the caller guarantees a valid x-carry (a site of a
// march after one that was evolved), so the recomputation of the carried values
// is not compiled in; the general instance keeps both and the compiler
// evaluates the recomputation alongside the carry where it predicates the
// choice, which costs the x-march kernels 4 % of their step time.
template <class S, int MODEL, bool ENERGY, int HF = kHfNone, bool STEADY = false, class A, class R, class LV>
__device__ __forceinline__ void site_step(const StepParams& P, const FConst& F, const A& acc, const Stencil<R>& n,
                                          PastSite<S, LV> ps,
                                          XCarry<S, (MODEL == kModelSM) ? 1 : 2>& carry, double (&obs)[kObsCount],
                                          unsigned& warn, bool count = true)
{
    const unsigned warn_in = warn;
    using C = S;  // FP64 form -> double, mixed form -> float
    constexpr int ND = (MODEL == kModelSM) ? 1 : 2;
    // Own-site past level: on non-logging steps loaded here, so that the
    // memory latency overlaps the force arithmetic below (the logging-step
    // variant has no registers to spare and loads it where it is used).
    Q<C> pst_f[ND], pst_u[3];
    C pst_t[3];
    if (!ENERGY) {
#pragma unroll
        for (int db = 0; db < ND; db++) pst_f[db] = ld4<C>(ps.L.ph[db], ps.s);
#pragma unroll
        for (int d = 0; d < 3; d++) {
            pst_u[d] = ld4<C>(ps.L.q[d], ps.s);
            pst_t[d] = ld1<C>(ps.L.th[d], ps.s);
        }
    }
    const bool have = STEADY || carry.valid;
    const C lap[3] = {pf<C>(F.lap[0], P.lap[0]), pf<C>(F.lap[1], P.lap[1]), pf<C>(F.lap[2], P.lap[2])};

    Q<C> U[3];
    C th[3];
#pragma unroll
    for (int a = 0; a < 3; a++) {
        U[a] = acc.q(a, n.c);
        th[a] = acc.th(a, n.c);
    }

    // ---- magnetic term: U(1) sines and SU(2) staple sums ----
    C MgY[3] = {(C)0, (C)0, (C)0};
    // lower U(1) loops of the links 1 and 2 in the planes with x: the x-1 site's (0,1), (0,2) angles
    const C prev01 = carry.s01, prev02 = carry.s02;
    Q<C> SA[3], SB[3];
#pragma unroll
    for (int a = 0; a < 3; a++) {
        SA[a] = {(C)0, (C)0, (C)0, (C)0};
        SB[a] = {(C)0, (C)0, (C)0, (C)0};
    }
    // logging-step terms: per-site partial sums in the form's arithmetic (a few
    // cancellation-free terms each), added to the FP64 block sums once per site
    C mag_e = (C)0, plaq2 = (C)0, plaq1 = (C)0;
#pragma unroll
    for (int pl = 0; pl < 3; pl++) {
        const int i = (pl == 2) ? 1 : 0;
        const int j = (pl == 0) ? 1 : 2;
        const Q<C> Uj_pi = acc.q(j, n.p[i]);
        const Q<C> Ui_pj = acc.q(i, n.p[j]);
        // F_ij(x) = theta_i(x) + theta_j(x+i) - theta_i(x+j) - theta_j(x); the reference's
        // local angle is -F for link i and +F for link j (StandardModel.cpp:348-353).
        const C Fa = th[i] + acc.th(j, n.p[i]) - acc.th(i, n.p[j]) - th[j];
        const C sF = gsin(Fa);
        MgY[i] -= sF * lap[j];
        MgY[j] += sF * lap[i];
        if (pl == 0) carry.s01 = sF;
        if (pl == 1) carry.s02 = sF;
        const Q<C> Cij = qmul(qconj(Uj_pi), Ui_pj);
        const Q<C> Aij = qmul(Cij, U[j]);
        const Q<C> Aji = qmul(qconj(Cij), U[i]);
        SA[i] = qadd_scaled(SA[i], lap[j], Aij);
        SA[j] = qadd_scaled(SA[j], lap[i], Aji);
        if (ENERGY) {
            // plaquette P1 = Aij U_i^dag: both orientations have the same trace;
            // 1 - cos F = 2 sin^2(F/2) (no cancellation for small F)
            const Q<C> P1 = qmul(Aij, qconj(U[i]));
            const C omt = one_minus_trace(P1);
            const C hF = gsin((C)0.5 * Fa);
            const C omc = (C)2 * hF * hF;
            mag_e += pf<C>(F.e_plaq[pl], 4.0 * P.lap[i] * P.lap[j]) *
                     (pf<C>(F.inv_g_sqr, P.inv_g_sqr) * omt + pf<C>(F.inv_gp_sqr, P.inv_gp_sqr) * omc);
            plaq2 += (C)1 - omt;
            plaq1 += (C)1 - omc;
        }
    }
#pragma unroll
    for (int i = 0; i < 3; i++) {
#pragma unroll
        for (int j = 0; j < 3; j++) {
            if (j == i) continue;
            const R mj = n.m[j];
            const R dg = n.dg(i, j);
            const Q<C> Uj_mj = acc.q(j, mj);
            const Q<C> Ui_mj = acc.q(i, mj);
            const Q<C> Uj_dg = acc.q(j, dg);
            if (j == 0 && have) {
                MgY[i] -= ((i == 1) ? prev01 : prev02) * lap[0];
            } else {
                const C neigh = -acc.th(j, dg) - acc.th(i, mj) + acc.th(j, mj) + th[i];
                MgY[i] -= gsin(neigh) * lap[j];
            }
            const Q<C> B = qmul(qmul(Uj_mj, qconj(Ui_mj)), qconj(Uj_dg));
            SB[i] = qadd_scaled(SB[i], lap[j], B);
        }
    }
    // ---- Higgs-family magnetic term (WilsonLoops/Source/TwoHDM.cpp:484-551): the same
    //      loops on theta_H (U(1)) or the family quaternion (SU(2)), coupling g'' ----
    C MgH[3][3];
#pragma unroll
    for (int i = 0; i < 3; i++) MgH[i][0] = MgH[i][1] = MgH[i][2] = (C)0;
    if constexpr (HF == kHfU1) {
        C hc[3];
#pragma unroll
        for (int a = 0; a < 3; a++) hc[a] = acc.hth(a, n.c);
#pragma unroll
        for (int pl = 0; pl < 3; pl++) {
            const int i = (pl == 2) ? 1 : 0;
            const int j = (pl == 0) ? 1 : 2;
            const C Fa = hc[i] + acc.hth(j, n.p[i]) - acc.hth(i, n.p[j]) - hc[j];
            const C sF = gsin(Fa);
            MgH[i][0] -= sF * lap[j];
            MgH[j][0] += sF * lap[i];
            if (ENERGY) {
                const C hF = gsin((C)0.5 * Fa);
                mag_e += pf<C>(F.e_plaq[pl], 4.0 * P.lap[i] * P.lap[j]) * pf<C>(F.inv_gpp_sqr, P.inv_gpp_sqr) *
                         ((C)2 * hF * hF);
            }
        }
#pragma unroll
        for (int i = 0; i < 3; i++) {
#pragma unroll
            for (int j = 0; j < 3; j++) {
                if (j == i) continue;
                const C neigh = -acc.hth(j, n.dg(i, j)) - acc.hth(i, n.m[j]) + acc.hth(j, n.m[j]) + hc[i];
                MgH[i][0] -= gsin(neigh) * lap[j];
            }
        }
    } else if constexpr (HF == kHfSU2) {
        Q<C> UH[3], SAH[3], SBH[3];
#pragma unroll
        for (int a = 0; a < 3; a++) {
            UH[a] = acc.hq(a, n.c);
            SAH[a] = {(C)0, (C)0, (C)0, (C)0};
            SBH[a] = {(C)0, (C)0, (C)0, (C)0};
        }
#pragma unroll
        for (int pl = 0; pl < 3; pl++) {
            const int i = (pl == 2) ? 1 : 0;
            const int j = (pl == 0) ? 1 : 2;
            const Q<C> Cij = qmul(qconj(acc.hq(j, n.p[i])), acc.hq(i, n.p[j]));
            const Q<C> Aij = qmul(Cij, UH[j]);
            const Q<C> Aji = qmul(qconj(Cij), UH[i]);
            SAH[i] = qadd_scaled(SAH[i], lap[j], Aij);
            SAH[j] = qadd_scaled(SAH[j], lap[i], Aji);
            if (ENERGY)
                mag_e += pf<C>(F.e_plaq[pl], 4.0 * P.lap[i] * P.lap[j]) * pf<C>(F.inv_gpp_sqr, P.inv_gpp_sqr) *
                         one_minus_trace(qmul(Aij, qconj(UH[i])));
        }
#pragma unroll
        for (int i = 0; i < 3; i++) {
#pragma unroll
            for (int j = 0; j < 3; j++) {
                if (j == i) continue;
                const Q<C> Bq = qmul(qmul(acc.hq(j, n.m[j]), qconj(acc.hq(i, n.m[j]))), qconj(acc.hq(j, n.dg(i, j))));
                SBH[i] = qadd_scaled(SBH[i], lap[j], Bq);
            }
        }
#pragma unroll
        for (int i = 0; i < 3; i++) {
            C a1, a2, a3, b1, b2, b3;
            qmul_vec(SAH[i], qconj(UH[i]), a1, a2, a3);
            qmul_vec(UH[i], SBH[i], b1, b2, b3);
            MgH[i][0] = a1 - b1;
            MgH[i][1] = a2 - b2;
            MgH[i][2] = a3 - b3;
        }
    }

    C Mg[3][3];
#pragma unroll
    for (int i = 0; i < 3; i++) {
        C a1, a2, a3, b1, b2, b3;
        qmul_vec(SA[i], qconj(U[i]), a1, a2, a3);
        qmul_vec(U[i], SB[i], b1, b2, b3);
        Mg[i][0] = a1 - b1;
        Mg[i][1] = a2 - b2;
        Mg[i][2] = a3 - b3;
    }

    // ---- scalar sector: covariant Laplacian D and currents J ----
    Q<C> fc[ND];
#pragma unroll
    for (int db = 0; db < ND; db++) fc[db] = acc.ph(db, n.c);
    Q<C> D[ND];
#pragma unroll
    for (int db = 0; db < ND; db++) {
        const C w = pf<C>(F.diag, -2.0 * (P.lap[0] + P.lap[1] + P.lap[2]));
        D[db] = {w * fc[db].w, w * fc[db].x, w * fc[db].y, w * fc[db].z};
    }
    C J[3][4];
    C JH[3][3];  // Higgs-family currents (Gradients/Source/TwoHDM.cpp:465-485)
    C grad_e = (C)0;
    if constexpr (HF != kHfNone) {
#pragma unroll
        for (int a = 0; a < 3; a++) {
            C sn, cs, smm, cmm;
            gsincos(th[a], sn, cs);
            gsincos(acc.th(a, n.m[a]), smm, cmm);
            const Q<C> Um = acc.q(a, n.m[a]);
            C hcs = (C)1, hsn = (C)0, hcm = (C)1, hsm = (C)0;
            Q<C> uh = {(C)1, (C)0, (C)0, (C)0}, uhm = {(C)1, (C)0, (C)0, (C)0};
            if constexpr (HF == kHfU1) {
                gsincos(acc.hth(a, n.c), hsn, hcs);
                gsincos(acc.hth(a, n.m[a]), hsm, hcm);
            } else {
                uh = acc.hq(a, n.c);
                uhm = acc.hq(a, n.m[a]);
            }
            Q<C> tm[2], tp[2], t[2], fp[2];
#pragma unroll
            for (int db = 0; db < 2; db++) {
                fp[db] = acc.ph(db, n.p[a]);
                tm[db] = transport(Um, cmm, smm, acc.ph(db, n.m[a]));
                tp[db] = transport(qconj(U[a]), cs, -sn, fp[db]);
                t[db] = transport(U[a], cs, sn, fc[db]);
            }
            hf_act<HF>(tm[0], tm[1], hcm, hsm, uhm);
            hf_act<HF>(tp[0], tp[1], hcs, -hsn, qconj(uh));
            hf_act<HF>(t[0], t[1], hcs, hsn, uh);
            C j0 = 0, j1 = 0, j2 = 0, j3 = 0;
#pragma unroll
            for (int db = 0; db < 2; db++) {
                D[db] = qadd_scaled(D[db], lap[a], tm[db]);
                D[db] = qadd_scaled(D[db], lap[a], tp[db]);
                const Q<C> u = t[db], f = fp[db];
                j0 += u.w * f.x - u.x * f.w + u.y * f.z - u.z * f.y;
                j1 += u.w * f.z - u.x * f.y + u.y * f.x - u.z * f.w;
                j2 += -u.w * f.y - u.x * f.z + u.y * f.w + u.z * f.x;
                j3 += u.w * f.x - u.x * f.w - u.y * f.z + u.z * f.y;
                if (ENERGY) {
                    const C e0 = f.w - u.w, e1 = f.x - u.x, e2 = f.y - u.y, e3 = f.z - u.z;
                    grad_e += pf<C>(F.e_grad[a], 0.5 * P.inv_dx[a] * P.inv_dx[a]) * (e0 * e0 + e1 * e1 + e2 * e2 + e3 * e3);
                }
            }
            J[a][0] = (C)0.25 * j0;
            J[a][1] = (C)0.25 * j1;
            J[a][2] = (C)0.25 * j2;
            J[a][3] = (C)0.25 * j3;
            // family pairs: components (i, i+1) of doublet 1 and of doublet 2, i = 0 (upper) and 2 (lower)
            const C t8[8] = {t[0].w, t[0].x, t[0].y, t[0].z, t[1].w, t[1].x, t[1].y, t[1].z};
            const C n8[8] = {fp[0].w, fp[0].x, fp[0].y, fp[0].z, fp[1].w, fp[1].x, fp[1].y, fp[1].z};
            C h4 = 0, h5 = 0, h6 = 0;
#pragma unroll
            for (int i = 0; i < 4; i += 2) {
                if constexpr (HF == kHfU1) {
                    h4 += t8[i] * n8[i + 1] - t8[i + 1] * n8[i] - t8[i + 4] * n8[i + 5] + t8[i + 5] * n8[i + 4];
                } else {
                    h4 += t8[i] * n8[i + 5] - t8[i + 1] * n8[i + 4] + t8[i + 4] * n8[i + 1] - t8[i + 5] * n8[i];
                    h5 += -t8[i] * n8[i + 4] - t8[i + 1] * n8[i + 5] + t8[i + 4] * n8[i] + t8[i + 5] * n8[i + 1];
                    h6 += t8[i] * n8[i + 1] - t8[i + 1] * n8[i] - t8[i + 4] * n8[i + 5] + t8[i + 5] * n8[i + 4];
                }
            }
            JH[a][0] = (C)0.25 * h4;
            JH[a][1] = (C)0.25 * h5;
            JH[a][2] = (C)0.25 * h6;
        }
    } else {
#pragma unroll
    for (int a = 0; a < 3; a++) {
        C sn, cs;
        gsincos(th[a], sn, cs);
        const Q<C> Uc = qconj(U[a]);
        C j0 = 0, j1 = 0, j2 = 0, j3 = 0;
        const bool from_carry = (a == 0) && have;
        C sm = (C)0, cm = (C)1;
        Q<C> Um = {(C)1, (C)0, (C)0, (C)0};
        if (!from_carry) {
            gsincos(acc.th(a, n.m[a]), sm, cm);
            Um = acc.q(a, n.m[a]);
        }
#pragma unroll
        for (int db = 0; db < ND; db++) {
            const Q<C> fp = acc.ph(db, n.p[a]);
            // D: U_a(x-a) phi(x-a) + U_a(x)^dag phi(x+a); the first is the x-1 site's transported doublet
            const Q<C> tm = from_carry ? carry.t0[db] : transport(Um, cm, sm, acc.ph(db, n.m[a]));
            const Q<C> tp = transport(Uc, cs, -sn, fp);
            D[db] = qadd_scaled(D[db], lap[a], tm);
            D[db] = qadd_scaled(D[db], lap[a], tp);
            // J: Im of (U_a(x) phi(x))^dag sigma phi(x+a)
            const Q<C> t = transport(U[a], cs, sn, fc[db]);
            if (a == 0) carry.t0[db] = t;
            j0 += t.w * fp.x - t.x * fp.w + t.y * fp.z - t.z * fp.y;
            j1 += t.w * fp.z - t.x * fp.y + t.y * fp.x - t.z * fp.w;
            j2 += -t.w * fp.y - t.x * fp.z + t.y * fp.w + t.z * fp.x;
            j3 += t.w * fp.x - t.x * fp.w - t.y * fp.z + t.z * fp.y;
            if (ENERGY) {
                const C e0 = fp.w - t.w, e1 = fp.x - t.x, e2 = fp.y - t.y, e3 = fp.z - t.z;
                grad_e += pf<C>(F.e_grad[a], 0.5 * P.inv_dx[a] * P.inv_dx[a]) * (e0 * e0 + e1 * e1 + e2 * e2 + e3 * e3);
            }
        }
        J[a][0] = (C)0.25 * j0;
        J[a][1] = (C)0.25 * j1;
        J[a][2] = (C)0.25 * j2;
        J[a][3] = (C)0.25 * j3;
    }
    }

    // ---- potential dV/dphi ----
    C Pot[ND][4];
    double pot_e = 0.0;
    if (MODEL == kModelSM) {
        const C fsq = fc[0].w * fc[0].w + fc[0].x * fc[0].x + fc[0].y * fc[0].y + fc[0].z * fc[0].z;
        const C k = pf<C>(F.lambda, P.lambda) * (fsq - pf<C>(F.eta_sqr, P.eta_sqr));
        Pot[0][0] = k * fc[0].w;
        Pot[0][1] = k * fc[0].x;
        Pot[0][2] = k * fc[0].y;
        Pot[0][3] = k * fc[0].z;
        if (ENERGY) {
            const double t = (double)fsq - P.eta_sqr;
            pot_e = 0.25 * P.lambda * t * t;
        }
    } else {
        const Q<C> f1 = fc[0], f2 = fc[ND - 1];
        const C s1 = f1.w * f1.w + f1.x * f1.x + f1.y * f1.y + f1.z * f1.z;
        const C s2 = f2.w * f2.w + f2.x * f2.x + f2.y * f2.y + f2.z * f2.z;
        const C dot = P.break_son ? f1.w * f2.w + f1.x * f2.x + f1.y * f2.y + f1.z * f2.z : (C)0;
        const C anti = (P.break_son && P.break_uhalfn) ? f1.w * f2.x - f1.x * f2.w + f1.y * f2.z - f1.z * f2.y : (C)0;
        const C l3x2 = pf<C>(F.l3x2, 2.0 * P.l3);
        const C a1 = pf<C>(F.m1x2n, -2.0 * P.m1) + pf<C>(F.l1x4, 4.0 * P.l1) * s1 + l3x2 * s2;
        const C a2 = pf<C>(F.m2x2n, -2.0 * P.m2) + pf<C>(F.l2x4, 4.0 * P.l2) * s2 + l3x2 * s1;
        // single SO(N): (-m12r + 2 l4p5 dot + l6r s1 + l7r s2) f_other + 2 l6r|l7r dot f_self
        const C bs = pf<C>(F.m12rn, -P.m12r) + pf<C>(F.l4p5x2, 2.0 * P.l4p5) * dot + pf<C>(F.l6r, P.l6r) * s1 +
                     pf<C>(F.l7r, P.l7r) * s2;
        const C b1 = pf<C>(F.l6rx2, 2.0 * P.l6r) * dot, b2 = pf<C>(F.l7rx2, 2.0 * P.l7r) * dot;
        // U(N/2): (m12i + 2 l4m5 anti - 2 l5i dot - l6i s1 - l7i s2) J f_other - 2 l5i anti f_other - 2 l6i|l7i anti f_self
        const C l5ix2 = pf<C>(F.l5ix2, 2.0 * P.l5i);
        const C cu = pf<C>(F.m12i, P.m12i) + pf<C>(F.l4m5x2, 2.0 * P.l4m5) * anti - l5ix2 * dot -
                     pf<C>(F.l6i, P.l6i) * s1 - pf<C>(F.l7i, P.l7i) * s2;
        const C c5 = l5ix2 * anti;
        const C c1 = pf<C>(F.l6ix2, 2.0 * P.l6i) * anti, c2 = pf<C>(F.l7ix2, 2.0 * P.l7i) * anti;
        const C f1v[4] = {f1.w, f1.x, f1.y, f1.z};
        const C f2v[4] = {f2.w, f2.x, f2.y, f2.z};
#pragma unroll
        for (int k = 0; k < 4; k++) {
            const int alt = 1 - 2 * (k % 2);
            C v1 = a1 * f1v[k];
            C v2 = a2 * f2v[k];
            if (P.break_son) {
                v1 += bs * f2v[k] + b1 * f1v[k];
                v2 += bs * f1v[k] + b2 * f2v[k];
                if (P.break_uhalfn) {
                    v1 += cu * (C)alt * f2v[k + alt] - c5 * f2v[k] - c1 * f1v[k];
                    v2 += -cu * (C)alt * f1v[k + alt] - c5 * f1v[k] - c2 * f2v[k];
                }
            }
            Pot[0][k] = v1;
            Pot[ND - 1][k] = v2;
        }
        if (ENERGY) {
            const double d1 = s1, d2 = s2, dd = dot, da = anti;
            double v = -P.m1 * d1 - P.m2 * d2 + P.l1 * d1 * d1 + P.l2 * d2 * d2 + P.l3 * d1 * d2;
            if (P.break_son) {
                v += -P.m12r * dd + P.l4p5 * dd * dd + P.l6r * d1 * dd + P.l7r * d2 * dd;
                if (P.break_uhalfn)
                    v += P.m12i * da + P.l4m5 * da * da - 2.0 * P.l5i * dd * da - P.l6i * d1 * da - P.l7i * d2 * da;
            }
            if (P.apply_norm) v += P.energy_offset;
            pot_e = v;
        }
    }

    // ---- scalar leapfrog (Model.cpp:347-356):
    //      phi(t+dt) = phi + [(phi - phi_past)(1 - damping) + dt^2 (D - dV)], one rounding at the end
    C kin_e = (C)0, phisq = (C)0;
    C check = (C)0;  // sum of every new value: non-finite iff one of them is
    const C dt2 = pf<C>(F.dt2, P.dt2);
    const C keep = pf<C>(F.keep, 1.0 - P.damping_step);
#pragma unroll
    for (int db = 0; db < ND; db++) {
        const Q<C> fpast = ENERGY ? ld4<C>(ps.L.ph[db], ps.s) : pst_f[db];
        const C fn[4] = {fc[db].w, fc[db].x, fc[db].y, fc[db].z};
        const C fo[4] = {fpast.w, fpast.x, fpast.y, fpast.z};
        const C dd[4] = {D[db].w, D[db].x, D[db].y, D[db].z};
        C out[4];
#pragma unroll
        for (int k = 0; k < 4; k++) {
            const C vel = fn[k] - fo[k];
            out[k] = fn[k] + (keep * vel + dt2 * (dd[k] - Pot[db][k]));
            check += out[k];
            if (ENERGY) {
                kin_e += vel * vel;  // x 0.5 / dt^2 below
                phisq += fn[k] * fn[k];
            }
        }
        st4(ps.L.ph[db], ps.s, out[0], out[1], out[2], out[3]);
    }

    // ---- link update (WilsonLoops/Source/StandardModel.cpp:456-514) ----
    C elec_e = (C)0;
    const C gY = pf<C>(F.gY, P.gsq[0]), gI = pf<C>(F.gI, P.gsq[1]);
#pragma unroll
    for (int d = 0; d < 3; d++) {
        const Q<C> Un = U[d];
        const Q<C> Up = ENERGY ? ld4<C>(ps.L.q[d], ps.s) : pst_u[d];
        const C thp = ENERGY ? ld1<C>(ps.L.th[d], ps.s) : pst_t[d];
        // link momentum vec(U_now U_past^dag) = vec((U_now - U_past) U_past^dag)
        const Q<C> dlt = {Un.w - Up.w, Un.x - Up.x, Un.y - Up.y, Un.z - Up.z};
        C E1, E2, E3;
        qmul_vec(dlt, qconj(Up), E1, E2, E3);
        const C dth = th[d] - thp;
        const C R0 = keep * gsin(dth) + dt2 * (MgY[d] + gY * J[d][0]);
        const C R1 = keep * E1 + dt2 * (Mg[d][0] + gI * J[d][1]);
        const C R2 = keep * E2 + dt2 * (Mg[d][1] + gI * J[d][2]);
        const C R3 = keep * E3 + dt2 * (Mg[d][2] + gI * J[d][3]);
        if (ENERGY) {
            // 1 - (U_now U_past^dag)_0 / |U_now U_past^dag| and 1 - cos(dtheta) = 2 sin^2(dtheta/2)
            const Q<C> Ed = {Un.w * Up.w + Un.x * Up.x + Un.y * Up.y + Un.z * Up.z, E1, E2, E3};
            const C h = gsin((C)0.5 * dth);
            elec_e += pf<C>(F.e_elec[d], 4.0 * P.lap[d] * P.inv_sqr_dt) *
                      (pf<C>(F.inv_g_sqr, P.inv_g_sqr) * one_minus_trace(Ed) + pf<C>(F.inv_gp_sqr, P.inv_gp_sqr) * (C)2 * h * h);
        }
        if (R0 * R0 > (C)1) warn |= kWarnAsin;
        if (fabs(th[d]) > (C)1e4) warn |= kWarnRange;
        // theta(t+dt) = theta(t) + asin(RHS_Y)
        const C thn = th[d] + gasin(R0);
        // u = (sqrt(1-|c|^2), c); U(t+dt) = normalise(u U(t)), written as U + correction:
        //   dU = (u - 1) U with u0 - 1 = -|c|^2 / (1 + sqrt(1 - |c|^2)),
        //   |U + dU|^2 - 1 = (|U|^2 - 1) + 2 U.dU + |dU|^2 =: e,  1/sqrt(1+e) - 1 = -e/2 + 3e^2/8
        const C cm = R1 * R1 + R2 * R2 + R3 * R3;
        if (cm > (C)1) warn |= kWarnSqrt;
        const C u0m1 = sqrt1m_minus1(cm);
        const Q<C> dU = qmul(Q<C>{u0m1, R1, R2, R3}, Un);
        C e = fma(Un.w, Un.w, (C)-1);
        e = fma(Un.x, Un.x, e);
        e = fma(Un.y, Un.y, e);
        e = fma(Un.z, Un.z, e);
        const C udu = Un.w * dU.w + Un.x * dU.x + Un.y * dU.y + Un.z * dU.z;
        const C dd = dU.w * dU.w + dU.x * dU.x + dU.y * dU.y + dU.z * dU.z;
        e += (C)2 * udu + dd;
        const C fm1 = e * ((C)0.375 * e - (C)0.5);
        const Q<C> Unew = {Un.w + (dU.w + fm1 * (Un.w + dU.w)), Un.x + (dU.x + fm1 * (Un.x + dU.x)),
                           Un.y + (dU.y + fm1 * (Un.y + dU.y)), Un.z + (dU.z + fm1 * (Un.z + dU.z))};
        check += thn + e;
        ps.L.th[d][ps.s] = thn;
        st4(ps.L.q[d], ps.s, Unew.w, Unew.x, Unew.y, Unew.z);

        // Higgs-family link (WilsonLoops/Source/TwoHDM.cpp:601-633, 702-745), coupling g''
        if constexpr (HF == kHfU1) {
            const C gH = (C)P.gsq_hf;
            const C hn = acc.hth(d, n.c);
            const C dh = hn - ld1<C>(ps.L.hth[d], ps.s);
            const C RH = keep * gsin(dh) + dt2 * (MgH[d][0] + gH * JH[d][0]);
            if (ENERGY) {
                const C h = gsin((C)0.5 * dh);
                elec_e += pf<C>(F.e_elec[d], 4.0 * P.lap[d] * P.inv_sqr_dt) * pf<C>(F.inv_gpp_sqr, P.inv_gpp_sqr) * ((C)2 * h * h);
            }
            if (RH * RH > (C)1) warn |= kWarnAsin;
            if (fabs(hn) > (C)1e4) warn |= kWarnRange;
            const C hnew = hn + gasin(RH);
            check += hnew;
            ps.L.hth[d][ps.s] = hnew;
        } else if constexpr (HF == kHfSU2) {
            const C gH = (C)P.gsq_hf;
            const Q<C> Hn = acc.hq(d, n.c);
            const Q<C> Hp = ld4<C>(ps.L.hq[d], ps.s);
            const Q<C> dH = {Hn.w - Hp.w, Hn.x - Hp.x, Hn.y - Hp.y, Hn.z - Hp.z};
            C F1, F2, F3;
            qmul_vec(dH, qconj(Hp), F1, F2, F3);
            const C H1 = keep * F1 + dt2 * (MgH[d][0] + gH * JH[d][0]);
            const C H2 = keep * F2 + dt2 * (MgH[d][1] + gH * JH[d][1]);
            const C H3 = keep * F3 + dt2 * (MgH[d][2] + gH * JH[d][2]);
            if (ENERGY) {
                const Q<C> Ed = {Hn.w * Hp.w + Hn.x * Hp.x + Hn.y * Hp.y + Hn.z * Hp.z, F1, F2, F3};
                elec_e += pf<C>(F.e_elec[d], 4.0 * P.lap[d] * P.inv_sqr_dt) * pf<C>(F.inv_gpp_sqr, P.inv_gpp_sqr) *
                          one_minus_trace(Ed);
            }
            const Q<C> Hnew = su2_advance(Hn, H1, H2, H3, warn, check);
            st4(ps.L.hq[d], ps.s, Hnew.w, Hnew.x, Hnew.y, Hnew.z);
        }
    }
    if (!isfinite(check)) warn |= kWarnNonFinite;
    carry.valid = true;
    if (!count) {
        warn = warn_in;
        return;
    }

    if (ENERGY) {
        const double ge = (double)grad_e, ke = 0.5 * P.inv_sqr_dt * (double)kin_e;
        const double me = (double)mag_e, ee = (double)elec_e;
        if (P.loc_energy) {  // Energy's local densities (Analysers/Source/Energy.cpp:137-143)
            float* o = P.loc_energy + 6 * (size_t)ps.s;
            o[0] = (float)(pot_e + ge + ke + me + ee);
            o[1] = (float)pot_e;
            o[2] = (float)ge;
            o[3] = (float)ke;
            o[4] = (float)me;
            o[5] = (float)ee;
        }
        obs[kObsPotential] += pot_e;
        obs[kObsGradient] += ge;
        obs[kObsKinetic] += ke;
        obs[kObsMagnetic] += me;
        obs[kObsElectric] += ee;
        obs[kObsPlaqSU2] += (double)plaq2;
        obs[kObsPlaqU1] += (double)plaq1;
        obs[kObsPhiSq] += (double)phisq;
    }
}

// Gauss-law residual at site c after a step (Analysers/Source/GaugeCondition.cpp:117-165,
// Core/Source/Model.cpp:323-337 semantics), in FP64 for every form; md[a] is
// the site x - e_a.  v[k] = v[4 + k] = |violation of constraint k| (the
// integrated and the maximum slot of the analyser).  sin is the library's
// double series.
// One link direction at one site, both levels, as FP64 values.
struct GLink {
    Q<double> now, fut;
    double tnow, tfut;
};

template <class S, class LV>
__device__ __forceinline__ GLink gauss_link(const LV& now, const LV& fut, int d, int s)
{
    return {ld4<double>(now.q[d], s), ld4<double>(fut.q[d], s), ld1<double>(now.th[d], s), ld1<double>(fut.th[d], s)};
}

// The residuals from the links at x (own[d]) and at x - e_d (back[d]) and the
// doublets at x (phn / phf: both levels; site c for the local output).
// NEQ_ALL: the local-violation stride (gaugeNum; the Higgs-family constraints follow)
template <int MODEL, int NEQ_ALL = 4>
__device__ __forceinline__ void gauss_core(const StepParams& P, const GLink (&own)[3], const GLink (&back)[3],
                                           const Q<double> (&phn)[2], const Q<double> (&phf)[2], int c,
                                           double (&v)[kGaussSlots])
{
    constexpr int ND = (MODEL == kModelSM) ? 1 : 2;
    double el[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
    for (int d = 0; d < 3; d++) {
        const double la = own[d].tfut - own[d].tnow;
        const double na = back[d].tfut - back[d].tnow;
        el[0] += (gsin(la) - gsin(na)) * P.lap[d];
        // vec(U_now(x)^dag U_fut(x)) - vec(U_fut(x-d) U_now(x-d)^dag)
        double a1, a2, a3, b1, b2, b3;
        qmul_vec(qconj(own[d].now), own[d].fut, a1, a2, a3);
        qmul_vec(back[d].fut, qconj(back[d].now), b1, b2, b3);
        el[1] += (a1 - b1) * P.lap[d];
        el[2] += (a2 - b2) * P.lap[d];
        el[3] += (a3 - b3) * P.lap[d];
    }
    double gr[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
    for (int db = 0; db < ND; db++) {
        const Q<double> p = phn[db];
        const Q<double> q = phf[db];
        gr[0] += 0.25 * (p.w * q.x - p.x * q.w + p.y * q.z - p.z * q.y);
        gr[1] += 0.25 * (p.w * q.z - p.x * q.y + p.y * q.x - p.z * q.w);
        gr[2] += 0.25 * (-p.w * q.y - p.x * q.z + p.y * q.w + p.z * q.x);
        gr[3] += 0.25 * (p.w * q.x - p.x * q.w - p.y * q.z + p.z * q.y);
    }
#pragma unroll
    for (int k = 0; k < 4; k++) {
        const double viol = el[k] - P.gsq[k] * gr[k];
        const double av = fabs(viol);
        v[k] = av;
        v[4 + k] = av;
        if (P.loc_gauss) P.loc_gauss[(size_t)NEQ_ALL * c + k] = (float)viol;  // GaugeCondition local violation
    }
}

// v = |violation| of the 2 * gaugeNum slots (integrated then maximum) per
// constraint; with a Higgs-family field (HF != 0) the constraints 4.. of
// WilsonLoops/Source/TwoHDM.cpp:357-392 and Gradients/Source/TwoHDM.cpp:355-372 follow.
template <class S, int MODEL, int HF = kHfNone, class LV>
__device__ __forceinline__ void gauss_site(const StepParams& P, const LV& now, const LV& fut,
                                           int c, int md0, int md1, int md2, double (&v)[2 * hf_neq(HF)])
{
    const GLink own[3] = {gauss_link<S>(now, fut, 0, c), gauss_link<S>(now, fut, 1, c), gauss_link<S>(now, fut, 2, c)};
    const GLink back[3] = {gauss_link<S>(now, fut, 0, md0), gauss_link<S>(now, fut, 1, md1), gauss_link<S>(now, fut, 2, md2)};
    Q<double> phn[2], phf[2];
#pragma unroll
    for (int db = 0; db < ((MODEL == kModelSM) ? 1 : 2); db++) {
        phn[db] = ld4<double>(now.ph[db], c);
        phf[db] = ld4<double>(fut.ph[db], c);
    }
    if constexpr (HF == kHfNone) {
        gauss_core<MODEL>(P, own, back, phn, phf, c, v);
    } else {
        constexpr int NEQ = hf_neq(HF);
        double vs[kGaussSlots];
        gauss_core<MODEL, NEQ>(P, own, back, phn, phf, c, vs);
#pragma unroll
        for (int k = 0; k < 4; k++) {
            v[k] = vs[k];
            v[NEQ + k] = vs[4 + k];
        }
        const int md[3] = {md0, md1, md2};
        double el[3] = {0.0, 0.0, 0.0};
#pragma unroll
        for (int d = 0; d < 3; d++) {
            if constexpr (HF == kHfU1) {
                const double la = ld1<double>(fut.hth[d], c) - ld1<double>(now.hth[d], c);
                const double na = ld1<double>(fut.hth[d], md[d]) - ld1<double>(now.hth[d], md[d]);
                el[0] += (gsin(la) - gsin(na)) * P.lap[d];
            } else {
                double a1, a2, a3, b1, b2, b3;
                qmul_vec(qconj(ld4<double>(now.hq[d], c)), ld4<double>(fut.hq[d], c), a1, a2, a3);
                qmul_vec(ld4<double>(fut.hq[d], md[d]), qconj(ld4<double>(now.hq[d], md[d])), b1, b2, b3);
                el[0] += (a1 - b1) * P.lap[d];
                el[1] += (a2 - b2) * P.lap[d];
                el[2] += (a3 - b3) * P.lap[d];
            }
        }
        const Q<double> p1 = ld4<double>(now.ph[0], c), p2 = ld4<double>(now.ph[1], c);
        const Q<double> q1 = ld4<double>(fut.ph[0], c), q2 = ld4<double>(fut.ph[1], c);
        const double a8[8] = {p1.w, p1.x, p1.y, p1.z, p2.w, p2.x, p2.y, p2.z};
        const double b8[8] = {q1.w, q1.x, q1.y, q1.z, q2.w, q2.x, q2.y, q2.z};
        double gr[3] = {0.0, 0.0, 0.0};
#pragma unroll
        for (int i = 0; i < 4; i += 2) {
            if constexpr (HF == kHfU1) {
                gr[0] += 0.25 * (a8[i] * b8[i + 1] - a8[i + 1] * b8[i] - a8[i + 4] * b8[i + 5] + a8[i + 5] * b8[i + 4]);
            } else {
                gr[0] += 0.25 * (a8[i] * b8[i + 5] - a8[i + 1] * b8[i + 4] + a8[i + 4] * b8[i + 1] - a8[i + 5] * b8[i]);
                gr[1] += 0.25 * (-a8[i] * b8[i + 4] - a8[i + 1] * b8[i + 5] + a8[i + 4] * b8[i] + a8[i + 5] * b8[i + 1]);
                gr[2] += 0.25 * (a8[i] * b8[i + 1] - a8[i + 1] * b8[i] - a8[i + 4] * b8[i + 5] + a8[i + 5] * b8[i + 4]);
            }
        }
#pragma unroll
        for (int k = 0; k < NEQ - 4; k++) {
            const double viol = el[k] - P.gsq_hf * gr[k];
            const double av = fabs(viol);
            v[4 + k] = av;
            v[NEQ + 4 + k] = av;
            if (P.loc_gauss) P.loc_gauss[(size_t)NEQ * c + 4 + k] = (float)viol;
        }
    }
}

}  // namespace gft
