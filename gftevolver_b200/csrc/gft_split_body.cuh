// gft_split_body.cuh -- the SM mixed form's plain site update divided between
// two threads, so that each holds about half of the live state.
//
// The one-site tiled step is limited by instruction issue with latency that its
// 16 resident warps per SM cannot hide (128 registers per thread, two CTAs per
// SM).  Here a site's work is split between a "links" thread (SU(2) staple sums
// and the SU(2) link update) and a "scalars" thread (U(1) plaquette sines, the
// covariant Laplacian and the Higgs currents, the potential, the scalar
// leapfrog, the U(1) link update, and the SU(2) link momentum E); the scalars
// thread hands E and the currents J to the links thread through shared memory.
// With about 85 registers per thread, three 256-thread CTAs fit per SM: 24
// warps.  The arithmetic is site_step's (gft_step_body.cuh) for MODEL = SM, no
// Higgs-family field, ENERGY = false, expression by expression, so the results
// agree with the one-site step to contraction-level rounding.  Physics it
// restates: Core/Source/Model.cpp:339-373, WilsonLoops/Source/StandardModel.cpp:324-514,
// Gradients/Source/StandardModel.cpp:72-100, 272-363, Potentials/Source/SO_N.cpp:57-75.
#pragma once

#include "gft_device.cuh"
#include "gft_math.cuh"
#include "gft_step_body.cuh"

namespace gft {
namespace split {

// What the scalars thread hands to the links thread for one site: the SU(2)
// link momentum E_d = vec((U_now - U_past) U_past^dag) and the currents J_d(1..3),
// 18 floats in shared memory, structure of arrays over the NT threads of a role
// (consecutive threads, consecutive words: no bank conflicts).
template <int NT>
struct Handoff {
    float* base;
    int t;
    __device__ __forceinline__ float& e(int a, int k) const { return base[(a * 3 + k) * NT + t]; }
    __device__ __forceinline__ float& j(int a, int k) const { return base[(9 + a * 3 + k) * NT + t]; }
    static constexpr int kBytes = 18 * NT * 4;
};

// Values the scalars thread carries along the x-march (XCarry's): the sines of
// the (0,1) and (0,2) plaquette angles and the doublet transported along the x link.
struct ScalarCarry {
    bool valid;
    float s01, s02;
    Q<float> t0;
};

// The scalars thread of a site: everything of site_step except the SU(2)
// staples and the SU(2) link update.  Writes the new doublet and the new U(1)
// phases, and fills `out` for the links thread.
template <class A, class R, class H>
__device__ __forceinline__ void site_scalars(const FConst& F, const A& acc, const Stencil<R>& n,
                                             const LevelPtrs<float>& past, int s, ScalarCarry& carry,
                                             const H& out, unsigned& warn)
{
    using C = float;
    Q<C> pst_u[3];
    C pst_t[3];
    const Q<C> pst_f = ld4<C>(past.ph[0], s);
#pragma unroll
    for (int d = 0; d < 3; d++) {
        pst_u[d] = ld4<C>(past.q[d], s);
        pst_t[d] = ld1<C>(past.th[d], s);
    }
    const bool have = carry.valid;
    const C lap[3] = {F.lap[0], F.lap[1], F.lap[2]};
    C th[3];
#pragma unroll
    for (int a = 0; a < 3; a++) th[a] = acc.th(a, n.c);

    // ---- U(1) magnetic term ----
    C MgY[3] = {(C)0, (C)0, (C)0};
    const C prev01 = carry.s01, prev02 = carry.s02;
#pragma unroll
    for (int pl = 0; pl < 3; pl++) {
        const int i = (pl == 2) ? 1 : 0;
        const int j = (pl == 0) ? 1 : 2;
        const C Fa = th[i] + acc.th(j, n.p[i]) - acc.th(i, n.p[j]) - th[j];
        const C sF = gsin(Fa);
        MgY[i] -= sF * lap[j];
        MgY[j] += sF * lap[i];
        if (pl == 0) carry.s01 = sF;
        if (pl == 1) carry.s02 = sF;
    }
#pragma unroll
    for (int i = 0; i < 3; i++) {
#pragma unroll
        for (int j = 0; j < 3; j++) {
            if (j == i) continue;
            if (j == 0 && have) {
                MgY[i] -= ((i == 1) ? prev01 : prev02) * lap[0];
            } else {
                const R mj = n.m[j];
                const C neigh = -acc.th(j, n.dg(i, j)) - acc.th(i, mj) + acc.th(j, mj) + th[i];
                MgY[i] -= gsin(neigh) * lap[j];
            }
        }
    }

    // ---- covariant Laplacian D and currents J ----
    const Q<C> fc = acc.ph(0, n.c);
    Q<C> D;
    {
        const C w = F.diag;
        D = {w * fc.w, w * fc.x, w * fc.y, w * fc.z};
    }
    C J0[3];
#pragma unroll
    for (int a = 0; a < 3; a++) {
        C sn, cs;
        gsincos(th[a], sn, cs);
        const Q<C> Ua = acc.q(a, n.c);
        const Q<C> Uc = qconj(Ua);
        C j0 = 0, j1 = 0, j2 = 0, j3 = 0;
        const bool from_carry = (a == 0) && have;
        C sm = (C)0, cm = (C)1;
        Q<C> Um = {(C)1, (C)0, (C)0, (C)0};
        if (!from_carry) {
            gsincos(acc.th(a, n.m[a]), sm, cm);
            Um = acc.q(a, n.m[a]);
        }
        const Q<C> fp = acc.ph(0, n.p[a]);
        const Q<C> tm = from_carry ? carry.t0 : transport(Um, cm, sm, acc.ph(0, n.m[a]));
        const Q<C> tp = transport(Uc, cs, -sn, fp);
        D = qadd_scaled(D, lap[a], tm);
        D = qadd_scaled(D, lap[a], tp);
        const Q<C> t = transport(Ua, cs, sn, fc);
        if (a == 0) carry.t0 = t;
        j0 += t.w * fp.x - t.x * fp.w + t.y * fp.z - t.z * fp.y;
        j1 += t.w * fp.z - t.x * fp.y + t.y * fp.x - t.z * fp.w;
        j2 += -t.w * fp.y - t.x * fp.z + t.y * fp.w + t.z * fp.x;
        j3 += t.w * fp.x - t.x * fp.w - t.y * fp.z + t.z * fp.y;
        J0[a] = (C)0.25 * j0;
        out.j(a, 0) = (C)0.25 * j1;
        out.j(a, 1) = (C)0.25 * j2;
        out.j(a, 2) = (C)0.25 * j3;
        // SU(2) link momentum vec(U_now U_past^dag) = vec((U_now - U_past) U_past^dag)
        const Q<C> Up = pst_u[a];
        const Q<C> dlt = {Ua.w - Up.w, Ua.x - Up.x, Ua.y - Up.y, Ua.z - Up.z};
        C e1, e2, e3;
        qmul_vec(dlt, qconj(Up), e1, e2, e3);
        out.e(a, 0) = e1;
        out.e(a, 1) = e2;
        out.e(a, 2) = e3;
    }

    // ---- potential dV/dphi (SO_N) and the scalar leapfrog ----
    const C fsq = fc.w * fc.w + fc.x * fc.x + fc.y * fc.y + fc.z * fc.z;
    const C k = F.lambda * (fsq - F.eta_sqr);
    const C pot[4] = {k * fc.w, k * fc.x, k * fc.y, k * fc.z};
    const C dt2 = F.dt2, keep = F.keep;
    C check = (C)0;
    {
        const C fn[4] = {fc.w, fc.x, fc.y, fc.z};
        const C fo[4] = {pst_f.w, pst_f.x, pst_f.y, pst_f.z};
        const C dd[4] = {D.w, D.x, D.y, D.z};
        C o[4];
#pragma unroll
        for (int c = 0; c < 4; c++) {
            const C vel = fn[c] - fo[c];
            o[c] = fn[c] + (keep * vel + dt2 * (dd[c] - pot[c]));
            check += o[c];
        }
        st4(past.ph[0], s, o[0], o[1], o[2], o[3]);
    }

    // ---- U(1) link update: theta(t+dt) = theta(t) + asin(RHS_Y) ----
    const C gY = F.gY;
#pragma unroll
    for (int d = 0; d < 3; d++) {
        const C dth = th[d] - pst_t[d];
        const C R0 = keep * gsin(dth) + dt2 * (MgY[d] + gY * J0[d]);
        if (R0 * R0 > (C)1) warn |= kWarnAsin;
        if (fabs(th[d]) > (C)1e4) warn |= kWarnRange;
        const C thn = th[d] + gasin(R0);
        check += thn;
        past.th[d][s] = thn;
    }
    if (!isfinite(check)) warn |= kWarnNonFinite;
    carry.valid = true;
}

// The links thread of a site: the SU(2) staple sums, then -- after wait(),
// which orders the scalars thread's handoff before the reads -- the SU(2) link
// update from E and J, written as site_step writes it.
template <class A, class R, class H, class Wait>
__device__ __forceinline__ void site_links(const FConst& F, const A& acc, const Stencil<R>& n,
                                           const LevelPtrs<float>& past, int s, const H& in, Wait&& wait,
                                           unsigned& warn)
{
    using C = float;
    const C lap[3] = {F.lap[0], F.lap[1], F.lap[2]};
    Q<C> U[3];
#pragma unroll
    for (int a = 0; a < 3; a++) U[a] = acc.q(a, n.c);
    Q<C> SA[3], SB[3];
#pragma unroll
    for (int a = 0; a < 3; a++) {
        SA[a] = {(C)0, (C)0, (C)0, (C)0};
        SB[a] = {(C)0, (C)0, (C)0, (C)0};
    }
#pragma unroll
    for (int pl = 0; pl < 3; pl++) {
        const int i = (pl == 2) ? 1 : 0;
        const int j = (pl == 0) ? 1 : 2;
        const Q<C> Uj_pi = acc.q(j, n.p[i]);
        const Q<C> Ui_pj = acc.q(i, n.p[j]);
        const Q<C> Cij = qmul(qconj(Uj_pi), Ui_pj);
        const Q<C> Aij = qmul(Cij, U[j]);
        const Q<C> Aji = qmul(qconj(Cij), U[i]);
        SA[i] = qadd_scaled(SA[i], lap[j], Aij);
        SA[j] = qadd_scaled(SA[j], lap[i], Aji);
    }
#pragma unroll
    for (int i = 0; i < 3; i++) {
#pragma unroll
        for (int j = 0; j < 3; j++) {
            if (j == i) continue;
            const R mj = n.m[j];
            const Q<C> B = qmul(qmul(acc.q(j, mj), qconj(acc.q(i, mj))), qconj(acc.q(j, n.dg(i, j))));
            SB[i] = qadd_scaled(SB[i], lap[j], B);
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

    wait();  // E and J of this site from the scalars thread
    const C dt2 = F.dt2, keep = F.keep, gI = F.gI;
    C check = (C)0;
#pragma unroll
    for (int d = 0; d < 3; d++) {
        const Q<C> Un = U[d];
        const C R1 = keep * in.e(d, 0) + dt2 * (Mg[d][0] + gI * in.j(d, 0));
        const C R2 = keep * in.e(d, 1) + dt2 * (Mg[d][1] + gI * in.j(d, 1));
        const C R3 = keep * in.e(d, 2) + dt2 * (Mg[d][2] + gI * in.j(d, 2));
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
        st4(past.q[d], s, Un.w + (dU.w + fm1 * (Un.w + dU.w)), Un.x + (dU.x + fm1 * (Un.x + dU.x)),
            Un.y + (dU.y + fm1 * (Un.y + dU.y)), Un.z + (dU.z + fm1 * (Un.z + dU.z)));
    }
    if (!isfinite(check)) warn |= kWarnNonFinite;
}

}  // namespace split
}  // namespace gft
