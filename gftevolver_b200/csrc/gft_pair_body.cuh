// gft_pair_body.cuh -- the SM mixed form's plain (non-logging) site update for
// TWO sites per thread, evaluated with Blackwell's paired FP32 instructions
// (fma.rn.f32x2 / add / mul: one instruction computes the same operation on
// both halves of a 64-bit register pair, each half rounded as the scalar
// instruction would round it).
//
// Why: the single-site tiled step issues ~1.7 k warp instructions per 32 sites
// and is limited by instruction issue, not by DRAM (its traffic is already the
// algorithmic 228 B per site-update).  Three quarters of those instructions are
// FP32 multiply-adds of the quaternion products, staple sums, transports and
// series; evaluating them on (site A, site B) pairs halves their count.
//
// The arithmetic is site_step's (gft_step_body.cuh) for MODEL = SM, no
// Higgs-family field, ENERGY = false -- the same reassociated staple sums, the
// same series (gft_math.cuh), the same rearranged FP32 leapfrog and link
// update -- with every float operation replaced by its paired form.  The
// physics it restates: Core/Source/Model.cpp:339-373,
// WilsonLoops/Source/StandardModel.cpp:324-514, Gradients/Source/StandardModel.cpp:72-100,
// 272-363, Potentials/Source/SO_N.cpp:57-75.
//
// V = float2 holds (site A, site B); the accessor returns both sites of a
// stencil position, so the neighbour structure of the two sites is identical
// and no value ever moves between halves.
#pragma once

#include "gft_device.cuh"
#include "gft_math.cuh"
#include "gft_step_body.cuh"

namespace gft {
namespace pair {

using V = float2;

__device__ __forceinline__ V bc(float s) { return make_float2(s, s); }
__device__ __forceinline__ V neg(V a) { return make_float2(-a.x, -a.y); }
__device__ __forceinline__ V add(V a, V b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ V sub(V a, V b) { return __fadd2_rn(a, neg(b)); }
__device__ __forceinline__ V mul(V a, V b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ V fma(V a, V b, V c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ V zero() { return make_float2(0.0f, 0.0f); }

using Q2 = Q<V>;

__device__ __forceinline__ Q2 qconj(Q2 a) { return {a.w, neg(a.x), neg(a.y), neg(a.z)}; }

// a0 b0 + a1 b1 + a2 b2 + a3 b3 summed from the left, each further term one
// fused multiply-add: the order in which the scalar kernels' expressions contract
__device__ __forceinline__ V dot4(V a0, V b0, V a1, V b1, V a2, V b2, V a3, V b3)
{
    return fma(a3, b3, fma(a2, b2, fma(a1, b1, mul(a0, b0))));
}

// (a0 b0 - a.b, a0 b + b0 a - a x b), the convention of WilsonLoops/Source/StandardModel.cpp:160-191
__device__ __forceinline__ Q2 qmul(Q2 a, Q2 b)
{
    Q2 r;
    r.w = dot4(a.w, b.w, neg(a.x), b.x, neg(a.y), b.y, neg(a.z), b.z);
    r.x = dot4(a.w, b.x, a.x, b.w, neg(a.y), b.z, a.z, b.y);
    r.y = dot4(a.w, b.y, a.y, b.w, neg(a.z), b.x, a.x, b.z);
    r.z = dot4(a.w, b.z, a.z, b.w, neg(a.x), b.y, a.y, b.x);
    return r;
}

__device__ __forceinline__ void qmul_vec(Q2 a, Q2 b, V& rx, V& ry, V& rz)
{
    rx = dot4(a.w, b.x, a.x, b.w, neg(a.y), b.z, a.z, b.y);
    ry = dot4(a.w, b.y, a.y, b.w, neg(a.z), b.x, a.x, b.z);
    rz = dot4(a.w, b.z, a.z, b.w, neg(a.x), b.y, a.y, b.x);
}

__device__ __forceinline__ Q2 qadd_scaled(Q2 acc, V s, Q2 a)
{
    return {fma(s, a.w, acc.w), fma(s, a.x, acc.x), fma(s, a.y, acc.y), fma(s, a.z, acc.z)};
}

__device__ __forceinline__ Q2 qzero() { return {zero(), zero(), zero(), zero()}; }

// Doublet f rotated by the hypercharge phase (cs, sn), then acted on by the
// SU(2) quaternion u as the real 4x4 of Gradients/Source/StandardModel.cpp:94-97.
__device__ __forceinline__ Q2 transport(Q2 u, V cs, V sn, Q2 f)
{
    const V h0 = fma(neg(sn), f.x, mul(cs, f.w));
    const V h1 = fma(sn, f.w, mul(cs, f.x));
    const V h2 = fma(neg(sn), f.z, mul(cs, f.y));
    const V h3 = fma(sn, f.y, mul(cs, f.z));
    Q2 t;
    t.w = dot4(u.w, h0, neg(u.z), h1, u.y, h2, neg(u.x), h3);
    t.x = dot4(u.z, h0, u.w, h1, u.x, h2, u.y, h3);
    t.y = dot4(neg(u.y), h0, neg(u.x), h1, u.w, h2, u.z, h3);
    t.z = dot4(u.x, h0, neg(u.y), h1, neg(u.z), h2, u.w, h3);
    return t;
}

// ---- elementary functions on pairs (the series and reduction of gft_math.cuh) ----

// x = k pi + r with the 1.5 * 2^23 rounding constant; the (-1)^k sign masks per half.
__device__ __forceinline__ V reduce_pi(V x, unsigned& sx, unsigned& sy)
{
    const V t = fma(x, bc(0.3183098861837907f), bc(12582912.0f));
    const V kf = sub(t, bc(12582912.0f));
    sx = __float_as_uint(t.x) << 31;
    sy = __float_as_uint(t.y) << 31;
    const V r = fma(neg(kf), bc(3.1415927410125732f), x);
    return fma(neg(kf), bc(-8.742277657347586e-08f), r);
}

__device__ __forceinline__ V flip(V v, unsigned sx, unsigned sy)
{
    return make_float2(__uint_as_float(__float_as_uint(v.x) ^ sx), __uint_as_float(__float_as_uint(v.y) ^ sy));
}

__device__ __forceinline__ V sin_poly(V r)
{
    const V r2 = mul(r, r);
    V ps = bc(GFT_FS9);
    ps = fma(ps, r2, bc(GFT_FS7));
    ps = fma(ps, r2, bc(GFT_FS5));
    ps = fma(ps, r2, bc(GFT_FS3));
    return fma(mul(ps, r2), r, r);
}

__device__ __forceinline__ V gsin(V x)
{
    unsigned sx, sy;
    const V r = reduce_pi(x, sx, sy);
    return flip(sin_poly(r), sx, sy);
}

__device__ __forceinline__ void gsincos(V x, V& s, V& c)
{
    unsigned sx, sy;
    const V r = reduce_pi(x, sx, sy);
    const V r2 = mul(r, r);
    V ps = bc(GFT_FS9);
    ps = fma(ps, r2, bc(GFT_FS7));
    ps = fma(ps, r2, bc(GFT_FS5));
    ps = fma(ps, r2, bc(GFT_FS3));
    s = flip(fma(mul(ps, r2), r, r), sx, sy);
    V pc = bc(GFT_FC10);
    pc = fma(pc, r2, bc(GFT_FC8));
    pc = fma(pc, r2, bc(GFT_FC6));
    pc = fma(pc, r2, bc(GFT_FC4));
    pc = fma(pc, r2, bc(GFT_FC2));
    c = flip(fma(pc, r2, bc(1.0f)), sx, sy);
}

// asin by its series for |x| <= 1/4 in both halves, else each half through the
// wide path (the link update's argument is dt * E ~ 1e-3)
__device__ __forceinline__ V gasin(V x)
{
    if (fabsf(x.x) > 0.25f || fabsf(x.y) > 0.25f) return make_float2(gft::gasin(x.x), gft::gasin(x.y));
    const V x2 = mul(x, x);
    V p = bc(924.0f / 53248.0f);
    p = fma(p, x2, bc(252.0f / 11264.0f));
    p = fma(p, x2, bc(70.0f / 2304.0f));
    p = fma(p, x2, bc(20.0f / 448.0f));
    p = fma(p, x2, bc(6.0f / 80.0f));
    p = fma(p, x2, bc(2.0f / 12.0f));
    return fma(mul(p, x2), x, x);
}

// sqrt(1 - c) - 1 by its series for c < 1/64 in both halves, else each half through the wide path
__device__ __forceinline__ V sqrt1m_minus1(V c)
{
    if (!(c.x < 0.015625f && c.y < 0.015625f)) return make_float2(gft::sqrt1m_minus1(c.x), gft::sqrt1m_minus1(c.y));
    return mul(c, fma(c, fma(c, fma(c, bc(-5.0f / 128.0f), bc(-1.0f / 16.0f)), bc(-1.0f / 8.0f)), bc(-0.5f)));
}

// ---- the paired site update ------------------------------------------------

// Values carried along the x-march to the +x site (as XCarry): the sines of
// the (0,1) and (0,2) plaquette angles and the doublet transported along the x link.
struct Carry2 {
    bool valid;
    V s01, s02;
    Q2 t0;
};

__device__ __forceinline__ Q2 ld_pair4(const float* p, int sa, int sb)
{
    const float4 a = __ldg(reinterpret_cast<const float4*>(p) + sa);
    const float4 b = __ldg(reinterpret_cast<const float4*>(p) + sb);
    return {make_float2(a.x, b.x), make_float2(a.y, b.y), make_float2(a.z, b.z), make_float2(a.w, b.w)};
}

__device__ __forceinline__ void st_pair4(float* p, int sa, int sb, Q2 v)
{
    reinterpret_cast<float4*>(p)[sa] = make_float4(v.w.x, v.x.x, v.y.x, v.z.x);
    reinterpret_cast<float4*>(p)[sb] = make_float4(v.w.y, v.x.y, v.y.y, v.z.y);
}

// A: pair accessor (q(d, R) -> Q2, th(d, R) -> V, ph(R) -> Q2 for the "now"
// level at stencil reference R, both sites).  past: the own sites' past level
// (read, then overwritten with t + dt) at site indices sa, sb.
template <class A, class R>
__device__ __forceinline__ void site_step2(const FConst& F, const A& acc, const Stencil<R>& n,
                                           const LevelPtrs<float>& past, int sa, int sb, Carry2& carry,
                                           unsigned& warn, bool count)
{
    const unsigned warn_in = warn;
    // own-site past level, loaded first so its latency overlaps the force arithmetic
    const Q2 pst_f = ld_pair4(past.ph[0], sa, sb);
    Q2 pst_u[3];
    V pst_t[3];
#pragma unroll
    for (int d = 0; d < 3; d++) {
        pst_u[d] = ld_pair4(past.q[d], sa, sb);
        pst_t[d] = make_float2(__ldg(past.th[d] + sa), __ldg(past.th[d] + sb));
    }
    const bool have = carry.valid;
    const V lap[3] = {bc(F.lap[0]), bc(F.lap[1]), bc(F.lap[2])};

    Q2 U[3];
    V th[3];
#pragma unroll
    for (int a = 0; a < 3; a++) {
        U[a] = acc.q(a, n.c);
        th[a] = acc.th(a, n.c);
    }

    // ---- magnetic term: U(1) sines and SU(2) staple sums ----
    V MgY[3] = {zero(), zero(), zero()};
    const V prev01 = carry.s01, prev02 = carry.s02;
    Q2 SA[3], SB[3];
#pragma unroll
    for (int a = 0; a < 3; a++) {
        SA[a] = qzero();
        SB[a] = qzero();
    }
#pragma unroll
    for (int pl = 0; pl < 3; pl++) {
        const int i = (pl == 2) ? 1 : 0;
        const int j = (pl == 0) ? 1 : 2;
        const Q2 Uj_pi = acc.q(j, n.p[i]);
        const Q2 Ui_pj = acc.q(i, n.p[j]);
        // F_ij(x) = theta_i(x) + theta_j(x+i) - theta_i(x+j) - theta_j(x)
        const V Fa = sub(sub(add(th[i], acc.th(j, n.p[i])), acc.th(i, n.p[j])), th[j]);
        const V sF = gsin(Fa);
        MgY[i] = fma(neg(sF), lap[j], MgY[i]);
        MgY[j] = fma(sF, lap[i], MgY[j]);
        if (pl == 0) carry.s01 = sF;
        if (pl == 1) carry.s02 = sF;
        const Q2 Cij = qmul(qconj(Uj_pi), Ui_pj);
        const Q2 Aij = qmul(Cij, U[j]);
        const Q2 Aji = qmul(qconj(Cij), U[i]);
        SA[i] = qadd_scaled(SA[i], lap[j], Aij);
        SA[j] = qadd_scaled(SA[j], lap[i], Aji);
    }
#pragma unroll
    for (int i = 0; i < 3; i++) {
#pragma unroll
        for (int j = 0; j < 3; j++) {
            if (j == i) continue;
            const R mj = n.m[j];
            const R dg = n.dg(i, j);
            const Q2 Uj_mj = acc.q(j, mj);
            const Q2 Ui_mj = acc.q(i, mj);
            const Q2 Uj_dg = acc.q(j, dg);
            if (j == 0 && have) {
                MgY[i] = fma(neg((i == 1) ? prev01 : prev02), lap[0], MgY[i]);
            } else {
                const V nb = add(add(sub(neg(acc.th(j, dg)), acc.th(i, mj)), acc.th(j, mj)), th[i]);
                MgY[i] = fma(neg(gsin(nb)), lap[j], MgY[i]);
            }
            const Q2 B = qmul(qmul(Uj_mj, qconj(Ui_mj)), qconj(Uj_dg));
            SB[i] = qadd_scaled(SB[i], lap[j], B);
        }
    }
    V Mg[3][3];
#pragma unroll
    for (int i = 0; i < 3; i++) {
        V a1, a2, a3, b1, b2, b3;
        qmul_vec(SA[i], qconj(U[i]), a1, a2, a3);
        qmul_vec(U[i], SB[i], b1, b2, b3);
        Mg[i][0] = sub(a1, b1);
        Mg[i][1] = sub(a2, b2);
        Mg[i][2] = sub(a3, b3);
    }

    // ---- scalar sector: covariant Laplacian D and currents J ----
    const Q2 fc = acc.ph(n.c);
    const V diag = bc(F.diag);
    Q2 D = {mul(diag, fc.w), mul(diag, fc.x), mul(diag, fc.y), mul(diag, fc.z)};
    V J[3][4];
#pragma unroll
    for (int a = 0; a < 3; a++) {
        V sn, cs;
        gsincos(th[a], sn, cs);
        const Q2 Uc = qconj(U[a]);
        const bool from_carry = (a == 0) && have;
        V sm = zero(), cm = bc(1.0f);
        Q2 Um = {bc(1.0f), zero(), zero(), zero()};
        if (!from_carry) {
            gsincos(acc.th(a, n.m[a]), sm, cm);
            Um = acc.q(a, n.m[a]);
        }
        const Q2 fp = acc.ph(n.p[a]);
        // D: U_a(x-a) phi(x-a) + U_a(x)^dag phi(x+a); the first is the x-1 site's transported doublet
        const Q2 tm = from_carry ? carry.t0 : transport(Um, cm, sm, acc.ph(n.m[a]));
        const Q2 tp = transport(Uc, cs, neg(sn), fp);
        D = qadd_scaled(D, lap[a], tm);
        D = qadd_scaled(D, lap[a], tp);
        // J: Im of (U_a(x) phi(x))^dag sigma phi(x+a)
        const Q2 t = transport(U[a], cs, sn, fc);
        if (a == 0) carry.t0 = t;
        const V q = bc(0.25f);
        J[a][0] = mul(q, dot4(t.w, fp.x, neg(t.x), fp.w, t.y, fp.z, neg(t.z), fp.y));
        J[a][1] = mul(q, dot4(t.w, fp.z, neg(t.x), fp.y, t.y, fp.x, neg(t.z), fp.w));
        J[a][2] = mul(q, dot4(neg(t.w), fp.y, neg(t.x), fp.z, t.y, fp.w, t.z, fp.x));
        J[a][3] = mul(q, dot4(t.w, fp.x, neg(t.x), fp.w, neg(t.y), fp.z, t.z, fp.y));
    }

    // ---- potential dV/dphi (SO_N) ----
    const V fsq = dot4(fc.w, fc.w, fc.x, fc.x, fc.y, fc.y, fc.z, fc.z);
    const V k = mul(bc(F.lambda), sub(fsq, bc(F.eta_sqr)));
    const V Pot[4] = {mul(k, fc.w), mul(k, fc.x), mul(k, fc.y), mul(k, fc.z)};

    // ---- scalar leapfrog: phi + [(phi - phi_past)(1 - damping) + dt^2 (D - dV)] ----
    const V dt2 = bc(F.dt2), keep = bc(F.keep);
    V check = zero();  // sum of every new value: non-finite iff one of them is
    {
        const V fn[4] = {fc.w, fc.x, fc.y, fc.z};
        const V fo[4] = {pst_f.w, pst_f.x, pst_f.y, pst_f.z};
        const V dd[4] = {D.w, D.x, D.y, D.z};
        V out[4];
#pragma unroll
        for (int c = 0; c < 4; c++) {
            const V vel = sub(fn[c], fo[c]);
            out[c] = add(fn[c], fma(keep, vel, mul(dt2, sub(dd[c], Pot[c]))));
            check = add(check, out[c]);
        }
        st_pair4(past.ph[0], sa, sb, {out[0], out[1], out[2], out[3]});
    }

    // ---- link update (WilsonLoops/Source/StandardModel.cpp:456-514) ----
    const V gY = bc(F.gY), gI = bc(F.gI);
#pragma unroll
    for (int d = 0; d < 3; d++) {
        const Q2 Un = U[d];
        const Q2 Up = pst_u[d];
        // link momentum vec(U_now U_past^dag) = vec((U_now - U_past) U_past^dag)
        const Q2 dlt = {sub(Un.w, Up.w), sub(Un.x, Up.x), sub(Un.y, Up.y), sub(Un.z, Up.z)};
        V E1, E2, E3;
        qmul_vec(dlt, qconj(Up), E1, E2, E3);
        const V dth = sub(th[d], pst_t[d]);
        const V R0 = fma(keep, gsin(dth), mul(dt2, fma(gY, J[d][0], MgY[d])));
        const V R1 = fma(keep, E1, mul(dt2, fma(gI, J[d][1], Mg[d][0])));
        const V R2 = fma(keep, E2, mul(dt2, fma(gI, J[d][2], Mg[d][1])));
        const V R3 = fma(keep, E3, mul(dt2, fma(gI, J[d][3], Mg[d][2])));
        const V r0sq = mul(R0, R0);
        if (r0sq.x > 1.0f || r0sq.y > 1.0f) warn |= kWarnAsin;
        if (fabsf(th[d].x) > 1e4f || fabsf(th[d].y) > 1e4f) warn |= kWarnRange;
        // theta(t+dt) = theta(t) + asin(RHS_Y)
        const V thn = add(th[d], gasin(R0));
        // U(t+dt) = normalise(u U(t)) as U + correction (site_step's form)
        const V cm = fma(R3, R3, fma(R2, R2, mul(R1, R1)));
        if (cm.x > 1.0f || cm.y > 1.0f) warn |= kWarnSqrt;
        const V u0m1 = sqrt1m_minus1(cm);
        const Q2 dU = qmul(Q2{u0m1, R1, R2, R3}, Un);
        V e = fma(Un.w, Un.w, bc(-1.0f));
        e = fma(Un.x, Un.x, e);
        e = fma(Un.y, Un.y, e);
        e = fma(Un.z, Un.z, e);
        const V udu = dot4(Un.w, dU.w, Un.x, dU.x, Un.y, dU.y, Un.z, dU.z);
        const V dd = dot4(dU.w, dU.w, dU.x, dU.x, dU.y, dU.y, dU.z, dU.z);
        e = add(e, fma(bc(2.0f), udu, dd));
        const V fm1 = mul(e, fma(bc(0.375f), e, bc(-0.5f)));
        const Q2 Unew = {add(Un.w, fma(fm1, add(Un.w, dU.w), dU.w)), add(Un.x, fma(fm1, add(Un.x, dU.x), dU.x)),
                         add(Un.y, fma(fm1, add(Un.y, dU.y), dU.y)), add(Un.z, fma(fm1, add(Un.z, dU.z), dU.z))};
        check = add(check, add(thn, e));
        past.th[d][sa] = thn.x;
        past.th[d][sb] = thn.y;
        st_pair4(past.q[d], sa, sb, Unew);
    }
    if (!isfinite(check.x) || !isfinite(check.y)) warn |= kWarnNonFinite;
    carry.valid = true;
    if (!count) warn = warn_in;  // ghost planes of an x-slab: no warnings
}

}  // namespace pair
}  // namespace gft
