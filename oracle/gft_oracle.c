/*
 * gft_oracle.c -- TEST INFRASTRUCTURE ONLY (see gft_oracle.h).
 *
 * A plain-C restatement of the reference's per-site leapfrog update and its
 * two analysers, written to reproduce the reference's arithmetic operation by
 * operation: fields are stored as S (float or double), every per-site quantity
 * is evaluated in double in the reference's order, and values the reference
 * keeps in `float` containers are kept in S.  Compile with
 *     -DORC_S=float  -DORC_PREFIX=orc32_     (reference as shipped)
 *     -DORC_S=double -DORC_PREFIX=orc64_     (reference with float -> double)
 * and never with FMA contraction (-ffp-contract=off), so that results match
 * the reference binary bit for bit except where libm differs.
 *
 * Layout (Core/Source/Lattice.cpp:358-367, 658-671): two time levels,
 *     scalars[((t*nx + x)*ny + y)*nz + z][nsc]     nsc = 4 (SM) or 8 (2HDM)
 *     vectors[((t*nx + x)*ny + y)*nz + z][3*dw]    per direction d: [theta_Y, c0, c1, c2, c3]
 *                                                  (+ theta_H, or + d0..d3, for the 2HDM
 *                                                  Higgs-family gauge field: dw = 5, 6 or 9);
 *                                                  generator representation: [theta_Y, w1..w3]
 *                                                  (+ theta_H or w'1..w'3: dw = 4, 5 or 7)
 * At step time_iter the "now" level is (time_iter + 1) % 2 and the update is
 * written in place into the other ("past") level (Lattice.cpp:773-774).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "gft_oracle.h"

#ifndef ORC_S
#define ORC_S float
#endif
#ifndef ORC_PREFIX
#define ORC_PREFIX orc32_
#endif

typedef ORC_S S;

#define ORC_CAT2(a, b) a##b
#define ORC_CAT(a, b) ORC_CAT2(a, b)
#define FN(name) ORC_CAT(ORC_PREFIX, name)

/* ----------------------------------------------------------------------------
 * Model context: the plugin parameters the reference keeps as members.
 * ------------------------------------------------------------------------- */
typedef struct {
    int model, nsc;
    int hf, dw, nv, neq;         /* Higgs family, words per direction, per site, gauge equations per direction */
    int gen;                     /* generator link representation */
    int hf_off;                  /* offset of the Higgs-family field in a direction block */
    long long nx, ny, nz, nsite;
    double dt;
    double stencil[3][3];        /* Gradients/Source/StandardModel.cpp:14-24 */
    double energy_stencil[3][3]; /* Gradients/Source/StandardModel.cpp:35-42 */
    double inv_sqr[3];           /* WilsonLoops/Source/StandardModel.cpp:51-53 */
    double inv_sqr_dt;           /* :55 */
    double g_sqr, gp_sqr, inv_g_sqr, inv_gp_sqr;
    double gpp_sqr, inv_gpp_sqr; /* WilsonLoops/Source/TwoHDM.cpp:17-39, 62-86 */
    double gsq_coupling[ORC_MAX_EQ]; /* getSqrCouplings(k) (returns float: :224-230; TwoHDM.cpp:258-267) */
    int store_energy;            /* WilsonLoops storeEnergy flag (:243-248) */
    double damping_step;         /* Core/Source/Model.cpp:345 */
    const orc_config* cfg;
} ctx_t;

/* stencil pointers at t_now: vp[a][0..4] = x-a, x, x+a, x+a-e_j0, x+a-e_j1 (j0 < j1
 * the other two axes), sp[a][0..2] = x-a, x, x+a (Lattice.cpp:572-655,
 * Periodic.cpp:18-170; periodic wrap on every axis). */
typedef struct {
    const S* vp[3][5];
    const S* sp[3][3];
} stencil_t;

/* ----------------------------------------------------------------------------
 * SU(2) helpers (WilsonLoops/Source/StandardModel.cpp:76-112, 160-191)
 * ------------------------------------------------------------------------- */

/* getSU2Representation (WilsonLoops/Source/StandardModel.cpp:76-112, TwoHDM.cpp:94-126):
 * quaternion branch c0 = v[d+off], c_a = conj*v[d+off+a]; generator branch from
 * w = v[d+off .. d+off+2]: c0 = cos|w|, c_a = conj*sin|w|*w_a/|w| (c1 = sin|w| when
 * |w| <= tol).  off = 1: the isospin link; the Higgs-family SU(2) link at hf_off. */
static int g_gen = 0;          /* the representation of the current run (set by ctx_init) */
static double g_gen_tol = 0.0; /* divisionByZeroTolerance */

static void su2_rep_at(const S* v, int d, int off, int conj, double c[4])
{
    if (g_gen) {
        double wm = 0.0;
        for (int k = 0; k < 3; k++) wm += (double)v[d + off + k] * (double)v[d + off + k];
        wm = sqrt(wm);
        c[0] = cos(wm);
        c[1] = c[2] = c[3] = 0.0;
        if (wm > g_gen_tol) {
            for (int k = 1; k < 4; k++) c[k] = ((double)(conj ? -1 : 1) * sin(wm)) * (double)v[d + off + k - 1] / wm;
        } else {
            c[1] = sin(wm);
        }
        return;
    }
    c[0] = (double)v[d + off];
    for (int k = 1; k < 4; k++) {
        S comp = conj ? (S)(-v[d + off + k]) : v[d + off + k];
        c[k] = (double)comp;
    }
}

static void su2_rep(const S* v, int d, int conj, double c[4]) { su2_rep_at(v, d, 1, conj, c); }

/* invertSU2Representation (WilsonLoops/Source/StandardModel.cpp:114-158): phase =
 * asin|c| (pi/2 when |c| > 1), pi - phase when c0 < 0; w = phase*c/|c| (w1 = phase when
 * |c| <= tol); stored in S. */
static void su2_invert(const double c[4], S w[3])
{
    double cm = 0.0;
    for (int k = 1; k < 4; k++) cm += c[k] * c[k];
    cm = sqrt(cm);
    double phase = (cm > 1) ? 1.5707963267948966 : asin(cm);
    if (c[0] < 0) phase = 3.141592653589793 - phase;
    if (cm > g_gen_tol) {
        for (int k = 0; k < 3; k++) w[k] = (S)(phase * c[k + 1] / cm);
    } else {
        w[0] = (S)phase;
        w[1] = w[2] = (S)0;
    }
}

/* offset of the Higgs-family field in a direction block (TwoHDM.cpp:362-368: 5 in the
 * quaternion representation, 4 in the generator representation) */
#define HF_OFF (m->hf_off)

/* SU2Product(U1, U2, calc_trace): vector part always, scalar part and
 * renormalisation only when calc_trace (component 0 stays 0 otherwise). */
static void su2_product(const double a[4], const double b[4], int calc_trace, double out[4])
{
    double p[4];
    p[0] = 0.0;
    p[1] = a[0] * b[1] + a[1] * b[0] - a[2] * b[3] + a[3] * b[2];
    p[2] = a[0] * b[2] + a[2] * b[0] - a[3] * b[1] + a[1] * b[3];
    p[3] = a[0] * b[3] + a[3] * b[0] - a[1] * b[2] + a[2] * b[1];
    if (calc_trace) {
        double dot = 0.0;
        for (int k = 1; k < 4; k++) dot += a[k] * b[k];
        p[0] = a[0] * b[0] - dot;
        double norm = sqrt(p[0] * p[0] + p[1] * p[1] + p[2] * p[2] + p[3] * p[3]);
        for (int k = 0; k < 4; k++) p[k] = p[k] / norm;
    }
    for (int k = 0; k < 4; k++) out[k] = p[k];
}

/* ----------------------------------------------------------------------------
 * Gradients (Gradients/Source/StandardModel.cpp:72-100, TwoHDM.cpp:72-149)
 * ------------------------------------------------------------------------- */

/* transform(phi, link, conj): U(1) phase on each complex pair, then the SU(2)
 * quaternion as a real 4x4 matrix, doublet by doublet; for the 2HDM with a
 * Higgs-family field, then its U(1) phase (+theta_H on doublet 1, -theta_H on
 * doublet 2) or its SU(2) acting on (doublet 1, doublet 2) component pairs
 * (Gradients/Source/TwoHDM.cpp:72-149). */
static void transform_sm(int nsc, const double* in, const S* v, int d, int conj, double* out);

static void transform(const ctx_t* m, const double* in, const S* v, int d, int conj, double* out)
{
    if (m->hf == ORC_HF_NONE) {
        transform_sm(m->nsc, in, v, d, conj, out);
        return;
    }
    double sm[8];
    transform_sm(8, in, v, d, conj, sm);
    const int conj_fac = conj ? -1 : 1;
    if (m->hf == ORC_HF_U1) {
        const double th = (double)v[d + HF_OFF];
        for (int c = 0; c < 8; c++) {
            int pm = -1 + 2 * (c % 2);
            int pm4 = 1 - 2 * (c / 4);
            out[c] = cos(th) * sm[c] + (double)pm * sin((double)(pm4 * conj_fac) * th) * sm[c - pm];
        }
    } else {
        double u[4];
        su2_rep_at(v, d, HF_OFF, conj, u);
        for (int inner = 0; inner < 2; inner++) {
            const int i = inner * 2;
            out[i]     =  u[0] * sm[i] - u[3] * sm[i + 1] + u[2] * sm[i + 4] - u[1] * sm[i + 5];
            out[i + 1] =  u[3] * sm[i] + u[0] * sm[i + 1] + u[1] * sm[i + 4] + u[2] * sm[i + 5];
            out[i + 4] = -u[2] * sm[i] - u[1] * sm[i + 1] + u[0] * sm[i + 4] + u[3] * sm[i + 5];
            out[i + 5] =  u[1] * sm[i] - u[2] * sm[i + 1] - u[3] * sm[i + 4] + u[0] * sm[i + 5];
        }
    }
}

static void transform_sm(int nsc, const double* in, const S* v, int d, int conj, double* out)
{
    double hyper[8];
    double th = (double)v[d];
    for (int c = 0; c < nsc; c++) {
        int pm = -1 + 2 * (c % 2);
        double s = sin((conj ? -1.0 : 1.0) * th);
        hyper[c] = cos(th) * in[c] + ((double)pm * s) * in[c - pm];
    }
    double u[4];
    su2_rep(v, d, conj, u);
    for (int db = 0; db < nsc; db += 4) {
        const double* h = hyper + db;
        out[db + 0] =  u[0] * h[0] - u[3] * h[1] + u[2] * h[2] - u[1] * h[3];
        out[db + 1] =  u[3] * h[0] + u[0] * h[1] + u[1] * h[2] + u[2] * h[3];
        out[db + 2] = -u[2] * h[0] - u[1] * h[1] + u[0] * h[2] + u[3] * h[3];
        out[db + 3] =  u[1] * h[0] - u[2] * h[1] - u[3] * h[2] + u[0] * h[3];
    }
}

static void load_scalar(int nsc, const S* p, double* out)
{
    for (int c = 0; c < nsc; c++) out[c] = (double)p[c];
}

/* calcDerivatives: 3-point covariant Laplacian, stencil-major order. */
static void calc_derivatives(const ctx_t* m, const stencil_t* st, double* D)
{
    int nsc = m->nsc;
    for (int c = 0; c < nsc; c++) D[c] = 0.0;
    for (int s = 0; s < 3; s++) {
        for (int a = 0; a < 3; a++) {
            int d = a * m->dw;
            double f[8], t[8];
            load_scalar(nsc, st->sp[a][s], f);
            if (s == 0) {
                transform(m, f, st->vp[a][0], d, 0, t);
                memcpy(f, t, sizeof(double) * (size_t)nsc);
            } else if (s == 2) {
                transform(m, f, st->vp[a][1], d, 1, t);
                memcpy(f, t, sizeof(double) * (size_t)nsc);
            }
            for (int c = 0; c < nsc; c++) D[c] += m->stencil[a][s] * f[c];
        }
    }
}

/* calcCurrents: J[neq*a + k] (hypercharge k = 0, isospin k = 1..3, Higgs family
 * k = 4 (U(1)) or 4..6 (SU(2))), summed over doublets (TwoHDM.cpp:424-489). */
static void calc_currents(const ctx_t* m, const stencil_t* st, double J[3 * ORC_MAX_EQ])
{
    int nsc = m->nsc;
    for (int k = 0; k < 3 * m->neq; k++) J[k] = 0.0;
    for (int a = 0; a < 3; a++) {
        int e = a * m->neq, d = a * m->dw;
        double f[8], t[8], n[8];
        load_scalar(nsc, st->sp[a][1], f);
        transform(m, f, st->vp[a][1], d, 0, t);
        load_scalar(nsc, st->sp[a][2], n);
        for (int db = 0; db < nsc; db += 4) {
            const double* p = t + db;
            const double* q = n + db;
            J[e + 0] += 0.25 * ( p[0] * q[1] - p[1] * q[0] + p[2] * q[3] - p[3] * q[2]);
            J[e + 1] += 0.25 * ( p[0] * q[3] - p[1] * q[2] + p[2] * q[1] - p[3] * q[0]);
            J[e + 2] += 0.25 * (-p[0] * q[2] - p[1] * q[3] + p[2] * q[0] + p[3] * q[1]);
            J[e + 3] += 0.25 * ( p[0] * q[1] - p[1] * q[0] - p[2] * q[3] + p[3] * q[2]);
            const int i = db / 2;  /* upper (0) or lower (2) component pair of both doublets */
            if (m->hf == ORC_HF_U1) {
                J[e + 4] += 0.25 * (t[i] * n[i + 1] - t[i + 1] * n[i] - t[i + 4] * n[i + 5] + t[i + 5] * n[i + 4]);
            } else if (m->hf == ORC_HF_SU2) {
                J[e + 4] += 0.25 * ( t[i] * n[i + 5] - t[i + 1] * n[i + 4] + t[i + 4] * n[i + 1] - t[i + 5] * n[i]);
                J[e + 5] += 0.25 * (-t[i] * n[i + 4] - t[i + 1] * n[i + 5] + t[i + 4] * n[i] + t[i + 5] * n[i + 1]);
                J[e + 6] += 0.25 * ( t[i] * n[i + 1] - t[i + 1] * n[i] - t[i + 4] * n[i + 5] + t[i + 5] * n[i + 4]);
            }
        }
    }
}

/* calcGradientEnergy: forward covariant difference, accumulated in S. */
static S gradient_energy(const ctx_t* m, const stencil_t* st)
{
    int nsc = m->nsc;
    S der[24];
    for (int k = 0; k < 3 * nsc; k++) der[k] = (S)0;
    for (int s = 1; s < 3; s++) {
        for (int a = 0; a < 3; a++) {
            double f[8], t[8];
            load_scalar(nsc, st->sp[a][s], f);
            if (s == 1) {
                transform(m, f, st->vp[a][1], a * m->dw, 0, t);
                memcpy(f, t, sizeof(double) * (size_t)nsc);
            }
            for (int c = 0; c < nsc; c++)
                der[a * nsc + c] = (S)((double)der[a * nsc + c] + m->energy_stencil[a][s] * f[c]);
        }
    }
    S ge = (S)0;
    for (int k = 0; k < 3 * nsc; k++) ge = (S)((double)ge + (double)der[k] * (double)der[k]);
    return (S)0.5f * ge;
}

/* calcKineticEnergy: powf((now - past)/float(dt), 2) in S. */
static S kinetic_energy(const ctx_t* m, const S* now, const S* past)
{
    S ke = (S)0;
    S dtS = (S)m->dt;
    for (int c = 0; c < m->nsc; c++) {
        S q = (S)(now[c] - past[c]) / dtS;
        ke = ke + q * q;
    }
    return (S)0.5f * ke;
}

/* Gradients::*::calcConstraintContributions (charge density of phi_future, phi_now). */
static void gradient_constraint(const ctx_t* m, const S* fut, const S* now, S out[ORC_MAX_EQ])
{
    for (int k = 0; k < m->neq; k++) out[k] = (S)0;
    for (int db = 0; db < m->nsc; db += 4) {
        const S* a = now + db;
        const S* b = fut + db;
        S t0 = a[0] * b[1] - a[1] * b[0] + a[2] * b[3] - a[3] * b[2];
        S t1 = a[0] * b[3] - a[1] * b[2] + a[2] * b[1] - a[3] * b[0];
        S t2 = -a[0] * b[2] - a[1] * b[3] + a[2] * b[0] + a[3] * b[1];
        S t3 = a[0] * b[1] - a[1] * b[0] - a[2] * b[3] + a[3] * b[2];
        if (m->nsc == 4) {
            /* SM: contribution[k] = 0.25*(...) assigned (StandardModel.cpp:255-267) */
            out[0] = (S)(0.25 * (double)t0);
            out[1] = (S)(0.25 * (double)t1);
            out[2] = (S)(0.25 * (double)t2);
            out[3] = (S)(0.25 * (double)t3);
        } else {
            /* TwoHDM: accumulated over doublets (TwoHDM.cpp:333-352) */
            out[0] = (S)((double)out[0] + 0.25 * (double)t0);
            out[1] = (S)((double)out[1] + 0.25 * (double)t1);
            out[2] = (S)((double)out[2] + 0.25 * (double)t2);
            out[3] = (S)((double)out[3] + 0.25 * (double)t3);
            /* Higgs-family charges (TwoHDM.cpp:355-372), over the full 8-vectors */
            const int i = db / 2;
            const S* A = now;
            const S* B = fut;
            if (m->hf == ORC_HF_U1) {
                S h = A[i] * B[i + 1] - A[i + 1] * B[i] - A[i + 4] * B[i + 5] + A[i + 5] * B[i + 4];
                out[4] = (S)((double)out[4] + 0.25 * (double)h);
            } else if (m->hf == ORC_HF_SU2) {
                S h4 = A[i] * B[i + 5] - A[i + 1] * B[i + 4] + A[i + 4] * B[i + 1] - A[i + 5] * B[i];
                S h5 = -A[i] * B[i + 4] - A[i + 1] * B[i + 5] + A[i + 4] * B[i] + A[i + 5] * B[i + 1];
                S h6 = A[i] * B[i + 1] - A[i + 1] * B[i] - A[i + 4] * B[i + 5] + A[i + 5] * B[i + 4];
                out[4] = (S)((double)out[4] + 0.25 * (double)h4);
                out[5] = (S)((double)out[5] + 0.25 * (double)h5);
                out[6] = (S)((double)out[6] + 0.25 * (double)h6);
            }
        }
    }
}

/* ----------------------------------------------------------------------------
 * Potentials (Potentials/Source/SO_N.cpp:57-87, Double_SO_N.cpp:157-368)
 * ------------------------------------------------------------------------- */

static void potential_derivatives(const ctx_t* m, const S* f, double* P)
{
    const orc_config* c = m->cfg;
    if (m->model == ORC_MODEL_SM) {
        double fsq = 0.0;
        for (int k = 0; k < 4; k++) fsq += (double)f[k] * (double)f[k];
        for (int k = 0; k < 4; k++) P[k] = c->lambda * (fsq - c->eta_sqr) * (double)f[k];
        return;
    }
    const int n0 = 4;
    double fsq[2] = {0.0, 0.0}, dot = 0.0, anti = 0.0;
    for (int fi = 0; fi < 2; fi++) {
        fsq[fi] = 0.0;
        for (int k = 0; k < 4; k++) fsq[fi] += (double)f[fi * n0 + k] * (double)f[fi * n0 + k];
        if (c->break_son) {
            dot = 0.0;
            for (int k = 0; k < n0; k++) dot += (double)f[k] * (double)f[n0 + k];
            if (c->break_uhalfn) {
                anti = 0.0;
                for (int k = 0; k < n0 / 2; k++)
                    anti += (double)f[2 * k] * (double)f[n0 + 2 * k + 1] - (double)f[2 * k + 1] * (double)f[n0 + 2 * k];
            }
        }
    }
    for (int k = 0; k < 8; k++) P[k] = 0.0;
    for (int k = 0; k < n0; k++) {
        int k2 = n0 + k;
        P[k] += (-2.0 * c->m1 + 4.0 * c->l1 * fsq[0] + 2.0 * c->l3 * fsq[1]) * (double)f[k];
        if (c->break_son) {
            P[k] += (-c->m12r + 2.0 * c->l4p5 * dot + c->l6r * fsq[0] + c->l7r * fsq[1]) * (double)f[k2]
                  + 2.0 * c->l6r * dot * (double)f[k];
            if (c->break_uhalfn) {
                int alt = 1 - 2 * (k % 2);
                P[k] += (c->m12i + 2.0 * c->l4m5 * anti - 2.0 * c->l5i * dot - c->l6i * fsq[0] - c->l7i * fsq[1])
                            * (double)alt * (double)f[k2 + alt]
                      - 2.0 * c->l5i * anti * (double)f[k2]
                      - 2.0 * c->l6i * anti * (double)f[k];
            }
        }
    }
    for (int k = 0; k < 4; k++) {
        int k2 = n0 + k;
        P[k2] += (-2.0 * c->m2 + 4.0 * c->l2 * fsq[1] + 2.0 * c->l3 * fsq[0]) * (double)f[k2];
        if (c->break_son) {
            P[k2] += (-c->m12r + 2.0 * c->l4p5 * dot + c->l6r * fsq[0] + c->l7r * fsq[1]) * (double)f[k]
                   + 2.0 * c->l7r * dot * (double)f[k2];
            if (c->break_uhalfn) {
                int alt = 1 - 2 * (k % 2);
                P[k2] += -(c->m12i + 2.0 * c->l4m5 * anti - 2.0 * c->l5i * dot - c->l6i * fsq[0] - c->l7i * fsq[1])
                             * (double)alt * (double)f[k + alt]
                       - 2.0 * c->l5i * anti * (double)f[k]
                       - 2.0 * c->l7i * anti * (double)f[k2];
            }
        }
    }
}

static S potential_energy(const ctx_t* m, const S* f)
{
    const orc_config* c = m->cfg;
    if (m->model == ORC_MODEL_SM) {
        double fsq = 0.0;
        for (int k = 0; k < 4; k++) fsq += (double)f[k] * (double)f[k];
        /* 0.25f*lambda*powf(fsq - etaSqr, 2): the square is taken in S */
        S t = (S)(fsq - c->eta_sqr);
        return (S)(0.25 * c->lambda * (double)(S)(t * t));
    }
    double fsq[2] = {0.0, 0.0};
    for (int fi = 0; fi < 2; fi++)
        for (int k = 0; k < 4; k++) fsq[fi] += (double)f[fi * 4 + k] * (double)f[fi * 4 + k];
    double dot = 0.0, anti = 0.0;
    if (c->break_son) {
        for (int k = 0; k < 4; k++) dot += (double)f[k] * (double)f[4 + k];
        if (c->break_uhalfn)
            for (int k = 0; k < 2; k++)
                anti += (double)f[2 * k] * (double)f[4 + 2 * k + 1] - (double)f[2 * k + 1] * (double)f[4 + 2 * k];
    }
    S v = (S)(-c->m1 * fsq[0] - c->m2 * fsq[1] + c->l1 * (fsq[0] * fsq[0]) + c->l2 * (fsq[1] * fsq[1])
              + c->l3 * fsq[0] * fsq[1]);
    if (c->break_son) {
        v = (S)((double)v + (-c->m12r * dot + c->l4p5 * (dot * dot) + c->l6r * fsq[0] * dot + c->l7r * fsq[1] * dot));
        if (c->break_uhalfn)
            v = (S)((double)v + (c->m12i * anti + c->l4m5 * (anti * anti) - 2.0 * c->l5i * dot * anti
                                 - c->l6i * fsq[0] * anti - c->l7i * fsq[1] * anti));
    }
    if (c->apply_norm) v = v + (S)c->energy_offset;
    return v;
}

/* ----------------------------------------------------------------------------
 * Wilson loops (WilsonLoops/Source/StandardModel.cpp:274-514; TwoHDM.cpp with
 * gaugeNum = 4 is the same arithmetic)
 * ------------------------------------------------------------------------- */

/* calcMagneticContributions: U(1) sines and SU(2) staples per (i, j != i).
 * *mag_energy is the reference's storedMagneticEnergy (accumulated in S);
 * plaq (if non-null) receives P1_0 and cos(local) for i < j. */
static void calc_magnetic(const ctx_t* m, const stencil_t* st, double Mg[3 * ORC_MAX_EQ], S* mag_energy,
                          double* plaq_su2, double* plaq_u1)
{
    for (int k = 0; k < 3 * m->neq; k++) Mg[k] = 0.0;
    for (int i = 0; i < 3; i++) {
        int e = i * m->neq, di = i * m->dw;
        int diag = 2;
        for (int j = 0; j < 3; j++) {
            if (j == i) continue;
            int dj = j * m->dw;
            diag += 1;
            double local = -(double)st->vp[i][2][dj] + (double)st->vp[j][2][di]
                           + (double)st->vp[i][1][dj] - (double)st->vp[j][1][di];
            double neigh = -(double)st->vp[i][diag][dj] - (double)st->vp[j][0][di]
                           + (double)st->vp[j][0][dj] + (double)st->vp[i][1][di];
            Mg[e] += (sin(local) - sin(neigh)) * m->inv_sqr[j];

            double p1[4], mul[4];
            su2_rep(st->vp[j][1], di, 1, p1);
            su2_rep(st->vp[i][1], dj, 0, mul);
            su2_product(mul, p1, 1, p1);
            su2_rep(st->vp[j][2], di, 0, mul);
            su2_product(mul, p1, 1, p1);
            su2_rep(st->vp[i][2], dj, 1, mul);
            su2_product(mul, p1, m->store_energy, p1);

            double p2[4];
            su2_rep(st->vp[i][diag], dj, 1, p2);
            su2_rep(st->vp[j][0], di, 1, mul);
            su2_product(mul, p2, 1, p2);
            su2_rep(st->vp[j][0], dj, 0, mul);
            su2_product(mul, p2, 1, p2);
            su2_rep(st->vp[i][1], di, 0, mul);
            su2_product(mul, p2, 0, p2);

            for (int k = 1; k < 4; k++) Mg[e + k] += (p1[k] - p2[k]) * m->inv_sqr[j];

            if (m->store_energy) {
                *mag_energy = (S)((double)*mag_energy
                    + 2.0 * m->inv_sqr[i] * m->inv_sqr[j]
                      * (m->inv_g_sqr * (1.0 - p1[0]) + m->inv_gp_sqr * (1.0 - cos(local))));
                if (plaq_su2 && i < j) {
                    *plaq_su2 += p1[0];
                    *plaq_u1 += cos(local);
                }
            }

            /* Higgs family (WilsonLoops/Source/TwoHDM.cpp:484-551): the same loops on
             * the family U(1) phase or SU(2) quaternion, coupling g'' */
            if (m->hf == ORC_HF_U1) {
                const int o = HF_OFF;
                double hl = -(double)st->vp[i][2][dj + o] + (double)st->vp[j][2][di + o]
                            + (double)st->vp[i][1][dj + o] - (double)st->vp[j][1][di + o];
                double hn = -(double)st->vp[i][diag][dj + o] - (double)st->vp[j][0][di + o]
                            + (double)st->vp[j][0][dj + o] + (double)st->vp[i][1][di + o];
                Mg[e + 4] += (sin(hl) - sin(hn)) * m->inv_sqr[j];
                if (m->store_energy)
                    *mag_energy = (S)((double)*mag_energy
                        + 2.0 * m->inv_sqr[i] * m->inv_sqr[j] * m->inv_gpp_sqr * (1.0 - cos(hl)));
            } else if (m->hf == ORC_HF_SU2) {
                double q1[4], q2[4], mq[4];
                su2_rep_at(st->vp[j][1], di, HF_OFF, 1, q1);
                su2_rep_at(st->vp[i][1], dj, HF_OFF, 0, mq);
                su2_product(mq, q1, 1, q1);
                su2_rep_at(st->vp[j][2], di, HF_OFF, 0, mq);
                su2_product(mq, q1, 1, q1);
                su2_rep_at(st->vp[i][2], dj, HF_OFF, 1, mq);
                su2_product(mq, q1, m->store_energy, q1);
                su2_rep_at(st->vp[i][diag], dj, HF_OFF, 1, q2);
                su2_rep_at(st->vp[j][0], di, HF_OFF, 1, mq);
                su2_product(mq, q2, 1, q2);
                su2_rep_at(st->vp[j][0], dj, HF_OFF, 0, mq);
                su2_product(mq, q2, 1, q2);
                su2_rep_at(st->vp[i][1], di, HF_OFF, 0, mq);
                su2_product(mq, q2, 0, q2);
                for (int k = 4; k < 7; k++) Mg[e + k] += (q1[k - 3] - q2[k - 3]) * m->inv_sqr[j];
                if (m->store_energy)
                    *mag_energy = (S)((double)*mag_energy
                        + 2.0 * m->inv_sqr[i] * m->inv_sqr[j] * m->inv_gpp_sqr * (1.0 - q1[0]));
            }
        }
    }
}

/* calcElectricContributions: sin(theta_now - theta_past), vec(U_now U_past^dag). */
static void calc_electric(const ctx_t* m, const S* now, const S* past, double El[3 * ORC_MAX_EQ], S* elec_energy)
{
    for (int d = 0; d < 3; d++) {
        int e = d * m->neq, dd = d * m->dw;
        double ang = (double)now[dd] - (double)past[dd];
        El[e] = sin(ang);
        double up[4], mul[4];
        su2_rep(past, dd, 1, up);
        su2_rep(now, dd, 0, mul);
        su2_product(mul, up, m->store_energy, up);
        for (int k = 1; k < 4; k++) El[e + k] = up[k];
        if (m->store_energy)
            *elec_energy = (S)((double)*elec_energy
                + 4.0 * m->inv_sqr[d] * (m->inv_g_sqr * (1.0 - up[0]) + m->inv_gp_sqr * (1.0 - cos(ang))));
        /* Higgs family (TwoHDM.cpp:601-633) */
        if (m->hf == ORC_HF_U1) {
            double ha = (double)now[dd + HF_OFF] - (double)past[dd + HF_OFF];
            El[e + 4] = sin(ha);
            if (m->store_energy)
                *elec_energy = (S)((double)*elec_energy + 4.0 * m->inv_sqr[d] * m->inv_gpp_sqr * (1.0 - cos(ha)));
        } else if (m->hf == ORC_HF_SU2) {
            double hp[4], hm[4];
            su2_rep_at(past, dd, HF_OFF, 1, hp);
            su2_rep_at(now, dd, HF_OFF, 0, hm);
            su2_product(hm, hp, m->store_energy, hp);
            for (int k = 4; k < 7; k++) El[e + k] = hp[k - 3];
            if (m->store_energy)
                *elec_energy = (S)((double)*elec_energy + 4.0 * m->inv_sqr[d] * m->inv_gpp_sqr * (1.0 - hp[0]));
        }
    }
}

/* WilsonLoops::StandardModel::evolve: theta <- asin(RHS) + theta_now;
 * U <- normalise((sqrt(1 - |c|^2), c) x U_now).  Returns domain-warning bits. */
static int evolve_links(const ctx_t* m, S* past, const S* now, const double R[3 * ORC_MAX_EQ])
{
    int warn = 0;
    for (int d = 0; d < 3; d++) {
        int e = d * m->neq, dd = d * m->dw;
        past[dd] = (S)(asin(R[e]) + (double)now[dd]);
        if (R[e] * R[e] > 1) warn |= 1;
        double cm = 0.0;
        for (int k = 1; k < 4; k++) cm += R[e + k] * R[e + k];
        if (cm > 1) warn |= 2;
        double u[4] = {sqrt(1.0 - cm), R[e + 1], R[e + 2], R[e + 3]};
        double up[4];
        su2_rep(now, dd, 0, up);
        su2_product(u, up, 1, up);
        if (m->gen) {
            S w[3];
            su2_invert(up, w);
            for (int k = 0; k < 3; k++) past[dd + 1 + k] = w[k];
        } else {
            for (int k = 0; k < 4; k++) past[dd + 1 + k] = (S)up[k];
        }
        /* Higgs family (TwoHDM.cpp:702-745) */
        if (m->hf == ORC_HF_U1) {
            past[dd + HF_OFF] = (S)(asin(R[e + 4]) + (double)now[dd + HF_OFF]);
            if (R[e + 4] * R[e + 4] > 1) warn |= 1;
        } else if (m->hf == ORC_HF_SU2) {
            double hm = 0.0;
            for (int k = 4; k < 7; k++) hm += R[e + k] * R[e + k];
            if (hm > 1) warn |= 2;
            double hu[4] = {sqrt(1.0 - hm), R[e + 4], R[e + 5], R[e + 6]};
            double hq[4];
            su2_rep_at(now, dd, HF_OFF, 0, hq);
            su2_product(hu, hq, 1, hq);
            if (m->gen) {
                S w[3];
                su2_invert(hq, w);
                for (int k = 0; k < 3; k++) past[dd + HF_OFF + k] = w[k];
            } else {
                for (int k = 0; k < 4; k++) past[dd + HF_OFF + k] = (S)hq[k];
            }
        }
    }
    return warn;
}

/* WilsonLoops::*::calcConstraintContributions over both levels (now, future). */
static void loop_constraint(const ctx_t* m, const S* x_now, const S* x_fut, const S* const xm_now[3],
                            const S* const xm_fut[3], S out[ORC_MAX_EQ])
{
    for (int k = 0; k < m->neq; k++) out[k] = (S)0;
    for (int d = 0; d < 3; d++) {
        int dd = d * m->dw;
        double la = (double)x_fut[dd] - (double)x_now[dd];
        double na = (double)xm_fut[d][dd] - (double)xm_now[d][dd];
        out[0] = (S)((double)out[0] + (sin(la) - sin(na)) * m->inv_sqr[d]);
        double p1[4], mul[4], p2[4];
        su2_rep(x_fut, dd, 0, p1);
        su2_rep(x_now, dd, 1, mul);
        su2_product(mul, p1, 0, p1);
        su2_rep(xm_now[d], dd, 1, p2);
        su2_rep(xm_fut[d], dd, 0, mul);
        su2_product(mul, p2, 0, p2);
        for (int k = 1; k < 4; k++) out[k] = out[k] + (S)((p1[k] - p2[k]) * m->inv_sqr[d]);
        /* Higgs family (TwoHDM.cpp:357-392) */
        if (m->hf == ORC_HF_U1) {
            double hl = (double)x_fut[dd + HF_OFF] - (double)x_now[dd + HF_OFF];
            double hn = (double)xm_fut[d][dd + HF_OFF] - (double)xm_now[d][dd + HF_OFF];
            out[4] = (S)((double)out[4] + (sin(hl) - sin(hn)) * m->inv_sqr[d]);
        } else if (m->hf == ORC_HF_SU2) {
            double q1[4], q2[4], mq[4];
            su2_rep_at(x_fut, dd, HF_OFF, 0, q1);
            su2_rep_at(x_now, dd, HF_OFF, 1, mq);
            su2_product(mq, q1, 0, q1);
            su2_rep_at(xm_now[d], dd, HF_OFF, 1, q2);
            su2_rep_at(xm_fut[d], dd, HF_OFF, 0, mq);
            su2_product(mq, q2, 0, q2);
            for (int k = 4; k < 7; k++) out[k] = out[k] + (S)((q1[k - 3] - q2[k - 3]) * m->inv_sqr[d]);
        }
    }
}

/* ----------------------------------------------------------------------------
 * Lattice loop
 * ------------------------------------------------------------------------- */

static long long wrap(long long v, long long n) { return ((v % n) + n) % n; }

/* A site on a Fixed face: Fixed::evolve does nothing there and no analyser
 * visits it (BoundaryConditions/Source/Fixed.cpp:159-251; a region touching a
 * Fixed face is Fixed, Core/Source/Lattice.cpp:292-306). */
static int frozen(const ctx_t* m, long long x, long long y, long long z)
{
    const int f = m->cfg->fixed_axes;
    return ((f & 1) && (x == 0 || x == m->nx - 1)) || ((f & 2) && (y == 0 || y == m->ny - 1)) ||
           ((f & 4) && (z == 0 || z == m->nz - 1));
}

static long long site_index(const ctx_t* m, long long x, long long y, long long z)
{
    return (x * m->ny + y) * m->nz + z;
}

static void build_stencil(const ctx_t* m, const S* sc_now, const S* ve_now, long long x, long long y, long long z,
                          stencil_t* st)
{
    long long n[3] = {m->nx, m->ny, m->nz};
    long long p[3] = {x, y, z};
    for (int a = 0; a < 3; a++) {
        for (int s = 0; s < 3; s++) {
            long long q[3] = {p[0], p[1], p[2]};
            q[a] = wrap(q[a] + s - 1, n[a]);
            long long idx = site_index(m, q[0], q[1], q[2]);
            st->vp[a][s] = ve_now + idx * m->nv;
            st->sp[a][s] = sc_now + idx * m->nsc;
        }
        int k = 3;
        for (int j = 0; j < 3; j++) {
            if (j == a) continue;
            long long q[3] = {p[0], p[1], p[2]};
            q[a] = wrap(q[a] + 1, n[a]);
            q[j] = wrap(q[j] - 1, n[j]);
            st->vp[a][k++] = ve_now + site_index(m, q[0], q[1], q[2]) * m->nv;
        }
    }
}

/* Site order of the reference: the 26 boundary regions (Lattice.cpp:262-356,
 * BoundaryCondition.cpp:21-70; empty regions dropped) then the interior
 * (Lattice.cpp:411-438).  It fixes the order of the float running sums. */
static long long* reference_site_order(const ctx_t* m)
{
    long long* order = (long long*)malloc(sizeof(long long) * (size_t)m->nsite);
    if (!order) return NULL;
    long long n[3] = {m->nx, m->ny, m->nz};
    const long long s = 1;
    long long pos = 0;
    for (int w = 0; w < 26; w++) {
        int bv[3] = {0, 0, 0};
        int alt = -1 + 2 * (w % 2);
        int sc = w / 2;
        int salt = 1 - 2 * (sc % 2);
        if (w < 6) {
            bv[sc] = alt;
        } else if (w < 18) {
            bv[1 + w / 10] = alt;
            bv[w / 14] = salt;
        } else {
            bv[0] = -1 + 2 * (w / 22);
            bv[1] = salt;
            bv[2] = alt;
        }
        long long lo[3], hi[3];
        int empty = 0;
        for (int a = 0; a < 3; a++) {
            if (bv[a] == -1) { lo[a] = 0; hi[a] = s; }
            else if (bv[a] == 0) { lo[a] = s; hi[a] = (n[a] < 2 * s) ? s : n[a] - s; }
            else { lo[a] = (n[a] < 2 * s) ? s : n[a] - s; hi[a] = n[a]; }
            if (lo[a] >= hi[a]) empty = 1;
        }
        if (empty) continue;
        for (long long x = lo[0]; x < hi[0]; x++)
            for (long long y = lo[1]; y < hi[1]; y++)
                for (long long z = lo[2]; z < hi[2]; z++) order[pos++] = site_index(m, x, y, z);
    }
    long long ilo = s, ihi[3];
    for (int a = 0; a < 3; a++) ihi[a] = (n[a] < s) ? 0 : n[a] - s;
    for (long long x = ilo; x < ihi[0]; x++)
        for (long long y = ilo; y < ihi[1]; y++)
            for (long long z = ilo; z < ihi[2]; z++) order[pos++] = site_index(m, x, y, z);
    if (pos != m->nsite) { free(order); return NULL; }
    return order;
}

static int ctx_init(ctx_t* m, const orc_config* c)
{
    memset(m, 0, sizeof(*m));
    if (c->model != ORC_MODEL_SM && c->model != ORC_MODEL_2HDM) return -1;
    if (c->nx < 1 || c->ny < 1 || c->nz < 1) return -1;
    if (c->hf < ORC_HF_NONE || c->hf > ORC_HF_SU2 || (c->hf != ORC_HF_NONE && c->model != ORC_MODEL_2HDM)) return -1;
    m->cfg = c;
    m->model = c->model;
    m->nsc = (c->model == ORC_MODEL_SM) ? 4 : 8;
    m->hf = c->hf;
    m->gen = c->generator_rep != 0;
    m->hf_off = m->gen ? 4 : 5;
    if (m->gen)
        m->dw = (c->hf == ORC_HF_U1) ? 5 : (c->hf == ORC_HF_SU2) ? 7 : 4;
    else
        m->dw = (c->hf == ORC_HF_U1) ? 6 : (c->hf == ORC_HF_SU2) ? 9 : 5;
    g_gen = m->gen;
    g_gen_tol = c->div_tol;
    m->nv = 3 * m->dw;
    m->neq = (c->hf == ORC_HF_U1) ? 5 : (c->hf == ORC_HF_SU2) ? 7 : 4;
    m->nx = c->nx; m->ny = c->ny; m->nz = c->nz;
    m->nsite = m->nx * m->ny * m->nz;
    m->dt = c->dt;
    double sp[3] = {c->dx, c->dy, c->dz};
    for (int a = 0; a < 3; a++) {
        m->stencil[a][0] = 1.0 / (sp[a] * sp[a]);
        m->stencil[a][1] = -2.0 / (sp[a] * sp[a]);
        m->stencil[a][2] = 1.0 / (sp[a] * sp[a]);
        m->energy_stencil[a][0] = 0.0;
        m->energy_stencil[a][1] = -1.0 / sp[a];
        m->energy_stencil[a][2] = 1.0 / sp[a];
        m->inv_sqr[a] = 1.0 / (sp[a] * sp[a]);
    }
    m->inv_sqr_dt = 1.0 / (c->dt * c->dt);
    m->g_sqr = c->g * c->g;
    m->gp_sqr = c->gp * c->gp;
    m->inv_g_sqr = (m->g_sqr > c->div_tol) ? 1.0 / m->g_sqr : 0.0;
    m->inv_gp_sqr = (m->gp_sqr > c->div_tol) ? 1.0 / m->gp_sqr : 0.0;
    /* getSqrCouplings returns float in the shipped build: the coupling enters as S */
    m->gpp_sqr = c->gpp * c->gpp;
    m->inv_gpp_sqr = (m->gpp_sqr > c->div_tol) ? 1.0 / m->gpp_sqr : 0.0;
    m->gsq_coupling[0] = (double)(S)m->gp_sqr;
    for (int k = 1; k < 4; k++) m->gsq_coupling[k] = (double)(S)m->g_sqr;
    for (int k = 4; k < ORC_MAX_EQ; k++) m->gsq_coupling[k] = (double)(S)m->gpp_sqr;
    return 0;
}

/* Reference damping schedule (Model.cpp:241-254); currentDamping is a float
 * member in the shipped build. */
static double damping_step(const ctx_t* m, int time_iter)
{
    S current = (time_iter < m->cfg->nt_damped) ? (S)m->cfg->damping : (S)0;
    return 0.5 * (double)current * m->dt;
}

/*
 * Gauss-law residual of the levels (now, fut) in the reference's site order
 * (GaugeCondition.cpp:117-165 with Model.cpp:323-337): per constraint the sum
 * of |violation| in the storage type (ref_int) and in double (gint), and its
 * maximum (gmax); loc_g (may be NULL) [nsite][gaugeNum] receives the signed
 * violations rounded to float.
 */
static void gauss_pass(ctx_t* m, const long long* order, const S* sc_now, const S* sc_fut, const S* ve_now,
                       const S* ve_fut, double* loc_g, double* gint, double* gmax, S* ref_int)
{
    const long long N = m->nsite;
    const int nsc = m->nsc, NV = m->nv, neq = m->neq;
    for (long long oi = 0; oi < N; oi++) {
        long long idx = order[oi];
        long long x = idx / (m->ny * m->nz), y = (idx / m->nz) % m->ny, z = idx % m->nz;
        if (frozen(m, x, y, z)) continue;
        long long p[3] = {x, y, z}, n[3] = {m->nx, m->ny, m->nz};
        const S* xm_now[3];
        const S* xm_fut[3];
        for (int d = 0; d < 3; d++) {
            long long q[3] = {p[0], p[1], p[2]};
            q[d] = wrap(q[d] - 1, n[d]);
            long long j = site_index(m, q[0], q[1], q[2]);
            xm_now[d] = ve_now + j * NV;
            xm_fut[d] = ve_fut + j * NV;
        }
        S el[ORC_MAX_EQ], gr[ORC_MAX_EQ];
        loop_constraint(m, ve_now + idx * NV, ve_fut + idx * NV, xm_now, xm_fut, el);
        gradient_constraint(m, sc_fut + idx * nsc, sc_now + idx * nsc, gr);
        for (int k = 0; k < neq; k++) {
            S viol = el[k] - (S)m->gsq_coupling[k] * gr[k];
            if (loc_g) loc_g[idx * neq + k] = (double)(float)viol;
            S v = viol < (S)0 ? -viol : viol;
            ref_int[k] = ref_int[k] + v;
            gint[k] += (double)v;
            if ((double)v > gmax[k]) gmax[k] = (double)v;
        }
    }
}

/*
 * Evolve nsteps steps starting at time step time_iter0, in place on the
 * two-level arrays.  Energy / Gauss rows are written on steps where
 * time_iter % every == 0 (the analysers' counters, Energy.cpp:212-219,
 * GaugeCondition.cpp:220-225, with the run starting at time_iter 0).
 * Returns the number of rows written (>= 0), or < 0 on error.  *warn receives
 * the OR of domain-warning bits (1: |RHS_Y| > 1, 2: |c|^2 > 1).  loc_e [nsite][6] and
 * loc_g [nsite][gaugeNum] (either may be NULL) receive the per-site densities and
 * signed violations of the last local-output step in the run, rounded to float as
 * the reference stores them; sites it does not visit are left untouched.
 */
int FN(evolve)(const orc_config* cfg, S* scalars, S* vectors, int time_iter0, int nsteps, orc_row* rows,
               int max_rows, int* warn, double* loc_e, double* loc_g)
{
    ctx_t m;
    if (ctx_init(&m, cfg) != 0) return -1;
    long long* order = reference_site_order(&m);
    if (!order) return -2;
    const long long N = m.nsite;
    const int nsc = m.nsc, NV = m.nv, neq = m.neq;
    int nrows = 0, w = 0;

    for (int step = 0; step < nsteps; step++) {
        int time_iter = time_iter0 + step;
        int t_now = (time_iter + 1) % 2, t_past = 1 - t_now;
        int do_energy = cfg->energy_every > 0 && time_iter % cfg->energy_every == 0;
        int do_gauss = cfg->gauss_every > 0 && time_iter % cfg->gauss_every == 0;
        int local_e = cfg->energy_local_every > 0 && time_iter % cfg->energy_local_every == 0;
        int local_g = cfg->gauss_local_every > 0 && time_iter % cfg->gauss_local_every == 0;
        m.store_energy = do_energy || local_e;
        m.damping_step = damping_step(&m, time_iter);

        S* sc_now = scalars + (long long)t_now * N * nsc;
        S* sc_past = scalars + (long long)t_past * N * nsc;
        S* ve_now = vectors + (long long)t_now * N * NV;
        S* ve_past = vectors + (long long)t_past * N * NV;

        orc_row row;
        memset(&row, 0, sizeof(row));
        row.time_iter = time_iter;
        S ref_sum[6] = {0, 0, 0, 0, 0, 0};
        double dsum[6] = {0, 0, 0, 0, 0, 0};
        double plaq2 = 0.0, plaq1 = 0.0, phisq = 0.0;

        long long nevolved = 0;
        for (long long oi = 0; oi < N; oi++) {
            long long idx = order[oi];
            long long x = idx / (m.ny * m.nz), y = (idx / m.nz) % m.ny, z = idx % m.nz;
            if (frozen(&m, x, y, z)) continue;
            nevolved++;
            stencil_t st;
            build_stencil(&m, sc_now, ve_now, x, y, z, &st);
            S* s_now = sc_now + idx * nsc;
            S* s_past = sc_past + idx * nsc;
            S* v_now = ve_now + idx * NV;
            S* v_past = ve_past + idx * NV;

            double P[8], D[8], J[3 * ORC_MAX_EQ], Mg[3 * ORC_MAX_EQ], El[3 * ORC_MAX_EQ];
            potential_derivatives(&m, s_now, P);
            calc_derivatives(&m, &st, D);
            calc_currents(&m, &st, J);
            S mag_e = (S)0, elec_e = (S)0;
            double pl2 = 0.0, pl1 = 0.0;
            calc_magnetic(&m, &st, Mg, &mag_e, &pl2, &pl1);
            calc_electric(&m, v_now, v_past, El, &elec_e);

            if (do_energy || local_e) {
                S pe = potential_energy(&m, s_now);
                S ge = gradient_energy(&m, &st);
                S ke = kinetic_energy(&m, s_now, s_past);
                S me = mag_e;
                S ee = (S)(m.inv_sqr_dt * (double)elec_e);
                S tot = pe + ge + ke + me + ee;
                S dens[6] = {tot, pe, ge, ke, me, ee};
                if (local_e && loc_e)
                    for (int k = 0; k < 6; k++) loc_e[idx * 6 + k] = (double)(float)dens[k];
                for (int k = 0; k < 6; k++) {
                    ref_sum[k] = ref_sum[k] + dens[k];
                    dsum[k] += (double)dens[k];
                }
                plaq2 += pl2;
                plaq1 += pl1;
                double fs = 0.0;
                for (int c = 0; c < nsc; c++) fs += (double)s_now[c] * (double)s_now[c];
                phisq += fs;
            }

            /* Model::evolve (Model.cpp:339-373) */
            for (int c = 0; c < nsc; c++) {
                double rhs = m.dt * m.dt * (D[c] - P[c])
                           - m.damping_step * ((double)s_now[c] - (double)s_past[c]);
                s_past[c] = (S)(2 * (double)s_now[c] - (double)s_past[c] + rhs);
            }
            double R[3 * ORC_MAX_EQ];
            for (int k = 0; k < 3 * neq; k++)
                R[k] = (1.0 - m.damping_step) * El[k] + m.dt * m.dt * (Mg[k] + m.gsq_coupling[k % neq] * J[k]);
            w |= evolve_links(&m, v_past, v_now, R);
        }

        if (do_energy) {
            double dv = cfg->dx * cfg->dy * cfg->dz;
            row.has_energy = 1;
            row.energy = dsum[0] * dv;
            row.potential = dsum[1] * dv;
            row.gradient = dsum[2] * dv;
            row.kinetic = dsum[3] * dv;
            row.magnetic = dsum[4] * dv;
            row.electric = dsum[5] * dv;
            for (int k = 0; k < 6; k++) row.ref_energy[k] = (double)ref_sum[k];
            const double ne = nevolved > 0 ? (double)nevolved : 1.0;
            row.plaq_su2 = plaq2 / (3.0 * ne);
            row.plaq_u1 = plaq1 / (3.0 * ne);
            row.phi_sq = phisq / ne;
        }

        if (do_gauss || local_g) {
            /* post-evolve: the past slot now holds t + dt (Lattice.cpp:441-541) */
            S ref_int[ORC_MAX_EQ] = {0};
            double gint[ORC_MAX_EQ] = {0}, gmax[ORC_MAX_EQ] = {0};
            gauss_pass(&m, order, sc_now, sc_past, ve_now, ve_past, local_g ? loc_g : NULL, gint, gmax, ref_int);
            double dv = cfg->dx * cfg->dy * cfg->dz;
            row.has_gauss = do_gauss;
            for (int k = 0; k < neq && do_gauss; k++) {
                row.gauss_int[k] = gint[k] * dv;
                row.gauss_max[k] = gmax[k];
                row.ref_gauss_int[k] = (double)ref_int[k];
            }
        }

        if ((do_energy || do_gauss) && rows && nrows < max_rows) rows[nrows] = row;
        if (do_energy || do_gauss) nrows++;
    }
    free(order);
    if (warn) *warn = w;
    return nrows;
}

/*
 * The Gauss row of the two levels as they stand after step time_iter (the
 * past slot of that step holding t + dt), computed as the post-evolve analyser
 * of FN(evolve) computes it, without stepping: gauss_int[k] (times the cell
 * volume) and gauss_max[k] for the gaugeNum constraints; loc_g as in FN(evolve)
 * (may be NULL).  Returns 0, or < 0 on error.
 */
int FN(gauss)(const orc_config* cfg, const S* scalars, const S* vectors, int time_iter, double* gauss_int,
              double* gauss_max, double* loc_g)
{
    ctx_t m;
    if (ctx_init(&m, cfg) != 0) return -1;
    long long* order = reference_site_order(&m);
    if (!order) return -2;
    const long long N = m.nsite;
    const int t_now = (time_iter + 1) % 2, t_past = 1 - t_now;
    S ref_int[ORC_MAX_EQ] = {0};
    double gint[ORC_MAX_EQ] = {0}, gmax[ORC_MAX_EQ] = {0};
    gauss_pass(&m, order, scalars + (long long)t_now * N * m.nsc, scalars + (long long)t_past * N * m.nsc,
               vectors + (long long)t_now * N * m.nv, vectors + (long long)t_past * N * m.nv, loc_g, gint, gmax,
               ref_int);
    const double dv = cfg->dx * cfg->dy * cfg->dz;
    for (int k = 0; k < m.neq; k++) {
        gauss_int[k] = gint[k] * dv;
        gauss_max[k] = gmax[k];
    }
    free(order);
    return 0;
}

/* ----------------------------------------------------------------------------
 * Initial conditions (no reference counterpart: the reference ships only
 * RandomUniform, InitialConditions/Source/RandomUniform.cpp:60-77).
 *
 * Counter-based generator: u(seed, stream, i) = ((mix64(seed, stream, i) >> 11) + 0.5) * 2^-53
 * with the SplitMix64 finaliser; Gaussian variate i of a stream from the
 * Box-Muller cosine branch of u(2i), u(2i+1).  The CUDA generator restates
 * the same algorithm; stream ids are fixed per field component.
 * ------------------------------------------------------------------------- */

static uint64_t mix64(uint64_t z)
{
    z += 0x9E3779B97F4A7C15ULL;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

static double uniform01(uint64_t seed, uint64_t stream, uint64_t i)
{
    uint64_t h = mix64(mix64(seed ^ (stream * 0xD1B54A32D192ED03ULL)) + i);
    return ((double)(h >> 11) + 0.5) * (1.0 / 9007199254740992.0);
}

static double gaussian(uint64_t seed, uint64_t stream, uint64_t i)
{
    const double two_pi = 6.283185307179586476925286766559;
    double u1 = uniform01(seed, stream, 2 * i), u2 = uniform01(seed, stream, 2 * i + 1);
    return sqrt(-2.0 * log(u1)) * cos(two_pi * u2);
}

/* Stream ids: scalars 0..7 (component c), theta_Y of direction d: 16 + d,
 * SU(2) angle eps: 32 + d, axis cos(polar): 48 + d, axis azimuth: 64 + d;
 * Higgs-family U(1) phase: 80 + d; Higgs-family SU(2): 96 + d, 112 + d, 128 + d
 * (eps, cos polar, azimuth). */
#define ORC_STREAM_SCALAR(c) (0 + (c))
#define ORC_STREAM_THETA(d) (16 + (d))
#define ORC_STREAM_EPS(d) (32 + (d))
#define ORC_STREAM_COSPOLAR(d) (48 + (d))
#define ORC_STREAM_AZIMUTH(d) (64 + (d))
#define ORC_STREAM_HF_THETA(d) (80 + (d))
#define ORC_STREAM_HF_EPS(d) (96 + (d))
#define ORC_STREAM_HF_COSPOLAR(d) (112 + (d))
#define ORC_STREAM_HF_AZIMUTH(d) (128 + (d))

/* Random unit quaternion q[0..3] = (cos eps, sin eps n), eps ~ N(0, eps_sigma^2), n uniform
 * on S^2, and its generators q[4..6] = eps n. */
static void random_link(uint64_t seed, int s_eps, int s_cos, int s_az, uint64_t i, double eps_sigma, double q[7])
{
    const double two_pi = 6.283185307179586476925286766559;
    q[0] = 1.0;
    q[1] = q[2] = q[3] = 0.0;
    q[4] = q[5] = q[6] = 0.0;
    if (eps_sigma > 0.0) {
        double eps = eps_sigma * gaussian(seed, (uint64_t)s_eps, i);
        double ct = 2.0 * uniform01(seed, (uint64_t)s_cos, i) - 1.0;
        double st = sqrt(1.0 - ct * ct);
        double ph = two_pi * uniform01(seed, (uint64_t)s_az, i);
        double se = sin(eps);
        q[0] = cos(eps);
        q[1] = se * st * cos(ph);
        q[2] = se * st * sin(ph);
        q[3] = se * ct;
        q[4] = eps * st * cos(ph);
        q[5] = eps * st * sin(ph);
        q[6] = eps * ct;
    }
}

/*
 * Fill both time levels (E = 0, pi = 0).  Scalars: component c ~ N(mean[c], sigma[c]^2)
 * (+ wall profile on component 0 when wall_width > 0).  Links: theta_Y ~ N(0, theta_sigma^2);
 * SU(2) = (cos eps, sin eps n) with eps ~ N(0, eps_sigma^2), n uniform on S^2; identity when
 * eps_sigma == 0 and theta_sigma == 0.  hf: a Higgs-family phase ~ N(0, theta_sigma^2)
 * (ORC_HF_U1) or quaternion drawn like the SU(2) link (ORC_HF_SU2).  gen: links stored
 * as generators, w = eps n (the same group element).
 */
void FN(init_fields)(int nx, int ny, int nz, int nsc, int hf, int gen, S* scalars, S* vectors,
                     unsigned long long seed, const double* mean, const double* sigma, double theta_sigma,
                     double eps_sigma, double wall_width, double wall_value)
{
    long long N = (long long)nx * ny * nz;
    const int dw = (gen ? 4 : 5) + (hf == ORC_HF_U1 ? 1 : (hf == ORC_HF_SU2 ? (gen ? 3 : 4) : 0));
    const int off = gen ? 4 : 5;
    const int NV = 3 * dw;
    for (long long i = 0; i < N; i++) {
        long long z = i % nz;
        for (int c = 0; c < nsc; c++) {
            double v = mean[c] + sigma[c] * gaussian(seed, ORC_STREAM_SCALAR(c), (uint64_t)i);
            if (c == 0 && wall_width > 0.0) {
                double zz = (double)z;
                v += wall_value * 0.5 * (tanh((zz - 0.25 * nz) / wall_width) - tanh((zz - 0.75 * nz) / wall_width));
            }
            scalars[i * nsc + c] = (S)v;
            scalars[(N + i) * nsc + c] = (S)v;
        }
        for (int d = 0; d < 3; d++) {
            double th = theta_sigma * gaussian(seed, ORC_STREAM_THETA(d), (uint64_t)i);
            double q[7];
            random_link(seed, ORC_STREAM_EPS(d), ORC_STREAM_COSPOLAR(d), ORC_STREAM_AZIMUTH(d), (uint64_t)i, eps_sigma, q);
            S* v0 = vectors + i * NV + d * dw;
            S* v1 = vectors + (N + i) * NV + d * dw;
            v0[0] = v1[0] = (S)th;
            if (gen)
                for (int k = 0; k < 3; k++) v0[1 + k] = v1[1 + k] = (S)q[4 + k];
            else
                for (int k = 0; k < 4; k++) v0[1 + k] = v1[1 + k] = (S)q[k];
            if (hf == ORC_HF_U1) {
                double hth = theta_sigma * gaussian(seed, ORC_STREAM_HF_THETA(d), (uint64_t)i);
                v0[off] = v1[off] = (S)hth;
            } else if (hf == ORC_HF_SU2) {
                double hq[7];
                random_link(seed, ORC_STREAM_HF_EPS(d), ORC_STREAM_HF_COSPOLAR(d), ORC_STREAM_HF_AZIMUTH(d),
                            (uint64_t)i, eps_sigma, hq);
                if (gen)
                    for (int k = 0; k < 3; k++) v0[off + k] = v1[off + k] = (S)hq[4 + k];
                else
                    for (int k = 0; k < 4; k++) v0[off + k] = v1[off + k] = (S)hq[k];
            }
        }
    }
}

int FN(storage_bytes)(void) { return (int)sizeof(S); }
