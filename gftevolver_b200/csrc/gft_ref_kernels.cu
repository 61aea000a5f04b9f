// gft_ref_kernels.cu -- the "reference arithmetic" form (GFT_FORM_REF).
//
// Every per-site quantity is evaluated in FP64 in the same operation order as
// the reference (GFTEvolver), values the reference keeps in `float` containers
// are kept in the storage type S, and this file is compiled with -fmad=false
// so that no multiply-add is contracted.  With S = float this is the reference
// exactly as shipped; with S = double it is the reference with FP64 storage.
// Results then differ from the reference only where CUDA's sin/cos/asin differ
// from the host libm in the last bit.
//
// One thread per site; each writes only its own site of the past level
// (Jacobi update in place, Core/Source/Lattice.cpp:773-841).
#include "gft_device.cuh"
#include "gft_launch.h"

namespace gft {
namespace {

template <class S>
struct RefView {
    const LevelPtrs<S>& L;
    bool gen;    // links stored as generators (w1, w2, w3, unused)
    double tol;  // divisionByZeroTolerance
    __device__ double th(int d, int s) const { return (double)L.th[d][s]; }
    // getSU2Representation (WilsonLoops/Source/StandardModel.cpp:76-112)
    __device__ void rep(int d, int s, bool conj, double c[4]) const { rep_of(L.q[d], s, conj, c); }
    // the same for the Higgs-family field (TwoHDM.cpp:94-126, 362-368)
    __device__ double hth(int d, int s) const { return (double)L.hth[d][s]; }
    __device__ void hrep(int d, int s, bool conj, double c[4]) const { rep_of(L.hq[d], s, conj, c); }
    __device__ void rep_of(const S* a, int s, bool conj, double c[4]) const
    {
        const S* p = a + 4 * (size_t)s;
        if (gen) {
            // generator branch: c0 = cos|w|, c_a = conj * sin|w| * w_a / |w| (c1 = sin|w| when |w| <= tol)
            double wm = 0.0;
            wm += (double)p[0] * (double)p[0];
            wm += (double)p[1] * (double)p[1];
            wm += (double)p[2] * (double)p[2];
            wm = sqrt(wm);
            c[0] = cos(wm);
            c[1] = c[2] = c[3] = 0.0;
            if (wm > tol) {
                const double cs = (double)(conj ? -1 : 1) * sin(wm);
                for (int k = 1; k < 4; k++) c[k] = cs * (double)p[k - 1] / wm;
            } else {
                c[1] = sin(wm);
            }
            return;
        }
        c[0] = (double)p[0];
        for (int k = 1; k < 4; k++) c[k] = conj ? -(double)p[k] : (double)p[k];
    }
    // Store a link: the quaternion, or (generator representation) invertSU2Representation
    // (WilsonLoops/Source/StandardModel.cpp:114-158): phase = asin|c| (pi/2 when |c| > 1),
    // pi - phase when c0 < 0, w = phase * c / |c| (w1 = phase when |c| <= tol).
    __device__ void store(S* a, int s, const double c[4], bool& finite) const
    {
        S o[4];
        if (gen) {
            double cm = 0.0;
            cm += c[1] * c[1];
            cm += c[2] * c[2];
            cm += c[3] * c[3];
            cm = sqrt(cm);
            double phase = (cm > 1) ? 1.5707963267948966 : asin(cm);
            if (c[0] < 0) phase = 3.141592653589793 - phase;
            if (cm > tol) {
                for (int k = 0; k < 3; k++) o[k] = (S)(phase * c[k + 1] / cm);
            } else {
                o[0] = (S)phase;
                o[1] = o[2] = (S)0;
            }
            o[3] = (S)0;
        } else {
            for (int k = 0; k < 4; k++) o[k] = (S)c[k];
        }
        st4(a, s, o[0], o[1], o[2], o[3]);
        for (int k = 0; k < 4; k++) finite = finite && isfinite((double)o[k]);
    }
};

// SU2Product (WilsonLoops/Source/StandardModel.cpp:160-191).
__device__ __forceinline__ void ref_su2_product(const double a[4], const double b[4], bool calc_trace, double out[4])
{
    double p0 = 0.0;
    double p1 = a[0] * b[1] + a[1] * b[0] - a[2] * b[3] + a[3] * b[2];
    double p2 = a[0] * b[2] + a[2] * b[0] - a[3] * b[1] + a[1] * b[3];
    double p3 = a[0] * b[3] + a[3] * b[0] - a[1] * b[2] + a[2] * b[1];
    if (calc_trace) {
        double dot = 0.0;
        dot += a[1] * b[1];
        dot += a[2] * b[2];
        dot += a[3] * b[3];
        p0 = a[0] * b[0] - dot;
        double norm = sqrt(p0 * p0 + p1 * p1 + p2 * p2 + p3 * p3);
        p0 = p0 / norm;
        p1 = p1 / norm;
        p2 = p2 / norm;
        p3 = p3 / norm;
    }
    out[0] = p0;
    out[1] = p1;
    out[2] = p2;
    out[3] = p3;
}

// Gradients::StandardModel::transform / TwoHDM::transform
// (Gradients/Source/StandardModel.cpp:72-100, TwoHDM.cpp:72-149): hypercharge
// phase, isospin SU(2), then the Higgs-family U(1) (+theta_H on doublet 1,
// -theta_H on doublet 2) or SU(2) (acting on doublet-1 / doublet-2 pairs).
template <int NSC, class S>
__device__ __forceinline__ void ref_transform_sm(const double* in, const RefView<S>& V, int d, int s, bool conj,
                                                 double* out);

template <int NSC, int HF, class S>
__device__ __forceinline__ void ref_transform(const double* in, const RefView<S>& V, int d, int s, bool conj,
                                              double* out)
{
    if (HF == kHfNone) {
        ref_transform_sm<NSC>(in, V, d, s, conj, out);
        return;
    }
    double sm[8];
    ref_transform_sm<8>(in, V, d, s, conj, sm);
    const int conj_fac = conj ? -1 : 1;
    if (HF == kHfU1) {
        const double th = V.hth(d, s);
#pragma unroll
        for (int c = 0; c < 8; c++) {
            const int pm = -1 + 2 * (c % 2);
            const int pm4 = 1 - 2 * (c / 4);
            out[c] = cos(th) * sm[c] + (double)pm * sin((double)(pm4 * conj_fac) * th) * sm[c - pm];
        }
    } else {
        double u[4];
        V.hrep(d, s, conj, u);
#pragma unroll
        for (int inner = 0; inner < 2; inner++) {
            const int i = inner * 2;
            out[i] = u[0] * sm[i] - u[3] * sm[i + 1] + u[2] * sm[i + 4] - u[1] * sm[i + 5];
            out[i + 1] = u[3] * sm[i] + u[0] * sm[i + 1] + u[1] * sm[i + 4] + u[2] * sm[i + 5];
            out[i + 4] = -u[2] * sm[i] - u[1] * sm[i + 1] + u[0] * sm[i + 4] + u[3] * sm[i + 5];
            out[i + 5] = u[1] * sm[i] - u[2] * sm[i + 1] - u[3] * sm[i + 4] + u[0] * sm[i + 5];
        }
    }
}

template <int NSC, class S>
__device__ __forceinline__ void ref_transform_sm(const double* in, const RefView<S>& V, int d, int s, bool conj,
                                                 double* out)
{
    const double th = V.th(d, s);
    const double sn = sin((conj ? -1.0 : 1.0) * th);
    const double cs = cos(th);
    double h[NSC];
#pragma unroll
    for (int c = 0; c < NSC; c++) {
        const int pm = -1 + 2 * (c % 2);
        h[c] = cs * in[c] + ((double)pm * sn) * in[c - pm];
    }
    double u[4];
    V.rep(d, s, conj, u);
#pragma unroll
    for (int db = 0; db < NSC; db += 4) {
        const double* g = h + db;
        out[db + 0] = u[0] * g[0] - u[3] * g[1] + u[2] * g[2] - u[1] * g[3];
        out[db + 1] = u[3] * g[0] + u[0] * g[1] + u[1] * g[2] + u[2] * g[3];
        out[db + 2] = -u[2] * g[0] - u[1] * g[1] + u[0] * g[2] + u[3] * g[3];
        out[db + 3] = u[1] * g[0] - u[2] * g[1] - u[3] * g[2] + u[0] * g[3];
    }
}

template <int NSC, class S>
__device__ __forceinline__ void ref_load_scalar(const LevelPtrs<S>& L, int s, double* f)
{
#pragma unroll
    for (int db = 0; db < NSC / 4; db++) {
        const S* p = L.ph[db] + 4 * (size_t)s;
#pragma unroll
        for (int k = 0; k < 4; k++) f[4 * db + k] = (double)p[k];
    }
}

template <int NSC, class S>
__device__ __forceinline__ void ref_load_scalar_S(const LevelPtrs<S>& L, int s, S* f)
{
#pragma unroll
    for (int db = 0; db < NSC / 4; db++) {
        const S* p = L.ph[db] + 4 * (size_t)s;
#pragma unroll
        for (int k = 0; k < 4; k++) f[4 * db + k] = p[k];
    }
}

// SO_N::calcPotentialDerivatives / Double_SO_N::calcPotentialDerivatives
// (Potentials/Source/SO_N.cpp:57-75, Double_SO_N.cpp:244-341).
template <int MODEL, class S>
__device__ __forceinline__ void ref_potential_derivs(const StepParams& P, const S* f, double* out)
{
    if (MODEL == kModelSM) {
        double fsq = 0.0;
#pragma unroll
        for (int k = 0; k < 4; k++) fsq += (double)f[k] * (double)f[k];
#pragma unroll
        for (int k = 0; k < 4; k++) out[k] = P.lambda * (fsq - P.eta_sqr) * (double)f[k];
    } else {
        double fsq0 = 0.0, fsq1 = 0.0, dot = 0.0, anti = 0.0;
#pragma unroll
        for (int k = 0; k < 4; k++) fsq0 += (double)f[k] * (double)f[k];
#pragma unroll
        for (int k = 0; k < 4; k++) fsq1 += (double)f[4 + k] * (double)f[4 + k];
        if (P.break_son) {
#pragma unroll
            for (int k = 0; k < 4; k++) dot += (double)f[k] * (double)f[4 + k];
            if (P.break_uhalfn) {
#pragma unroll
                for (int k = 0; k < 2; k++)
                    anti += (double)f[2 * k] * (double)f[4 + 2 * k + 1] - (double)f[2 * k + 1] * (double)f[4 + 2 * k];
            }
        }
#pragma unroll
        for (int k = 0; k < 4; k++) {
            const int k2 = 4 + k;
            double v = 0.0;
            v += (-2.0 * P.m1 + 4.0 * P.l1 * fsq0 + 2.0 * P.l3 * fsq1) * (double)f[k];
            if (P.break_son) {
                v += (-P.m12r + 2.0 * P.l4p5 * dot + P.l6r * fsq0 + P.l7r * fsq1) * (double)f[k2]
                     + 2.0 * P.l6r * dot * (double)f[k];
                if (P.break_uhalfn) {
                    const int alt = 1 - 2 * (k % 2);
                    v += (P.m12i + 2.0 * P.l4m5 * anti - 2.0 * P.l5i * dot - P.l6i * fsq0 - P.l7i * fsq1)
                             * (double)alt * (double)f[k2 + alt]
                         - 2.0 * P.l5i * anti * (double)f[k2] - 2.0 * P.l6i * anti * (double)f[k];
                }
            }
            out[k] = v;
        }
#pragma unroll
        for (int k = 0; k < 4; k++) {
            const int k2 = 4 + k;
            double v = 0.0;
            v += (-2.0 * P.m2 + 4.0 * P.l2 * fsq1 + 2.0 * P.l3 * fsq0) * (double)f[k2];
            if (P.break_son) {
                v += (-P.m12r + 2.0 * P.l4p5 * dot + P.l6r * fsq0 + P.l7r * fsq1) * (double)f[k]
                     + 2.0 * P.l7r * dot * (double)f[k2];
                if (P.break_uhalfn) {
                    const int alt = 1 - 2 * (k % 2);
                    v += -(P.m12i + 2.0 * P.l4m5 * anti - 2.0 * P.l5i * dot - P.l6i * fsq0 - P.l7i * fsq1)
                             * (double)alt * (double)f[k + alt]
                         - 2.0 * P.l5i * anti * (double)f[k] - 2.0 * P.l7i * anti * (double)f[k2];
                }
            }
            out[k2] = v;
        }
    }
}

// SO_N::calcPotentialEnergy / Double_SO_N::calcPotentialEnergy, value in S.
template <int MODEL, class S>
__device__ __forceinline__ S ref_potential_energy(const StepParams& P, const S* f)
{
    if (MODEL == kModelSM) {
        double fsq = 0.0;
#pragma unroll
        for (int k = 0; k < 4; k++) fsq += (double)f[k] * (double)f[k];
        const S t = (S)(fsq - P.eta_sqr);
        const S t2 = t * t;
        return (S)(0.25 * P.lambda * (double)t2);
    } else {
        double fsq0 = 0.0, fsq1 = 0.0, dot = 0.0, anti = 0.0;
#pragma unroll
        for (int k = 0; k < 4; k++) fsq0 += (double)f[k] * (double)f[k];
#pragma unroll
        for (int k = 0; k < 4; k++) fsq1 += (double)f[4 + k] * (double)f[4 + k];
        if (P.break_son) {
#pragma unroll
            for (int k = 0; k < 4; k++) dot += (double)f[k] * (double)f[4 + k];
            if (P.break_uhalfn) {
#pragma unroll
                for (int k = 0; k < 2; k++)
                    anti += (double)f[2 * k] * (double)f[4 + 2 * k + 1] - (double)f[2 * k + 1] * (double)f[4 + 2 * k];
            }
        }
        S v = (S)(-P.m1 * fsq0 - P.m2 * fsq1 + P.l1 * (fsq0 * fsq0) + P.l2 * (fsq1 * fsq1) + P.l3 * fsq0 * fsq1);
        if (P.break_son) {
            v = (S)((double)v + (-P.m12r * dot + P.l4p5 * (dot * dot) + P.l6r * fsq0 * dot + P.l7r * fsq1 * dot));
            if (P.break_uhalfn)
                v = (S)((double)v + (P.m12i * anti + P.l4m5 * (anti * anti) - 2.0 * P.l5i * dot * anti
                                     - P.l6i * fsq0 * anti - P.l7i * fsq1 * anti));
        }
        if (P.apply_norm) v = v + (S)P.energy_offset;
        return v;
    }
}

template <class S, int MODEL, int HF, bool ENERGY>
__global__ void __launch_bounds__(128) ref_step_kernel(StepParams P, LevelPtrs<S> now, LevelPtrs<S> past,
                                                       unsigned* status, double* partials)
{
    constexpr int NSC = (MODEL == kModelSM) ? 4 : 8;
    constexpr int NEQ = hf_neq(HF);  // gauge equations per direction
    const int z = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    const int x = blockIdx.z;
    const bool active = (z < P.nz) && (y < P.ny) && !frozen(P, x, y, z);  // Fixed faces: not evolved
    double obs[kObsCount];
#pragma unroll
    for (int k = 0; k < kObsCount; k++) obs[k] = 0.0;
    unsigned warn = 0;

    if (active) {
        const Nbr n = neighbours(P, x, y, z);
        const RefView<S> V{now, P.gen != 0, P.div_tol};
        const RefView<S> Vp{past, P.gen != 0, P.div_tol};
        const bool store = ENERGY;

        // ---- potential (Model::calcPotentialContributions) ----
        S f_now[NSC], f_past[NSC];
        ref_load_scalar_S<NSC>(now, n.c, f_now);
        ref_load_scalar_S<NSC>(past, n.c, f_past);
        double Pot[NSC];
        ref_potential_derivs<MODEL>(P, f_now, Pot);

        // ---- calcDerivatives (Gradients/Source/StandardModel.cpp:272-320) ----
        double D[NSC];
#pragma unroll
        for (int c = 0; c < NSC; c++) D[c] = 0.0;
        for (int st = 0; st < 3; st++) {
            for (int a = 0; a < 3; a++) {
                double f[NSC], t[NSC];
                const int s = (st == 0) ? n.m[a] : (st == 1 ? n.c : n.p[a]);
                ref_load_scalar<NSC>(now, s, f);
                const double w = (st == 1) ? -2.0 * P.lap[a] : P.lap[a];
                if (st == 0) {
                    ref_transform<NSC, HF>(f, V, a, n.m[a], false, t);
                } else if (st == 2) {
                    ref_transform<NSC, HF>(f, V, a, n.c, true, t);
                } else {
#pragma unroll
                    for (int c = 0; c < NSC; c++) t[c] = f[c];
                }
#pragma unroll
                for (int c = 0; c < NSC; c++) D[c] += w * t[c];
            }
        }

        // ---- calcCurrents (:323-363) and, on energy steps, calcGradientEnergy (:192-235) ----
        double J[3 * NEQ];
        S der[3 * NSC];
        for (int a = 0; a < 3; a++) {
            double f[NSC], t[NSC], nb[NSC];
            ref_load_scalar<NSC>(now, n.c, f);
            ref_transform<NSC, HF>(f, V, a, n.c, false, t);
            ref_load_scalar<NSC>(now, n.p[a], nb);
            double jj[NEQ];
#pragma unroll
            for (int k = 0; k < NEQ; k++) jj[k] = 0.0;
#pragma unroll
            for (int db = 0; db < NSC; db += 4) {
                const double* p = t + db;
                const double* q = nb + db;
                jj[0] += 0.25 * (p[0] * q[1] - p[1] * q[0] + p[2] * q[3] - p[3] * q[2]);
                jj[1] += 0.25 * (p[0] * q[3] - p[1] * q[2] + p[2] * q[1] - p[3] * q[0]);
                jj[2] += 0.25 * (-p[0] * q[2] - p[1] * q[3] + p[2] * q[0] + p[3] * q[1]);
                jj[3] += 0.25 * (p[0] * q[1] - p[1] * q[0] - p[2] * q[3] + p[3] * q[2]);
                // Higgs-family currents (Gradients/Source/TwoHDM.cpp:465-485), i = upper or lower pair
                const int i = db / 2;
                if (HF == kHfU1) {
                    jj[4 % NEQ] += 0.25 * (t[i] * nb[i + 1] - t[i + 1] * nb[i] - t[i + 4] * nb[i + 5] + t[i + 5] * nb[i + 4]);
                } else if (HF == kHfSU2) {
                    jj[4 % NEQ] += 0.25 * (t[i] * nb[i + 5] - t[i + 1] * nb[i + 4] + t[i + 4] * nb[i + 1] - t[i + 5] * nb[i]);
                    jj[5 % NEQ] += 0.25 * (-t[i] * nb[i + 4] - t[i + 1] * nb[i + 5] + t[i + 4] * nb[i] + t[i + 5] * nb[i + 1]);
                    jj[6 % NEQ] += 0.25 * (t[i] * nb[i + 1] - t[i + 1] * nb[i] - t[i + 4] * nb[i + 5] + t[i + 5] * nb[i + 4]);
                }
            }
#pragma unroll
            for (int k = 0; k < NEQ; k++) J[NEQ * a + k] = jj[k];
            if (ENERGY) {
                // stencil_iter 1 (-1/dx * U phi(x)) then stencil_iter 2 (+1/dx * phi(x+a)), accumulated in S
#pragma unroll
                for (int c = 0; c < NSC; c++) der[a * NSC + c] = (S)0;
#pragma unroll
                for (int c = 0; c < NSC; c++) der[a * NSC + c] = (S)((double)der[a * NSC + c] + (-P.inv_dx[a]) * t[c]);
            }
        }
        S grad_e = (S)0;
        if (ENERGY) {
            // the reference loops stencil_iter outer, axis inner; each entry sees -U phi then +phi(x+a)
            for (int a = 0; a < 3; a++) {
                double nb[NSC];
                ref_load_scalar<NSC>(now, n.p[a], nb);
#pragma unroll
                for (int c = 0; c < NSC; c++) der[a * NSC + c] = (S)((double)der[a * NSC + c] + P.inv_dx[a] * nb[c]);
            }
#pragma unroll
            for (int k = 0; k < 3 * NSC; k++) grad_e = (S)((double)grad_e + (double)der[k] * (double)der[k]);
            grad_e = (S)0.5f * grad_e;
        }

        // ---- calcMagneticContributions (WilsonLoops/Source/StandardModel.cpp:324-409) ----
        double Mg[3 * NEQ];
#pragma unroll
        for (int k = 0; k < 3 * NEQ; k++) Mg[k] = 0.0;
        S mag_e = (S)0;
        double plaq2 = 0.0, plaq1 = 0.0;
        for (int i = 0; i < 3; i++) {
            for (int j = 0; j < 3; j++) {
                if (j == i) continue;
                const int di = n.dg[i][j];
                const double local = -V.th(j, n.p[i]) + V.th(i, n.p[j]) + V.th(j, n.c) - V.th(i, n.c);
                const double neigh = -V.th(j, di) - V.th(i, n.m[j]) + V.th(j, n.m[j]) + V.th(i, n.c);
                Mg[NEQ * i] += (sin(local) - sin(neigh)) * P.lap[j];

                double p1[4], mul[4];
                V.rep(i, n.c, true, p1);
                V.rep(j, n.c, false, mul);
                ref_su2_product(mul, p1, true, p1);
                V.rep(i, n.p[j], false, mul);
                ref_su2_product(mul, p1, true, p1);
                V.rep(j, n.p[i], true, mul);
                ref_su2_product(mul, p1, store, p1);

                double p2[4];
                V.rep(j, di, true, p2);
                V.rep(i, n.m[j], true, mul);
                ref_su2_product(mul, p2, true, p2);
                V.rep(j, n.m[j], false, mul);
                ref_su2_product(mul, p2, true, p2);
                V.rep(i, n.c, false, mul);
                ref_su2_product(mul, p2, false, p2);

#pragma unroll
                for (int k = 1; k < 4; k++) Mg[NEQ * i + k] += (p1[k] - p2[k]) * P.lap[j];

                if (ENERGY) {
                    const double cl = cos(local);
                    mag_e = (S)((double)mag_e + 2.0 * P.lap[i] * P.lap[j]
                                                   * (P.inv_g_sqr * (1.0 - p1[0]) + P.inv_gp_sqr * (1.0 - cl)));
                    if (i < j) {
                        plaq2 += p1[0];
                        plaq1 += cl;
                    }
                }

                // Higgs family (WilsonLoops/Source/TwoHDM.cpp:484-551)
                if (HF == kHfU1) {
                    const double hl = -V.hth(j, n.p[i]) + V.hth(i, n.p[j]) + V.hth(j, n.c) - V.hth(i, n.c);
                    const double hn = -V.hth(j, di) - V.hth(i, n.m[j]) + V.hth(j, n.m[j]) + V.hth(i, n.c);
                    Mg[NEQ * i + 4 % NEQ] += (sin(hl) - sin(hn)) * P.lap[j];
                    if (ENERGY)
                        mag_e = (S)((double)mag_e + 2.0 * P.lap[i] * P.lap[j] * P.inv_gpp_sqr * (1.0 - cos(hl)));
                } else if (HF == kHfSU2) {
                    double q1[4], q2[4], mq[4];
                    V.hrep(i, n.c, true, q1);
                    V.hrep(j, n.c, false, mq);
                    ref_su2_product(mq, q1, true, q1);
                    V.hrep(i, n.p[j], false, mq);
                    ref_su2_product(mq, q1, true, q1);
                    V.hrep(j, n.p[i], true, mq);
                    ref_su2_product(mq, q1, store, q1);
                    V.hrep(j, di, true, q2);
                    V.hrep(i, n.m[j], true, mq);
                    ref_su2_product(mq, q2, true, q2);
                    V.hrep(j, n.m[j], false, mq);
                    ref_su2_product(mq, q2, true, q2);
                    V.hrep(i, n.c, false, mq);
                    ref_su2_product(mq, q2, false, q2);
#pragma unroll
                    for (int k = 4; k < 7; k++) Mg[NEQ * i + k % NEQ] += (q1[k - 3] - q2[k - 3]) * P.lap[j];
                    if (ENERGY)
                        mag_e = (S)((double)mag_e + 2.0 * P.lap[i] * P.lap[j] * P.inv_gpp_sqr * (1.0 - q1[0]));
                }
            }
        }

        // ---- calcElectricContributions (:412-453) ----
        double El[3 * NEQ];
        S elec_e = (S)0;
        for (int d = 0; d < 3; d++) {
            const double ang = V.th(d, n.c) - Vp.th(d, n.c);
            El[NEQ * d] = sin(ang);
            double up[4], mul[4];
            Vp.rep(d, n.c, true, up);
            V.rep(d, n.c, false, mul);
            ref_su2_product(mul, up, store, up);
#pragma unroll
            for (int k = 1; k < 4; k++) El[NEQ * d + k] = up[k];
            if (ENERGY)
                elec_e = (S)((double)elec_e
                             + 4.0 * P.lap[d] * (P.inv_g_sqr * (1.0 - up[0]) + P.inv_gp_sqr * (1.0 - cos(ang))));
            // Higgs family (TwoHDM.cpp:601-633)
            if (HF == kHfU1) {
                const double ha = V.hth(d, n.c) - Vp.hth(d, n.c);
                El[NEQ * d + 4 % NEQ] = sin(ha);
                if (ENERGY) elec_e = (S)((double)elec_e + 4.0 * P.lap[d] * P.inv_gpp_sqr * (1.0 - cos(ha)));
            } else if (HF == kHfSU2) {
                double hp[4], hm[4];
                Vp.hrep(d, n.c, true, hp);
                V.hrep(d, n.c, false, hm);
                ref_su2_product(hm, hp, store, hp);
#pragma unroll
                for (int k = 4; k < 7; k++) El[NEQ * d + k % NEQ] = hp[k - 3];
                if (ENERGY) elec_e = (S)((double)elec_e + 4.0 * P.lap[d] * P.inv_gpp_sqr * (1.0 - hp[0]));
            }
        }

        // ---- Energy::preEvolveLocationAnalysis (Analysers/Source/Energy.cpp:117-163) ----
        if (ENERGY) {
            const S pe = ref_potential_energy<MODEL>(P, f_now);
            S ke = (S)0;
            const S dtS = (S)P.dt;
#pragma unroll
            for (int c = 0; c < NSC; c++) {
                const S q = (S)(f_now[c] - f_past[c]) / dtS;
                ke = ke + q * q;
            }
            ke = (S)0.5f * ke;
            const S ee = (S)(P.inv_sqr_dt * (double)elec_e);
            const S tot = pe + grad_e + ke + mag_e + ee;
            obs[kObsEnergy] = (double)tot;
            obs[kObsPotential] = (double)pe;
            obs[kObsGradient] = (double)grad_e;
            obs[kObsKinetic] = (double)ke;
            obs[kObsMagnetic] = (double)mag_e;
            obs[kObsElectric] = (double)ee;
            if (P.loc_energy && counts(P, x)) {  // Energy's local densities (Analysers/Source/Energy.cpp:137-143)
                float* o = P.loc_energy + 6 * (size_t)n.c;
                o[0] = (float)tot;
                o[1] = (float)pe;
                o[2] = (float)grad_e;
                o[3] = (float)ke;
                o[4] = (float)mag_e;
                o[5] = (float)ee;
            }
            obs[kObsPlaqSU2] = plaq2;
            obs[kObsPlaqU1] = plaq1;
            double fs = 0.0;
#pragma unroll
            for (int c = 0; c < NSC; c++) fs += (double)f_now[c] * (double)f_now[c];
            obs[kObsPhiSq] = fs;
        }

        // ---- Model::evolve (Core/Source/Model.cpp:339-373) ----
        S f_new[NSC];
        bool finite = true;
#pragma unroll
        for (int c = 0; c < NSC; c++) {
            const double rhs = P.dt * P.dt * (D[c] - Pot[c]) - P.damping_step * ((double)f_now[c] - (double)f_past[c]);
            f_new[c] = (S)(2 * (double)f_now[c] - (double)f_past[c] + rhs);
            finite = finite && isfinite((double)f_new[c]);
        }
#pragma unroll
        for (int db = 0; db < NSC / 4; db++)
            st4(past.ph[db], n.c, f_new[4 * db], f_new[4 * db + 1], f_new[4 * db + 2], f_new[4 * db + 3]);

        // ---- WilsonLoops::StandardModel::evolve (:456-514) ----
        for (int d = 0; d < 3; d++) {
            double R[NEQ];
#pragma unroll
            for (int k = 0; k < NEQ; k++)
                R[k] = (1.0 - P.damping_step) * El[NEQ * d + k]
                       + P.dt * P.dt * (Mg[NEQ * d + k] + (k < 4 ? P.gsq[k & 3] : P.gsq_hf) * J[NEQ * d + k]);
            const S th_new = (S)(asin(R[0]) + V.th(d, n.c));
            if (R[0] * R[0] > 1) warn |= kWarnAsin;
            double cm = 0.0;
            cm += R[1] * R[1];
            cm += R[2] * R[2];
            cm += R[3] * R[3];
            if (cm > 1) warn |= kWarnSqrt;
            const double u[4] = {sqrt(1.0 - cm), R[1], R[2], R[3]};
            double up[4];
            V.rep(d, n.c, false, up);
            ref_su2_product(u, up, true, up);
            past.th[d][n.c] = th_new;
            V.store(past.q[d], n.c, up, finite);
            finite = finite && isfinite((double)th_new);
            // Higgs family (TwoHDM.cpp:702-745)
            if (HF == kHfU1) {
                const double r4 = R[4 % NEQ];
                const S h_new = (S)(asin(r4) + V.hth(d, n.c));
                if (r4 * r4 > 1) warn |= kWarnAsin;
                past.hth[d][n.c] = h_new;
                finite = finite && isfinite((double)h_new);
            } else if (HF == kHfSU2) {
                double hm = 0.0;
                hm += R[4 % NEQ] * R[4 % NEQ];
                hm += R[5 % NEQ] * R[5 % NEQ];
                hm += R[6 % NEQ] * R[6 % NEQ];
                if (hm > 1) warn |= kWarnSqrt;
                const double hu[4] = {sqrt(1.0 - hm), R[4 % NEQ], R[5 % NEQ], R[6 % NEQ]};
                double hq[4];
                V.hrep(d, n.c, false, hq);
                ref_su2_product(hu, hq, true, hq);
                V.store(past.hq[d], n.c, hq, finite);
            }
        }
        if (!finite) warn |= kWarnNonFinite;
        if (!counts(P, x)) {  // ghost plane of an x-slab: no observables, no warnings
            warn = 0;
#pragma unroll
            for (int k = 0; k < kObsCount; k++) obs[k] = 0.0;
        }
    }

    if (ENERGY) {
        const int b = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z);
        block_reduce_store<kObsCount>(obs, partials + (size_t)b * kObsCount, kObsCount);
    }
    if (warn) atomicOr(status, warn);
}

// GaugeCondition::postEvolveLocationAnalysis + Model::calcConstraintViolation
// (Analysers/Source/GaugeCondition.cpp:117-165, Core/Source/Model.cpp:323-337).
template <class S, int MODEL, int HF>
__global__ void __launch_bounds__(128) ref_gauss_kernel(StepParams P, LevelPtrs<S> now, LevelPtrs<S> fut,
                                                        double* partials)
{
    constexpr int NSC = (MODEL == kModelSM) ? 4 : 8;
    constexpr int NEQ = hf_neq(HF);
    constexpr int NG = 2 * NEQ;  // integrated then max |violation| per constraint
    const int z = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    const int x = blockIdx.z;
    double v[NG];
#pragma unroll
    for (int k = 0; k < NG; k++) v[k] = 0.0;
    if (z < P.nz && y < P.ny && counts(P, x) && !frozen(P, x, y, z)) {
        const Nbr n = neighbours(P, x, y, z);
        const RefView<S> Vn{now, P.gen != 0, P.div_tol};
        const RefView<S> Vf{fut, P.gen != 0, P.div_tol};
        // WilsonLoops::*::calcConstraintContributions (WilsonLoops/Source/StandardModel.cpp:274-322,
        // TwoHDM.cpp:312-396)
        S el[NEQ];
#pragma unroll
        for (int k = 0; k < NEQ; k++) el[k] = (S)0;
        for (int d = 0; d < 3; d++) {
            const double la = Vf.th(d, n.c) - Vn.th(d, n.c);
            const double na = Vf.th(d, n.m[d]) - Vn.th(d, n.m[d]);
            el[0] = (S)((double)el[0] + (sin(la) - sin(na)) * P.lap[d]);
            double p1[4], mul[4], p2[4];
            Vf.rep(d, n.c, false, p1);
            Vn.rep(d, n.c, true, mul);
            ref_su2_product(mul, p1, false, p1);
            Vn.rep(d, n.m[d], true, p2);
            Vf.rep(d, n.m[d], false, mul);
            ref_su2_product(mul, p2, false, p2);
#pragma unroll
            for (int k = 1; k < 4; k++) el[k] = el[k] + (S)((p1[k] - p2[k]) * P.lap[d]);
            if (HF == kHfU1) {
                const double hl = Vf.hth(d, n.c) - Vn.hth(d, n.c);
                const double hn = Vf.hth(d, n.m[d]) - Vn.hth(d, n.m[d]);
                el[4 % NEQ] = (S)((double)el[4 % NEQ] + (sin(hl) - sin(hn)) * P.lap[d]);
            } else if (HF == kHfSU2) {
                double q1[4], q2[4], mq[4];
                Vf.hrep(d, n.c, false, q1);
                Vn.hrep(d, n.c, true, mq);
                ref_su2_product(mq, q1, false, q1);
                Vn.hrep(d, n.m[d], true, q2);
                Vf.hrep(d, n.m[d], false, mq);
                ref_su2_product(mq, q2, false, q2);
#pragma unroll
                for (int k = 4; k < 7; k++) el[k % NEQ] = el[k % NEQ] + (S)((q1[k - 3] - q2[k - 3]) * P.lap[d]);
            }
        }
        // Gradients::*::calcConstraintContributions (Gradients/Source/StandardModel.cpp:250-270, TwoHDM.cpp:329-373)
        S a[NSC], b[NSC];
        ref_load_scalar_S<NSC>(now, n.c, a);
        ref_load_scalar_S<NSC>(fut, n.c, b);
        S gr[NEQ];
#pragma unroll
        for (int k = 0; k < NEQ; k++) gr[k] = (S)0;
#pragma unroll
        for (int db = 0; db < NSC; db += 4) {
            const S* p = a + db;
            const S* q = b + db;
            const S t0 = p[0] * q[1] - p[1] * q[0] + p[2] * q[3] - p[3] * q[2];
            const S t1 = p[0] * q[3] - p[1] * q[2] + p[2] * q[1] - p[3] * q[0];
            const S t2 = -p[0] * q[2] - p[1] * q[3] + p[2] * q[0] + p[3] * q[1];
            const S t3 = p[0] * q[1] - p[1] * q[0] - p[2] * q[3] + p[3] * q[2];
            if (NSC == 4) {
                gr[0] = (S)(0.25 * (double)t0);
                gr[1] = (S)(0.25 * (double)t1);
                gr[2] = (S)(0.25 * (double)t2);
                gr[3] = (S)(0.25 * (double)t3);
            } else {
                gr[0] = (S)((double)gr[0] + 0.25 * (double)t0);
                gr[1] = (S)((double)gr[1] + 0.25 * (double)t1);
                gr[2] = (S)((double)gr[2] + 0.25 * (double)t2);
                gr[3] = (S)((double)gr[3] + 0.25 * (double)t3);
                // Higgs-family charges (Gradients/Source/TwoHDM.cpp:355-372) over the full 8-vectors
                const int i = db / 2;
                if (HF == kHfU1) {
                    const S h = a[i] * b[i + 1] - a[i + 1] * b[i] - a[i + 4] * b[i + 5] + a[i + 5] * b[i + 4];
                    gr[4 % NEQ] = (S)((double)gr[4 % NEQ] + 0.25 * (double)h);
                } else if (HF == kHfSU2) {
                    const S h4 = a[i] * b[i + 5] - a[i + 1] * b[i + 4] + a[i + 4] * b[i + 1] - a[i + 5] * b[i];
                    const S h5 = -a[i] * b[i + 4] - a[i + 1] * b[i + 5] + a[i + 4] * b[i] + a[i + 5] * b[i + 1];
                    const S h6 = a[i] * b[i + 1] - a[i + 1] * b[i] - a[i + 4] * b[i + 5] + a[i + 5] * b[i + 4];
                    gr[4 % NEQ] = (S)((double)gr[4 % NEQ] + 0.25 * (double)h4);
                    gr[5 % NEQ] = (S)((double)gr[5 % NEQ] + 0.25 * (double)h5);
                    gr[6 % NEQ] = (S)((double)gr[6 % NEQ] + 0.25 * (double)h6);
                }
            }
        }
#pragma unroll
        for (int k = 0; k < NEQ; k++) {
            const S viol = el[k] - (S)(k < 4 ? P.gsq[k & 3] : P.gsq_hf) * gr[k];
            const double av = (double)(viol < (S)0 ? -viol : viol);
            v[k] = av;
            v[NEQ + k] = av;
            if (P.loc_gauss) P.loc_gauss[(size_t)NEQ * n.c + k] = (float)viol;  // GaugeCondition local violation
        }
    }
    const int blk = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z);
    block_reduce_store<NG>(v, partials + (size_t)blk * NG, NEQ);
}

template <class S, int MODEL, int HF>
void ref_step_launch(const StepParams& P, const LevelPtrs<S>& now, const LevelPtrs<S>& past, unsigned* status,
                     double* partials, bool energy, cudaStream_t stream)
{
    const dim3 block(32, 4, 1);
    const dim3 grid((P.nz + 31) / 32, (P.ny + 3) / 4, P.nx);
    if (energy)
        ref_step_kernel<S, MODEL, HF, true><<<grid, block, 0, stream>>>(P, now, past, status, partials);
    else
        ref_step_kernel<S, MODEL, HF, false><<<grid, block, 0, stream>>>(P, now, past, status, partials);
}

template <class S, int MODEL, int HF>
void ref_gauss_launch(const StepParams& P, const LevelPtrs<S>& now, const LevelPtrs<S>& fut, double* partials,
                      cudaStream_t stream)
{
    const dim3 block(32, 4, 1);
    const dim3 grid((P.nz + 31) / 32, (P.ny + 3) / 4, P.nx);
    ref_gauss_kernel<S, MODEL, HF><<<grid, block, 0, stream>>>(P, now, fut, partials);
}

}  // namespace

// P.hf selects the Higgs-family variant (2HDM only); the Gauss kernel writes
// 2 * gaugeNum partial slots per block.
template <class S, int MODEL>
cudaError_t launch_ref_step(const StepParams& P, const LevelPtrs<S>& now, const LevelPtrs<S>& past, unsigned* status,
                            double* partials, bool energy, cudaStream_t stream)
{
    if constexpr (MODEL == kModel2HDM) {
        if (P.hf == kHfU1)
            ref_step_launch<S, MODEL, kHfU1>(P, now, past, status, partials, energy, stream);
        else if (P.hf == kHfSU2)
            ref_step_launch<S, MODEL, kHfSU2>(P, now, past, status, partials, energy, stream);
        else
            ref_step_launch<S, MODEL, kHfNone>(P, now, past, status, partials, energy, stream);
    } else {
        ref_step_launch<S, MODEL, kHfNone>(P, now, past, status, partials, energy, stream);
    }
    return cudaGetLastError();
}

template <class S, int MODEL>
cudaError_t launch_ref_gauss(const StepParams& P, const LevelPtrs<S>& now, const LevelPtrs<S>& fut, double* partials,
                             cudaStream_t stream)
{
    if constexpr (MODEL == kModel2HDM) {
        if (P.hf == kHfU1)
            ref_gauss_launch<S, MODEL, kHfU1>(P, now, fut, partials, stream);
        else if (P.hf == kHfSU2)
            ref_gauss_launch<S, MODEL, kHfSU2>(P, now, fut, partials, stream);
        else
            ref_gauss_launch<S, MODEL, kHfNone>(P, now, fut, partials, stream);
    } else {
        ref_gauss_launch<S, MODEL, kHfNone>(P, now, fut, partials, stream);
    }
    return cudaGetLastError();
}

int ref_launch_blocks(const StepParams& P) { return ((P.nz + 31) / 32) * ((P.ny + 3) / 4) * P.nx; }

#define GFT_INSTANTIATE_REF(S, M)                                                                                    \
    template cudaError_t launch_ref_step<S, M>(const StepParams&, const LevelPtrs<S>&, const LevelPtrs<S>&,          \
                                               unsigned*, double*, bool, cudaStream_t);                               \
    template cudaError_t launch_ref_gauss<S, M>(const StepParams&, const LevelPtrs<S>&, const LevelPtrs<S>&, double*, \
                                                cudaStream_t);
GFT_INSTANTIATE_REF(float, kModelSM)
GFT_INSTANTIATE_REF(float, kModel2HDM)
GFT_INSTANTIATE_REF(double, kModelSM)
GFT_INSTANTIATE_REF(double, kModel2HDM)

}  // namespace gft
