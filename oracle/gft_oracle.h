/*
 * gft_oracle.h -- TEST INFRASTRUCTURE ONLY.
 *
 * CPU restatement of GFTEvolver's real-time leapfrog step (the per-site loop
 * body of Lattice::evolve, Core/Source/Lattice.cpp:755-876) used as the parity
 * checker for the CUDA path.  Nothing in the product links or calls this code;
 * only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg do.
 *
 * The same source (gft_oracle.c) is compiled twice:
 *   - storage float  (symbols orc32_*): the reference exactly as shipped
 *     (std::vector<float> fields, double per-site arithmetic);
 *   - storage double (symbols orc64_*): the reference with every `float`
 *     replaced by `double` (the FP64 plain form).
 *
 * Pinning: the float build is checked against the unmodified reference
 * compiled from its own sources (oracle/_ref/ref32) and the double build
 * against the same sources compiled with float->double (oracle/_ref/ref64),
 * through the golden fixtures in tests/golden/.
 */
#ifndef GFT_ORACLE_H
#define GFT_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* Model selector: which Potential / Gradient / WilsonLoop plugins are active
 * (Core/Header/Model.hpp:19-21).  Only the quaternion link representation and
 * periodic faces are restated (the paths the benchmark configurations use). */
#define ORC_MODEL_SM    1   /* SO_N potential, Gradients::StandardModel, WilsonLoops::StandardModel */
#define ORC_MODEL_2HDM  2   /* Double_SO_N, Gradients::TwoHDM, WilsonLoops::TwoHDM (gaugeNum 4, 5 or 7) */

/* Higgs-family gauge field of the 2HDM (WilsonLoops/Source/TwoHDM.cpp:210-242):
 * none (gaugeNum 4, 5 link words per direction), a U(1) phase theta_H (gaugeNum 5,
 * 6 words: [theta_Y, c0..c3, theta_H]) or an SU(2) quaternion d (gaugeNum 7,
 * 9 words: [theta_Y, c0..c3, d0..d3]). */
#define ORC_HF_NONE 0
#define ORC_HF_U1   1
#define ORC_HF_SU2  2
#define ORC_MAX_EQ  7

typedef struct orc_config {
    int model;
    int nx, ny, nz;
    double dx, dy, dz, dt;
    /* WilsonLoops/*.cfg */
    double g, gp;
    double div_tol;             /* "Tolerance for division by zero" (inverse couplings) */
    /* Core/Config/Model.cfg damping schedule */
    double damping;
    int nt_damped;
    /* Potentials/Config/SO_N.cfg */
    double lambda, eta_sqr;
    /* Potentials/Config/Double_SO_N.cfg */
    double m1, m2, l1, l2, l3;
    double m12r, l4p5, l6r, l7r;
    double m12i, l4m5, l5i, l6i, l7i;
    int break_son, break_uhalfn, apply_norm;
    double energy_offset;
    /* Analysers/Config/Energy.cfg and GaugeCondition.cfg output frequencies; 0 = analyser off */
    int energy_every, gauss_every;
    /* Core/Config/Lattice.cfg face types: bit a set = both faces of axis a are
     * Fixed (type 1; Core/Source/Lattice.cpp:217-300 pairs faces per axis),
     * clear = periodic.  Sites on a Fixed face are not evolved and are not part
     * of the analysers' domain (BoundaryConditions/Source/Fixed.cpp:159-251). */
    int fixed_axes;
    /* 2HDM Higgs-family gauge group (ORC_HF_*) and its coupling g'' (WilsonLoops/Config/TwoHDM.cfg) */
    int hf;
    double gpp;
    /* generator link representation: each SU(2) link stored as its 3 generators w, U =
     * (cos|w|, sin|w| w/|w|) (WilsonLoops/Source/StandardModel.cpp:76-160); 4 words per
     * direction [theta_Y, w1, w2, w3] (+ theta_H, or + w'1..w'3 for the Higgs family) */
    int generator_rep;
    /* Energy / GaugeCondition local-output frequencies (0 = none): per-site densities and
     * signed violations on those steps; the energy pass (storeEnergy) runs on the union of
     * the global and local Energy cadences (Analysers/Source/Energy.cpp:212-219) */
    int energy_local_every, gauss_local_every;
} orc_config;

/* One row of global observables, written on every step where an analyser logs.
 * Energies are integrated (sum x dx dy dz, Analysers/Source/Energy.cpp:181);
 * Gauss entries follow Analysers/Source/GaugeCondition.cpp:167-193.  The
 * plaquette and <phi^dag phi> means have no reference counterpart. */
typedef struct orc_row {
    int time_iter;
    int has_energy, has_gauss;
    double energy, potential, gradient, kinetic, magnetic, electric;
    double gauss_int[ORC_MAX_EQ], gauss_max[ORC_MAX_EQ];  /* gaugeNum entries used */
    double plaq_su2, plaq_u1, phi_sq;
    /* reference-precision running sums (float in the shipped build), as the
     * reference accumulates them site by site in its own region order */
    double ref_energy[6];
    double ref_gauss_int[ORC_MAX_EQ];
} orc_row;

#ifdef __cplusplus
}
#endif
#endif
