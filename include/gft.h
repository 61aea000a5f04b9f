/*
 * gft.h -- C ABI of the B200 lattice evolver (libgft_b200.so).
 *
 * Drop-in boundary for GFTEvolver's time stepper.  The reference evolves the
 * lattice through per-site virtual calls (Potential, Gradient, WilsonLoop,
 * BoundaryCondition, Analyser) from the loop in Lattice::evolve
 * (Core/Source/Lattice.cpp:755-876) and each Periodic::evolve
 * (BoundaryConditions/Source/Periodic.cpp:205-268).  This library replaces that
 * loop for the whole lattice at once: the plugin choices become a model
 * selector plus parameters, the periodic boundary becomes index wrap, and the
 * Energy / GaugeCondition analysers become fused device reductions that fill
 * gft_observables rows.
 *
 * Conventions
 *   - Host field buffers use the reference layout (Lattice.cpp:358-367,
 *     658-671): scalars[2][nx][ny][nz][nsc], vectors[2][nx][ny][nz][3 * dw] with
 *     per direction [theta_Y, c0, c1, c2, c3] (quaternion representation, dw = 5),
 *     followed for a 2HDM Higgs-family gauge field by theta_H (dw = 6) or the
 *     family quaternion d0..d3 (dw = 9) (WilsonLoops/Source/TwoHDM.cpp:210-242); with
 *     generator_rep, [theta_Y, w1, w2, w3] (dw = 4, 5 or 7).  The reference-arithmetic
 *     form keeps the generators on the device and converts on every access as the
 *     reference does; the throughput forms convert at upload / download and evolve
 *     quaternions (the same group elements, different rounding).
 *     Level index = the reference's time slot; at time step time_iter the
 *     "now" slot is (time_iter + 1) % 2 (Lattice.cpp:773-774).
 *   - Device memory is owned by the handle; host buffers are caller-owned and
 *     copied.  One handle per CUDA stream; thread-safe across handles, not
 *     within one handle.
 *   - Return value: 0 = success, < 0 = error (see GFT_E_*), > 0 = warning
 *     bitmask (GFT_W_*).  The reference prints "Panic" and continues when an
 *     asin or sqrt argument leaves its domain
 *     (WilsonLoops/Source/StandardModel.cpp:474-491); here the condition is
 *     counted on the device and reported as a warning bit.
 */
#ifndef GFT_H
#define GFT_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define GFT_OK 0
#define GFT_E_INVALID (-1)      /* bad argument / configuration (reference: std::runtime_error at construction) */
#define GFT_E_UNSUPPORTED (-2)  /* combination not built (e.g. a Higgs-family field in an ensemble) */
#define GFT_E_CUDA (-3)         /* CUDA runtime error; see gft_last_error */
#define GFT_E_NOMEM (-4)        /* device allocation failed */
#define GFT_E_STATE (-5)        /* call out of order (e.g. evolve before upload) */
#define GFT_E_TIMEOUT (-6)      /* a bounded device-side wait gave up; the step's results are invalid */

#define GFT_W_ASIN_DOMAIN 1     /* |RHS_Y| > 1 somewhere (theta update used asin outside [-1,1]) */
#define GFT_W_SQRT_DOMAIN 2     /* |c|^2 > 1 somewhere (SU(2) update used sqrt of a negative number) */
#define GFT_W_NONFINITE 4       /* a non-finite value was written */
#define GFT_W_RANGE 16          /* a link phase |theta| > 1e4: the throughput forms' sin/cos lose accuracy */

/* ---- model / form selectors -------------------------------------------- */
/* Model.cfg plugin triples (Core/Header/Model.hpp:19-21) that are built. */
#define GFT_MODEL_SM 1    /* SO_N potential + Gradients::StandardModel + WilsonLoops::StandardModel */
#define GFT_MODEL_2HDM 2  /* Double_SO_N + Gradients::TwoHDM + WilsonLoops::TwoHDM (gaugeNum 4, 5 or 7) */

/* 2HDM Higgs-family gauge field (gft_config.higgs_family; WilsonLoops/Source/TwoHDM.cpp:210-242). */
#define GFT_HF_NONE 0     /* gaugeNum 4: SU(2) x U(1) only (5 link words per direction) */
#define GFT_HF_U1 1       /* gaugeNum 5: + a family U(1) phase theta_H (6 words) */
#define GFT_HF_SU2 2      /* gaugeNum 7: + a family SU(2) quaternion (9 words) */
#define GFT_MAX_GAUSS 7   /* Gauss constraint equations at most (gaugeNum) */

/* Arithmetic forms. */
#define GFT_FORM_REF 0    /* reference arithmetic: per-site math in FP64 in the reference's operation
                             order; storage = `storage_bytes` (4: the reference as shipped, 8: FP64 storage) */
#define GFT_FORM_FP64 1   /* plain FP64 form: FP64 storage and math, reassociated for throughput */
#define GFT_FORM_MIXED 2  /* FP32 storage and FP32 per-site math throughout (forces, link momentum,
                             leapfrog and link update, renormalisation), rearranged so that no step
                             subtracts nearly equal FP32 values; FP64 only for the energy, plaquette,
                             <phi^2> and Gauss reductions (the Gauss residual itself in FP64) */

typedef struct gft_config {
    int model;                     /* GFT_MODEL_* */
    int form;                      /* GFT_FORM_* */
    int storage_bytes;             /* GFT_FORM_REF only: 4 or 8 */
    int device;                    /* CUDA device ordinal */
    int nx, ny, nz;                /* Core/Config/Lattice.cfg */
    double dx, dy, dz, dt;
    double g, gp;                  /* WilsonLoops/Config/*.cfg */
    double div_tol;                /* division-by-zero tolerance for the inverse couplings */
    double damping;                /* Core/Config/Model.cfg: damping factor */
    int nt_damped;                 /*   number of damped time steps */
    double lambda, eta_sqr;        /* Potentials/Config/SO_N.cfg */
    double m1, m2, l1, l2, l3;     /* Potentials/Config/Double_SO_N.cfg */
    double m12r, l4p5, l6r, l7r;
    double m12i, l4m5, l5i, l6i, l7i;
    int break_son, break_uhalfn, apply_norm;
    double energy_offset;
    int energy_every;              /* Analysers/Config/Energy.cfg output frequency; 0 = no Energy analyser */
    int gauss_every;               /* Analysers/Config/GaugeCondition.cfg frequency; 0 = off */
    int fixed_axes;                /* Core/Config/Lattice.cfg face types: bit a set = both faces of axis a
                                      are Fixed (type 1), clear = periodic (type 3).  Sites on a Fixed
                                      face are not evolved and not counted by the analysers
                                      (BoundaryConditions/Source/Fixed.cpp:159-251, Core/Source/Lattice.cpp:217-306). */
    int higgs_family;              /* GFT_HF_*: 2HDM Higgs-family gauge field (model 2 only) */
    double gpp;                    /* its coupling g'' (WilsonLoops/Config/TwoHDM.cfg) */
    int generator_rep;             /* 1: host vectors hold each SU(2) link as its 3 generators w,
                                      U = (cos|w|, sin|w| w/|w|) (WilsonLoops/Source/StandardModel.cpp:76-160):
                                      4 words per direction [theta_Y, w1, w2, w3] (+ theta_H or w'1..w'3) */
    int energy_local_every;        /* Energy.cfg local-output frequency (0 = none): on those steps the
                                      per-site densities are kept for gft_local_fields */
    int gauss_local_every;         /* GaugeCondition.cfg local-output frequency (0 = none) */
} gft_config;

/* One row of global observables (Analysers/Source/Energy.cpp:169-220,
 * Analysers/Source/GaugeCondition.cpp:167-226).  Energies are integrated over
 * the lattice (sum x dx dy dz); the Gauss entries are the integrated and the
 * maximum |violation| per constraint equation (gaugeNum of them: hypercharge,
 * isospin 1..3, then the Higgs family; unused entries 0).  plaq_* and phi_sq
 * are means with no reference counterpart. */
typedef struct gft_observables {
    int time_iter;
    int has_energy, has_gauss;
    double energy, potential, gradient, kinetic, magnetic, electric;
    double gauss_int[GFT_MAX_GAUSS], gauss_max[GFT_MAX_GAUSS];
    double plaq_su2, plaq_u1, phi_sq;
} gft_observables;

/* Initial data generated on the device (no reference counterpart: the
 * reference ships only RandomUniform, InitialConditions/Source/RandomUniform.cpp:60-77).
 * Both time levels are set equal (E = 0, pi = 0).  Scalars: component c ~
 * N(mean[c], sigma[c]^2), plus a periodic tanh double wall on component 0 when
 * wall_width > 0.  Links: theta_Y ~ N(0, theta_sigma^2); SU(2) =
 * (cos eps, sin eps n), eps ~ N(0, eps_sigma^2), n uniform on S^2; a
 * Higgs-family phase ~ N(0, theta_sigma^2) or quaternion drawn like the SU(2) link. */
typedef struct gft_ic {
    uint64_t seed;
    double mean[8], sigma[8];
    double theta_sigma, eps_sigma;
    double wall_width, wall_value;
} gft_ic;

typedef struct gft_handle gft_handle;

/* Lattice construction (replaces Lattice::Lattice, Core/Source/Lattice.cpp:679-722,
 * and Model::configure, Core/Source/Model.cpp:145-234). */
int gft_create(const gft_config* cfg, gft_handle** out);
void gft_destroy(gft_handle* h);

/* Field transfer in the reference layout (both levels).  `time_iter` is the
 * reference step counter the data belongs to (0 for initial data). */
int gft_upload_f32(gft_handle* h, const float* scalars, const float* vectors, int time_iter);
int gft_upload_f64(gft_handle* h, const double* scalars, const double* vectors, int time_iter);
int gft_download_f32(gft_handle* h, float* scalars, float* vectors);
int gft_download_f64(gft_handle* h, double* scalars, double* vectors);

/* The same transfers with the reference-layout buffers in device memory of the
 * handle's device (no host copy, no staging buffer): for callers that keep the
 * fields on the GPU.  Synchronous with respect to the handle's stream. */
int gft_upload_device_f32(gft_handle* h, const float* d_scalars, const float* d_vectors, int time_iter);
int gft_upload_device_f64(gft_handle* h, const double* d_scalars, const double* d_vectors, int time_iter);
int gft_download_device_f32(gft_handle* h, float* d_scalars, float* d_vectors);
int gft_download_device_f64(gft_handle* h, double* d_scalars, double* d_vectors);

/* Generate initial data on the device (InitialCondition::setInitialFields,
 * InitialConditions/Header/InitialCondition.hpp:24). */
int gft_init_fields(gft_handle* h, const gft_ic* ic);

/* Evolve n_steps time steps (the body of Lattice::evolve's time loop).  Rows
 * are written for every step on which an analyser logs (time_iter % every ==
 * 0); *n_rows receives the number written (at most max_rows). */
int gft_evolve(gft_handle* h, int n_steps, gft_observables* rows, int max_rows, int* n_rows);

/* Observables of the current state without stepping (energy terms at the
 * current level pair, plaquette means, <phi^dag phi>). */
int gft_observe(gft_handle* h, gft_observables* row);

/* Current reference step counter. */
int gft_time_iter(const gft_handle* h);
/* Per-site analyser outputs of the most recent local-output step (Energy's and
 * GaugeCondition's local options, Analysers/Source/Energy.cpp:117-163, 191-207,
 * Analysers/Source/GaugeCondition.cpp:117-140, 194-212): energy[nsite][6] =
 * (energy, potential, gradient, kinetic, magnetic, electric) densities at
 * step *energy_step (before its update), gauss[nsite][gaugeNum] = the signed
 * constraint violations after step *gauss_step, sites in the reference's index
 * order (x slowest), float as the reference stores them; sites on Fixed faces
 * are 0.  Either buffer may be NULL; a step is -1 when none was computed yet.
 * A local-output step also renormalises as an energy step does (the reference's
 * storeEnergy covers both cadences). */
int gft_local_fields(gft_handle* h, float* energy, float* gauss, int* energy_step, int* gauss_step);

/* Device-resident access for callers that keep the state on the GPU:
 * the stream the handle launches on, and the number of device bytes it holds. */
void* gft_stream(gft_handle* h);
size_t gft_device_bytes(const gft_handle* h);

/* Average duration in milliseconds of the step kernel over the launches since
 * the last call (CUDA events on the handle's stream); 0 if none. */
double gft_step_kernel_ms(gft_handle* h, int* launches);

/* Name of the step kernel gft_evolve launches for this handle's form, lattice and
 * gft_set_kernel choice ("ref_step_kernel", "fast_step_kernel" or
 * "tiled_step_kernel"; no reference counterpart). */
const char* gft_step_kernel_name(const gft_handle* h);

/* Number of kernels gft_evolve has launched on this handle so far (step
 * kernels, analyser reductions); a diagnostic with no reference counterpart. */
long long gft_launch_count(const gft_handle* h);

/* ---- x-slabs of a lattice split over ranks ------------------------------ */
/* A handle can hold one x-slab of a larger periodic lattice (no reference
 * counterpart; the reference only notes where an MPI halo exchange would go,
 * Core/Source/Lattice.cpp:779).
 * Its lattice is the slab plus one ghost plane on each side (nx = own planes +
 * 2); the kernels run unchanged on it and the ghost planes' own updates are
 * discarded: observables, Gauss residuals and warnings count only planes
 * [x_begin, x_end), and the device initial data of local plane x is that of
 * global plane (x + x_offset) mod nx_global.  Means in the rows are over the
 * slab's own sites (a caller combines ranks by site-weighted sums). */
int gft_set_slab(gft_handle* h, int x_offset, int nx_global, int x_begin, int x_end);

/* Called by gft_evolve after each step's kernels are enqueued on the handle's
 * stream and before anything reads the level just written (`level`): the
 * caller refreshes that level's ghost planes (e.g. NCCL send/recv of the
 * boundary planes, ordered on gft_stream(h)).  Nonzero return aborts gft_evolve. */
typedef int (*gft_exchange_fn)(gft_handle* h, int level, void* user);
int gft_set_exchange(gft_handle* h, gft_exchange_fn fn, void* user);

/* Device addresses and byte sizes of plane x of every field array of a level
 * (3 quaternion arrays, 3 phase arrays, 1 or 2 doublet arrays, then 3
 * Higgs-family arrays when present, in that order); returns the number of
 * arrays (7, 8 or 11). */
int gft_level_planes(gft_handle* h, int level, int x, void** ptrs, size_t* bytes, int max);

/* The ghost-plane exchange inside the library, over NCCL (no reference
 * counterpart; the reference's Core/Source/Lattice.cpp:779 marks where an
 * overlapped send / late receive would go).  gft_nccl_unique_id writes the
 * 128-byte id of a new communicator (one rank calls it and shares the bytes
 * with the others); gft_set_slab_nccl joins it as `rank` of `nranks` (ring
 * neighbours rank - 1 and rank + 1 mod nranks; one rank exchanges with itself).
 * The slab must have been set with gft_set_slab(h, ..., 1, nx - 1) and no
 * exchange callback.  From then on gft_evolve posts the exchange itself: on
 * plain steps of the tiled kernels it computes the two boundary planes, sends
 * them on a second stream while the interior planes are computed, and makes
 * the next work wait for the ghost planes; on other steps it exchanges after
 * the whole step.  Its final wait is bounded by timeout_s seconds (and watches
 * the communicator for errors): a rank whose peer is gone gets GFT_E_TIMEOUT or
 * GFT_E_CUDA, and the communicator is aborted.  NCCL is loaded at run time
 * (libnccl.so.2); GFT_E_UNSUPPORTED if it cannot be. */
int gft_nccl_unique_id(unsigned char* id);
int gft_set_slab_nccl(gft_handle* h, const unsigned char* id, int nranks, int rank, double timeout_s);

/* Allocation-free observables (no counterpart in the reference).  For callers
 * that cannot allocate device memory where they need the numbers -- a fixed
 * memory budget, a region that must stay asynchronous (cudaMalloc/cudaFree
 * synchronise the device), or fields owned by another framework's allocator.
 * Computes the energy terms, plaquette means and <phi^dag phi> of the state
 * at step `time_iter` from the caller's device buffers in the reference layout
 * (float: scalars[2][nx][ny][nz][nsc], vectors[2][nx][ny][nz][3 * w], w = 5
 * words per direction, 6 or 9 with a 2HDM Higgs-family field) and writes
 * 9 doubles to the caller's device buffer d_out (energy, potential, gradient,
 * kinetic, magnetic, electric, plaq_su2, plaq_u1, phi_sq; the units of
 * gft_observables), asynchronously on `stream` (NULL: the default stream).
 * Allocates nothing: its scratch is a fixed 1.2 MB device array compiled into
 * the library, so lattices above 67,108,864 sites return GFT_E_UNSUPPORTED.
 * The first call on a device looks up that array's address (do it before any
 * stream capture) and keeps it for the life of the process, so a device that
 * has been reset with cudaDeviceReset must not be used with it again.  Calls
 * that overlap on the GPU share the array and race, so the caller serialises
 * them.  Only cfg's lattice, model, coupling and Higgs-family fields are read
 * (form and storage_bytes are ignored); periodic lattices with quaternion links
 * (generator_rep = 0) only, otherwise GFT_E_UNSUPPORTED. */
int gft_observe_static(const gft_config* cfg, const float* d_scalars, const float* d_vectors, int time_iter,
                       double* d_out, void* stream);

/* Step-kernel selection for the throughput forms (no reference counterpart):
 * kind 0 = automatic (for the SM model, the tiled kernel when the lattice
 * divides into a built tile and the tiles fill at least 0.8 of a wave of
 * resident CTAs -- 5 waves in the FP64 form --, else the one-thread-per-site
 * kernel), 1 = one
 * thread per site with neighbours read through L1/L2, 2 = TMA-staged tiles
 * marching along x (mixed form; FP64 form of the SM model), 3 = as 2, with two sites per thread in paired
 * FP32 arithmetic on the plain (non-logging) steps (periodic SM model, tiles 0
 * and 3).  tile = tile shape (0: 8 x 32, 1: 4 x 32,
 * 2: 4 x 16, 3: 16 x 16 sites in y x z); march = planes per CTA along x.  Returns
 * GFT_E_UNSUPPORTED when the lattice does not divide into the tile or carries a
 * Higgs-family field (one thread per site serves those). */
int gft_set_kernel(gft_handle* h, int kind, int tile, int march);

/* Launch mode of gft_evolve (no reference counterpart).  on != 0 (the default):
 * lattices of up to 4,194,304 sites (160^3), without an x-slab exchange or local
 * analyser outputs, replay each whole logging period (lcm of 2 and the analyser
 * cadences, after the damped steps) from a CUDA graph captured once, so short
 * steps pay no host launch each; the results are those of the launches one by
 * one.  For such periods gft_step_kernel_ms averages the whole period's device
 * time per step (step kernels, reductions and Gauss passes).  on = 0 launches
 * every kernel directly. */
int gft_set_graphs(gft_handle* h, int on);

/* Diagnostic with no reference counterpart: the time limit, in nanoseconds, of
 * the tiled kernel's waits for its staged planes, at most 4e9 (0 restores the
 * default, 2 s).
 * When a wait gives up, the tile still waits, with the 2 s bound, for its copies
 * in flight, then the step returns GFT_E_TIMEOUT and the fields are invalid
 * until the next upload.  A limit below 1 us makes each wait a single
 * non-blocking test, which fails whenever the copy has not yet landed: a way to
 * exercise that error path with copies that do complete. */
int gft_set_wait_limit(gft_handle* h, unsigned long long ns);

/* Diagnostic with no reference counterpart: evaluates the library's own
 * sin/cos/asin (range-reduced series used by the throughput forms) against
 * CUDA's functions on `device`.  out[9] = max abs error of float sincos.sin,
 * float sincos.cos, float sin, double sincos.sin, double sincos.cos, double sin;
 * max relative error of float asin, double asin, and of the float 1 - a0/|a| of
 * the energy terms (Newton-refined reciprocal square root and reciprocal) against
 * the same expression in double. */
int gft_selftest_math(int device, double* out);

/* ---- ensembles ---------------------------------------------------------- */
/* Many independent lattices (realisations: own seeds, couplings and sizes) in
 * one object, evolved together by ONE persistent kernel launch per time step
 * (no reference counterpart: the reference runs one lattice per process,
 * Core/Source/Lattice.cpp:755-876).  All members share the model, the device,
 * the analysers' cadence, the Higgs-family field and the step counter; the form
 * is GFT_FORM_MIXED; the members' (ny, nz) must share a tile shape (ny % 4 == 0
 * and nz % 16 == 0 at least).  Each member evolves exactly as a single handle
 * would with the same tile shape and march depth (gft_set_kernel).  2HDM members
 * with a Higgs-family field (gaugeNum 5 or 7) take the single handle's
 * one-thread-per-site launches instead, member after member (any shape; no tile
 * shape: gft_batch_set_kernel applies only its use_graphs, gft_batch_autotune
 * returns GFT_E_UNSUPPORTED), and evolve bit for bit as single handles do. */
typedef struct gft_batch gft_batch;

int gft_batch_create(const gft_config* cfgs, int n, gft_batch** out);
void gft_batch_destroy(gft_batch* b);
int gft_batch_size(const gft_batch* b);
/* Device initial data, one gft_ic per member. */
int gft_batch_init_fields(gft_batch* b, const gft_ic* ics);
/* Member transfer in the reference layout (float); an upload sets the shared step counter. */
int gft_batch_upload_f32(gft_batch* b, int member, const float* scalars, const float* vectors, int time_iter);
int gft_batch_download_f32(gft_batch* b, int member, float* scalars, float* vectors);
/* Evolve every member n_steps.  rows[m * max_rows + r] receives member m's r-th
 * logged row; *n_rows the rows written per member.  Whole logging periods run
 * as one CUDA graph replay. */
int gft_batch_evolve(gft_batch* b, int n_steps, gft_observables* rows, int max_rows, int* n_rows);
/* Tile shape (0: 8 x 32, 1: 4 x 32, 2: 4 x 16, 3: 16 x 16), planes per tile along x, and
 * whether whole logging periods are replayed from a CUDA graph. */
int gft_batch_set_kernel(gft_batch* b, int tile, int march, int use_graphs);
/* Times every tile shape the members admit with march depths 8..64 for
 * trial_steps steps each on the ensemble itself (fields and step counter are
 * restored afterwards) and keeps the fastest; reports the choice. */
int gft_batch_autotune(gft_batch* b, int trial_steps, int* tile, int* march);
/* Device time in milliseconds of the last gft_batch_evolve call (CUDA events on its stream). */
double gft_batch_last_ms(const gft_batch* b);
long long gft_batch_launch_count(const gft_batch* b);
int gft_batch_time_iter(const gft_batch* b);
void* gft_batch_stream(gft_batch* b);
size_t gft_batch_device_bytes(const gft_batch* b);
const char* gft_batch_last_error(const gft_batch* b);

/* Message for the last error on this handle (or the last global error if h is NULL). */
const char* gft_last_error(const gft_handle* h);

/* Library / build information. */
const char* gft_version(void);

#ifdef __cplusplus
}
#endif
#endif
