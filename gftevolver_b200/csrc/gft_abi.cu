// gft_abi.cu -- the C ABI (include/gft.h): handle, device memory, step loop.
//
// The handle plays the role of the reference's Lattice + Model objects
// (Core/Header/Lattice.hpp:22-212, Core/Header/Model.hpp:23-266): it owns both
// time levels of the fields on the device, the model parameters, the step
// counter and the analysers' logging cadence.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <numeric>
#include <string>
#include <vector>

#include "gft.h"
#include "gft_launch.h"

using namespace gft;

namespace {

std::mutex g_err_mu;
std::string g_err;

void set_global_error(const std::string& s)
{
    std::lock_guard<std::mutex> lk(g_err_mu);
    g_err = s;
}

// Slots of one device row: kObsCount energy slots, then gaugeNum integrated and
// gaugeNum maximum Gauss slots (room for gaugeNum = 7).
constexpr int kRowSlots = kRowSlotCount;
constexpr int kMaxProfiled = 8192;
// Single handles replay whole logging periods from a CUDA graph up to this many
// sites (160^3 and below: a step is short enough that launching it costs), for
// periods up to kMaxGraphPeriod steps.
constexpr int kGraphMaxSites = 1 << 22;
constexpr int kMaxGraphPeriod = 256;

}  // namespace

namespace gft {
void set_last_error(const std::string& msg) { set_global_error(msg); }
}  // namespace gft

struct gft_handle {
    gft_config cfg{};
    int nsc = 4;
    int hf = 0;             // Higgs-family field (kHf*)
    int nve = 15;           // link words per site in the reference layout (15, 18, 27; generators 12, 15, 21)
    LinkCodec codec;        // generator representation: how host links map to device records
    int neq = 4;            // gauge equations per direction = Gauss constraints (gaugeNum)
    int nsite = 0;
    int nsm = 148;          // the device's SMs (the automatic kernel choice counts waves of tiles)
    int sbytes = 4;         // storage bytes per word (4 or 8)
    void* level_mem[2] = {nullptr, nullptr};
    LevelPtrs<float> lf[2]{};
    LevelPtrs<double> ld[2]{};
    unsigned* d_status = nullptr;
    double* d_part_e = nullptr;
    double* d_part_g = nullptr;
    int part_cap = 0;           // blocks the partial buffers hold
    double* d_scale = nullptr;  // kRowSlots scale factors
    double* d_mid = nullptr;    // stage-one rows of the two-stage finalize (kFinMidCapacity doubles)
    double* d_rows = nullptr;
    int rows_cap = 0;
    void* d_stage = nullptr;
    size_t stage_bytes = 0;
    cudaStream_t stream = nullptr;
    int time_iter = 0;
    bool has_data = false;
    bool profile = true;
    std::vector<cudaEvent_t> ev;
    std::vector<int> ev_steps;  // steps each profiled interval covers (a graph replay: its period)
    int ev_used = 0;
    // CUDA graph of one logging period (graph_period)
    bool use_graphs = true;
    cudaGraphExec_t graph = nullptr;
    int graph_period = 0, graph_rows = 0;
    long long graph_launches = 0;
    double* d_graph_rows = nullptr;
    int graph_rows_cap = 0;
    long long launches = 0;  // kernels launched by gft_evolve / gft_observe
    std::string err;
    size_t dev_bytes = 0;
    // step kernel selection for the throughput forms
    int kernel_kind = 0;    // 0 auto, 1 global-memory kernel, 2 tiled (TMA) kernel, 3 tiled with two
                            // sites per thread on plain steps (SM), 4 tiled with each site split
                            // between two threads on plain steps (SM)
    int tile_variant = 0;   // tiled: index into the built tile shapes
    int march = 32;         // tiled: planes per CTA along x
    unsigned wait_limit_ns = 0;  // gft_set_wait_limit (0: the 2 s default)
    bool tiled_ready = false;
    TMaps tm[2];   // staged "now" planes (with halo), per level
    TMaps tp[2];   // past-level L2 prefetch boxes (no halo), per level
    TMaps tm_split[2], tp_split[2];  // the same for the split-site kernel's tile (kernel kind 4)
    // x-slab of a larger lattice (gft_set_slab): planes [x_begin, x_end) are
    // this handle's own, the others are ghost copies of the neighbours' planes
    int x_begin = 0, x_end = 0;  // x_end = 0: all planes
    int x_offset = 0, nx_global = 0;
    gft_exchange_fn exchange = nullptr;
    void* exchange_user = nullptr;
    // gft_set_slab_nccl: the ghost-plane exchange posted by gft_evolve itself over
    // NCCL, on comm_stream, overlapped with the interior planes
    SlabComm* comm = nullptr;
    cudaStream_t comm_stream = nullptr;
    cudaEvent_t ev_bound = nullptr, ev_comm = nullptr;
    double comm_timeout_s = 300.0;
    // per-site analyser outputs (gft_local_fields)
    float* d_loc_e = nullptr;   // [nsite][6]
    float* d_loc_g = nullptr;   // [nsite][neq]
    int loc_e_step = -1, loc_g_step = -1;

    int fail(int code, const std::string& msg)
    {
        err = msg;
        set_global_error(msg);
        return code;
    }
    int cuda_fail(cudaError_t e, const char* what)
    {
        std::string m = std::string(what) + ": " + cudaGetErrorString(e);
        return fail(GFT_E_CUDA, m);
    }
};

namespace {

bool is_f64_storage(const gft_handle* h) { return h->sbytes == 8; }

// Whether step `ti` writes an analyser row.
bool logs_row(const gft_config& c, int ti)
{
    return (c.energy_every > 0 && ti % c.energy_every == 0) || (c.gauss_every > 0 && ti % c.gauss_every == 0);
}

// Forget the captured period (its launches bake in the kernel choice, tensor maps,
// buffers and parameters that the caller is about to change).
void drop_graph(gft_handle* h)
{
    if (h->graph) {
        cudaStreamSynchronize(h->stream);
        cudaGraphExecDestroy(h->graph);
    }
    h->graph = nullptr;
    h->graph_period = 0;
}

// Parameters of one launch.  For the reference-arithmetic form with float
// storage, the couplings and the damping factor take the values the shipped
// reference sees: getSqrCouplings returns float (WilsonLoops/Source/StandardModel.cpp:224-230)
// and currentDamping is a float member (Core/Header/Model.hpp:38-40).
}  // namespace

StepParams gft::config_params(const gft_config& c, int nsite, bool f32ref, int time_iter, bool energy)
{
    StepParams P{};
    P.nx = c.nx;
    P.ny = c.ny;
    P.nz = c.nz;
    P.nsite = nsite;
    P.dt = c.dt;
    P.dt2 = c.dt * c.dt;
    const double sp[3] = {c.dx, c.dy, c.dz};
    for (int a = 0; a < 3; a++) {
        P.lap[a] = 1.0 / (sp[a] * sp[a]);
        P.inv_dx[a] = 1.0 / sp[a];
    }
    P.inv_sqr_dt = 1.0 / (c.dt * c.dt);
    const double g2 = c.g * c.g, gp2 = c.gp * c.gp;
    P.gsq[0] = f32ref ? (double)(float)gp2 : gp2;
    for (int k = 1; k < 4; k++) P.gsq[k] = f32ref ? (double)(float)g2 : g2;
    P.inv_g_sqr = (g2 > c.div_tol) ? 1.0 / g2 : 0.0;
    P.inv_gp_sqr = (gp2 > c.div_tol) ? 1.0 / gp2 : 0.0;
    P.hf = (c.model == GFT_MODEL_2HDM) ? c.higgs_family : kHfNone;
    P.gen = (c.generator_rep && c.form == GFT_FORM_REF) ? 1 : 0;  // the throughput forms hold quaternions
    P.div_tol = c.div_tol;
    const double gpp2 = c.gpp * c.gpp;
    P.gsq_hf = f32ref ? (double)(float)gpp2 : gpp2;
    P.inv_gpp_sqr = (gpp2 > c.div_tol) ? 1.0 / gpp2 : 0.0;
    double damp = (time_iter < c.nt_damped) ? c.damping : 0.0;
    if (f32ref) damp = (double)(float)damp;
    P.damping_step = 0.5 * damp * c.dt;
    P.lambda = c.lambda;
    P.eta_sqr = c.eta_sqr;
    P.m1 = c.m1;
    P.m2 = c.m2;
    P.l1 = c.l1;
    P.l2 = c.l2;
    P.l3 = c.l3;
    P.m12r = c.m12r;
    P.l4p5 = c.l4p5;
    P.l6r = c.l6r;
    P.l7r = c.l7r;
    P.m12i = c.m12i;
    P.l4m5 = c.l4m5;
    P.l5i = c.l5i;
    P.l6i = c.l6i;
    P.l7i = c.l7i;
    P.break_son = c.break_son;
    P.break_uhalfn = c.break_uhalfn;
    P.apply_norm = c.apply_norm;
    P.energy_offset = c.energy_offset;
    P.store_energy = energy ? 1 : 0;
    P.obs_x0 = 0;
    P.obs_x1 = c.nx;
    P.fixed_axes = c.fixed_axes;
    return P;
}

void gft::row_scales(const gft_config& c, int nsite, double* scale)
{
    // means over the evolved sites (nsite = nx * ny * nz of c): a Fixed axis loses its two face planes
    if (c.fixed_axes) {
        const long long n[3] = {c.nx, c.ny, c.nz};
        long long e = 1;
        for (int a = 0; a < 3; a++) e *= ((c.fixed_axes >> a) & 1) ? (n[a] > 2 ? n[a] - 2 : 0) : n[a];
        nsite = (int)(e > 0 ? e : 1);
    }
    const double dv = c.dx * c.dy * c.dz;
    for (int k = 0; k < kRowSlots; k++) scale[k] = 1.0;
    for (int k = kObsEnergy; k <= kObsElectric; k++) scale[k] = dv;
    scale[kObsPlaqSU2] = 1.0 / (3.0 * nsite);
    scale[kObsPlaqU1] = 1.0 / (3.0 * nsite);
    scale[kObsPhiSq] = 1.0 / (double)nsite;
    for (int k = 0; k < config_neq(c); k++) scale[kObsCount + k] = dv;  // integrated |violation|; maxima unscaled
}

namespace {

StepParams make_params(const gft_handle* h, int time_iter, bool energy)
{
    StepParams P = config_params(h->cfg, h->nsite, (h->cfg.form == GFT_FORM_REF) && h->sbytes == 4, time_iter, energy);
    if (h->x_end > 0) {
        P.obs_x0 = h->x_begin;
        P.obs_x1 = h->x_end;
    }
    P.wait_limit_ns = h->wait_limit_ns;
    return P;
}


// Every array of a level starts on a 64-word boundary (256 B for float,
// 512 B for double) so that the 16-byte vector accesses of q[] and ph[] are
// aligned for any lattice size.
size_t padded_sites(int nsite) { return ((size_t)nsite + 63) / 64 * 64; }

// hf: Higgs-family arrays after the doublets (3 phase arrays or 3 quaternion arrays).
template <class S>
void carve(void* mem, int nsite, int nsc, LevelPtrs<S>& L, int hf = kHfNone)
{
    const size_t np = padded_sites(nsite);
    S* p = static_cast<S*>(mem);
    for (int d = 0; d < 3; d++) {
        L.q[d] = p;
        p += 4 * np;
    }
    for (int d = 0; d < 3; d++) {
        L.th[d] = p;
        p += np;
    }
    L.ph[0] = p;
    p += 4 * np;
    L.ph[1] = (nsc == 8) ? p : nullptr;
    p += (nsc == 8) ? 4 * np : 0;
    for (int d = 0; d < 3; d++) {
        L.hth[d] = (hf == kHfU1) ? p + d * np : nullptr;
        L.hq[d] = (hf == kHfSU2) ? p + 4 * d * np : nullptr;
    }
}

size_t level_words(int nsite, int nsc, int hf = kHfNone)
{
    return padded_sites(nsite) * (15 + (size_t)nsc + (hf == kHfU1 ? 3 : (hf == kHfSU2 ? 12 : 0)));
}

// Tensor maps of both levels for a tile shape: staged planes and past prefetch.
bool encode_tiled(const gft_handle* h, const StepParams& P, int tile, TMaps* tm, TMaps* tp)
{
    int ty, tz;
    tiled_tile(tile, ty, tz);
    for (int t = 0; t < 2; t++) {
        if (h->sbytes == 8) {
            if (!tiled_encode_maps<double>(P, h->ld[t], h->nsc / 4, ty, tz, true, &tm[t])) return false;
            if (!tiled_encode_maps<double>(P, h->ld[t], h->nsc / 4, ty, tz, false, &tp[t])) return false;
        } else {
            if (!tiled_encode_maps<float>(P, h->lf[t], h->nsc / 4, ty, tz, true, &tm[t])) return false;
            if (!tiled_encode_maps<float>(P, h->lf[t], h->nsc / 4, ty, tz, false, &tp[t])) return false;
        }
    }
    return true;
}

// Automatic choice (kernel_kind 0), from B200 measurements at 192^3-448^3: the
// tiled kernel for SM (46 % of HBM against 42 % for one thread per site);
// one thread per site for 2HDM, whose four staged plane buffers (two doublets)
// need 130 KB of shared memory and leave one CTA per SM (30 % against 45 %).
// The automatic choice (kernel kind 0) takes the staged step for the SM model
// when its tiles fill enough waves of resident CTAs: fewer tiles leave SMs idle
// while each CTA marches its planes, and one thread per site is faster there
// (mixed form at 32^3: 14x, 64^3 (0.11 waves): 3.6x; 128^3 (0.86 waves): the
// staged step 2 % faster, 192^3 (2.9 waves): 15 %.  FP64, one CTA per SM: one
// thread per site 11 % faster at 128^3 (1.7 waves) and 7.5 % at 160^3 (3.4
// waves); the staged step 1.6 % faster at 192^3 (5.8 waves) and 7 % at 256^3
// (13.8 waves)).
constexpr double kAutoWavesMixed = 0.8, kAutoWavesFP64 = 5.0;

bool use_tiled(const gft_handle* h, const StepParams& P)
{
    if (!h->tiled_ready || h->kernel_kind == 1 || h->hf != kHfNone) return false;
    const bool fp64 = h->cfg.form == GFT_FORM_FP64;
    // the FP64 form: the staged SM step only (kinds 0 and 2)
    if (fp64 && (h->cfg.model != GFT_MODEL_SM || h->kernel_kind > 2)) return false;
    if (h->cfg.form != GFT_FORM_MIXED && !fp64) return false;
    if (!tiled_supported(P, h->tile_variant)) return false;
    if (h->kernel_kind != 0) return true;
    if (h->cfg.model != GFT_MODEL_SM) return false;
    const long long slots = (long long)h->nsm * tiled_ctas_per_sm(h->tile_variant, fp64);
    return tiled_blocks(P, h->tile_variant, h->march) >= (fp64 ? kAutoWavesFP64 : kAutoWavesMixed) * (double)slots;
}

// Plain steps of the SM mixed form with two sites per thread (kernel kind 3):
// periodic lattices (no Fixed faces) in a tile shape the paired kernel is built for.
bool use_pair(const gft_handle* h, const StepParams& P)
{
    return h->kernel_kind == 3 && h->cfg.model == GFT_MODEL_SM && P.fixed_axes == 0 &&
           tiled_pair_tile(h->tile_variant);
}

// Plain steps of the SM mixed form with each site split between two threads
// (kernel kind 4): periodic lattices whose (ny, nz) divide into its tile.
bool use_split(const gft_handle* h, const StepParams& P)
{
    return h->kernel_kind == 4 && h->cfg.model == GFT_MODEL_SM && P.fixed_axes == 0 && P.ny % kSplitTileY == 0 &&
           P.nz % kSplitTileZ == 0;
}

int step_blocks(const gft_handle* h, const StepParams& P)
{
    if (h->cfg.form == GFT_FORM_REF) return ref_launch_blocks(P);
    if (use_tiled(h, P)) return tiled_blocks(P, h->tile_variant, h->march);
    return fast_launch_blocks(P, 0);
}

// `tn` is the index (0 or 1) of the handle level passed as `now`.
// xa, xn: planes [xa, xa + xn) only (the tiled kernels; xn < 0: every plane);
// st: the stream of a tiled launch (null: the handle's).
template <class S>
cudaError_t launch_step(gft_handle* h, const StepParams& P, int tn, const LevelPtrs<S>& now, const LevelPtrs<S>& past,
                        bool energy, int xa = 0, int xn = -1, cudaStream_t st = nullptr)
{
    const int model = h->cfg.model;
    if (h->cfg.form == GFT_FORM_REF) {
        if (model == GFT_MODEL_SM) return launch_ref_step<S, kModelSM>(P, now, past, h->d_status, h->d_part_e, energy, h->stream);
        return launch_ref_step<S, kModel2HDM>(P, now, past, h->d_status, h->d_part_e, energy, h->stream);
    }
    if constexpr (sizeof(S) == 8) {
        if (model == GFT_MODEL_SM && use_tiled(h, P))
            return launch_tiled_step<S, kModelSM>(h->tm[tn], h->tp[1 - tn], P, now, past, h->tile_variant, h->march,
                                                  h->d_status, h->d_part_e, energy, st ? st : h->stream, xa, xn);
    }
    if constexpr (sizeof(S) == 4) {
        if (use_tiled(h, P)) {
            cudaStream_t s = st ? st : h->stream;
            if (!energy && use_split(h, P))
                return launch_tiled_split_step(h->tm_split[tn], h->tp_split[1 - tn], P, now, past, h->march,
                                               h->d_status, s, xa, xn);
            if (!energy && use_pair(h, P))
                return launch_tiled_pair_step(h->tm[tn], h->tp[1 - tn], P, now, past, h->tile_variant, h->march,
                                              h->d_status, s, xa, xn);
            if (model == GFT_MODEL_SM)
                return launch_tiled_step<S, kModelSM>(h->tm[tn], h->tp[1 - tn], P, now, past, h->tile_variant, h->march,
                                                      h->d_status, h->d_part_e, energy, s, xa, xn);
            return launch_tiled_step<S, kModel2HDM>(h->tm[tn], h->tp[1 - tn], P, now, past, h->tile_variant, h->march,
                                                    h->d_status, h->d_part_e, energy, s, xa, xn);
        }
    }
    if (model == GFT_MODEL_SM)
        return launch_fast_step<S, kModelSM>(P, now, past, h->d_status, h->d_part_e, energy, 0, h->stream);
    return launch_fast_step<S, kModel2HDM>(P, now, past, h->d_status, h->d_part_e, energy, 0, h->stream);
}

// Partial rows the Gauss kernel of this handle's form writes.
int gauss_blocks(const gft_handle* h, const StepParams& P)
{
    return (h->cfg.form == GFT_FORM_REF) ? ref_launch_blocks(P) : fast_gauss_blocks(P);
}

template <class S>
cudaError_t launch_gauss(gft_handle* h, const StepParams& P, const LevelPtrs<S>& now, const LevelPtrs<S>& fut)
{
    const int model = h->cfg.model;
    if (h->cfg.form == GFT_FORM_REF) {
        if (model == GFT_MODEL_SM) return launch_ref_gauss<S, kModelSM>(P, now, fut, h->d_part_g, h->stream);
        return launch_ref_gauss<S, kModel2HDM>(P, now, fut, h->d_part_g, h->stream);
    }
    if (model == GFT_MODEL_SM) return launch_fast_gauss<S, kModelSM>(P, now, fut, h->d_part_g, h->stream);
    return launch_fast_gauss<S, kModel2HDM>(P, now, fut, h->d_part_g, h->stream);
}

int validate(const gft_config* c, std::string& why)
{
    if (!c) {
        why = "gft_create: null config";
        return GFT_E_INVALID;
    }
    if (c->model != GFT_MODEL_SM && c->model != GFT_MODEL_2HDM) {
        why = "gft_create: unsupported model " + std::to_string(c->model);
        return GFT_E_UNSUPPORTED;
    }
    if (c->form != GFT_FORM_REF && c->form != GFT_FORM_FP64 && c->form != GFT_FORM_MIXED) {
        why = "gft_create: unknown form " + std::to_string(c->form);
        return GFT_E_INVALID;
    }
    if (c->form == GFT_FORM_REF && c->storage_bytes != 4 && c->storage_bytes != 8) {
        why = "gft_create: storage_bytes must be 4 or 8 for the reference-arithmetic form";
        return GFT_E_INVALID;
    }
    if (c->nx < 1 || c->ny < 1 || c->nz < 1) {
        why = "gft_create: lattice dimensions must be >= 1";
        return GFT_E_INVALID;
    }
    if (c->nx > 65535) {
        why = "gft_create: nx > 65535 is not supported (one grid row per x plane)";
        return GFT_E_UNSUPPORTED;
    }
    const long long n = (long long)c->nx * c->ny * c->nz;
    if (n > (long long)0x7fffffff / 4) {
        why = "gft_create: lattice too large for 32-bit site indices";
        return GFT_E_UNSUPPORTED;
    }
    if (!(c->dx > 0 && c->dy > 0 && c->dz > 0 && c->dt > 0)) {
        why = "gft_create: spacings and time step must be positive";
        return GFT_E_INVALID;
    }
    if (c->energy_every < 0 || c->gauss_every < 0 || c->energy_local_every < 0 || c->gauss_local_every < 0) {
        why = "gft_create: analyser frequencies must be >= 0";
        return GFT_E_INVALID;
    }
    if (c->fixed_axes < 0 || c->fixed_axes > 7) {
        why = "gft_create: fixed_axes is a bitmask of the three axes (0..7)";
        return GFT_E_INVALID;
    }
    if (c->higgs_family < GFT_HF_NONE || c->higgs_family > GFT_HF_SU2) {
        why = "gft_create: higgs_family must be GFT_HF_NONE, GFT_HF_U1 or GFT_HF_SU2";
        return GFT_E_INVALID;
    }
    if (c->higgs_family != GFT_HF_NONE && c->model != GFT_MODEL_2HDM) {
        why = "gft_create: a Higgs-family gauge field needs the 2HDM (WilsonLoops::TwoHDM)";
        return GFT_E_INVALID;
    }
    if (c->generator_rep != 0 && c->generator_rep != 1) {
        why = "gft_create: generator_rep is 0 (quaternion links) or 1 (generators)";
        return GFT_E_INVALID;
    }
    return GFT_OK;
}

}  // namespace

extern "C" {

const char* gft_version(void) { return "gft_b200 1.0 (sm_100a)"; }

const char* gft_last_error(const gft_handle* h)
{
    if (h) return h->err.c_str();
    std::lock_guard<std::mutex> lk(g_err_mu);
    static thread_local std::string copy;
    copy = g_err;
    return copy.c_str();
}

int gft_create(const gft_config* cfg, gft_handle** out)
{
    if (!out) return GFT_E_INVALID;
    *out = nullptr;
    std::string why;
    int rc = validate(cfg, why);
    if (rc != GFT_OK) {
        set_global_error(why);
        return rc;
    }
    gft_handle* h = new gft_handle();
    h->cfg = *cfg;
    h->nsc = (cfg->model == GFT_MODEL_SM) ? 4 : 8;
    h->hf = (cfg->model == GFT_MODEL_2HDM) ? cfg->higgs_family : kHfNone;
    h->codec.gen = cfg->generator_rep;
    h->codec.convert = (cfg->form != GFT_FORM_REF) ? 1 : 0;
    h->codec.tol = cfg->div_tol;
    {
        const int lw = cfg->generator_rep ? 3 : 4;  // words of one SU(2) link
        h->nve = 3 * (1 + lw + (h->hf == kHfU1 ? 1 : (h->hf == kHfSU2 ? lw : 0)));
    }
    h->neq = config_neq(*cfg);
    h->nsite = cfg->nx * cfg->ny * cfg->nz;
    h->sbytes = (cfg->form == GFT_FORM_REF) ? cfg->storage_bytes : (cfg->form == GFT_FORM_FP64 ? 8 : 4);
    cudaError_t e = cudaSetDevice(cfg->device);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&h->nsm, cudaDevAttrMultiProcessorCount, cfg->device);
    if (e != cudaSuccess) {
        int r = h->cuda_fail(e, "cudaSetDevice");
        delete h;
        return r;
    }
    e = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        int r = h->cuda_fail(e, "cudaStreamCreate");
        delete h;
        return r;
    }
    const size_t lbytes = level_words(h->nsite, h->nsc, h->hf) * (size_t)h->sbytes;
    for (int t = 0; t < 2; t++) {
        e = cudaMalloc(&h->level_mem[t], lbytes);
        if (e != cudaSuccess) {
            h->fail(GFT_E_NOMEM, std::string("cudaMalloc(level): ") + cudaGetErrorString(e));
            gft_destroy(h);
            return GFT_E_NOMEM;
        }
        h->dev_bytes += lbytes;
        if (h->sbytes == 4)
            carve<float>(h->level_mem[t], h->nsite, h->nsc, h->lf[t], h->hf);
        else
            carve<double>(h->level_mem[t], h->nsite, h->nsc, h->ld[t], h->hf);
    }
    const StepParams P = make_params(h, 0, false);
    if (cfg->form == GFT_FORM_MIXED || (cfg->form == GFT_FORM_FP64 && cfg->model == GFT_MODEL_SM)) {
        // default tile: the largest built shape the lattice divides
        h->tile_variant = 0;
        while (h->tile_variant < kTiledVariants && !tiled_supported(P, h->tile_variant)) h->tile_variant++;
        h->tiled_ready = h->tile_variant < kTiledVariants && encode_tiled(h, P, h->tile_variant, h->tm, h->tp);
    }
    int nb = std::max(fast_launch_blocks(P, 0), fast_gauss_blocks(P));
    nb = std::max(nb, ref_launch_blocks(P));
    const size_t pe = (size_t)nb * kObsCount * sizeof(double), pg = (size_t)nb * 2 * h->neq * sizeof(double);
    h->rows_cap = 64;
    if ((e = cudaMalloc(&h->d_status, sizeof(unsigned))) != cudaSuccess ||
        (e = cudaMalloc(&h->d_part_e, pe)) != cudaSuccess || (e = cudaMalloc(&h->d_part_g, pg)) != cudaSuccess ||
        (e = cudaMalloc(&h->d_scale, kRowSlots * sizeof(double))) != cudaSuccess ||
        (e = cudaMalloc(&h->d_mid, kFinMidCapacity * sizeof(double))) != cudaSuccess ||
        (e = cudaMalloc(&h->d_rows, (size_t)h->rows_cap * kRowSlots * sizeof(double))) != cudaSuccess) {
        h->fail(GFT_E_NOMEM, std::string("cudaMalloc(scratch): ") + cudaGetErrorString(e));
        gft_destroy(h);
        return GFT_E_NOMEM;
    }
    h->part_cap = nb;
    h->dev_bytes += pe + pg + sizeof(unsigned) + kRowSlots * sizeof(double) * (1 + h->rows_cap) +
                    kFinMidCapacity * sizeof(double);
    // per-site analyser outputs, zeroed (sites on Fixed faces stay 0, as in the reference)
    const size_t le = cfg->energy_local_every > 0 ? (size_t)h->nsite * 6 * sizeof(float) : 0;
    const size_t lg = cfg->gauss_local_every > 0 ? (size_t)h->nsite * h->neq * sizeof(float) : 0;
    if ((le && ((e = cudaMalloc(&h->d_loc_e, le)) != cudaSuccess || (e = cudaMemset(h->d_loc_e, 0, le)) != cudaSuccess)) ||
        (lg && ((e = cudaMalloc(&h->d_loc_g, lg)) != cudaSuccess || (e = cudaMemset(h->d_loc_g, 0, lg)) != cudaSuccess))) {
        h->fail(GFT_E_NOMEM, std::string("cudaMalloc(local outputs): ") + cudaGetErrorString(e));
        gft_destroy(h);
        return GFT_E_NOMEM;
    }
    h->dev_bytes += le + lg;
    double scale[kRowSlots];
    row_scales(*cfg, h->nsite, scale);
    cudaMemcpy(h->d_scale, scale, sizeof(scale), cudaMemcpyHostToDevice);
    cudaMemset(h->d_status, 0, sizeof(unsigned));
    h->ev.resize(2 * (size_t)kMaxProfiled);
    h->ev_steps.assign(kMaxProfiled, 1);
    for (auto& x : h->ev) {
        if ((e = cudaEventCreate(&x)) != cudaSuccess) {
            x = nullptr;
            h->cuda_fail(e, "cudaEventCreate");
            gft_destroy(h);
            return GFT_E_CUDA;
        }
    }
    e = cudaDeviceSynchronize();
    if (e != cudaSuccess) {
        int r = h->cuda_fail(e, "gft_create");
        gft_destroy(h);
        return r;
    }
    *out = h;
    return GFT_OK;
}

void gft_destroy(gft_handle* h)
{
    if (!h) return;
    cudaSetDevice(h->cfg.device);
    if (h->stream) cudaStreamSynchronize(h->stream);
    if (h->comm_stream) cudaStreamSynchronize(h->comm_stream);
    drop_graph(h);
    cudaFree(h->d_graph_rows);
    slab_comm_destroy(h->comm, false);
    if (h->ev_bound) cudaEventDestroy(h->ev_bound);
    if (h->ev_comm) cudaEventDestroy(h->ev_comm);
    if (h->comm_stream) cudaStreamDestroy(h->comm_stream);
    for (auto& x : h->ev)
        if (x) cudaEventDestroy(x);
    for (int t = 0; t < 2; t++)
        if (h->level_mem[t]) cudaFree(h->level_mem[t]);
    cudaFree(h->d_status);
    cudaFree(h->d_part_e);
    cudaFree(h->d_part_g);
    cudaFree(h->d_scale);
    cudaFree(h->d_mid);
    cudaFree(h->d_rows);
    cudaFree(h->d_stage);
    cudaFree(h->d_loc_e);
    cudaFree(h->d_loc_g);
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
}

int gft_time_iter(const gft_handle* h) { return h ? h->time_iter : -1; }
void* gft_stream(gft_handle* h) { return h ? (void*)h->stream : nullptr; }
size_t gft_device_bytes(const gft_handle* h) { return h ? h->dev_bytes : 0; }

}  // extern "C"

namespace {

int ensure_stage(gft_handle* h, size_t bytes)
{
    if (h->stage_bytes >= bytes) return GFT_OK;
    if (h->d_stage) {
        cudaStreamSynchronize(h->stream);
        cudaFree(h->d_stage);
        h->dev_bytes -= h->stage_bytes;
        h->d_stage = nullptr;
        h->stage_bytes = 0;
    }
    cudaError_t e = cudaMalloc(&h->d_stage, bytes);
    if (e != cudaSuccess) return h->fail(GFT_E_NOMEM, std::string("cudaMalloc(stage): ") + cudaGetErrorString(e));
    h->stage_bytes = bytes;
    h->dev_bytes += bytes;
    return GFT_OK;
}

// `on_device`: sc/ve are device buffers (converted in place, no staging copy).
template <class H>
int upload_impl(gft_handle* h, const H* sc, const H* ve, int time_iter, bool on_device = false)
{
    if (!h || !sc || !ve) return GFT_E_INVALID;
    if (time_iter < 0) return h->fail(GFT_E_INVALID, "gft_upload: time_iter must be >= 0");
    cudaSetDevice(h->cfg.device);
    const size_t nsc_w = 2 * (size_t)h->nsite * h->nsc, nve_w = 2 * (size_t)h->nsite * h->nve;
    const H* dsc = sc;
    const H* dve = ve;
    cudaError_t e = cudaSuccess;
    if (!on_device) {
        int rc = ensure_stage(h, (nsc_w + nve_w) * sizeof(H));
        if (rc != GFT_OK) return rc;
        H* st = static_cast<H*>(h->d_stage);
        e = cudaMemcpyAsync(st, sc, nsc_w * sizeof(H), cudaMemcpyHostToDevice, h->stream);
        if (e == cudaSuccess) e = cudaMemcpyAsync(st + nsc_w, ve, nve_w * sizeof(H), cudaMemcpyHostToDevice, h->stream);
        dsc = st;
        dve = st + nsc_w;
    }
    for (int t = 0; t < 2 && e == cudaSuccess; t++) {
        const H* s_t = dsc + (size_t)t * h->nsite * h->nsc;
        const H* v_t = dve + (size_t)t * h->nsite * h->nve;
        e = is_f64_storage(h) ? launch_aos_to_soa<double, H>(s_t, v_t, h->nsite, h->nsc, h->ld[t], h->stream, h->codec)
                              : launch_aos_to_soa<float, H>(s_t, v_t, h->nsite, h->nsc, h->lf[t], h->stream, h->codec);
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) return h->cuda_fail(e, "gft_upload");
    h->time_iter = time_iter;
    h->has_data = true;
    return GFT_OK;
}

template <class H>
int download_impl(gft_handle* h, H* sc, H* ve, bool on_device = false)
{
    if (!h || !sc || !ve) return GFT_E_INVALID;
    if (!h->has_data) return h->fail(GFT_E_STATE, "gft_download: no field data on the device");
    cudaSetDevice(h->cfg.device);
    const size_t nsc_w = 2 * (size_t)h->nsite * h->nsc, nve_w = 2 * (size_t)h->nsite * h->nve;
    H* dsc = sc;
    H* dve = ve;
    if (!on_device) {
        int rc = ensure_stage(h, (nsc_w + nve_w) * sizeof(H));
        if (rc != GFT_OK) return rc;
        dsc = static_cast<H*>(h->d_stage);
        dve = dsc + nsc_w;
    }
    cudaError_t e = cudaSuccess;
    for (int t = 0; t < 2 && e == cudaSuccess; t++) {
        H* s_t = dsc + (size_t)t * h->nsite * h->nsc;
        H* v_t = dve + (size_t)t * h->nsite * h->nve;
        e = is_f64_storage(h) ? launch_soa_to_aos<double, H>(h->ld[t], h->nsite, h->nsc, s_t, v_t, h->stream, h->codec)
                              : launch_soa_to_aos<float, H>(h->lf[t], h->nsite, h->nsc, s_t, v_t, h->stream, h->codec);
    }
    if (!on_device) {
        if (e == cudaSuccess) e = cudaMemcpyAsync(sc, dsc, nsc_w * sizeof(H), cudaMemcpyDeviceToHost, h->stream);
        if (e == cudaSuccess) e = cudaMemcpyAsync(ve, dve, nve_w * sizeof(H), cudaMemcpyDeviceToHost, h->stream);
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) return h->cuda_fail(e, "gft_download");
    return GFT_OK;
}

int ensure_rows(gft_handle* h, int n)
{
    if (n <= h->rows_cap) return GFT_OK;
    cudaStreamSynchronize(h->stream);
    double* p = nullptr;
    cudaError_t e = cudaMalloc(&p, (size_t)n * kRowSlots * sizeof(double));
    if (e != cudaSuccess) return h->fail(GFT_E_NOMEM, std::string("cudaMalloc(rows): ") + cudaGetErrorString(e));
    h->dev_bytes += (size_t)(n - h->rows_cap) * kRowSlots * sizeof(double);
    cudaFree(h->d_rows);
    h->d_rows = p;
    h->rows_cap = n;
    return GFT_OK;
}

void fill_row(gft_observables* r, int time_iter, bool e, bool g, const double* v, int neq)
{
    std::memset(r, 0, sizeof(*r));
    r->time_iter = time_iter;
    r->has_energy = e;
    r->has_gauss = g;
    if (e) {
        r->energy = v[kObsEnergy];
        r->potential = v[kObsPotential];
        r->gradient = v[kObsGradient];
        r->kinetic = v[kObsKinetic];
        r->magnetic = v[kObsMagnetic];
        r->electric = v[kObsElectric];
        r->plaq_su2 = v[kObsPlaqSU2];
        r->plaq_u1 = v[kObsPlaqU1];
        r->phi_sq = v[kObsPhiSq];
    }
    if (g) {
        for (int k = 0; k < neq; k++) {
            r->gauss_int[k] = v[kObsCount + k];
            r->gauss_max[k] = v[kObsCount + neq + k];
        }
    }
}

// The four planes of every field array of `level` that one slab exchange moves.
int fill_slab_planes(gft_handle* h, int level, SlabPlanes& pl)
{
    size_t b[kMaxPlaneArrays];
    int n = gft_level_planes(h, level, h->x_begin, pl.send_lo, pl.bytes, kMaxPlaneArrays);
    if (n < 0) return n;
    if (gft_level_planes(h, level, h->x_end - 1, pl.send_hi, b, kMaxPlaneArrays) < 0 ||
        gft_level_planes(h, level, h->x_begin - 1, pl.recv_lo, b, kMaxPlaneArrays) < 0 ||
        gft_level_planes(h, level, h->x_end, pl.recv_hi, b, kMaxPlaneArrays) < 0)
        return GFT_E_INVALID;
    pl.n = n;
    return GFT_OK;
}

// A plain step of an x-slab with the exchange in the library (tiled kernels).
// The first and the last x-chunk of own planes (march planes each, so that no
// CTA pays the ring's start-up for fewer planes than usual) are computed on
// comm_stream, created with the highest priority so that their CTAs are
// scheduled first, and the two boundary planes are sent from there while the
// interior chunks are computed concurrently on the handle's stream; the plane
// sets are disjoint and all read only the "now" level, so the kernels may
// overlap.  The handle's stream then waits for the exchange before anything
// reads the ghost planes.  `launches` counts the step kernels; `why` receives
// an NCCL error.
template <class S>
cudaError_t split_slab_step(gft_handle* h, const StepParams& P, int tn, const LevelPtrs<S>* lv, int& launches,
                            int& rc, std::string& why)
{
    const int tp = 1 - tn;
    const int a = h->x_begin, b = h->x_end, nloc = b - a;  // own planes [a, b)
    // everything before this step (the previous step's writes and exchange) precedes the boundary planes
    cudaError_t err = cudaEventRecord(h->ev_bound, h->stream);
    if (err == cudaSuccess) err = cudaStreamWaitEvent(h->comm_stream, h->ev_bound, 0);
    if (err != cudaSuccess) return err;
    const int m = h->march;  // boundary chunks [a, a + m) and [b - m, b); interior [a + m, b - m)
    const bool interior = nloc > 2 * m;
    if (!interior) {
        err = launch_step<S>(h, P, tn, lv[tn], lv[tp], false, a, nloc, h->comm_stream);
        launches += 1;
    } else {
        err = launch_step<S>(h, P, tn, lv[tn], lv[tp], false, a, m, h->comm_stream);
        if (err == cudaSuccess) err = launch_step<S>(h, P, tn, lv[tn], lv[tp], false, b - m, m, h->comm_stream);
        launches += 2;
    }
    if (err != cudaSuccess) return err;
    SlabPlanes pl;
    rc = fill_slab_planes(h, tp, pl);
    if (rc == GFT_OK) rc = slab_comm_exchange(h->comm, pl, h->comm_stream, why);
    if (rc != GFT_OK) return cudaSuccess;
    err = cudaEventRecord(h->ev_comm, h->comm_stream);
    if (err == cudaSuccess && interior) {
        err = launch_step<S>(h, P, tn, lv[tn], lv[tp], false, a + m, nloc - 2 * m);
        launches += 1;
    }
    if (err == cudaSuccess) err = cudaStreamWaitEvent(h->stream, h->ev_comm, 0);
    return err;
}

// The launches of one step at time_iter `ti`: the step kernel (split for an
// x-slab with the library's exchange), the energy row into `out`, the ghost
// exchange, the Gauss pass and its row.  prof: record the step kernel's events.
// Returns a CUDA error, or sets rc / why (exchange failures).
template <class S>
cudaError_t issue_step(gft_handle* h, const LevelPtrs<S>* lv, int ti, double* out, bool prof, int& rc,
                       std::string& why)
{
    const gft_config& c = h->cfg;
    const int tn = (ti + 1) % 2, tp = 1 - tn;
    const bool e = c.energy_every > 0 && ti % c.energy_every == 0;  // rows
    const bool g = c.gauss_every > 0 && ti % c.gauss_every == 0;
    // local outputs: the energy pass (and its renormalisation) also runs on their steps
    const bool el = c.energy_local_every > 0 && ti % c.energy_local_every == 0;
    const bool gl = c.gauss_local_every > 0 && ti % c.gauss_local_every == 0;
    StepParams P = make_params(h, ti, e || el);
    P.loc_energy = el ? h->d_loc_e : nullptr;
    P.loc_gauss = gl ? h->d_loc_g : nullptr;
    if (el) h->loc_e_step = ti;
    if (gl) h->loc_g_step = ti;
    if (prof) cudaEventRecord(h->ev[2 * (size_t)h->ev_used], h->stream);
    // an x-slab with the exchange in the library overlaps it with the interior on plain steps
    const bool split = h->comm && !(e || el) && sizeof(S) == 4 && use_tiled(h, P) && h->x_begin == 1 &&
                       h->x_end == c.nx - 1;
    int nstep = 1;
    cudaError_t err;
    if (split) {
        nstep = 0;
        err = split_slab_step<S>(h, P, tn, lv, nstep, rc, why);
        if (rc != GFT_OK) return cudaSuccess;
    } else {
        err = launch_step<S>(h, P, tn, lv[tn], lv[tp], e || el);
    }
    h->launches += nstep + (e ? finalize_launches(step_blocks(h, P), true) : 0) + ((g || gl) ? 1 : 0) +
                   (g ? finalize_launches(gauss_blocks(h, P), true) : 0);
    if (prof) {
        cudaEventRecord(h->ev[2 * (size_t)h->ev_used + 1], h->stream);
        h->ev_steps[h->ev_used] = 1;
        h->ev_used++;
    }
    if (err != cudaSuccess) return err;
    if (e) err = launch_finalize(h->d_part_e, step_blocks(h, P), kObsCount, kObsCount, h->d_scale, out, h->d_mid,
                                 h->stream);
    if (h->comm && !split && err == cudaSuccess) {
        // logging steps (and forms without the split): the exchange after the whole step
        SlabPlanes pl;
        rc = fill_slab_planes(h, tp, pl);
        if (rc == GFT_OK) rc = slab_comm_exchange(h->comm, pl, h->stream, why);
        if (rc != GFT_OK) return cudaSuccess;
    }
    if (h->exchange && err == cudaSuccess) {
        // refresh the ghost planes of the level just written before anything reads them
        const int xr = h->exchange(h, tp, h->exchange_user);
        if (xr != 0) {
            rc = GFT_E_STATE;
            why = "the exchange callback failed (" + std::to_string(xr) + ")";
            return cudaSuccess;
        }
    }
    if ((g || gl) && err == cudaSuccess) {
        err = launch_gauss<S>(h, P, lv[tn], lv[tp]);
        if (err == cudaSuccess && g)
            err = launch_finalize(h->d_part_g, gauss_blocks(h, P), 2 * h->neq, h->neq, h->d_scale + kObsCount,
                                  out + kObsCount, h->d_mid, h->stream);
    }
    return err;
}

// Logging period replayed from a CUDA graph (lcm of 2 and the analysers'
// cadences), or 0 where a single handle steps launch by launch: lattices large
// enough that launching is no cost, x-slabs (per-step exchange), local outputs.
int graph_period(const gft_handle* h)
{
    const gft_config& c = h->cfg;
    if (!h->use_graphs || h->nsite > kGraphMaxSites || h->exchange || h->comm || c.energy_local_every > 0 ||
        c.gauss_local_every > 0)
        return 0;
    int p = 2;
    if (c.energy_every > 0) p = std::lcm(p, c.energy_every);
    if (c.gauss_every > 0) p = std::lcm(p, c.gauss_every);
    return p <= kMaxGraphPeriod ? p : 0;
}

// Capture the period starting at ti0 (a multiple of the period; the launches
// depend on time_iter only through its parity and the logging cadence).
template <class S>
int build_graph(gft_handle* h, const LevelPtrs<S>* lv, int ti0, int period)
{
    int nrows = 0;
    for (int s = 0; s < period; s++) nrows += logs_row(h->cfg, ti0 + s) ? 1 : 0;
    if (nrows > h->graph_rows_cap) {
        cudaStreamSynchronize(h->stream);
        cudaFree(h->d_graph_rows);
        h->d_graph_rows = nullptr;
        if (cudaMalloc(&h->d_graph_rows, (size_t)std::max(nrows, 1) * kRowSlots * sizeof(double)) != cudaSuccess)
            return h->fail(GFT_E_NOMEM, "gft_evolve: graph rows allocation failed");
        h->graph_rows_cap = nrows;
    }
    const long long l0 = h->launches;
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return h->cuda_fail(e, "gft_evolve: begin capture");
    cudaError_t ie = cudaSuccess;
    int rc = GFT_OK, row = 0;
    std::string why;
    for (int s = 0; s < period && ie == cudaSuccess && rc == GFT_OK; s++) {
        const int ti = ti0 + s;
        ie = issue_step<S>(h, lv, ti, h->d_graph_rows + (size_t)row * kRowSlots, false, rc, why);
        if (logs_row(h->cfg, ti)) row++;
    }
    e = cudaStreamEndCapture(h->stream, &g);
    const long long nl = h->launches - l0;
    h->launches = l0;
    if (ie != cudaSuccess || e != cudaSuccess || rc != GFT_OK) {
        if (g) cudaGraphDestroy(g);
        if (rc != GFT_OK) return h->fail(rc, "gft_evolve: " + why);
        return h->cuda_fail(ie != cudaSuccess ? ie : e, "gft_evolve: capture");
    }
    cudaGraphExec_t x = nullptr;
    e = cudaGraphInstantiate(&x, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return h->cuda_fail(e, "gft_evolve: graph instantiate");
    drop_graph(h);
    h->graph = x;
    h->graph_period = period;
    h->graph_rows = nrows;
    h->graph_launches = nl;
    return GFT_OK;
}

template <class S>
int evolve_impl(gft_handle* h, const LevelPtrs<S>* lv, int n_steps, gft_observables* rows, int max_rows, int* n_rows)
{
    const gft_config& c = h->cfg;
    struct Meta {
        int ti;
        bool e, g;
    };
    std::vector<Meta> meta;
    int nlog = 0;
    for (int s = 0; s < n_steps; s++)
        if (logs_row(c, h->time_iter + s)) nlog++;
    int rc = ensure_rows(h, std::max(nlog, 1));
    if (rc != GFT_OK) return rc;
    const int period = graph_period(h);
    cudaError_t err = cudaSuccess;
    int row = 0;
    for (int s = 0; s < n_steps && err == cudaSuccess;) {
        const int ti = h->time_iter;
        if (period > 0 && ti % period == 0 && n_steps - s >= period && ti >= c.nt_damped) {
            // a whole logging period from the graph (no host launch per kernel)
            if (!h->graph || h->graph_period != period) {
                rc = build_graph<S>(h, lv, ti, period);
                if (rc != GFT_OK) return rc;
            }
            const bool prof = h->profile && h->ev_used < kMaxProfiled;
            if (prof) cudaEventRecord(h->ev[2 * (size_t)h->ev_used], h->stream);
            err = cudaGraphLaunch(h->graph, h->stream);
            if (prof) {
                cudaEventRecord(h->ev[2 * (size_t)h->ev_used + 1], h->stream);
                h->ev_steps[h->ev_used] = period;
                h->ev_used++;
            }
            h->launches += h->graph_launches;
            if (err == cudaSuccess && h->graph_rows > 0)
                err = cudaMemcpyAsync(h->d_rows + (size_t)row * kRowSlots, h->d_graph_rows,
                                      (size_t)h->graph_rows * kRowSlots * sizeof(double), cudaMemcpyDeviceToDevice,
                                      h->stream);
            for (int k = 0; k < period; k++) {
                const int t = ti + k;
                const bool e = c.energy_every > 0 && t % c.energy_every == 0;
                const bool g = c.gauss_every > 0 && t % c.gauss_every == 0;
                if (e || g) {
                    meta.push_back({t, e, g});
                    row++;
                }
            }
            h->time_iter += period;
            s += period;
            continue;
        }
        const bool e = c.energy_every > 0 && ti % c.energy_every == 0;
        const bool g = c.gauss_every > 0 && ti % c.gauss_every == 0;
        std::string why;
        err = issue_step<S>(h, lv, ti, h->d_rows + (size_t)row * kRowSlots, h->profile && h->ev_used < kMaxProfiled,
                            rc, why);
        if (rc != GFT_OK) {
            h->time_iter++;
            return h->fail(rc, "gft_evolve: " + why);
        }
        if (e || g) {
            meta.push_back({ti, e, g});
            row++;
        }
        h->time_iter++;
        s++;
    }
    if (err != cudaSuccess) return h->cuda_fail(err, "gft_evolve(launch)");
    std::vector<double> host((size_t)std::max(row, 1) * kRowSlots);
    unsigned status = 0;
    if (row > 0) err = cudaMemcpyAsync(host.data(), h->d_rows, (size_t)row * kRowSlots * sizeof(double),
                                       cudaMemcpyDeviceToHost, h->stream);
    if (err == cudaSuccess) err = cudaMemcpyAsync(&status, h->d_status, sizeof(unsigned), cudaMemcpyDeviceToHost, h->stream);
    if (err == cudaSuccess) err = cudaMemsetAsync(h->d_status, 0, sizeof(unsigned), h->stream);
    if (err == cudaSuccess && h->comm) {
        // bounded: a peer that is gone must not hold this rank for good
        std::string why;
        const int wrc = slab_comm_wait(h->comm, h->stream, h->comm_timeout_s, why);
        if (wrc != GFT_OK) return h->fail(wrc, "gft_evolve: " + why);
    }
    if (err == cudaSuccess) err = cudaStreamSynchronize(h->stream);
    if (err != cudaSuccess) return h->cuda_fail(err, "gft_evolve");
    if (status & 8u) return h->fail(GFT_E_TIMEOUT, "gft_evolve: a device wait timed out (tensor-copy barrier)");
    const int nw = rows ? std::min(row, std::max(max_rows, 0)) : 0;
    for (int r = 0; r < nw; r++)
        fill_row(&rows[r], meta[r].ti, meta[r].e, meta[r].g, host.data() + (size_t)r * kRowSlots, h->neq);
    if (n_rows) *n_rows = nw;
    return (int)(status & (GFT_W_ASIN_DOMAIN | GFT_W_SQRT_DOMAIN | GFT_W_NONFINITE | GFT_W_RANGE));
}

}  // namespace

int gft::validate_config(const gft_config* c, std::string& why) { return validate(c, why); }
void gft::fill_observables(gft_observables* r, int time_iter, bool e, bool g, const double* v, int neq)
{
    fill_row(r, time_iter, e, g, v, neq);
}
size_t gft::level_bytes_f32(int nsite, int nsc, int hf) { return level_words(nsite, nsc, hf) * sizeof(float); }
void gft::carve_level_f32(void* mem, int nsite, int nsc, LevelPtrs<float>& L, int hf)
{
    carve<float>(mem, nsite, nsc, L, hf);
}
void gft::set_error(const std::string& msg) { set_global_error(msg); }

extern "C" {

int gft_upload_f32(gft_handle* h, const float* sc, const float* ve, int time_iter) { return upload_impl(h, sc, ve, time_iter); }
int gft_upload_f64(gft_handle* h, const double* sc, const double* ve, int time_iter) { return upload_impl(h, sc, ve, time_iter); }
int gft_download_f32(gft_handle* h, float* sc, float* ve) { return download_impl(h, sc, ve); }
int gft_download_f64(gft_handle* h, double* sc, double* ve) { return download_impl(h, sc, ve); }
int gft_upload_device_f32(gft_handle* h, const float* sc, const float* ve, int time_iter)
{
    return upload_impl(h, sc, ve, time_iter, true);
}
int gft_upload_device_f64(gft_handle* h, const double* sc, const double* ve, int time_iter)
{
    return upload_impl(h, sc, ve, time_iter, true);
}
int gft_download_device_f32(gft_handle* h, float* sc, float* ve) { return download_impl(h, sc, ve, true); }
int gft_download_device_f64(gft_handle* h, double* sc, double* ve) { return download_impl(h, sc, ve, true); }

int gft_init_fields(gft_handle* h, const gft_ic* ic)
{
    if (!h || !ic) return GFT_E_INVALID;
    cudaSetDevice(h->cfg.device);
    ICParams p{};
    p.seed = ic->seed;
    for (int k = 0; k < 8; k++) {
        p.mean[k] = ic->mean[k];
        p.sigma[k] = ic->sigma[k];
    }
    p.theta_sigma = ic->theta_sigma;
    p.eps_sigma = ic->eps_sigma;
    p.wall_width = ic->wall_width;
    p.wall_value = ic->wall_value;
    p.x_offset = h->x_offset;
    p.nx_global = h->nx_global;
    p.store_generators = (h->codec.gen && !h->codec.convert) ? 1 : 0;
    const StepParams P = make_params(h, 0, false);
    cudaError_t e = is_f64_storage(h) ? launch_init_fields<double>(P, h->nsc, p, h->ld[0], h->ld[1], h->stream)
                                      : launch_init_fields<float>(P, h->nsc, p, h->lf[0], h->lf[1], h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) return h->cuda_fail(e, "gft_init_fields");
    h->time_iter = 0;
    h->has_data = true;
    return GFT_OK;
}

int gft_evolve(gft_handle* h, int n_steps, gft_observables* rows, int max_rows, int* n_rows)
{
    if (n_rows) *n_rows = 0;
    if (!h) return GFT_E_INVALID;
    if (n_steps < 0) return h->fail(GFT_E_INVALID, "gft_evolve: n_steps must be >= 0");
    if (!h->has_data) return h->fail(GFT_E_STATE, "gft_evolve: upload or initialise the fields first");
    cudaSetDevice(h->cfg.device);
    if (is_f64_storage(h)) return evolve_impl<double>(h, h->ld, n_steps, rows, max_rows, n_rows);
    return evolve_impl<float>(h, h->lf, n_steps, rows, max_rows, n_rows);
}

int gft_observe(gft_handle* h, gft_observables* row)
{
    if (!h || !row) return GFT_E_INVALID;
    if (!h->has_data) return h->fail(GFT_E_STATE, "gft_observe: no field data on the device");
    // Observe = one energy-logging step computed into scratch levels is not
    // side-effect free; instead evaluate with a copy of the past level.
    cudaSetDevice(h->cfg.device);
    const int ti = h->time_iter;
    const int tn = (ti + 1) % 2, tp = 1 - tn;
    const size_t lbytes = level_words(h->nsite, h->nsc, h->hf) * (size_t)h->sbytes;
    int rc = ensure_stage(h, lbytes);
    if (rc != GFT_OK) return rc;
    cudaError_t e = cudaMemcpyAsync(h->d_stage, h->level_mem[tp], lbytes, cudaMemcpyDeviceToDevice, h->stream);
    const StepParams P = make_params(h, ti, true);
    if (e == cudaSuccess) {
        if (is_f64_storage(h)) {
            LevelPtrs<double> tmp;
            carve<double>(h->d_stage, h->nsite, h->nsc, tmp, h->hf);
            e = launch_step<double>(h, P, tn, h->ld[tn], tmp, true);
        } else {
            LevelPtrs<float> tmp;
            carve<float>(h->d_stage, h->nsite, h->nsc, tmp, h->hf);
            e = launch_step<float>(h, P, tn, h->lf[tn], tmp, true);
        }
    }
    // the step wrote into the copy; restore nothing (the levels are untouched)
    if (e == cudaSuccess) e = launch_finalize(h->d_part_e, step_blocks(h, P), kObsCount, kObsCount, h->d_scale, h->d_rows,
                                                  h->d_mid, h->stream);
    std::vector<double> host(kRowSlots, 0.0);
    if (e == cudaSuccess) e = cudaMemcpyAsync(host.data(), h->d_rows, kObsCount * sizeof(double), cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(h->d_status, 0, sizeof(unsigned), h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) return h->cuda_fail(e, "gft_observe");
    fill_row(row, ti, true, false, host.data(), h->neq);
    return GFT_OK;
}

int gft_set_graphs(gft_handle* h, int on)
{
    if (!h) return GFT_E_INVALID;
    drop_graph(h);
    h->use_graphs = on != 0;
    return GFT_OK;
}

int gft_set_wait_limit(gft_handle* h, unsigned long long ns)
{
    if (!h) return GFT_E_INVALID;
    if (ns > 4000000000ull) return h->fail(GFT_E_INVALID, "gft_set_wait_limit: the limit is at most 4 s");
    drop_graph(h);
    h->wait_limit_ns = (unsigned)ns;
    return GFT_OK;
}

int gft_set_kernel(gft_handle* h, int kind, int tile, int march)
{
    if (!h) return GFT_E_INVALID;
    if (kind < 0 || kind > 4 || march < 1) return h->fail(GFT_E_INVALID, "gft_set_kernel: bad kind or march");
    if (kind == 4 && (h->cfg.model != GFT_MODEL_SM || h->cfg.fixed_axes != 0 || h->cfg.ny % kSplitTileY != 0 ||
                      h->cfg.nz % kSplitTileZ != 0))
        return h->fail(GFT_E_UNSUPPORTED,
                       "gft_set_kernel: the split-site step serves the periodic SM model with ny % 8 == 0 and "
                       "nz % 16 == 0");
    if (kind == 3 && (h->cfg.model != GFT_MODEL_SM || h->cfg.fixed_axes != 0 || !tiled_pair_tile(tile)))
        return h->fail(GFT_E_UNSUPPORTED,
                       "gft_set_kernel: two sites per thread serve the periodic SM model in 8 x 32 or 16 x 16 tiles");
    if (kind == 1) {
        drop_graph(h);
        h->kernel_kind = 1;
        return GFT_OK;
    }
    if (kind >= 2 && h->hf != kHfNone)
        return h->fail(GFT_E_UNSUPPORTED, "gft_set_kernel: the tiled kernel has no Higgs-family field");
    // the FP64 form of the SM model takes tiles too (kind 2, and kind 0's automatic choice)
    const bool fp64_sm = h->cfg.form == GFT_FORM_FP64 && h->cfg.model == GFT_MODEL_SM && (kind == 2 || kind == 0);
    if (h->cfg.form != GFT_FORM_MIXED && !fp64_sm) {
        if (kind >= 2)
            return h->fail(GFT_E_UNSUPPORTED,
                           "gft_set_kernel: the tiled kernel serves the mixed form and the FP64 form of the SM model");
        drop_graph(h);
        h->kernel_kind = 0;
        return GFT_OK;
    }
    if (tile < 0 || tile >= kTiledVariants) return h->fail(GFT_E_INVALID, "gft_set_kernel: bad tile index");
    cudaSetDevice(h->cfg.device);
    drop_graph(h);
    const StepParams P = make_params(h, h->time_iter, false);
    if (!tiled_supported(P, tile)) {
        if (kind == 0) {  // automatic: the tile shape chosen at creation, or one thread per site
            h->kernel_kind = 0;
            return GFT_OK;
        }
        return h->fail(GFT_E_UNSUPPORTED, "gft_set_kernel: the lattice shape does not divide into this tile");
    }
    TMaps tm[2], tp[2];
    if (!encode_tiled(h, P, tile, tm, tp))
        return h->fail(GFT_E_UNSUPPORTED, "gft_set_kernel: tensor map encoding failed");
    if (kind == 4) {
        for (int t = 0; t < 2; t++)
            if (!tiled_encode_maps<float>(P, h->lf[t], 1, kSplitTileY, kSplitTileZ, true, &h->tm_split[t]) ||
                !tiled_encode_maps<float>(P, h->lf[t], 1, kSplitTileY, kSplitTileZ, false, &h->tp_split[t]))
                return h->fail(GFT_E_UNSUPPORTED, "gft_set_kernel: tensor map encoding failed (split tile)");
    }
    const int nb = tiled_blocks(P, tile, march);
    if (nb > h->part_cap) {
        cudaStreamSynchronize(h->stream);
        double* pe = nullptr;
        if (cudaMalloc(&pe, (size_t)nb * kObsCount * sizeof(double)) != cudaSuccess)
            return h->fail(GFT_E_NOMEM, "gft_set_kernel: partials allocation failed");
        cudaFree(h->d_part_e);
        h->d_part_e = pe;
        h->dev_bytes += (size_t)(nb - h->part_cap) * kObsCount * sizeof(double);
        h->part_cap = nb;
    }
    h->tm[0] = tm[0];
    h->tm[1] = tm[1];
    h->tp[0] = tp[0];
    h->tp[1] = tp[1];
    h->tiled_ready = true;
    h->tile_variant = tile;
    h->march = march;
    h->kernel_kind = kind;
    return GFT_OK;
}

int gft_selftest_math(int device, double* out)
{
    if (!out) return GFT_E_INVALID;
    cudaError_t e = cudaSetDevice(device);
    if (e == cudaSuccess) e = run_math_selftest(1 << 22, out);
    if (e != cudaSuccess) {
        set_global_error(std::string("gft_selftest_math: ") + cudaGetErrorString(e));
        return GFT_E_CUDA;
    }
    return GFT_OK;
}

double gft_step_kernel_ms(gft_handle* h, int* launches)
{
    if (launches) *launches = 0;
    if (!h || h->ev_used == 0) return 0.0;
    cudaEventSynchronize(h->ev[2 * (size_t)h->ev_used - 1]);
    double total = 0.0;
    int n = 0;
    for (int i = 0; i < h->ev_used; i++) {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, h->ev[2 * (size_t)i], h->ev[2 * (size_t)i + 1]);
        total += ms;
        n += h->ev_steps[i];
    }
    h->ev_used = 0;
    if (launches) *launches = n;
    return total / n;
}

long long gft_launch_count(const gft_handle* h) { return h ? h->launches : 0; }

int gft_local_fields(gft_handle* h, float* energy, float* gauss, int* energy_step, int* gauss_step)
{
    if (!h) return GFT_E_INVALID;
    if (energy_step) *energy_step = h->loc_e_step;
    if (gauss_step) *gauss_step = h->loc_g_step;
    if ((energy && !h->d_loc_e) || (gauss && !h->d_loc_g))
        return h->fail(GFT_E_STATE, "gft_local_fields: no local-output cadence was configured for that analyser");
    cudaSetDevice(h->cfg.device);
    cudaError_t e = cudaSuccess;
    if (energy)
        e = cudaMemcpyAsync(energy, h->d_loc_e, (size_t)h->nsite * 6 * sizeof(float), cudaMemcpyDeviceToHost, h->stream);
    if (gauss && e == cudaSuccess)
        e = cudaMemcpyAsync(gauss, h->d_loc_g, (size_t)h->nsite * h->neq * sizeof(float), cudaMemcpyDeviceToHost,
                            h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) return h->cuda_fail(e, "gft_local_fields");
    return GFT_OK;
}

int gft_set_slab(gft_handle* h, int x_offset, int nx_global, int x_begin, int x_end)
{
    if (!h) return GFT_E_INVALID;
    const int nx = h->cfg.nx;
    if (nx_global < 1 || x_begin < 0 || x_end > nx || x_begin >= x_end)
        return h->fail(GFT_E_INVALID, "gft_set_slab: need 0 <= x_begin < x_end <= nx and nx_global >= 1");
    if (h->cfg.fixed_axes & 1)
        return h->fail(GFT_E_UNSUPPORTED, "gft_set_slab: x-slabs need a periodic x axis (Fixed x faces given)");
    drop_graph(h);
    h->x_offset = x_offset;
    h->nx_global = nx_global;
    h->x_begin = x_begin;
    h->x_end = x_end;
    // means over this handle's own sites
    gft_config c = h->cfg;
    c.nx = x_end - x_begin;
    double scale[kRowSlots];
    row_scales(c, c.nx * c.ny * c.nz, scale);
    cudaSetDevice(h->cfg.device);
    cudaStreamSynchronize(h->stream);
    cudaError_t e = cudaMemcpy(h->d_scale, scale, sizeof(scale), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return h->cuda_fail(e, "gft_set_slab");
    return GFT_OK;
}

int gft_nccl_unique_id(unsigned char* id)
{
    if (!id) return GFT_E_INVALID;
    std::string why;
    const int rc = nccl_unique_id(id, why);
    if (rc != GFT_OK) set_global_error("gft_nccl_unique_id: " + why);
    return rc;
}

int gft_set_slab_nccl(gft_handle* h, const unsigned char* id, int nranks, int rank, double timeout_s)
{
    if (!h) return GFT_E_INVALID;
    if (!id || nranks < 1 || rank < 0 || rank >= nranks || !(timeout_s > 0))
        return h->fail(GFT_E_INVALID, "gft_set_slab_nccl: need an id, 0 <= rank < nranks and a positive timeout");
    if (h->x_end == 0 || h->x_begin != 1 || h->x_end != h->cfg.nx - 1)
        return h->fail(GFT_E_STATE, "gft_set_slab_nccl: call gft_set_slab first, with one ghost plane on each side");
    if (h->exchange) return h->fail(GFT_E_STATE, "gft_set_slab_nccl: an exchange callback is set");
    if (h->comm) return h->fail(GFT_E_STATE, "gft_set_slab_nccl: the exchange is already set up");
    cudaSetDevice(h->cfg.device);
    cudaError_t e = cudaSuccess;
    int prio_lo = 0, prio_hi = 0;  // the boundary planes' kernels ahead of the interior's CTAs
    if (!h->comm_stream && (e = cudaDeviceGetStreamPriorityRange(&prio_lo, &prio_hi)) == cudaSuccess)
        e = cudaStreamCreateWithPriority(&h->comm_stream, cudaStreamNonBlocking, prio_hi);
    if (e == cudaSuccess && !h->ev_bound) e = cudaEventCreateWithFlags(&h->ev_bound, cudaEventDisableTiming);
    if (e == cudaSuccess && !h->ev_comm) e = cudaEventCreateWithFlags(&h->ev_comm, cudaEventDisableTiming);
    if (e != cudaSuccess) return h->cuda_fail(e, "gft_set_slab_nccl");
    std::string why;
    SlabComm* c = nullptr;
    const int rc = slab_comm_create(id, nranks, rank, &c, why);
    if (rc != GFT_OK) return h->fail(rc, "gft_set_slab_nccl: " + why);
    drop_graph(h);
    h->comm = c;
    h->comm_timeout_s = timeout_s;
    return GFT_OK;
}

int gft_set_exchange(gft_handle* h, gft_exchange_fn fn, void* user)
{
    if (!h) return GFT_E_INVALID;
    if (fn && h->comm) return h->fail(GFT_E_STATE, "gft_set_exchange: the NCCL exchange of gft_set_slab_nccl is set");
    drop_graph(h);
    h->exchange = fn;
    h->exchange_user = user;
    return GFT_OK;
}

int gft_level_planes(gft_handle* h, int level, int x, void** ptrs, size_t* bytes, int max)
{
    if (!h || level < 0 || level > 1 || x < 0 || x >= h->cfg.nx || !ptrs || !bytes) return GFT_E_INVALID;
    const int n = 7 + (h->nsc == 8 ? 1 : 0) + (h->hf != kHfNone ? 3 : 0);
    if (max < n) return h->fail(GFT_E_INVALID, "gft_level_planes: need room for " + std::to_string(n) + " arrays");
    const size_t plane = (size_t)h->cfg.ny * h->cfg.nz;
    const size_t w = (size_t)h->sbytes;
    int k = 0;
    if (h->sbytes == 4) {
        const LevelPtrs<float>& L = h->lf[level];
        for (int d = 0; d < 3; d++, k++) { ptrs[k] = L.q[d] + 4 * plane * x; bytes[k] = 4 * plane * w; }
        for (int d = 0; d < 3; d++, k++) { ptrs[k] = L.th[d] + plane * x; bytes[k] = plane * w; }
        for (int db = 0; db < h->nsc / 4; db++, k++) { ptrs[k] = L.ph[db] + 4 * plane * x; bytes[k] = 4 * plane * w; }
        for (int d = 0; d < 3 && h->hf == kHfU1; d++, k++) { ptrs[k] = L.hth[d] + plane * x; bytes[k] = plane * w; }
        for (int d = 0; d < 3 && h->hf == kHfSU2; d++, k++) { ptrs[k] = L.hq[d] + 4 * plane * x; bytes[k] = 4 * plane * w; }
    } else {
        const LevelPtrs<double>& L = h->ld[level];
        for (int d = 0; d < 3; d++, k++) { ptrs[k] = L.q[d] + 4 * plane * x; bytes[k] = 4 * plane * w; }
        for (int d = 0; d < 3; d++, k++) { ptrs[k] = L.th[d] + plane * x; bytes[k] = plane * w; }
        for (int db = 0; db < h->nsc / 4; db++, k++) { ptrs[k] = L.ph[db] + 4 * plane * x; bytes[k] = 4 * plane * w; }
        for (int d = 0; d < 3 && h->hf == kHfU1; d++, k++) { ptrs[k] = L.hth[d] + plane * x; bytes[k] = plane * w; }
        for (int d = 0; d < 3 && h->hf == kHfSU2; d++, k++) { ptrs[k] = L.hq[d] + 4 * plane * x; bytes[k] = 4 * plane * w; }
    }
    return n;
}

const char* gft_step_kernel_name(const gft_handle* h)
{
    if (!h) return "";
    if (h->cfg.form == GFT_FORM_REF) return "ref_step_kernel";
    const StepParams P = make_params(h, 0, false);
    if (!use_tiled(h, P)) return "fast_step_kernel";
    if (use_split(h, P)) return "tiled_split_kernel";
    return use_pair(h, P) ? "tiled_pair_kernel" : "tiled_step_kernel";
}

}  // extern "C"
