// gft_ensemble.cu -- an ensemble of independent lattices (realisations with
// their own seeds, couplings and sizes) evolved together on one GPU.
//
// The reference evolves one lattice per process (Lattice::evolve,
// Core/Source/Lattice.cpp:755-876); an ensemble of realisations is a loop of
// processes.  Here every member's step is one work list of tiles -- (member,
// y0, z0, x0) of the TMA-staged pipeline of gft_tiled_tile.cuh -- consumed by
// ONE persistent launch per time step: a grid of (SMs x resident CTAs) that
// strides over the list, so small members do not leave the GPU idle and the
// launch count does not grow with the number of members.  Members' step
// parameters and level pointers travel as kernel parameters (up to kGroup
// members per launch); their tensor maps live in global memory.
//
// Logging steps add a Gauss kernel over the same tiles and one reduction
// kernel that writes one observables row per member.  A whole logging period
// of launches is captured once in a CUDA graph and replayed.  The tile shape
// and the x-march depth are chosen by gft_batch_autotune, which times every
// candidate on the ensemble itself and restores the fields afterwards.
#include <algorithm>
#include <array>
#include <cstring>
#include <numeric>
#include <string>
#include <vector>

#include "gft.h"
#include "gft_launch.h"
#include "gft_reduce.cuh"
#include "gft_tiled_tile.cuh"

namespace gft {
namespace {

using namespace tiled;

constexpr int kGroup = 64;  // members per launch: their parameters are kernel parameters

// A member's level arrays (the ensemble runs gaugeNum-4 models: no Higgs-family
// arrays, so the kernel-parameter copy omits those pointers).  The step and
// Gauss bodies read them from the parameter space in place.
struct EnsLevel {
    float* q[3];
    float* th[3];
    float* ph[2];
    EnsLevel& operator=(const LevelPtrs<float>& L)
    {
        for (int d = 0; d < 3; d++) {
            q[d] = L.q[d];
            th[d] = L.th[d];
        }
        ph[0] = L.ph[0];
        ph[1] = L.ph[1];
        return *this;
    }
};

struct EnsParams {
    StepParams P[kGroup];
    EnsLevel lv[kGroup][2];
    // Members with the same physics parameters (the usual ensemble: own seeds and
    // sizes, shared couplings): their common StepParams and float constants, read
    // as by-value kernel parameters (constant operands) instead of through the
    // member index.
    StepParams common;
    FConst fcommon;
};
// Kernel parameter space (sm_70 and later, CUDA 12.1+): 32,764 bytes; the kernel's
// other parameters take 48.
static_assert(sizeof(EnsParams) + 64 <= 32764, "ensemble parameters exceed the kernel parameter space");

// Tensor maps of one member (global memory, 64-byte aligned by CUtensorMap).
struct EnsMaps {
    TMaps tm[2];  // staged "now" planes when level t is "now"
    TMaps tp[2];  // past-level prefetch boxes of level t
};

__device__ __forceinline__ void tmap_acquire(const TMaps& m)
{
    // the descriptors were written by a host copy before the launch; order them
    // with this CTA's tensor copies (cheap, once per tile)
#pragma unroll
    for (int d = 0; d < 3; d++) {
        asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"(&m.q[d]) : "memory");
        asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"(&m.th[d]) : "memory");
    }
#pragma unroll
    for (int k = 0; k < 2; k++)
        asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"(&m.ph[k]) : "memory");
}

// One persistent launch per step.  CTA b evolves the tiles of its list,
// order[start[b]] .. order[start[b + 1] - 1] (balanced by the host: tile costs
// differ with the planes of the x-chunk), when the grid has the list count
// nlist; otherwise tiles b, b + G, b + 2G, ...  items[i] = {member within the
// group, y0, z0, x0}; tile i's energy partials go to partials row i.  UNIFORM:
// the members share ep.common but for their geometry (the per-member fields
// copied below).
// Plain steps stage the wrapped halo sites (run_tile's STAGE) where the staging
// area leaves the resident CTAs per SM unchanged; the dynamic shared memory
// then includes it.
template <int MODEL, int TY, int TZ, bool ENERGY>
constexpr bool ens_stage()
{
    return !ENERGY && HaloStage<float, TY, TZ, (MODEL == kModelSM) ? 1 : 2>::kUse;
}
template <int MODEL, int TY, int TZ, bool ENERGY>
constexpr int ens_smem()
{
    constexpr int ND = (MODEL == kModelSM) ? 1 : 2;
    return ens_stage<MODEL, TY, TZ, ENERGY>() ? HaloStage<float, TY, TZ, ND>::SMEM : Geom<float, TY, TZ, ND>::SMEM;
}

template <int MODEL, int TY, int TZ, bool ENERGY, bool UNIFORM>
__global__ void __launch_bounds__(TY * TZ, 512 / (TY * TZ))
    ensemble_step_kernel(const __grid_constant__ EnsParams ep, const EnsMaps* __restrict__ maps,
                         const int4* __restrict__ items, int nitems, const int* __restrict__ order,
                         const int* __restrict__ start, int nlist, int lx, int tn, unsigned* status,
                         double* partials)
{
    constexpr int ND = (MODEL == kModelSM) ? 1 : 2;
    using G = Geom<float, TY, TZ, ND>;
    extern __shared__ unsigned char smem_raw[];
    unsigned char* smem =
        reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 127) & ~(uintptr_t)127);
    unsigned long long* bars = reinterpret_cast<unsigned long long*>(smem + G::NBUF * G::BUF);
    const int tid = threadIdx.y * TZ + threadIdx.x;

    __shared__ int s_abort;
    if (tid == 0) {
        s_abort = 0;
        for (int b = 0; b < G::NBUF; b++) mbar_init(&bars[b], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();

    RingPhase ring = {0u};
    unsigned warn = 0;
    const bool listed = order != nullptr && (int)gridDim.x == nlist;
    const int k0 = listed ? start[blockIdx.x] : (int)blockIdx.x;
    const int k1 = listed ? start[blockIdx.x + 1] : nitems;
    const int kstep = listed ? 1 : (int)gridDim.x;
    for (int k = k0; k < k1; k += kstep) {
        const int it = listed ? order[k] : k;
        const int4 w = items[it];
        const int m = w.x;
        const EnsMaps& mp = maps[m];
        if (tid == 0) {
            tmap_acquire(mp.tm[tn]);
            tmap_acquire(mp.tp[1 - tn]);
        }
        double obs[kObsCount];
#pragma unroll
        for (int k = 0; k < kObsCount; k++) obs[k] = 0.0;
        StepParams Pu;
        if constexpr (UNIFORM) {
            Pu = ep.common;
            const StepParams& Pm = ep.P[m];
            Pu.nx = Pm.nx;
            Pu.ny = Pm.ny;
            Pu.nz = Pm.nz;
            Pu.nsite = Pm.nsite;
            Pu.obs_x0 = Pm.obs_x0;
            Pu.obs_x1 = Pm.obs_x1;
            Pu.fixed_axes = Pm.fixed_axes;
        }
        const StepParams& P = UNIFORM ? Pu : ep.P[m];
        FConst Fm;
        if constexpr (!UNIFORM) Fm = make_fconst(P);
        const FConst& F = UNIFORM ? ep.fcommon : Fm;
        const bool ok = run_tile<float, MODEL, TY, TZ, ENERGY, EnsLevel, ens_stage<MODEL, TY, TZ, ENERGY>()>(
            mp.tm[tn], mp.tp[1 - tn], P, F, ep.lv[m][tn], ep.lv[m][1 - tn], w.y, w.z, w.w, min(lx, P.nx - w.w), smem,
            bars, ring, &s_abort, obs, warn, smem + HaloStage<float, TY, TZ, ND>::OFFSET);
        if (!ok) {
            if (tid == 0) atomicOr(status, kErrTimeout);
            break;
        }
        if (ENERGY) {
            energy_total(obs);
            block_reduce_store<kObsCount>(obs, partials + (size_t)it * kObsCount, kObsCount);
        }
        __syncthreads();  // the reduction scratch and the plane ring are reused by the next tile
    }
    if (warn) atomicOr(status, warn);
}

// Gauss-law residual over the same tiles: CTA (tile, i) takes plane i of the
// tile's x-chunk, one thread per site (independent loads; a march of the
// chunk's planes per thread serialises them: 0.948 against 0.866 ms on the
// 64-member benchmark with 16 x 16 tiles, march 64), and writes partial row
// tile * gridDim.y + i (zeros past the chunk's end).
template <int MODEL, int TY, int TZ>
__global__ void __launch_bounds__(TY * TZ) ensemble_gauss_kernel(const __grid_constant__ EnsParams ep,
                                                                 const int4* __restrict__ items, int lx, int tn,
                                                                 double* partials)
{
    const int it = blockIdx.x, i = blockIdx.y;
    const int4 w = items[it];
    const int m = w.x;
    const StepParams& P = ep.P[m];
    const int y = w.y + threadIdx.y, z = w.z + threadIdx.x;
    const int ym = (y == 0) ? P.ny - 1 : y - 1, zm = (z == 0) ? P.nz - 1 : z - 1;
    double v[kGaussSlots];
#pragma unroll
    for (int k = 0; k < kGaussSlots; k++) v[k] = 0.0;
    const int x = w.w + i, xm = (x == 0) ? P.nx - 1 : x - 1;
    if (i < min(lx, P.nx - w.w) && counts(P, x) && !frozen(P, x, y, z)) {
        gauss_site<float, MODEL>(P, ep.lv[m][tn], ep.lv[m][1 - tn], (x * P.ny + y) * P.nz + z,
                                 (xm * P.ny + y) * P.nz + z, (x * P.ny + ym) * P.nz + z, (x * P.ny + y) * P.nz + zm,
                                 v);
    }
    block_reduce_store<kGaussSlots>(v, partials + ((size_t)it * gridDim.y + i) * kGaussSlots, 4);
}

// One block per member: reduce its tiles' partial rows [first[m] * rpt,
// first[m+1] * rpt) (rpt rows per tile) into slots [off, off + nslots) of its
// observables row.
__global__ void __launch_bounds__(kFinThreads) ensemble_finalize_kernel(const double* __restrict__ partials,
                                                                        const int* __restrict__ first, int rpt,
                                                                        int nslots, int max_from,
                                                                        const double* scales, int off, double* rows)
{
    const int m = blockIdx.x;
    const double t = reduce_rows_block(partials, first[m] * rpt, first[m + 1] * rpt, nslots, max_from);
    if (threadIdx.x < (unsigned)nslots) {
        const size_t o = (size_t)m * kRowSlotCount + off + threadIdx.x;
        rows[o] = t * scales[o];
    }
}

// Resident CTAs per SM of a step-kernel instance (also sets its shared-memory
// limit); evaluated outside any stream capture, by configure().
template <int MODEL, int TY, int TZ, bool ENERGY, bool UNIFORM>
int resident_ctas()
{
    constexpr int SMEM = ens_smem<MODEL, TY, TZ, ENERGY>();
    static int per_sm = 0;
    if (per_sm == 0) {
        auto k = ensemble_step_kernel<MODEL, TY, TZ, ENERGY, UNIFORM>;
        cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM);
        int n = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k, TY * TZ, SMEM) != cudaSuccess || n < 1) n = 1;
        per_sm = n;
    }
    return per_sm;
}

// A group's tiles and their per-CTA lists (balance_tiles): CTA c of a grid of
// nlist evolves items[order[k]] for k in [start[c], start[c + 1]).
struct GroupTiles {
    const int4* items;
    int nitems;
    const int* order;
    const int* start;
    int nlist;
};

template <int MODEL, int TY, int TZ, bool ENERGY, bool UNIFORM>
cudaError_t launch_step_u(const EnsParams& ep, const EnsMaps* maps, const GroupTiles& gt, int lx, int tn,
                          unsigned* status, double* partials, int nsm, cudaStream_t s)
{
    const int grid = std::min(gt.nitems, nsm * resident_ctas<MODEL, TY, TZ, ENERGY, UNIFORM>());
    if (grid < 1) return cudaSuccess;
    ensemble_step_kernel<MODEL, TY, TZ, ENERGY, UNIFORM><<<grid, dim3(TZ, TY, 1), ens_smem<MODEL, TY, TZ, ENERGY>(), s>>>(
        ep, maps, gt.items, gt.nitems, gt.order, gt.start, gt.nlist, lx, tn, status, partials);
    return cudaGetLastError();
}

template <int MODEL, int TY, int TZ, bool ENERGY>
cudaError_t launch_step_t(bool uniform, const EnsParams& ep, const EnsMaps* maps, const GroupTiles& gt, int lx,
                          int tn, unsigned* status, double* partials, int nsm, cudaStream_t s)
{
    return uniform ? launch_step_u<MODEL, TY, TZ, ENERGY, true>(ep, maps, gt, lx, tn, status, partials, nsm, s)
                   : launch_step_u<MODEL, TY, TZ, ENERGY, false>(ep, maps, gt, lx, tn, status, partials, nsm, s);
}

template <int MODEL, int TY, int TZ>
void prime_tile()
{
    resident_ctas<MODEL, TY, TZ, false, false>();
    resident_ctas<MODEL, TY, TZ, true, false>();
    resident_ctas<MODEL, TY, TZ, false, true>();
    resident_ctas<MODEL, TY, TZ, true, true>();
}

template <int MODEL>
void prime_variant(int variant)
{
    switch (variant) {
    case 0: prime_tile<MODEL, 8, 32>(); break;
    case 1: prime_tile<MODEL, 4, 32>(); break;
    case 2: prime_tile<MODEL, 4, 16>(); break;
    default: prime_tile<MODEL, 16, 16>(); break;
    }
}

// Resident CTAs per SM of the plain-step (uniform) instance of a tile shape.
template <int MODEL>
int resident_m(int variant)
{
    switch (variant) {
    case 0: return resident_ctas<MODEL, 8, 32, false, true>();
    case 1: return resident_ctas<MODEL, 4, 32, false, true>();
    case 2: return resident_ctas<MODEL, 4, 16, false, true>();
    default: return resident_ctas<MODEL, 16, 16, false, true>();
    }
}

template <int MODEL, int TY, int TZ>
cudaError_t launch_gauss_t(const EnsParams& ep, const int4* items, int nitems, int lx, int rows, int tn,
                           double* partials, cudaStream_t s)
{
    if (nitems < 1) return cudaSuccess;
    ensemble_gauss_kernel<MODEL, TY, TZ><<<dim3(nitems, rows, 1), dim3(TZ, TY, 1), 0, s>>>(ep, items, lx, tn, partials);
    return cudaGetLastError();
}

template <int MODEL>
cudaError_t launch_step_m(int variant, bool energy, bool uniform, const EnsParams& ep, const EnsMaps* maps,
                          const GroupTiles& gt, int lx, int tn, unsigned* status, double* partials, int nsm,
                          cudaStream_t s)
{
#define GFT_ENS_STEP(TY, TZ)                                                                                    \
    return energy ? launch_step_t<MODEL, TY, TZ, true>(uniform, ep, maps, gt, lx, tn, status, partials, nsm, s) \
                  : launch_step_t<MODEL, TY, TZ, false>(uniform, ep, maps, gt, lx, tn, status, partials, nsm, s)
    switch (variant) {
    case 0: GFT_ENS_STEP(8, 32);
    case 1: GFT_ENS_STEP(4, 32);
    case 2: GFT_ENS_STEP(4, 16);
    default: GFT_ENS_STEP(16, 16);
    }
#undef GFT_ENS_STEP
}

template <int MODEL>
cudaError_t launch_gauss_m(int variant, const EnsParams& ep, const int4* items, int nitems, int lx, int rows, int tn,
                           double* partials, cudaStream_t s)
{
    switch (variant) {
    case 0: return launch_gauss_t<MODEL, 8, 32>(ep, items, nitems, lx, rows, tn, partials, s);
    case 1: return launch_gauss_t<MODEL, 4, 32>(ep, items, nitems, lx, rows, tn, partials, s);
    case 2: return launch_gauss_t<MODEL, 4, 16>(ep, items, nitems, lx, rows, tn, partials, s);
    default: return launch_gauss_t<MODEL, 16, 16>(ep, items, nitems, lx, rows, tn, partials, s);
    }
}

constexpr int kMaxGraphPeriod = 256;

int gcd_i(int a, int b) { return b == 0 ? a : gcd_i(b, a % b); }
int lcm_i(int a, int b) { return a / gcd_i(a, b) * b; }

}  // namespace
}  // namespace gft

using namespace gft;

struct gft_batch {
    int n = 0;
    int model = GFT_MODEL_SM;
    int device = 0;
    int nsc = 4;
    int hf = kHfNone;  // 2HDM Higgs-family field shared by every member (then one launch per member and step)
    int nve = 15;      // link words per site in the reference layout (15, 18 or 27)
    int neq = 4;       // Gauss constraints per row (gaugeNum)
    // family ensembles: per-member partial rows (reused member after member on the stream) and
    // the two-stage reduction scratch
    double* d_part_f = nullptr;
    double* d_mid = nullptr;
    int nsm = 148;
    std::vector<gft_config> cfg;
    std::vector<int> nsite;
    std::vector<size_t> level_off;  // byte offset of each member's level 0 in the arena (level 1 follows)
    size_t level_bytes_total = 0;
    void* arena = nullptr;
    size_t arena_bytes = 0;
    std::vector<std::array<LevelPtrs<float>, 2>> lv;
    EnsMaps* d_maps = nullptr;
    int variant = -1;
    int lx = 32;
    int4* d_items = nullptr;
    int nitems = 0;
    int* d_order = nullptr;       // per-CTA tile lists of each group (group-local item indices)
    int* d_start = nullptr;       // list bounds: group g's nlist + 1 entries from group_start[g]
    std::vector<int> group_start, group_nlist;
    std::vector<int> group_item;  // first item of each group (+ end)
    int* d_first = nullptr;       // first item of each member (+ end)
    double* d_part_e = nullptr;
    double* d_part_g = nullptr;
    int part_cap = 0;           // tiles the energy partials hold
    long long part_cap_g = 0;   // rows the Gauss partials hold (tiles x gauss_rows)
    int gauss_rows = 32;        // Gauss partial rows per tile: planes of the longest chunk, min(lx, max nx)
    double* d_scale = nullptr;  // [n][kRowSlotCount]
    double* d_rows = nullptr;   // [rows_cap][n][kRowSlotCount]
    int rows_cap = 0;
    unsigned* d_status = nullptr;
    void* d_stage = nullptr;
    size_t stage_bytes = 0;
    cudaStream_t stream = nullptr;
    int time_iter = 0;
    bool has_data = false;
    long long launches = 0;
    std::string err;
    // CUDA graph of one logging period
    bool use_graphs = true;
    cudaGraphExec_t graph = nullptr;
    int graph_period = 0;
    int graph_rows = 0;       // logging rows the period writes
    long long graph_launches = 0;
    double* d_graph_rows = nullptr;
    int graph_rows_cap = 0;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    double last_ms = 0.0;

    int fail(int code, const std::string& m)
    {
        err = m;
        set_error(m);
        return code;
    }
    int cuda_fail(cudaError_t e, const char* what) { return fail(GFT_E_CUDA, std::string(what) + ": " + cudaGetErrorString(e)); }
    int ngroups() const { return (n + kGroup - 1) / kGroup; }
};

namespace {

void tile_of(int variant, int& ty, int& tz) { tiled_tile(variant, ty, tz); }

bool variant_fits(const gft_batch* b, int v)
{
    int ty, tz;
    tile_of(v, ty, tz);
    for (int m = 0; m < b->n; m++)
        if (b->cfg[m].ny % ty != 0 || b->cfg[m].nz % tz != 0) return false;
    return true;
}

void drop_graph(gft_batch* b)
{
    if (b->graph) cudaGraphExecDestroy(b->graph);
    b->graph = nullptr;
    b->graph_period = 0;
}

// Every StepParams field except the geometry ones (nx, ny, nz, nsite, obs_x0,
// obs_x1, fixed_axes) equal, compared field by field (the struct has padding).
bool same_physics(const StepParams& a, const StepParams& b)
{
    auto eq = [](const double* x, const double* y, int n) {
        for (int k = 0; k < n; k++)
            if (std::memcmp(&x[k], &y[k], sizeof(double)) != 0) return false;
        return true;
    };
    const double da[] = {a.dt, a.dt2, a.inv_sqr_dt, a.inv_g_sqr, a.inv_gp_sqr, a.gsq_hf, a.inv_gpp_sqr, a.div_tol,
                         a.damping_step, a.lambda, a.eta_sqr, a.m1, a.m2, a.l1, a.l2, a.l3, a.m12r, a.l4p5, a.l6r,
                         a.l7r, a.m12i, a.l4m5, a.l5i, a.l6i, a.l7i, a.energy_offset};
    const double db[] = {b.dt, b.dt2, b.inv_sqr_dt, b.inv_g_sqr, b.inv_gp_sqr, b.gsq_hf, b.inv_gpp_sqr, b.div_tol,
                         b.damping_step, b.lambda, b.eta_sqr, b.m1, b.m2, b.l1, b.l2, b.l3, b.m12r, b.l4p5, b.l6r,
                         b.l7r, b.m12i, b.l4m5, b.l5i, b.l6i, b.l7i, b.energy_offset};
    return eq(da, db, (int)(sizeof(da) / sizeof(double))) && eq(a.lap, b.lap, 3) && eq(a.inv_dx, b.inv_dx, 3) &&
           eq(a.gsq, b.gsq, 4) && a.hf == b.hf && a.gen == b.gen && a.loc_energy == b.loc_energy &&
           a.loc_gauss == b.loc_gauss && a.break_son == b.break_son && a.break_uhalfn == b.break_uhalfn &&
           a.apply_norm == b.apply_norm && a.store_energy == b.store_energy;
}

// Fills the group's parameters; returns whether its members share everything
// but their geometry (then ep->common holds member 0's values, whose geometry
// fields the kernel replaces by each member's).
bool fill_params(const gft_batch* b, int g, int ti, bool energy, EnsParams* ep)
{
    std::memset(ep, 0, sizeof(*ep));
    bool uniform = true;
    for (int j = 0; j < kGroup; j++) {
        const int m = g * kGroup + j;
        if (m >= b->n) break;
        ep->P[j] = config_params(b->cfg[m], b->nsite[m], false, ti, energy);
        ep->lv[j][0] = b->lv[m][0];
        ep->lv[j][1] = b->lv[m][1];
        if (j == 0) {
            ep->common = ep->P[0];
            ep->fcommon = make_fconst(ep->P[0]);
        }
        else if (!same_physics(ep->P[j], ep->common))
            uniform = false;
    }
    return uniform;
}

// Per-CTA tile lists of one group for a grid of G CTAs: the tiles by
// decreasing cost, each to the CTA with the least work so far (cost: the planes
// of its x-chunk plus three for filling the plane ring), then each CTA's tiles
// in item order.  Static striding over tiles of uneven x-chunks (a 48-plane
// member in chunks of 32 and 16) leaves the busiest CTA 13 % above the mean on
// the 64-member benchmark; these lists bring it within 1 %.
void balance_tiles(const std::vector<int4>& items, int i0, int ni, const std::vector<gft_config>& cfg, int m0, int lx,
                   int G, std::vector<int>& order, std::vector<int>& start)
{
    std::vector<int> cost(ni), idx(ni);
    for (int i = 0; i < ni; i++) {
        const int4 w = items[i0 + i];
        cost[i] = std::min(lx, cfg[m0 + w.x].nx - w.w) + 3;
        idx[i] = i;
    }
    std::stable_sort(idx.begin(), idx.end(), [&](int a, int c) { return cost[a] > cost[c]; });
    std::vector<long long> load(G, 0);
    std::vector<std::vector<int>> lists(G);
    for (int i : idx) {
        const int c = (int)(std::min_element(load.begin(), load.end()) - load.begin());
        load[c] += cost[i];
        lists[c].push_back(i);
    }
    start.assign(1, (int)order.size());
    for (auto& l : lists) {
        std::sort(l.begin(), l.end());
        order.insert(order.end(), l.begin(), l.end());
        start.push_back((int)order.size());
    }
}

// Tile list, tensor maps and partial buffers for a tile shape and march depth.
int configure(gft_batch* b, int variant, int lx)
{
    int ty, tz;
    tile_of(variant, ty, tz);
    std::vector<int4> items;
    std::vector<int> first(b->n + 1, 0);
    b->group_item.assign(b->ngroups() + 1, 0);
    for (int m = 0; m < b->n; m++) {
        if (m % kGroup == 0) b->group_item[m / kGroup] = (int)items.size();
        first[m] = (int)items.size();
        const gft_config& c = b->cfg[m];
        for (int x0 = 0; x0 < c.nx; x0 += lx)
            for (int y0 = 0; y0 < c.ny; y0 += ty)
                for (int z0 = 0; z0 < c.nz; z0 += tz) items.push_back(make_int4(m % kGroup, y0, z0, x0));
    }
    first[b->n] = (int)items.size();
    b->group_item[b->ngroups()] = (int)items.size();
    std::vector<EnsMaps> maps(b->n);
    for (int m = 0; m < b->n; m++) {
        const StepParams P = config_params(b->cfg[m], b->nsite[m], false, 0, false);
        for (int t = 0; t < 2; t++) {
            if (!tiled_encode_maps<float>(P, b->lv[m][t], b->nsc / 4, ty, tz, true, &maps[m].tm[t]) ||
                !tiled_encode_maps<float>(P, b->lv[m][t], b->nsc / 4, ty, tz, false, &maps[m].tp[t]))
                return b->fail(GFT_E_UNSUPPORTED, "gft_batch: tensor map encoding failed");
        }
    }
    cudaStreamSynchronize(b->stream);
    cudaFree(b->d_items);
    cudaFree(b->d_first);
    b->d_items = nullptr;
    b->d_first = nullptr;
    cudaError_t e = cudaMalloc(&b->d_items, items.size() * sizeof(int4));
    if (e == cudaSuccess) e = cudaMalloc(&b->d_first, first.size() * sizeof(int));
    if (e == cudaSuccess) e = cudaMemcpy(b->d_items, items.data(), items.size() * sizeof(int4), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(b->d_first, first.data(), first.size() * sizeof(int), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(b->d_maps, maps.data(), maps.size() * sizeof(EnsMaps), cudaMemcpyHostToDevice);
    // energy partials: a row per tile; Gauss partials: a row per tile and plane of its chunk
    int maxnx = 1;
    for (const auto& c : b->cfg) maxnx = std::max(maxnx, c.nx);
    const int grows = std::min(lx, maxnx);
    if (e == cudaSuccess && ((int)items.size() > b->part_cap || (long long)items.size() * grows > b->part_cap_g)) {
        cudaFree(b->d_part_e);
        cudaFree(b->d_part_g);
        b->d_part_e = b->d_part_g = nullptr;
        e = cudaMalloc(&b->d_part_e, items.size() * kObsCount * sizeof(double));
        if (e == cudaSuccess) e = cudaMalloc(&b->d_part_g, items.size() * (size_t)grows * kGaussSlots * sizeof(double));
        b->part_cap = (e == cudaSuccess) ? (int)items.size() : 0;
        b->part_cap_g = (e == cudaSuccess) ? (long long)items.size() * grows : 0;
    }
    b->gauss_rows = grows;
    if (e != cudaSuccess) return b->cuda_fail(e, "gft_batch: configure");
    b->nitems = (int)items.size();
    b->variant = variant;
    b->lx = lx;
    if (b->model == GFT_MODEL_SM)
        prime_variant<kModelSM>(variant);
    else
        prime_variant<kModel2HDM>(variant);
    // per-CTA lists for the plain-step grid (a launch with another grid strides)
    const int per_sm = (b->model == GFT_MODEL_SM) ? resident_m<kModelSM>(variant) : resident_m<kModel2HDM>(variant);
    std::vector<int> order, starts;
    b->group_start.assign(b->ngroups(), 0);
    b->group_nlist.assign(b->ngroups(), 0);
    for (int g = 0; g < b->ngroups(); g++) {  // group g's lists fill order[group_item[g] ..]
        const int i0 = b->group_item[g], ni = b->group_item[g + 1] - i0;
        const int G = std::max(1, std::min(ni, b->nsm * per_sm));
        std::vector<int> st;
        balance_tiles(items, i0, ni, b->cfg, g * kGroup, lx, G, order, st);
        b->group_start[g] = (int)starts.size();
        b->group_nlist[g] = G;
        starts.insert(starts.end(), st.begin(), st.end());
    }
    cudaFree(b->d_order);
    cudaFree(b->d_start);
    b->d_order = b->d_start = nullptr;
    e = cudaMalloc(&b->d_order, std::max<size_t>(order.size(), 1) * sizeof(int));
    if (e == cudaSuccess) e = cudaMalloc(&b->d_start, std::max<size_t>(starts.size(), 1) * sizeof(int));
    if (e == cudaSuccess && !order.empty())
        e = cudaMemcpy(b->d_order, order.data(), order.size() * sizeof(int), cudaMemcpyHostToDevice);
    if (e == cudaSuccess && !starts.empty())
        e = cudaMemcpy(b->d_start, starts.data(), starts.size() * sizeof(int), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return b->cuda_fail(e, "gft_batch: configure");
    drop_graph(b);
    return GFT_OK;
}

// A Higgs-family ensemble: no tiled or persistent step carries the family
// fields, so each member takes the launches a single handle makes -- the
// one-thread-per-site step, its energy row, the Gauss pass and its row --
// member after member on the ensemble's stream (one partial buffer serves them
// in turn).
cudaError_t issue_step_family(gft_batch* b, int ti, bool e, bool g, double* rows, long long* nlaunch)
{
    const int tn = (ti + 1) % 2, tp = 1 - tn;
    cudaError_t err = cudaSuccess;
    for (int m = 0; m < b->n && err == cudaSuccess; m++) {
        const StepParams P = config_params(b->cfg[m], b->nsite[m], false, ti, e);
        const double* scale = b->d_scale + (size_t)m * kRowSlotCount;
        double* row = rows + (size_t)m * kRowSlotCount;
        err = launch_fast_step<float, kModel2HDM>(P, b->lv[m][tn], b->lv[m][tp], b->d_status, b->d_part_f, e, 0,
                                                  b->stream);
        (*nlaunch)++;
        if (err == cudaSuccess && e) {
            const int nb = fast_launch_blocks(P, 0);
            err = launch_finalize(b->d_part_f, nb, kObsCount, kObsCount, scale, row, b->d_mid, b->stream);
            *nlaunch += finalize_launches(nb, true);
        }
        if (err == cudaSuccess && g) {
            const int nb = fast_gauss_blocks(P);
            err = launch_fast_gauss<float, kModel2HDM>(P, b->lv[m][tn], b->lv[m][tp], b->d_part_f, b->stream);
            if (err == cudaSuccess)
                err = launch_finalize(b->d_part_f, nb, 2 * b->neq, b->neq, scale + kObsCount, row + kObsCount,
                                      b->d_mid, b->stream);
            *nlaunch += 1 + finalize_launches(nb, true);
        }
    }
    return err;
}

// Launches of one step (time_iter ti); rows go to `rows` when a row is logged.
cudaError_t issue_step(gft_batch* b, int ti, bool e, bool g, double* rows, long long* nlaunch)
{
    if (b->hf != kHfNone) return issue_step_family(b, ti, e, g, rows, nlaunch);
    const int tn = (ti + 1) % 2;
    static thread_local EnsParams ep;
    cudaError_t err = cudaSuccess;
    for (int gr = 0; gr < b->ngroups() && err == cudaSuccess; gr++) {
        const bool uniform = fill_params(b, gr, ti, e, &ep);
        const int i0 = b->group_item[gr], ni = b->group_item[gr + 1] - i0;
        const EnsMaps* maps = b->d_maps + (size_t)gr * kGroup;
        const GroupTiles gt{b->d_items + i0, ni, b->d_order, b->d_start + b->group_start[gr], b->group_nlist[gr]};
        err = (b->model == GFT_MODEL_SM)
                  ? launch_step_m<kModelSM>(b->variant, e, uniform, ep, maps, gt, b->lx, tn, b->d_status,
                                            b->d_part_e + (size_t)i0 * kObsCount, b->nsm, b->stream)
                  : launch_step_m<kModel2HDM>(b->variant, e, uniform, ep, maps, gt, b->lx, tn, b->d_status,
                                              b->d_part_e + (size_t)i0 * kObsCount, b->nsm, b->stream);
        (*nlaunch)++;
    }
    if (err == cudaSuccess && e) {
        ensemble_finalize_kernel<<<b->n, kFinThreads, 0, b->stream>>>(b->d_part_e, b->d_first, 1, kObsCount, kObsCount,
                                                                      b->d_scale, 0, rows);
        err = cudaGetLastError();
        (*nlaunch)++;
    }
    if (err == cudaSuccess && g) {
        for (int gr = 0; gr < b->ngroups() && err == cudaSuccess; gr++) {
            fill_params(b, gr, ti, false, &ep);
            const int i0 = b->group_item[gr], ni = b->group_item[gr + 1] - i0;
            err = (b->model == GFT_MODEL_SM)
                      ? launch_gauss_m<kModelSM>(b->variant, ep, b->d_items + i0, ni, b->lx, b->gauss_rows, tn,
                                                 b->d_part_g + (size_t)i0 * b->gauss_rows * kGaussSlots, b->stream)
                      : launch_gauss_m<kModel2HDM>(b->variant, ep, b->d_items + i0, ni, b->lx, b->gauss_rows, tn,
                                                   b->d_part_g + (size_t)i0 * b->gauss_rows * kGaussSlots,
                                                   b->stream);
            (*nlaunch)++;
        }
        if (err == cudaSuccess) {
            ensemble_finalize_kernel<<<b->n, kFinThreads, 0, b->stream>>>(b->d_part_g, b->d_first, b->gauss_rows, kGaussSlots, 4,
                                                                          b->d_scale, kObsCount, rows);
            err = cudaGetLastError();
            (*nlaunch)++;
        }
    }
    return err;
}

int ensure_rows(gft_batch* b, int nrows)
{
    if (nrows <= b->rows_cap) return GFT_OK;
    cudaStreamSynchronize(b->stream);
    cudaFree(b->d_rows);
    b->d_rows = nullptr;
    const size_t bytes = (size_t)nrows * b->n * kRowSlotCount * sizeof(double);
    cudaError_t e = cudaMalloc(&b->d_rows, bytes);
    if (e != cudaSuccess) {
        b->rows_cap = 0;
        return b->fail(GFT_E_NOMEM, "gft_batch: rows allocation failed");
    }
    cudaMemset(b->d_rows, 0, bytes);
    b->rows_cap = nrows;
    return GFT_OK;
}

bool logs_energy(const gft_batch* b, int ti) { return b->cfg[0].energy_every > 0 && ti % b->cfg[0].energy_every == 0; }
bool logs_gauss(const gft_batch* b, int ti) { return b->cfg[0].gauss_every > 0 && ti % b->cfg[0].gauss_every == 0; }

int max_damped(const gft_batch* b)
{
    int t = 0;
    for (const auto& c : b->cfg) t = std::max(t, c.nt_damped);
    return t;
}

int graph_period_of(const gft_batch* b)
{
    int p = 2;
    if (b->cfg[0].energy_every > 0) p = lcm_i(p, b->cfg[0].energy_every);
    if (b->cfg[0].gauss_every > 0) p = lcm_i(p, b->cfg[0].gauss_every);
    return p;
}

// Capture one logging period starting at a time_iter that is a multiple of the period.
int build_graph(gft_batch* b, int ti0)
{
    const int period = graph_period_of(b);
    int nrows = 0;
    for (int s = 0; s < period; s++) nrows += (logs_energy(b, ti0 + s) || logs_gauss(b, ti0 + s)) ? 1 : 0;
    if (nrows > b->graph_rows_cap) {
        cudaFree(b->d_graph_rows);
        b->d_graph_rows = nullptr;
        if (cudaMalloc(&b->d_graph_rows, (size_t)std::max(nrows, 1) * b->n * kRowSlotCount * sizeof(double)) != cudaSuccess)
            return b->fail(GFT_E_NOMEM, "gft_batch: graph rows allocation failed");
        b->graph_rows_cap = nrows;
    }
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return b->cuda_fail(e, "gft_batch: begin capture");
    long long nl = 0;
    int row = 0;
    cudaError_t ie = cudaSuccess;
    for (int s = 0; s < period && ie == cudaSuccess; s++) {
        const int ti = ti0 + s;
        const bool le = logs_energy(b, ti), lg = logs_gauss(b, ti);
        ie = issue_step(b, ti, le, lg, b->d_graph_rows + (size_t)row * b->n * kRowSlotCount, &nl);
        if (le || lg) row++;
    }
    e = cudaStreamEndCapture(b->stream, &g);
    if (ie != cudaSuccess || e != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        return b->cuda_fail(ie != cudaSuccess ? ie : e, "gft_batch: capture");
    }
    cudaGraphExec_t x = nullptr;
    e = cudaGraphInstantiate(&x, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return b->cuda_fail(e, "gft_batch: graph instantiate");
    drop_graph(b);
    b->graph = x;
    b->graph_period = period;
    b->graph_rows = nrows;
    b->graph_launches = nl;
    return GFT_OK;
}

int ensure_stage(gft_batch* b, size_t bytes)
{
    if (b->stage_bytes >= bytes) return GFT_OK;
    cudaStreamSynchronize(b->stream);
    cudaFree(b->d_stage);
    b->d_stage = nullptr;
    if (cudaMalloc(&b->d_stage, bytes) != cudaSuccess) {
        b->stage_bytes = 0;
        return b->fail(GFT_E_NOMEM, "gft_batch: staging allocation failed");
    }
    b->stage_bytes = bytes;
    return GFT_OK;
}

}  // namespace

extern "C" {

int gft_batch_create(const gft_config* cfgs, int n, gft_batch** out)
{
    if (!out) return GFT_E_INVALID;
    *out = nullptr;
    if (!cfgs || n < 1) {
        set_error("gft_batch_create: need at least one member");
        return GFT_E_INVALID;
    }
    for (int m = 0; m < n; m++) {
        std::string why;
        int rc = validate_config(&cfgs[m], why);
        if (rc != GFT_OK) {
            set_error("gft_batch_create: member " + std::to_string(m) + ": " + why);
            return rc;
        }
        if (cfgs[m].form != GFT_FORM_MIXED) {
            set_error("gft_batch_create: the ensemble evolves the mixed form only");
            return GFT_E_UNSUPPORTED;
        }
        if (cfgs[m].higgs_family != cfgs[0].higgs_family) {
            set_error("gft_batch_create: all members must share the Higgs-family field (gaugeNum)");
            return GFT_E_INVALID;
        }
        if (cfgs[m].generator_rep) {
            set_error("gft_batch_create: the ensemble transfers quaternion links only (generator_rep = 0)");
            return GFT_E_UNSUPPORTED;
        }
        if (cfgs[m].model != cfgs[0].model || cfgs[m].device != cfgs[0].device) {
            set_error("gft_batch_create: all members must share the model and the device");
            return GFT_E_INVALID;
        }
        if (cfgs[m].energy_every != cfgs[0].energy_every || cfgs[m].gauss_every != cfgs[0].gauss_every) {
            set_error("gft_batch_create: all members must share the analysers' logging cadence");
            return GFT_E_INVALID;
        }
    }
    gft_batch* b = new gft_batch();
    b->n = n;
    b->model = cfgs[0].model;
    b->device = cfgs[0].device;
    b->nsc = (b->model == GFT_MODEL_SM) ? 4 : 8;
    b->hf = (b->model == GFT_MODEL_2HDM) ? cfgs[0].higgs_family : kHfNone;
    b->nve = 3 * (5 + (b->hf == kHfSU2 ? 4 : (b->hf == kHfU1 ? 1 : 0)));
    b->neq = config_neq(cfgs[0]);
    b->cfg.assign(cfgs, cfgs + n);
    for (int v = 0; v < kTiledVariants && b->variant < 0; v++)
        if (variant_fits(b, v)) b->variant = v;
    if (b->variant < 0 && b->hf == kHfNone) {
        delete b;
        set_error("gft_batch_create: the members' (ny, nz) share no built tile shape (4 x 16, the smallest, needs ny % 4 == 0 and nz % 16 == 0)");
        return GFT_E_UNSUPPORTED;
    }
    cudaError_t e = cudaSetDevice(b->device);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&b->nsm, cudaDevAttrMultiProcessorCount, b->device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreate(&b->ev0);
    if (e == cudaSuccess) e = cudaEventCreate(&b->ev1);
    if (e != cudaSuccess) {
        int rc = b->cuda_fail(e, "gft_batch_create");
        gft_batch_destroy(b);
        return rc;
    }
    size_t off = 0;
    for (int m = 0; m < n; m++) {
        b->nsite.push_back(cfgs[m].nx * cfgs[m].ny * cfgs[m].nz);
        b->level_off.push_back(off);
        off += 2 * ((level_bytes_f32(b->nsite[m], b->nsc, b->hf) + 255) / 256 * 256);
    }
    b->arena_bytes = off;
    e = cudaMalloc(&b->arena, b->arena_bytes);
    if (e == cudaSuccess) e = cudaMalloc(&b->d_maps, (size_t)n * sizeof(EnsMaps));
    if (e == cudaSuccess) e = cudaMalloc(&b->d_scale, (size_t)n * kRowSlotCount * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&b->d_status, sizeof(unsigned));
    if (e != cudaSuccess) {
        b->fail(GFT_E_NOMEM, std::string("gft_batch_create: ") + cudaGetErrorString(e));
        gft_batch_destroy(b);
        return GFT_E_NOMEM;
    }
    cudaMemset(b->d_status, 0, sizeof(unsigned));
    b->lv.resize(n);
    std::vector<double> scale((size_t)n * kRowSlotCount);
    for (int m = 0; m < n; m++) {
        const size_t lb = (level_bytes_f32(b->nsite[m], b->nsc, b->hf) + 255) / 256 * 256;
        for (int t = 0; t < 2; t++)
            carve_level_f32(static_cast<unsigned char*>(b->arena) + b->level_off[m] + t * lb, b->nsite[m], b->nsc,
                            b->lv[m][t], b->hf);
        row_scales(b->cfg[m], b->nsite[m], scale.data() + (size_t)m * kRowSlotCount);
    }
    cudaMemcpy(b->d_scale, scale.data(), scale.size() * sizeof(double), cudaMemcpyHostToDevice);
    if (b->hf != kHfNone) {
        // one thread per site, member after member: partial rows for the largest member
        int rows = 0;
        for (int m = 0; m < n; m++) {
            const StepParams P = config_params(b->cfg[m], b->nsite[m], false, 0, false);
            rows = std::max(rows, std::max(fast_launch_blocks(P, 0), fast_gauss_blocks(P)));
        }
        e = cudaMalloc(&b->d_part_f, (size_t)rows * kMaxSlots * sizeof(double));
        if (e == cudaSuccess) e = cudaMalloc(&b->d_mid, (size_t)kFinMidCapacity * sizeof(double));
        if (e != cudaSuccess) {
            b->fail(GFT_E_NOMEM, std::string("gft_batch_create: ") + cudaGetErrorString(e));
            gft_batch_destroy(b);
            return GFT_E_NOMEM;
        }
        *out = b;
        return GFT_OK;
    }
    int rc = configure(b, b->variant, 32);
    if (rc != GFT_OK) {
        gft_batch_destroy(b);
        return rc;
    }
    *out = b;
    return GFT_OK;
}

void gft_batch_destroy(gft_batch* b)
{
    if (!b) return;
    cudaSetDevice(b->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    drop_graph(b);
    cudaFree(b->arena);
    cudaFree(b->d_maps);
    cudaFree(b->d_items);
    cudaFree(b->d_order);
    cudaFree(b->d_start);
    cudaFree(b->d_first);
    cudaFree(b->d_part_e);
    cudaFree(b->d_part_g);
    cudaFree(b->d_scale);
    cudaFree(b->d_rows);
    cudaFree(b->d_status);
    cudaFree(b->d_stage);
    cudaFree(b->d_graph_rows);
    cudaFree(b->d_part_f);
    cudaFree(b->d_mid);
    if (b->ev0) cudaEventDestroy(b->ev0);
    if (b->ev1) cudaEventDestroy(b->ev1);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
}

int gft_batch_size(const gft_batch* b) { return b ? b->n : 0; }

int gft_batch_init_fields(gft_batch* b, const gft_ic* ics)
{
    if (!b || !ics) return GFT_E_INVALID;
    cudaSetDevice(b->device);
    cudaError_t e = cudaSuccess;
    for (int m = 0; m < b->n && e == cudaSuccess; m++) {
        ICParams p{};
        p.seed = ics[m].seed;
        for (int k = 0; k < 8; k++) {
            p.mean[k] = ics[m].mean[k];
            p.sigma[k] = ics[m].sigma[k];
        }
        p.theta_sigma = ics[m].theta_sigma;
        p.eps_sigma = ics[m].eps_sigma;
        p.wall_width = ics[m].wall_width;
        p.wall_value = ics[m].wall_value;
        const StepParams P = config_params(b->cfg[m], b->nsite[m], false, 0, false);
        e = launch_init_fields<float>(P, b->nsc, p, b->lv[m][0], b->lv[m][1], b->stream);
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
    if (e != cudaSuccess) return b->cuda_fail(e, "gft_batch_init_fields");
    b->time_iter = 0;
    b->has_data = true;
    return GFT_OK;
}

int gft_batch_upload_f32(gft_batch* b, int member, const float* sc, const float* ve, int time_iter)
{
    if (!b || !sc || !ve || member < 0 || member >= b->n || time_iter < 0) return GFT_E_INVALID;
    cudaSetDevice(b->device);
    const size_t nsc_w = 2 * (size_t)b->nsite[member] * b->nsc, nve_w = 2 * (size_t)b->nsite[member] * b->nve;
    int rc = ensure_stage(b, (nsc_w + nve_w) * sizeof(float));
    if (rc != GFT_OK) return rc;
    float* dsc = static_cast<float*>(b->d_stage);
    float* dve = dsc + nsc_w;
    cudaError_t e = cudaMemcpyAsync(dsc, sc, nsc_w * sizeof(float), cudaMemcpyHostToDevice, b->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dve, ve, nve_w * sizeof(float), cudaMemcpyHostToDevice, b->stream);
    for (int t = 0; t < 2 && e == cudaSuccess; t++)
        e = launch_aos_to_soa<float, float>(dsc + (size_t)t * b->nsite[member] * b->nsc,
                                            dve + (size_t)t * b->nsite[member] * b->nve, b->nsite[member], b->nsc,
                                            b->lv[member][t], b->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
    if (e != cudaSuccess) return b->cuda_fail(e, "gft_batch_upload_f32");
    b->time_iter = time_iter;
    b->has_data = true;
    return GFT_OK;
}

int gft_batch_download_f32(gft_batch* b, int member, float* sc, float* ve)
{
    if (!b || !sc || !ve || member < 0 || member >= b->n) return GFT_E_INVALID;
    if (!b->has_data) return b->fail(GFT_E_STATE, "gft_batch_download_f32: no field data");
    cudaSetDevice(b->device);
    const size_t nsc_w = 2 * (size_t)b->nsite[member] * b->nsc, nve_w = 2 * (size_t)b->nsite[member] * b->nve;
    int rc = ensure_stage(b, (nsc_w + nve_w) * sizeof(float));
    if (rc != GFT_OK) return rc;
    float* dsc = static_cast<float*>(b->d_stage);
    float* dve = dsc + nsc_w;
    cudaError_t e = cudaSuccess;
    for (int t = 0; t < 2 && e == cudaSuccess; t++)
        e = launch_soa_to_aos<float, float>(b->lv[member][t], b->nsite[member], b->nsc,
                                            dsc + (size_t)t * b->nsite[member] * b->nsc,
                                            dve + (size_t)t * b->nsite[member] * b->nve, b->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(sc, dsc, nsc_w * sizeof(float), cudaMemcpyDeviceToHost, b->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(ve, dve, nve_w * sizeof(float), cudaMemcpyDeviceToHost, b->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
    if (e != cudaSuccess) return b->cuda_fail(e, "gft_batch_download_f32");
    return GFT_OK;
}

int gft_batch_evolve(gft_batch* b, int n_steps, gft_observables* rows, int max_rows, int* n_rows)
{
    if (n_rows) *n_rows = 0;
    if (!b) return GFT_E_INVALID;
    if (n_steps < 0) return b->fail(GFT_E_INVALID, "gft_batch_evolve: n_steps must be >= 0");
    if (!b->has_data) return b->fail(GFT_E_STATE, "gft_batch_evolve: no field data");
    cudaSetDevice(b->device);
    int nlog = 0;
    for (int s = 0; s < n_steps; s++) nlog += (logs_energy(b, b->time_iter + s) || logs_gauss(b, b->time_iter + s)) ? 1 : 0;
    int rc = ensure_rows(b, std::max(nlog, 1));
    if (rc != GFT_OK) return rc;
    struct Meta {
        int ti;
        bool e, g;
    };
    std::vector<Meta> meta;
    cudaMemsetAsync(b->d_status, 0, sizeof(unsigned), b->stream);
    cudaEventRecord(b->ev0, b->stream);
    const int period = graph_period_of(b);
    const bool graphs_ok = b->use_graphs && period <= kMaxGraphPeriod;
    cudaError_t err = cudaSuccess;
    int row = 0, s = 0;
    while (s < n_steps && err == cudaSuccess) {
        const int ti = b->time_iter;
        if (graphs_ok && ti >= max_damped(b) && ti % period == 0 && n_steps - s >= period) {
            if (!b->graph) {
                rc = build_graph(b, ti);
                if (rc != GFT_OK) return rc;
            }
            err = cudaGraphLaunch(b->graph, b->stream);
            b->launches += b->graph_launches;
            if (err == cudaSuccess && b->graph_rows > 0)
                err = cudaMemcpyAsync(b->d_rows + (size_t)row * b->n * kRowSlotCount, b->d_graph_rows,
                                      (size_t)b->graph_rows * b->n * kRowSlotCount * sizeof(double),
                                      cudaMemcpyDeviceToDevice, b->stream);
            for (int k = 0; k < period; k++) {
                const bool le = logs_energy(b, ti + k), lg = logs_gauss(b, ti + k);
                if (le || lg) {
                    meta.push_back({ti + k, le, lg});
                    row++;
                }
            }
            b->time_iter += period;
            s += period;
            continue;
        }
        const bool le = logs_energy(b, ti), lg = logs_gauss(b, ti);
        err = issue_step(b, ti, le, lg, b->d_rows + (size_t)row * b->n * kRowSlotCount, &b->launches);
        if (le || lg) {
            meta.push_back({ti, le, lg});
            row++;
        }
        b->time_iter++;
        s++;
    }
    cudaEventRecord(b->ev1, b->stream);
    if (err != cudaSuccess) return b->cuda_fail(err, "gft_batch_evolve: launch");
    std::vector<double> host((size_t)row * b->n * kRowSlotCount);
    unsigned status = 0;
    if (row > 0)
        err = cudaMemcpyAsync(host.data(), b->d_rows, host.size() * sizeof(double), cudaMemcpyDeviceToHost, b->stream);
    if (err == cudaSuccess) err = cudaMemcpyAsync(&status, b->d_status, sizeof(unsigned), cudaMemcpyDeviceToHost, b->stream);
    if (err == cudaSuccess) err = cudaStreamSynchronize(b->stream);
    if (err != cudaSuccess) return b->cuda_fail(err, "gft_batch_evolve");
    float ms = 0.f;
    cudaEventElapsedTime(&ms, b->ev0, b->ev1);
    b->last_ms = ms;
    if (status & 8u) return b->fail(GFT_E_TIMEOUT, "gft_batch_evolve: a device-side wait gave up; fields are invalid");
    const int nw = rows ? std::min(row, max_rows) : 0;
    for (int m = 0; m < b->n && rows; m++)
        for (int r = 0; r < nw; r++)
            fill_observables(&rows[(size_t)m * max_rows + r], meta[r].ti, meta[r].e, meta[r].g,
                             host.data() + ((size_t)r * b->n + m) * kRowSlotCount, b->neq);
    if (n_rows) *n_rows = nw;
    return (int)(status & (GFT_W_ASIN_DOMAIN | GFT_W_SQRT_DOMAIN | GFT_W_NONFINITE | GFT_W_RANGE));
}

int gft_batch_set_kernel(gft_batch* b, int tile, int march, int use_graphs)
{
    if (!b) return GFT_E_INVALID;
    if (b->hf != kHfNone) {  // one thread per site: no tile shape or march; only the graph switch applies
        b->use_graphs = use_graphs != 0;
        if (!b->use_graphs) drop_graph(b);
        return GFT_OK;
    }
    if (tile < 0 || tile >= kTiledVariants || march < 1) return b->fail(GFT_E_INVALID, "gft_batch_set_kernel: bad tile or march");
    if (!variant_fits(b, tile)) return b->fail(GFT_E_UNSUPPORTED, "gft_batch_set_kernel: a member does not divide into this tile");
    cudaSetDevice(b->device);
    b->use_graphs = use_graphs != 0;
    if (tile == b->variant && march == b->lx) {
        if (!b->use_graphs) drop_graph(b);
        return GFT_OK;
    }
    return configure(b, tile, march);
}

int gft_batch_autotune(gft_batch* b, int trial_steps, int* tile, int* march)
{
    if (!b) return GFT_E_INVALID;
    if (b->hf != kHfNone)
        return b->fail(GFT_E_UNSUPPORTED, "gft_batch_autotune: a Higgs-family ensemble runs one thread per site (no tiles)");
    if (!b->has_data) return b->fail(GFT_E_STATE, "gft_batch_autotune: no field data");
    if (trial_steps < 1) trial_steps = 4;
    cudaSetDevice(b->device);
    void* backup = nullptr;
    if (cudaMalloc(&backup, b->arena_bytes) != cudaSuccess)
        return b->fail(GFT_E_NOMEM, "gft_batch_autotune: no room for the field backup");
    cudaError_t e = cudaMemcpyAsync(backup, b->arena, b->arena_bytes, cudaMemcpyDeviceToDevice, b->stream);
    int maxnx = 0;
    for (const auto& c : b->cfg) maxnx = std::max(maxnx, c.nx);
    const int ti0 = b->time_iter;
    float best = 1e30f;
    int bv = b->variant, bl = b->lx, rc = GFT_OK;
    const int marches[] = {8, 16, 32, 64};
    for (int v = 0; v < kTiledVariants && e == cudaSuccess && rc == GFT_OK; v++) {
        if (!variant_fits(b, v)) continue;
        for (int lx : marches) {
            if (lx > std::max(maxnx, 8)) continue;
            rc = configure(b, v, lx);
            if (rc != GFT_OK) break;
            long long nl = 0;
            e = issue_step(b, ti0, false, false, b->d_rows, &nl);  // warm-up
            if (e == cudaSuccess) e = cudaEventRecord(b->ev0, b->stream);
            for (int s = 0; s < trial_steps && e == cudaSuccess; s++)
                e = issue_step(b, ti0 + 1 + s, false, false, b->d_rows, &nl);
            if (e == cudaSuccess) e = cudaEventRecord(b->ev1, b->stream);
            if (e == cudaSuccess) e = cudaEventSynchronize(b->ev1);
            float ms = 0.f;
            if (e == cudaSuccess) cudaEventElapsedTime(&ms, b->ev0, b->ev1);
            if (e == cudaSuccess && ms < best) {
                best = ms;
                bv = v;
                bl = lx;
            }
            if (e == cudaSuccess)
                e = cudaMemcpyAsync(b->arena, backup, b->arena_bytes, cudaMemcpyDeviceToDevice, b->stream);
        }
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
    unsigned status = 0;
    cudaMemcpy(&status, b->d_status, sizeof(unsigned), cudaMemcpyDeviceToHost);
    cudaMemset(b->d_status, 0, sizeof(unsigned));
    cudaFree(backup);
    b->time_iter = ti0;
    if (e != cudaSuccess) return b->cuda_fail(e, "gft_batch_autotune");
    if (rc != GFT_OK) return rc;
    if (status & 8u) return b->fail(GFT_E_TIMEOUT, "gft_batch_autotune: a device-side wait gave up");
    rc = configure(b, bv, bl);
    if (rc != GFT_OK) return rc;
    if (tile) *tile = bv;
    if (march) *march = bl;
    return GFT_OK;
}

double gft_batch_last_ms(const gft_batch* b) { return b ? b->last_ms : 0.0; }
long long gft_batch_launch_count(const gft_batch* b) { return b ? b->launches : 0; }
int gft_batch_time_iter(const gft_batch* b) { return b ? b->time_iter : 0; }
void* gft_batch_stream(gft_batch* b) { return b ? (void*)b->stream : nullptr; }
size_t gft_batch_device_bytes(const gft_batch* b) { return b ? b->arena_bytes : 0; }

const char* gft_batch_last_error(const gft_batch* b) { return b ? b->err.c_str() : ""; }

}  // extern "C"
