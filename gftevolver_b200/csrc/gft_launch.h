// gft_launch.h -- host-side launchers of the device kernels (internal).
#pragma once

#include <cuda.h>
#include <string>
#include <cuda_runtime.h>

#include "gft.h"
#include "gft_device.cuh"

namespace gft {

// Reference-arithmetic form (gft_ref_kernels.cu, compiled with -fmad=false).
template <class S, int MODEL>
cudaError_t launch_ref_step(const StepParams& P, const LevelPtrs<S>& now, const LevelPtrs<S>& past, unsigned* status,
                            double* partials, bool energy, cudaStream_t stream);
template <class S, int MODEL>
cudaError_t launch_ref_gauss(const StepParams& P, const LevelPtrs<S>& now, const LevelPtrs<S>& fut, double* partials,
                             cudaStream_t stream);
int ref_launch_blocks(const StepParams& P);

// Throughput forms (gft_fast_kernels.cu): FP64 plain form (S = double) and
// mixed form (S = float).
template <class S, int MODEL>
cudaError_t launch_fast_step(const StepParams& P, const LevelPtrs<S>& now, const LevelPtrs<S>& past, unsigned* status,
                             double* partials, bool energy, int variant, cudaStream_t stream);
template <class S, int MODEL>
cudaError_t launch_fast_gauss(const StepParams& P, const LevelPtrs<S>& now, const LevelPtrs<S>& fut, double* partials,
                              cudaStream_t stream);
int fast_launch_blocks(const StepParams& P, int variant);
int fast_gauss_blocks(const StepParams& P);

// Tiled throughput kernel (gft_tiled_kernels.cu): TMA-staged planes, x-march.
// Tensor maps of the "now" level: quaternions and doublets as {4, nz, ny, nx},
// hypercharge phases as {nz, ny, nx}.
struct TMaps {
    CUtensorMap q[3];
    CUtensorMap th[3];
    CUtensorMap ph[2];
};
// halo = true: boxes with the one-site halo (staged "now" planes); false: the
// bare tile (L2 prefetch of the own-site past level).
template <class S>
bool tiled_encode_maps(const StepParams& P, const LevelPtrs<S>& L, int nd, int ty, int tz, bool halo, TMaps* out);
bool tiled_supported(const StepParams& P, int variant);
int tiled_blocks(const StepParams& P, int variant, int lx);
// Resident CTAs per SM the SM-model tiled step asks for (its launch bounds).
int tiled_ctas_per_sm(int variant, bool fp64);
template <class S, int MODEL>
cudaError_t launch_tiled_step(const TMaps& maps, const TMaps& pmaps, const StepParams& P, const LevelPtrs<S>& now,
                              const LevelPtrs<S>& past, int variant, int lx, unsigned* status, double* partials,
                              bool energy, cudaStream_t stream, int xa = 0, int xn = -1);
// The SM mixed form's plain steps with two sites per thread (rows ty and ty + TY/2
// of the tile) in paired FP32 arithmetic; same tiles, ring and tensor maps.
cudaError_t launch_tiled_pair_step(const TMaps& maps, const TMaps& pmaps, const StepParams& P,
                                   const LevelPtrs<float>& now, const LevelPtrs<float>& past, int variant, int lx,
                                   unsigned* status, cudaStream_t stream, int xa = 0, int xn = -1);
// The SM mixed form's plain steps with each site's update split between two
// threads (links / scalars), kSplitTileY x kSplitTileZ tiles, 256 threads,
// three CTAs per SM; its tensor maps are encoded for that tile.
constexpr int kSplitTileY = 8, kSplitTileZ = 16;
cudaError_t launch_tiled_split_step(const TMaps& maps, const TMaps& pmaps, const StepParams& P,
                                    const LevelPtrs<float>& now, const LevelPtrs<float>& past, int lx,
                                    unsigned* status, cudaStream_t stream, int xa = 0, int xn = -1);
constexpr int kTiledVariants = 4;  // 8x32, 4x32, 4x16, 16x16 (TY x TZ)
// Tile shapes the two-sites-per-thread kernel is built for (8 x 32 and 16 x 16:
// 128 threads per CTA, two CTAs per SM).
inline bool tiled_pair_tile(int variant) { return variant == 0 || variant == 3; }
inline void tiled_tile(int variant, int& ty, int& tz)
{
    static const int shapes[4][2] = {{8, 32}, {4, 32}, {4, 16}, {16, 16}};
    const int v = (variant >= 0 && variant < 4) ? variant : 0;
    ty = shapes[v][0];
    tz = shapes[v][1];
}

// x-slab ghost-plane exchange over NCCL (gft_slab_nccl.cu).
constexpr int kNcclIdBytes = 128;
constexpr int kMaxPlaneArrays = 11;  // field arrays of a level at most (2HDM with a Higgs-family SU(2))
struct SlabComm;
// Plane ranges of one exchange: per field array, the first and last own planes
// (sent left and right) and the two ghost planes (received from right and left).
struct SlabPlanes {
    int n = 0;
    void* send_lo[kMaxPlaneArrays];
    void* send_hi[kMaxPlaneArrays];
    void* recv_lo[kMaxPlaneArrays];
    void* recv_hi[kMaxPlaneArrays];
    size_t bytes[kMaxPlaneArrays];
};
int nccl_unique_id(unsigned char* out, std::string& why);
int slab_comm_create(const unsigned char* id, int nranks, int rank, SlabComm** out, std::string& why);
void slab_comm_destroy(SlabComm* c, bool abort);
int slab_comm_exchange(SlabComm* c, const SlabPlanes& pl, cudaStream_t stream, std::string& why);
int slab_comm_wait(SlabComm* c, cudaStream_t stream, double seconds, std::string& why);
bool slab_comm_alive(const SlabComm* c);

// Auxiliary kernels (gft_aux_kernels.cu).
// The reference record has 3 x 5 link words per site, 3 x 6 with a Higgs-family
// phase (lv.hth set) or 3 x 9 with a Higgs-family quaternion (lv.hq set); in the
// generator representation 3 x 4, 3 x 5 or 3 x 7.
struct LinkCodec {
    int gen = 0;       // host links are generators w (WilsonLoops/Source/StandardModel.cpp:76-160)
    int convert = 0;   // gen: the device holds quaternions (convert w <-> q), else the raw generators
    double tol = 0.0;  // divisionByZeroTolerance of the conversions
};
template <class S, class H>
cudaError_t launch_aos_to_soa(const H* aos_sc, const H* aos_ve, int nsite, int nsc, LevelPtrs<S> lv, cudaStream_t s,
                              LinkCodec codec = LinkCodec());
template <class S, class H>
cudaError_t launch_soa_to_aos(LevelPtrs<S> lv, int nsite, int nsc, H* aos_sc, H* aos_ve, cudaStream_t s,
                              LinkCodec codec = LinkCodec());

struct ICParams {
    unsigned long long seed;
    double mean[8], sigma[8];
    double theta_sigma, eps_sigma, wall_width, wall_value;
    // x-slab: local plane x draws the random numbers of global plane
    // (x + x_offset) mod nx_global, so slabs reproduce the whole lattice's data
    int x_offset, nx_global;
    // store the SU(2) links as their generators w = eps n (reference-arithmetic
    // form in the generator representation)
    int store_generators;
};
template <class S>
cudaError_t launch_init_fields(const StepParams& P, int nsc, const ICParams& ic, LevelPtrs<S> a, LevelPtrs<S> b,
                               cudaStream_t s);

// Sum (slots < max_from, compensated) or max (slots >= max_from) the per-block
// partials [nblocks][nslots] into out[nslots], scaled by scale[slot].
// Deterministic FP64 reduction of per-block partials into one row (scaled by
// scale[k]); `mid` (kFinMidRows x 16 doubles, may be null) enables a two-stage
// reduction for large block counts.
cudaError_t launch_finalize(const double* partials, int nblocks, int nslots, int max_from, const double* scale_dev,
                            double* out, double* mid, cudaStream_t s);
// Kernel launches launch_finalize makes for nblocks partial rows.
int finalize_launches(int nblocks, bool have_mid);
constexpr int kFinMidCapacity = 512 * 16;

// Record the library-wide last error message (gft_last_error(NULL)).
void set_last_error(const std::string& msg);
void set_error(const std::string& msg);

// Shared by the single-lattice handle (gft_abi.cu) and the ensemble (gft_ensemble.cu).
// Launch parameters of one step for a configuration (f32ref: the reference-
// arithmetic form with float storage, whose couplings are rounded to float).
StepParams config_params(const gft_config& c, int nsite, bool f32ref, int time_iter, bool energy);
// Per-slot scale of an observables row: energies and Gauss integrals x dV, means / N.
// (kRowSlotCount slots: kObsCount energy slots, then gaugeNum integrated and
// gaugeNum maximum Gauss slots.)
void row_scales(const gft_config& c, int nsite, double* scale);
int validate_config(const gft_config* c, std::string& why);
// neq = gaugeNum (Gauss constraints per row).
void fill_observables(gft_observables* r, int time_iter, bool e, bool g, const double* v, int neq = 4);
// One time level of float storage (with the Higgs-family arrays of hf): bytes, and the array pointers within it.
size_t level_bytes_f32(int nsite, int nsc, int hf = kHfNone);
void carve_level_f32(void* mem, int nsite, int nsc, LevelPtrs<float>& L, int hf = kHfNone);
constexpr int kRowSlotCount = kObsCount + kGaussSlotsMax;
// Gauge equations per direction (gaugeNum) of a configuration.
inline int config_neq(const gft_config& c) { return c.model == GFT_MODEL_2HDM ? hf_neq(c.higgs_family) : 4; }

// Elementary-function self-test (gft_math.cuh vs CUDA's functions) on the current device.
cudaError_t run_math_selftest(int n, double* out9);

}  // namespace gft
