// gft_static_observe.cu -- observables of a lattice state without allocating.
//
// gft_observe_static() computes the same global observables as gft_observe()
// (energy terms, plaquette means, <phi^dag phi>) for fields the caller already
// holds on the device, and allocates nothing: no cudaMalloc, no cudaFree, no
// handle.  It exists for callers that cannot allocate device memory at the
// point where they need the numbers -- code running under a memory budget
// fixed up front, or inside a region that must stay asynchronous (cudaMalloc
// and cudaFree synchronise the device), or on memory owned by another
// framework's allocator.
//
// Its scratch (one row of partial sums per thread block) is a file-scope
// __device__ array of fixed size, kStaticBlocks rows of kStaticSlots doubles
// (1.2 MB on every device that loads the library, held until the process
// exits).  One block covers kSitesPerBlock sites, so lattices of more than
// kStaticBlocks * kSitesPerBlock = 67,108,864 sites are rejected.  Every call
// shares the array: calls that overlap on the GPU (two streams, or two host
// threads) race on it and must be serialised by the caller.  Each call writes
// every row it reads before reading it, so nothing needs clearing between
// calls.
//
// In host code the array's name is only a host-side stand-in; its device
// address is obtained with cudaGetSymbolAddress once per device, on the first
// call made with that device current.  That first call therefore issues a
// runtime query and should come before any stream capture.  The address is kept
// per device ordinal for the life of the process: after cudaDeviceReset on a
// device, the library must not be called on that device again.
#include <mutex>
#include <string>

#include "gft.h"
#include "gft_device.cuh"
#include "gft_launch.h"
#include "gft_step_body.cuh"

namespace gft {
namespace {

constexpr int kStaticThreads = 256;
constexpr int kSitesPerThread = 16;
constexpr int kSitesPerBlock = kStaticThreads * kSitesPerThread;  // 4096
constexpr int kStaticBlocks = 16384;
constexpr int kStaticSlots = kObsCount;                            // 9
constexpr long long kStaticMaxSites = (long long)kStaticBlocks * kSitesPerBlock;

static __device__ __align__(256) double g_static_partials[kStaticBlocks * kStaticSlots];

constexpr int kMaxDevices = 64;
std::mutex g_static_mu;
double* g_static_addr[kMaxDevices] = {};

// Observables of the state at the level pair (now, past), read from the
// reference AoS layout: scalars[2][N][nsc], vectors[2][N][3 dw], per direction
// dw words: theta, the SU(2) quaternion, then the 2HDM Higgs-family field --
// none (dw = 5), its U(1) phase (6) or its SU(2) quaternion (9)
// (WilsonLoops/Source/TwoHDM.cpp:210-242).
struct AosView {
    const float* sc;
    const float* ve;
    int nsc, N, dw, hf;
    __device__ __forceinline__ const float* link(int lvl, int s, int d) const
    {
        return ve + ((size_t)lvl * N + s) * (3 * dw) + dw * d;
    }
    __device__ __forceinline__ Q<double> q(int lvl, int s, int d) const
    {
        const float* v = link(lvl, s, d);
        return {(double)v[1], (double)v[2], (double)v[3], (double)v[4]};
    }
    __device__ __forceinline__ double th(int lvl, int s, int d) const { return (double)link(lvl, s, d)[0]; }
    __device__ __forceinline__ double hth(int lvl, int s, int d) const { return (double)link(lvl, s, d)[5]; }
    __device__ __forceinline__ Q<double> hq(int lvl, int s, int d) const
    {
        const float* v = link(lvl, s, d);
        return {(double)v[5], (double)v[6], (double)v[7], (double)v[8]};
    }
    __device__ __forceinline__ Q<double> ph(int lvl, int s, int db) const
    {
        const float* f = sc + ((size_t)lvl * N + s) * nsc + 4 * db;
        return {(double)f[0], (double)f[1], (double)f[2], (double)f[3]};
    }
};

__device__ __forceinline__ double omt(Q<double> a)
{
    const double v2 = a.x * a.x + a.y * a.y + a.z * a.z;
    const double n = sqrt(a.w * a.w + v2);
    return v2 / (n * (n + a.w));
}

__device__ __forceinline__ Q<double> transport_d(Q<double> u, double cs, double sn, Q<double> f)
{
    const double h0 = cs * f.w - sn * f.x, h1 = cs * f.x + sn * f.w;
    const double h2 = cs * f.y - sn * f.z, h3 = cs * f.z + sn * f.y;
    return {u.w * h0 - u.z * h1 + u.y * h2 - u.x * h3, u.z * h0 + u.w * h1 + u.x * h2 + u.y * h3,
            -u.y * h0 - u.x * h1 + u.w * h2 + u.z * h3, u.x * h0 - u.y * h1 - u.z * h2 + u.w * h3};
}

__global__ void __launch_bounds__(kStaticThreads) static_observe_kernel(StepParams P, AosView A, int tn, int model,
                                                                         double* partials)
{
    const int tp = 1 - tn;
    const int nd = (model == kModelSM) ? 1 : 2;
    double obs[kObsCount];
#pragma unroll
    for (int k = 0; k < kObsCount; k++) obs[k] = 0.0;
    const int base = blockIdx.x * kSitesPerBlock;
    for (int r = 0; r < kSitesPerThread; r++) {
        const int s = base + r * kStaticThreads + threadIdx.x;
        if (s >= P.nsite) break;
        const int z = s % P.nz, y = (s / P.nz) % P.ny, x = s / (P.nz * P.ny);
        int pa[3];
        pa[0] = (((x + 1 == P.nx) ? 0 : x + 1) * P.ny + y) * P.nz + z;
        pa[1] = (x * P.ny + ((y + 1 == P.ny) ? 0 : y + 1)) * P.nz + z;
        pa[2] = (x * P.ny + y) * P.nz + ((z + 1 == P.nz) ? 0 : z + 1);
        Q<double> U[3];
        double th[3];
        for (int d = 0; d < 3; d++) {
            U[d] = A.q(tn, s, d);
            th[d] = A.th(tn, s, d);
        }
        // magnetic energy and plaquettes: P1 = U_j(x+i)^dag U_i(x+j) U_j(x) U_i(x)^dag, i < j
        for (int pl = 0; pl < 3; pl++) {
            const int i = (pl == 2) ? 1 : 0, j = (pl == 0) ? 1 : 2;
            const Q<double> P1 =
                qmul(qmul(qmul(qconj(A.q(tn, pa[i], j)), A.q(tn, pa[j], i)), U[j]), qconj(U[i]));
            const double F = th[i] + A.th(tn, pa[i], j) - A.th(tn, pa[j], i) - th[j];
            const double o = omt(P1), h = sin(0.5 * F);
            obs[kObsMagnetic] += 4.0 * P.lap[i] * P.lap[j] * (P.inv_g_sqr * o + P.inv_gp_sqr * 2.0 * h * h);
            obs[kObsPlaqSU2] += 1.0 - o;
            obs[kObsPlaqU1] += cos(F);
        }
        // Higgs-family loops, coupling g'' (WilsonLoops/Source/TwoHDM.cpp:484-551)
        if (A.hf == kHfU1) {
            for (int pl = 0; pl < 3; pl++) {
                const int i = (pl == 2) ? 1 : 0, j = (pl == 0) ? 1 : 2;
                const double F = A.hth(tn, s, i) + A.hth(tn, pa[i], j) - A.hth(tn, pa[j], i) - A.hth(tn, s, j);
                const double h = sin(0.5 * F);
                obs[kObsMagnetic] += 4.0 * P.lap[i] * P.lap[j] * P.inv_gpp_sqr * 2.0 * h * h;
            }
        } else if (A.hf == kHfSU2) {
            for (int pl = 0; pl < 3; pl++) {
                const int i = (pl == 2) ? 1 : 0, j = (pl == 0) ? 1 : 2;
                const Q<double> P1 = qmul(qmul(qmul(qconj(A.hq(tn, pa[i], j)), A.hq(tn, pa[j], i)), A.hq(tn, s, j)),
                                          qconj(A.hq(tn, s, i)));
                obs[kObsMagnetic] += 4.0 * P.lap[i] * P.lap[j] * P.inv_gpp_sqr * omt(P1);
            }
        }
        // electric energy: U_now U_past^dag and 1 - cos(dtheta)
        for (int d = 0; d < 3; d++) {
            const Q<double> E = qmul(U[d], qconj(A.q(tp, s, d)));
            const double h = sin(0.5 * (th[d] - A.th(tp, s, d)));
            obs[kObsElectric] += 4.0 * P.lap[d] * P.inv_sqr_dt * (P.inv_g_sqr * omt(E) + P.inv_gp_sqr * 2.0 * h * h);
            if (A.hf == kHfU1) {  // (WilsonLoops/Source/TwoHDM.cpp:601-633)
                const double hh = sin(0.5 * (A.hth(tn, s, d) - A.hth(tp, s, d)));
                obs[kObsElectric] += 4.0 * P.lap[d] * P.inv_sqr_dt * P.inv_gpp_sqr * 2.0 * hh * hh;
            } else if (A.hf == kHfSU2) {  // (WilsonLoops/Source/TwoHDM.cpp:702-745)
                obs[kObsElectric] += 4.0 * P.lap[d] * P.inv_sqr_dt * P.inv_gpp_sqr *
                                     omt(qmul(A.hq(tn, s, d), qconj(A.hq(tp, s, d))));
            }
        }
        // scalar sector: kinetic, <phi^dag phi>, gradient, potential
        double fsq[2] = {0.0, 0.0}, dot = 0.0, anti = 0.0;
        const Q<double> f0 = A.ph(tn, s, 0), f1 = (nd == 2) ? A.ph(tn, s, 1) : f0;
        for (int db = 0; db < nd; db++) {
            const Q<double> f = (db == 0) ? f0 : f1;
            const Q<double> fo = A.ph(tp, s, db);
            fsq[db] = f.w * f.w + f.x * f.x + f.y * f.y + f.z * f.z;
            const double v0 = (f.w - fo.w) / P.dt, v1 = (f.x - fo.x) / P.dt, v2 = (f.y - fo.y) / P.dt,
                         v3 = (f.z - fo.z) / P.dt;
            obs[kObsKinetic] += 0.5 * (v0 * v0 + v1 * v1 + v2 * v2 + v3 * v3);
            obs[kObsPhiSq] += fsq[db];
        }
        // the doublets transported along each link, then acted on by the Higgs-family
        // field of that link (Gradients/Source/TwoHDM.cpp:118-146)
        for (int a = 0; a < 3; a++) {
            const double cs = cos(th[a]), sn = sin(th[a]);
            Q<double> t[2] = {transport_d(U[a], cs, sn, f0), transport_d(U[a], cs, sn, f1)};
            if (A.hf == kHfU1) {
                const double ha = A.hth(tn, s, a);
                hf_act<kHfU1>(t[0], t[1], cos(ha), sin(ha), Q<double>{1.0, 0.0, 0.0, 0.0});
            } else if (A.hf == kHfSU2) {
                hf_act<kHfSU2>(t[0], t[1], 1.0, 0.0, A.hq(tn, s, a));
            }
            for (int db = 0; db < nd; db++) {
                const Q<double> n = A.ph(tn, pa[a], db);
                const double e0 = n.w - t[db].w, e1 = n.x - t[db].x, e2 = n.y - t[db].y, e3 = n.z - t[db].z;
                obs[kObsGradient] += 0.5 * P.inv_dx[a] * P.inv_dx[a] * (e0 * e0 + e1 * e1 + e2 * e2 + e3 * e3);
            }
        }
        double pot;
        if (model == kModelSM) {
            const double t = fsq[0] - P.eta_sqr;
            pot = 0.25 * P.lambda * t * t;
        } else {
            if (P.break_son) {
                dot = f0.w * f1.w + f0.x * f1.x + f0.y * f1.y + f0.z * f1.z;
                if (P.break_uhalfn) anti = f0.w * f1.x - f0.x * f1.w + f0.y * f1.z - f0.z * f1.y;
            }
            pot = -P.m1 * fsq[0] - P.m2 * fsq[1] + P.l1 * fsq[0] * fsq[0] + P.l2 * fsq[1] * fsq[1] +
                  P.l3 * fsq[0] * fsq[1];
            if (P.break_son) {
                pot += -P.m12r * dot + P.l4p5 * dot * dot + P.l6r * fsq[0] * dot + P.l7r * fsq[1] * dot;
                if (P.break_uhalfn)
                    pot += P.m12i * anti + P.l4m5 * anti * anti - 2.0 * P.l5i * dot * anti - P.l6i * fsq[0] * anti -
                           P.l7i * fsq[1] * anti;
            }
            if (P.apply_norm) pot += P.energy_offset;
        }
        obs[kObsPotential] += pot;
    }
    obs[kObsEnergy] = obs[kObsPotential] + obs[kObsGradient] + obs[kObsKinetic] + obs[kObsMagnetic] + obs[kObsElectric];
    block_reduce_store<kObsCount>(obs, partials + (size_t)blockIdx.x * kStaticSlots, kObsCount);
}

// One block sums the rows in block order (deterministic) and scales.
__global__ void __launch_bounds__(kStaticThreads) static_finalize_kernel(const double* partials, int nblocks,
                                                                          double dv, double inv3n, double invn,
                                                                          double* out)
{
    __shared__ double red[kStaticSlots][kStaticThreads];
    for (int k = 0; k < kStaticSlots; k++) {
        double sum = 0.0, comp = 0.0;
        for (int b = threadIdx.x; b < nblocks; b += blockDim.x) {
            const double v = partials[(size_t)b * kStaticSlots + k];
            const double t = sum + v;
            comp += (fabs(sum) >= fabs(v)) ? (sum - t) + v : (v - t) + sum;
            sum = t;
        }
        red[k][threadIdx.x] = sum + comp;
    }
    __syncthreads();
    if (threadIdx.x < kStaticSlots) {
        const int k = threadIdx.x;
        double sum = 0.0;
        for (int t = 0; t < kStaticThreads; t++) sum += red[k][t];
        double scale = dv;
        if (k == kObsPlaqSU2 || k == kObsPlaqU1) scale = inv3n;
        if (k == kObsPhiSq) scale = invn;
        out[k] = sum * scale;
    }
}

}  // namespace
}  // namespace gft

using namespace gft;

extern "C" int gft_observe_static(const gft_config* c, const float* d_scalars, const float* d_vectors, int time_iter,
                                  double* d_out, void* stream)
{
    if (!c || !d_scalars || !d_vectors || !d_out || time_iter < 0) {
        set_last_error("gft_observe_static: null configuration or buffer, or negative time_iter");
        return GFT_E_INVALID;
    }
    {
        // the same checks as gft_create (lattice extents, spacings, time step, couplings, model)
        // form and storage_bytes are not read here: validate as the mixed form
        gft_config v = *c;
        v.form = GFT_FORM_MIXED;
        v.storage_bytes = 4;
        std::string why;
        const int rc = validate_config(&v, why);
        if (rc != GFT_OK) {
            const std::string pre = "gft_create: ";
            if (why.compare(0, pre.size(), pre) == 0) why = why.substr(pre.size());
            set_last_error("gft_observe_static: " + why);
            return rc;
        }
    }
    if (c->fixed_axes != 0) {
        set_last_error("gft_observe_static: periodic lattices only (fixed_axes must be 0)");
        return GFT_E_UNSUPPORTED;
    }
    if (c->generator_rep) {
        set_last_error("gft_observe_static: quaternion links only (generator_rep = 0)");
        return GFT_E_UNSUPPORTED;
    }
    const long long n = (long long)c->nx * c->ny * c->nz;
    if (n > kStaticMaxSites) {
        set_last_error("gft_observe_static: lattice of " + std::to_string(n) +
                       " sites exceeds the fixed scratch limit of 67108864 sites (16384 blocks x 4096 sites)");
        return GFT_E_UNSUPPORTED;
    }
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
        set_last_error("gft_observe_static: no current CUDA device, or its ordinal is beyond " +
                       std::to_string(kMaxDevices - 1));
        return GFT_E_CUDA;
    }
    double* scratch = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_static_mu);
        if (!g_static_addr[dev]) {
            void* p = nullptr;
            const cudaError_t e = cudaGetSymbolAddress(&p, g_static_partials);
            if (e != cudaSuccess || !p) {
                set_last_error(std::string("gft_observe_static: cudaGetSymbolAddress: ") + cudaGetErrorString(e));
                return GFT_E_CUDA;
            }
            g_static_addr[dev] = static_cast<double*>(p);
        }
        scratch = g_static_addr[dev];
    }
    StepParams P{};
    P.nx = c->nx;
    P.ny = c->ny;
    P.nz = c->nz;
    P.nsite = (int)n;
    P.dt = c->dt;
    const double sp[3] = {c->dx, c->dy, c->dz};
    for (int a = 0; a < 3; a++) {
        P.lap[a] = 1.0 / (sp[a] * sp[a]);
        P.inv_dx[a] = 1.0 / sp[a];
    }
    P.inv_sqr_dt = 1.0 / (c->dt * c->dt);
    const double g2 = c->g * c->g, gp2 = c->gp * c->gp;
    P.inv_g_sqr = (g2 > c->div_tol) ? 1.0 / g2 : 0.0;
    P.inv_gp_sqr = (gp2 > c->div_tol) ? 1.0 / gp2 : 0.0;
    P.lambda = c->lambda;
    P.eta_sqr = c->eta_sqr;
    P.m1 = c->m1;
    P.m2 = c->m2;
    P.l1 = c->l1;
    P.l2 = c->l2;
    P.l3 = c->l3;
    P.m12r = c->m12r;
    P.l4p5 = c->l4p5;
    P.l6r = c->l6r;
    P.l7r = c->l7r;
    P.m12i = c->m12i;
    P.l4m5 = c->l4m5;
    P.l5i = c->l5i;
    P.l6i = c->l6i;
    P.l7i = c->l7i;
    P.break_son = c->break_son;
    P.break_uhalfn = c->break_uhalfn;
    P.apply_norm = c->apply_norm;
    P.energy_offset = c->energy_offset;
    const int hf = (c->model == GFT_MODEL_2HDM) ? c->higgs_family : GFT_HF_NONE;
    const double gpp2 = c->gpp * c->gpp;
    P.inv_gpp_sqr = (gpp2 > c->div_tol) ? 1.0 / gpp2 : 0.0;
    const int nsc = (c->model == GFT_MODEL_SM) ? 4 : 8;
    const int dw = (hf == GFT_HF_SU2) ? 9 : (hf == GFT_HF_U1) ? 6 : 5;  // words per direction
    const AosView A{d_scalars, d_vectors, nsc, (int)n, dw, hf};
    const int tn = (time_iter + 1) % 2;
    const int nblocks = (int)((n + kSitesPerBlock - 1) / kSitesPerBlock);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    static_observe_kernel<<<nblocks, kStaticThreads, 0, s>>>(P, A, tn, c->model, scratch);
    static_finalize_kernel<<<1, kStaticThreads, 0, s>>>(scratch, nblocks, c->dx * c->dy * c->dz, 1.0 / (3.0 * n),
                                                        1.0 / (double)n, d_out);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        set_last_error(std::string("gft_observe_static: launch: ") + cudaGetErrorString(e));
        return GFT_E_CUDA;
    }
    return GFT_OK;
}
