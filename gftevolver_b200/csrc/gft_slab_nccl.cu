// gft_slab_nccl.cu -- the x-slab ghost-plane exchange over NCCL, inside the library.
//
// The reference marks where a distributed run would exchange boundary data
// ("send here without blocking ... recv just before", Core/Source/Lattice.cpp:779).
// With an x-slab decomposition each rank sends its first own plane to the left
// neighbour and its last own plane to the right one, and receives the
// neighbours' planes into its two ghost planes, once per step.  gft_evolve
// posts that exchange itself, as one NCCL group of point-to-point operations on
// a stream of its own, so that the interior planes are computed while the
// boundary planes are in flight, and no host callback runs per step.
//
// NCCL is loaded at run time (dlopen of libnccl.so.2; in a process that has
// already loaded it, e.g. through torch.distributed, that copy is reused), so
// the library does not depend on it unless this path is used.
#include <dlfcn.h>
#include <nccl.h>

#include <chrono>
#include <cstring>
#include <mutex>
#include <string>
#include <thread>

#include "gft_launch.h"

namespace gft {

namespace {

struct NcclApi {
    ncclResult_t (*get_unique_id)(ncclUniqueId*) = nullptr;
    ncclResult_t (*comm_init_rank)(ncclComm_t*, int, ncclUniqueId, int) = nullptr;
    ncclResult_t (*comm_destroy)(ncclComm_t) = nullptr;
    ncclResult_t (*comm_abort)(ncclComm_t) = nullptr;
    ncclResult_t (*comm_get_async_error)(ncclComm_t, ncclResult_t*) = nullptr;
    ncclResult_t (*group_start)() = nullptr;
    ncclResult_t (*group_end)() = nullptr;
    ncclResult_t (*send)(const void*, size_t, ncclDataType_t, int, ncclComm_t, cudaStream_t) = nullptr;
    ncclResult_t (*recv)(void*, size_t, ncclDataType_t, int, ncclComm_t, cudaStream_t) = nullptr;
    const char* (*error_string)(ncclResult_t) = nullptr;
};

std::mutex g_nccl_mu;
NcclApi g_nccl;
bool g_nccl_tried = false;
std::string g_nccl_why;

const NcclApi* nccl_api(std::string& why)
{
    std::lock_guard<std::mutex> lk(g_nccl_mu);
    if (!g_nccl_tried) {
        g_nccl_tried = true;
        void* lib = dlopen("libnccl.so.2", RTLD_NOW | RTLD_GLOBAL | RTLD_NOLOAD);  // already in the process
        if (!lib) lib = dlopen("libnccl.so.2", RTLD_NOW | RTLD_GLOBAL);
        if (!lib) {
            g_nccl_why = std::string("libnccl.so.2 could not be loaded: ") + dlerror();
        } else {
            auto sym = [&](const char* name) { return dlsym(lib, name); };
            NcclApi a;
            a.get_unique_id = reinterpret_cast<decltype(a.get_unique_id)>(sym("ncclGetUniqueId"));
            a.comm_init_rank = reinterpret_cast<decltype(a.comm_init_rank)>(sym("ncclCommInitRank"));
            a.comm_destroy = reinterpret_cast<decltype(a.comm_destroy)>(sym("ncclCommDestroy"));
            a.comm_abort = reinterpret_cast<decltype(a.comm_abort)>(sym("ncclCommAbort"));
            a.comm_get_async_error = reinterpret_cast<decltype(a.comm_get_async_error)>(sym("ncclCommGetAsyncError"));
            a.group_start = reinterpret_cast<decltype(a.group_start)>(sym("ncclGroupStart"));
            a.group_end = reinterpret_cast<decltype(a.group_end)>(sym("ncclGroupEnd"));
            a.send = reinterpret_cast<decltype(a.send)>(sym("ncclSend"));
            a.recv = reinterpret_cast<decltype(a.recv)>(sym("ncclRecv"));
            a.error_string = reinterpret_cast<decltype(a.error_string)>(sym("ncclGetErrorString"));
            if (a.get_unique_id && a.comm_init_rank && a.comm_destroy && a.comm_abort && a.comm_get_async_error &&
                a.group_start && a.group_end && a.send && a.recv && a.error_string)
                g_nccl = a;
            else
                g_nccl_why = "libnccl.so.2 lacks a point-to-point entry point (NCCL >= 2.7 is needed)";
        }
    }
    if (!g_nccl.send) {
        why = g_nccl_why;
        return nullptr;
    }
    return &g_nccl;
}

std::string nccl_msg(const NcclApi* a, const char* what, ncclResult_t r)
{
    return std::string(what) + ": " + (a ? a->error_string(r) : "NCCL");
}

}  // namespace

struct SlabComm {
    const NcclApi* api = nullptr;
    ncclComm_t comm = nullptr;
    int nranks = 1, rank = 0, left = 0, right = 0;
};

int nccl_unique_id(unsigned char* out, std::string& why)
{
    const NcclApi* a = nccl_api(why);
    if (!a) return GFT_E_UNSUPPORTED;
    static_assert(sizeof(ncclUniqueId) == kNcclIdBytes, "ncclUniqueId size");
    ncclUniqueId id;
    const ncclResult_t r = a->get_unique_id(&id);
    if (r != ncclSuccess) {
        why = nccl_msg(a, "ncclGetUniqueId", r);
        return GFT_E_CUDA;
    }
    std::memcpy(out, &id, sizeof(id));
    return GFT_OK;
}

int slab_comm_create(const unsigned char* id_bytes, int nranks, int rank, SlabComm** out, std::string& why)
{
    const NcclApi* a = nccl_api(why);
    if (!a) return GFT_E_UNSUPPORTED;
    ncclUniqueId id;
    std::memcpy(&id, id_bytes, sizeof(id));
    SlabComm* c = new SlabComm;
    c->api = a;
    c->nranks = nranks;
    c->rank = rank;
    c->left = (rank + nranks - 1) % nranks;
    c->right = (rank + 1) % nranks;
    const ncclResult_t r = a->comm_init_rank(&c->comm, nranks, id, rank);
    if (r != ncclSuccess) {
        why = nccl_msg(a, "ncclCommInitRank", r);
        delete c;
        return GFT_E_CUDA;
    }
    *out = c;
    return GFT_OK;
}

void slab_comm_destroy(SlabComm* c, bool abort)
{
    if (!c) return;
    if (c->comm) (abort ? c->api->comm_abort : c->api->comm_destroy)(c->comm);
    delete c;
}

// One group per exchange; per field array, in the same order on every rank:
// send the first own plane left, receive the right ghost from the right,
// send the last own plane right, receive the left ghost from the left.
// Messages between two ranks match in posting order, so the pairs line up also
// when left and right are the same rank (two ranks) or this rank (one).
int slab_comm_exchange(SlabComm* c, const SlabPlanes& pl, cudaStream_t stream, std::string& why)
{
    const NcclApi* a = c->api;
    ncclResult_t r = a->group_start();
    for (int k = 0; k < pl.n && r == ncclSuccess; k++) {
        const size_t b = pl.bytes[k];
        if ((r = a->send(pl.send_lo[k], b, ncclChar, c->left, c->comm, stream)) != ncclSuccess) break;
        if ((r = a->recv(pl.recv_hi[k], b, ncclChar, c->right, c->comm, stream)) != ncclSuccess) break;
        if ((r = a->send(pl.send_hi[k], b, ncclChar, c->right, c->comm, stream)) != ncclSuccess) break;
        r = a->recv(pl.recv_lo[k], b, ncclChar, c->left, c->comm, stream);
    }
    const ncclResult_t e = a->group_end();
    if (r == ncclSuccess) r = e;
    if (r != ncclSuccess) {
        why = nccl_msg(a, "slab exchange", r);
        return GFT_E_CUDA;
    }
    return GFT_OK;
}

// Waits for `stream` with a time limit, watching the communicator for
// asynchronous errors; on either the communicator is aborted (its operations
// in flight are cancelled), so the caller returns an error instead of waiting
// for good on a peer that is gone.
int slab_comm_wait(SlabComm* c, cudaStream_t stream, double seconds, std::string& why)
{
    const auto t0 = std::chrono::steady_clock::now();
    for (;;) {
        const cudaError_t q = cudaStreamQuery(stream);
        if (q == cudaSuccess) return GFT_OK;
        if (q != cudaErrorNotReady) {
            why = std::string("slab exchange: ") + cudaGetErrorString(q);
            return GFT_E_CUDA;
        }
        if (c) {
            ncclResult_t ae = ncclSuccess;
            c->api->comm_get_async_error(c->comm, &ae);
            if (ae != ncclSuccess && ae != ncclInProgress) {
                why = nccl_msg(c->api, "slab exchange (asynchronous)", ae);
                c->api->comm_abort(c->comm);
                c->comm = nullptr;
                return GFT_E_CUDA;
            }
        }
        const double el = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        if (el > seconds) {
            why = "slab exchange: no completion within " + std::to_string((int)seconds) + " s (a peer is gone?)";
            if (c && c->comm) {
                c->api->comm_abort(c->comm);
                c->comm = nullptr;
            }
            return GFT_E_TIMEOUT;
        }
        std::this_thread::sleep_for(std::chrono::microseconds(50));
    }
}

bool slab_comm_alive(const SlabComm* c) { return c && c->comm; }

}  // namespace gft
