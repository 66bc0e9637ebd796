// shard.cu - row-block sharding of the FP64 system over GPUs.
//
// The system's rows belong to target fibers, and the rows of target fiber i
// depend only on the (replicated, small) positions and orientations: shard r
// of R owns the target fibers [t0(r), t1(r)) = [r M / R, (r + 1) M / R) and
// assembles only their rows (3 N (t1 - t0) rows x n columns), with no
// communication.  Everything else stays replicated on every shard: the state,
// the full-length Krylov vectors and the GMRES control (every shard takes the
// same decisions on the same numbers).  Exchanges, all over NCCL on the
// handle's stream:
//   the product  y = A x     each shard's rows, then one all-gather of the
//                            row blocks (the only per-iteration exchange);
//   the right-hand side      one all-gather per assembly;
//   the velocities           one all-gather of V and one of W per step.
// The all-gather wants equal counts: each shard's block is padded to the
// largest block, and a compaction kernel puts the blocks in row order.
//
// NCCL is loaded at run time (dlopen: RF_NCCL_LIBRARY, or an already loaded
// copy, or libnccl.so.2), so the library itself has no link dependency on it.
#include <dlfcn.h>
#include <nccl.h>

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <string>

#include "handle.h"

namespace rf {

struct NcclApi {
    void *lib = nullptr;
    ncclResult_t (*getUniqueId)(ncclUniqueId *) = nullptr;
    ncclResult_t (*commInitRank)(ncclComm_t *, int, ncclUniqueId, int) = nullptr;
    ncclResult_t (*allGather)(const void *, void *, size_t, ncclDataType_t, ncclComm_t, cudaStream_t) = nullptr;
    ncclResult_t (*commDestroy)(ncclComm_t) = nullptr;
    const char *(*getErrorString)(ncclResult_t) = nullptr;
};

namespace {

NcclApi g_nccl;
std::string g_nccl_err;

// The NCCL library: RF_NCCL_LIBRARY (a path) if set, else the copy already in
// the process (e.g. the one PyTorch loads: a second, older copy under the same
// name would break a later import of PyTorch), else libnccl.so.2.
bool load_nccl() {
    if (g_nccl.lib) return true;
    void *lib = nullptr;
    if (const char *path = getenv("RF_NCCL_LIBRARY")) lib = dlopen(path, RTLD_NOW | RTLD_GLOBAL);
    if (!lib) lib = dlopen("libnccl.so.2", RTLD_NOW | RTLD_NOLOAD);
    if (!lib) lib = dlopen("libnccl.so.2", RTLD_NOW | RTLD_GLOBAL);
    if (!lib) lib = dlopen("libnccl.so", RTLD_NOW | RTLD_GLOBAL);
    if (!lib) {
        const char *m = dlerror();
        g_nccl_err = std::string("cannot load libnccl.so.2: ") + (m ? m : "unknown");
        return false;
    }
    NcclApi a;
    a.lib = lib;
    a.getUniqueId = reinterpret_cast<decltype(a.getUniqueId)>(dlsym(lib, "ncclGetUniqueId"));
    a.commInitRank = reinterpret_cast<decltype(a.commInitRank)>(dlsym(lib, "ncclCommInitRank"));
    a.allGather = reinterpret_cast<decltype(a.allGather)>(dlsym(lib, "ncclAllGather"));
    a.commDestroy = reinterpret_cast<decltype(a.commDestroy)>(dlsym(lib, "ncclCommDestroy"));
    a.getErrorString = reinterpret_cast<decltype(a.getErrorString)>(dlsym(lib, "ncclGetErrorString"));
    if (!a.getUniqueId || !a.commInitRank || !a.allGather || !a.commDestroy || !a.getErrorString) {
        g_nccl_err = "libnccl.so.2 lacks an NCCL entry point";
        return false;
    }
    g_nccl = a;
    return true;
}

// full[e] = gathered[r * pad + e - unit * t0(r)] with r the shard of fiber e / unit
__global__ void compact_kernel(const double *__restrict__ gathered, int64_t pad, int M, int R, int unit,
                               double *__restrict__ full) {
    const int64_t len = (int64_t)unit * M;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < len; e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = e / unit;
        const int r = (int)(((i + 1) * R - 1) / M);  // t0(r) <= i < t0(r + 1)
        const int64_t t0 = (int64_t)r * M / R;
        full[e] = gathered[(int64_t)r * pad + e - (int64_t)unit * t0];
    }
}

}  // namespace

void shard_range(int M, int R, int r, int *t0, int *t1) {
    *t0 = (int)((int64_t)r * M / R);
    *t1 = (int)((int64_t)(r + 1) * M / R);
}

int shard_pad(int M, int R) {
    int pad = 0;
    for (int r = 0; r < R; ++r) {
        int a, b;
        shard_range(M, R, r, &a, &b);
        pad = std::max(pad, b - a);
    }
    return pad;
}

// The local segment of `full` (unit values per fiber of this shard) is copied
// to the send buffer, all shards' segments are gathered and put in order.
cudaError_t shard_allgather(rf_handle *h, double *full, int unit, const double *send_ready) {
    const int R = h->shards;
    const int64_t pad = (int64_t)unit * h->tpad;
    const int64_t len = (int64_t)unit * (h->t1 - h->t0);
    const double *send = send_ready;
    cudaError_t e = cudaSuccess;
    if (!send) {
        e = cudaMemcpyAsync(h->shard_send, full + (int64_t)unit * h->t0, sizeof(double) * len,
                            cudaMemcpyDeviceToDevice, h->stream);
        if (e != cudaSuccess) return e;
        send = h->shard_send;
    }
    const ncclResult_t nr = g_nccl.allGather(send, h->shard_gather, (size_t)pad, ncclFloat64,
                                             reinterpret_cast<ncclComm_t>(h->comm), h->stream);
    if (nr != ncclSuccess) {
        h->err = std::string("ncclAllGather: ") + g_nccl.getErrorString(nr);
        return cudaErrorUnknown;
    }
    compact_kernel<<<(unsigned)std::min<int64_t>(4096, ((int64_t)unit * h->M + 255) / 256), 256, 0, h->stream>>>(
        h->shard_gather, pad, h->M, R, unit, full);
    h->launches++;
    return cudaGetLastError();
}

rf_status shard_attach(rf_handle *h, const uint8_t *id) {
    if (!load_nccl()) return fail(h, RF_ERR_CUDA, g_nccl_err);
    ncclUniqueId uid;
    std::memcpy(uid.internal, id, NCCL_UNIQUE_ID_BYTES);
    ncclComm_t comm = nullptr;
    const ncclResult_t nr = g_nccl.commInitRank(&comm, h->shards, uid, h->shard);
    if (nr != ncclSuccess) return fail(h, RF_ERR_CUDA, std::string("ncclCommInitRank: ") + g_nccl.getErrorString(nr));
    h->comm = comm;
    const size_t pad = (size_t)std::max<int64_t>(3LL * h->N, 3) * h->tpad;  // the largest unit is 3 N
    if (cudaMalloc(&h->shard_send, sizeof(double) * pad) != cudaSuccess ||
        cudaMalloc(&h->shard_gather, sizeof(double) * pad * h->shards) != cudaSuccess)
        return fail(h, RF_ERR_OOM, "shard exchange buffers");
    return RF_OK;
}

void shard_detach(rf_handle *h) {
    if (h->comm && g_nccl.commDestroy) g_nccl.commDestroy(reinterpret_cast<ncclComm_t>(h->comm));
    h->comm = nullptr;
    cudaFree(h->shard_send);
    cudaFree(h->shard_gather);
    h->shard_send = h->shard_gather = nullptr;
}

}  // namespace rf

extern "C" rf_status rf_shard_unique_id(uint8_t *id) {
    if (!id) return rf::fail(nullptr, RF_ERR_INVALID_ARG, "id is null");
    if (!rf::load_nccl()) return rf::fail(nullptr, RF_ERR_CUDA, rf::g_nccl_err);
    ncclUniqueId uid;
    const ncclResult_t nr = rf::g_nccl.getUniqueId(&uid);
    if (nr != ncclSuccess)
        return rf::fail(nullptr, RF_ERR_CUDA, std::string("ncclGetUniqueId: ") + rf::g_nccl.getErrorString(nr));
    std::memcpy(id, uid.internal, NCCL_UNIQUE_ID_BYTES);
    return RF_OK;
}

extern "C" rf_status rf_shard_range(int32_t M, int32_t shard_count, int32_t shard_index, int32_t *t0, int32_t *t1) {
    if (!t0 || !t1 || M < 1 || shard_count < 1 || shard_count > M || shard_index < 0 || shard_index >= shard_count)
        return rf::fail(nullptr, RF_ERR_INVALID_ARG, "rf_shard_range: need 1 <= shard_count <= M, 0 <= index < count");
    int a, b;
    rf::shard_range(M, shard_count, shard_index, &a, &b);
    *t0 = a;
    *t1 = b;
    return RF_OK;
}
