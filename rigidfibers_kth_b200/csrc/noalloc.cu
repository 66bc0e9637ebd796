// noalloc.cu - a matrix-vector product for callers that cannot allocate
// device memory.
//
// Who needs it: a host application whose device memory is owned by its own
// allocator or memory pool (the cudaMalloc of a library would compete with
// that pool, or fail when the pool holds the memory), and a caller inside a
// loop that must not stall, since cudaMalloc and cudaFree can synchronise the
// device.  Such callers hand in their own device buffers for A, x and y; the
// partial sums the product needs live in one fixed array inside this
// library.  With CUDA's default lazy module loading the driver reserves the
// array on a device when this file's device code is first used there: at the
// cudaGetSymbolAddress of the first call on that device.
//
// The product is the streaming column-major GEMV of the solver (linalg.cu):
// column ranges are split across the grid and the per-split partial sums are
// added in a fixed order by a second kernel.  Here the partial sums go to
// g_noalloc_scratch instead of a buffer allocated with the handle.
#include <mutex>
#include <string>

#include "handle.h"

namespace {

// 8 MiB of partial sums (1,048,576 doubles).  Every GPU on which the entry
// point has been called keeps this array resident until the process exits.
constexpr int64_t kScratchDoubles = 1 << 20;
static __device__ __align__(256) double g_noalloc_scratch[kScratchDoubles];

// Device address of the array per device ordinal.  The symbol's host-side
// name is only a stand-in; a kernel needs the address returned by
// cudaGetSymbolAddress with that device current.
constexpr int kMaxDevices = 64;
std::mutex g_mu;
double *g_scratch_ptr[kMaxDevices] = {};
int g_sm_count[kMaxDevices] = {};

// the message is read back with rf_last_error(NULL)
rf_status fail(rf_status s, const std::string &msg) { return rf::fail(nullptr, s, msg); }

// GEMV row tile for FP64 storage: 256 threads x 2 rows
constexpr int64_t kRowTile = 512;

}  // namespace

extern "C" rf_status rf_matvec_noalloc(const double *A, int64_t lda, int64_t n, const double *x, double *y,
                                       void *stream) {
    // argument checks come first and touch no device state
    if (!A || !x || !y) return fail(RF_ERR_INVALID_ARG, "rf_matvec_noalloc: null pointer");
    if (n < 1 || lda < n) return fail(RF_ERR_INVALID_ARG, "rf_matvec_noalloc: need n >= 1 and lda >= n");
    if (lda % 2 != 0 || (reinterpret_cast<uintptr_t>(A) & 15) != 0)
        return fail(RF_ERR_INVALID_ARG, "rf_matvec_noalloc: lda must be even and A 16-byte aligned");
    const int64_t mpad = (lda + kRowTile - 1) / kRowTile * kRowTile;
    if (mpad > kScratchDoubles)
        return fail(RF_ERR_INVALID_ARG,
                    "rf_matvec_noalloc: lda exceeds the 1048576-row limit of the built-in scratch array");

    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(RF_ERR_NO_DEVICE, std::string("rf_matvec_noalloc: ") + cudaGetErrorString(e));
    }
    if (dev < 0 || dev >= kMaxDevices) return fail(RF_ERR_INVALID_ARG, "rf_matvec_noalloc: device ordinal too large");
    double *scratch = nullptr;
    int sms = 0;
    {
        // first call on a device: resolve the array's address with that device current
        std::lock_guard<std::mutex> lock(g_mu);
        if (!g_scratch_ptr[dev]) {
            void *p = nullptr;
            e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
            if (e != cudaSuccess) {
                cudaGetLastError();
                return fail(RF_ERR_CUDA, std::string("rf_matvec_noalloc: cudaGetSymbolAddress: ") +
                                             cudaGetErrorString(e));
            }
            int count = 0;
            e = cudaDeviceGetAttribute(&count, cudaDevAttrMultiProcessorCount, dev);
            if (e != cudaSuccess) {
                cudaGetLastError();
                return fail(RF_ERR_CUDA, std::string("rf_matvec_noalloc: ") + cudaGetErrorString(e));
            }
            g_scratch_ptr[dev] = static_cast<double *>(p);
            g_sm_count[dev] = count;
        }
        scratch = g_scratch_ptr[dev];
        sms = g_sm_count[dev];
    }
    // every partial sum that the reduction reads is written earlier in the
    // same call, so nothing in the array needs to start at zero
    e = rf::launch_gemv<double, double, double, double>(A, lda, n, n, x, y, nullptr, scratch, kScratchDoubles, sms,
                                                       static_cast<cudaStream_t>(stream));
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(RF_ERR_CUDA, std::string("rf_matvec_noalloc: launch: ") + cudaGetErrorString(e));
    }
    return RF_OK;
}
