// Allocation-free entry point: the blocked LDL' of one dense front with all
// of its scratch in a fixed, file-scope device array.
//
// Who needs it: callers that must not call cudaMalloc/cudaFree themselves or
// through this library -- e.g. a host application whose allocator owns every
// byte of device memory (a pool handed out by another framework), or a
// time-critical loop where an allocation would synchronise the device.  They
// pass the matrix and the pivot vector (device memory they already own); the
// scratch (diagonal copy, inverses of the 64x64 diagonal blocks, job
// descriptors, status words) lives in g_dense_scratch below.
//
// Limits and sharing:
//  * n <= kNoAllocMaxN (8192); larger fronts are rejected with -3.
//  * g_dense_scratch (5 MiB) is a file-scope __device__ array: every GPU that
//    loads the library holds it until the process exits.
//  * All calls share it and it keeps the last call's contents; each call
//    re-initialises what must start at zero.  Calls that overlap on the GPU
//    (different streams, or several host threads) race on it: serialise them.
//  * The first call on a device looks up the array's device address
//    (cudaGetSymbolAddress) with that device current; make that first call
//    before any stream capture.
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>

#include "engine.h"

namespace {

constexpr int64_t kNoAllocMaxN = 8192;
constexpr size_t kNoAllocBytes = (size_t)5 << 20;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_dense_scratch[kNoAllocBytes];

std::mutex g_setup_mu;
void* g_scratch_ptr[kMaxDevices] = {nullptr};

// Device address of g_dense_scratch on the current device (set up once per device).
void* scratch_address(int& err) {
    err = 0;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
        err = -4;
        return nullptr;
    }
    std::lock_guard<std::mutex> lk(g_setup_mu);
    if (!g_scratch_ptr[dev]) {
        void* p = nullptr;
        if (cudaGetSymbolAddress(&p, g_dense_scratch) != cudaSuccess || !p) {
            err = -4;
            return nullptr;
        }
        // the kernels' shared-memory opt-in, so that the first call in a
        // process (before any other entry point of this library) runs too
        if (sprb::dense_factor_setup() != 0) {
            err = -4;
            return nullptr;
        }
        g_scratch_ptr[dev] = p;
    }
    return g_scratch_ptr[dev];
}

}  // namespace

extern "C" {

// LDL' factorisation of a dense symmetric n x n matrix on the device, in
// place, without allocating device memory.  See include/spr_b200.h.
int spr_b200_dense_ldlt_noalloc(double* d_a, int64_t n, int64_t lda, double tol1, double* d_d, void* stream,
                                double* out) {
    if (n > kNoAllocMaxN || sprb::dense_scratch_bytes(n) > kNoAllocBytes) return -3;
    int err = 0;
    void* scratch = scratch_address(err);
    if (!scratch) return err;
    return sprb::dense_factor_with_scratch(d_a, n, lda, tol1, d_d, scratch, kNoAllocBytes, (cudaStream_t)stream,
                                           out);
}

}  // extern "C"
