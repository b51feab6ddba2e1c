// chemgen_getrates_noalloc: FP64 getrates that allocates no device memory.
//
// Some callers cannot call cudaMalloc while they run: solvers that own the
// whole device memory pool (or forbid allocation inside their time-step
// loop) and code that must not synchronise the device, which cudaMalloc and
// cudaFree can do.  For them this entry point runs the FP64 kernel whose
// per-point state lives in global scratch (the variant used for large
// mechanisms) with that scratch in a fixed, file-scope device array instead
// of a library allocation.
//
// Limits and behaviour:
// * the array holds kNoallocScratchBytes (16 MiB) on every GPU where the
//   module of this file has been loaded, until the process exits.  Under
//   CUDA's lazy module loading (the default) that happens at the first use of
//   the module on a device -- at the latest at this entry point's first call
//   there, which may then allocate the array and synchronise the device.  A
//   caller that must not allocate or synchronise in its loop makes one call
//   per device during set-up;
// * the kernel keeps 3*ns*64 doubles of state per resident block; a
//   mechanism whose single block slice exceeds the array (ns > 10922) is
//   rejected with CHEMGEN_ERR_TOO_LARGE; fewer slices than the GPU could run
//   only lower the number of persistent blocks;
// * the first call on a device also looks up the array's device address
//   (cudaGetSymbolAddress) with that device current; make that first call
//   during set-up, before any stream capture;
// * every call shares the one array: calls that overlap on the GPU (two
//   streams, two host threads) race on it.  Each call writes every state
//   value before reading it, so nothing has to start at zero.
#include <cuda_runtime.h>

#include <mutex>

#include "../../include/chemgen_b200.h"
#include "dev_mech.cuh"

namespace cg {
cudaError_t launch_getrates_fp64(const DevMech& m, const double* P, const double* T, const double* Y, double* wdot,
                                 int64_t ng, int block, double* scratch, int64_t scratch_blocks, cudaStream_t s);
size_t fp64_global_slice_bytes(int ns);
const DevMech* handle_mech(const chemgen_handle* h, int* device, int64_t* max_slices);
}  // namespace cg

namespace {

constexpr size_t kNoallocScratchBytes = (size_t)16 << 20;
__device__ __align__(256) double g_noalloc_scratch[kNoallocScratchBytes / sizeof(double)];

constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mu;
double* g_noalloc_ptr[kMaxDevices] = {};

// Device address of the array on `device` (which is current); once per device.
cudaError_t noalloc_scratch(int device, double** out) {
    if (device < 0 || device >= kMaxDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_ptr[device]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return e;
        g_noalloc_ptr[device] = static_cast<double*>(p);
    }
    *out = g_noalloc_ptr[device];
    return cudaSuccess;
}

}  // namespace

extern "C" int chemgen_getrates_noalloc(chemgen_handle* h, const double* P, const double* T, int64_t ng,
                                        const double* Y, double* wdot, void* stream) {
    if (!h || ng < 0) return CHEMGEN_ERR_INVALID_ARGUMENT;
    if (ng == 0) return CHEMGEN_OK;
    if (!P || !T || !Y || !wdot) return CHEMGEN_ERR_INVALID_ARGUMENT;
    auto misaligned = [](const void* p) { return (reinterpret_cast<uintptr_t>(p) & 7u) != 0; };
    if (misaligned(P) || misaligned(T) || misaligned(Y) || misaligned(wdot)) return CHEMGEN_ERR_MISALIGNED;
    int device = 0;
    int64_t max_slices = 0;
    const cg::DevMech* m = cg::handle_mech(h, &device, &max_slices);
    const size_t slice = cg::fp64_global_slice_bytes(m->ns);
    if (slice > kNoallocScratchBytes) return CHEMGEN_ERR_TOO_LARGE;
    int prev = -1;
    if (cudaGetDevice(&prev) != cudaSuccess) return CHEMGEN_ERR_CUDA;
    if (prev != device && cudaSetDevice(device) != cudaSuccess) return CHEMGEN_ERR_CUDA;
    double* scratch = nullptr;
    cudaError_t e = noalloc_scratch(device, &scratch);
    if (e == cudaSuccess) {
        int64_t slices = (int64_t)(kNoallocScratchBytes / slice);
        if (slices > max_slices) slices = max_slices;
        e = cg::launch_getrates_fp64(*m, P, T, Y, wdot, ng, 0, scratch, slices, (cudaStream_t)stream);
    }
    if (prev != device) cudaSetDevice(prev);
    return e == cudaSuccess ? CHEMGEN_OK : CHEMGEN_ERR_CUDA;
}
