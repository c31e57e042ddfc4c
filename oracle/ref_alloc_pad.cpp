/*
 * ref_alloc_pad.cpp -- every cudaMalloc of the reference build made larger.
 * TEST INFRASTRUCTURE ONLY (oracle/Makefile.ref, linked into
 * oracle/_ref/ref_engine with the shared CUDA runtime).
 *
 * The reference's setupDeadCells kernel tests `idx <= frameH * frameW`
 * (FDTDSolver.cu:823), so when frameH * frameW is not a multiple of its
 * 256-thread blocks one thread writes the cell_type of element
 * frameH * frameW, one past the end of PV_N (resized to frameH * frameW,
 * FDTDSolver.cu:564).  This definition of cudaMalloc takes precedence over the
 * runtime library's for every call made from the executable (thrust's
 * device_vector allocates through cudaMalloc, thrust/system/cuda/
 * memory_resource.h), forwards to the runtime with kPad extra bytes, and
 * counts the calls, so that write lands inside the same allocation.
 * ref_engine checks, before any reference code runs, that a thrust
 * device_vector allocation came through here.
 */
#include <cuda_runtime_api.h>
#include <dlfcn.h>

#include <cstddef>

namespace {
constexpr size_t kPad = 4096;
using MallocFn = cudaError_t (*)(void**, size_t);
}  // namespace

extern "C" {

unsigned long long ref_pad_calls = 0;
size_t ref_pad_last_request = 0;

cudaError_t cudaMalloc(void** ptr, size_t bytes) {
    static MallocFn real = reinterpret_cast<MallocFn>(dlsym(RTLD_NEXT, "cudaMalloc"));
    if (!real) return cudaErrorInitializationError;
    ++ref_pad_calls;
    ref_pad_last_request = bytes;
    return real(ptr, bytes + kPad);
}

}  // extern "C"
