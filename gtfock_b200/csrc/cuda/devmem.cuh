// devmem.cuh -- stream-ordered device buffers, pinned host blocks and leased
// cuBLAS / cuSOLVER handles (devmem.cu)
#pragma once

#include <cublas_v2.h>
#include <cuda_runtime.h>
#include <cusolverDn.h>

extern "C" {
// device buffer from the current device's memory pool, ordered on `st`
cudaError_t gtf_dmalloc(void **p, size_t bytes, cudaStream_t st);
// free ordered on `st`: every use of p must be ordered before it on `st`,
// or have completed (host-synchronized) before the call
void gtf_dfree(void *p, cudaStream_t st);
// unallocated bytes cached in the current device's pool
size_t gtf_pool_cached_bytes(void);
// pinned host block (never returned to the driver; reused by later calls)
void *gtf_pinned_alloc(size_t bytes);
void gtf_pinned_free(void *p);
}

// A cuBLAS / cuSOLVER handle of the current device for the lifetime of the
// object, bound to `st`; h is null if none could be created.  Handles return
// to a process-wide pool instead of being destroyed, since a destruction
// synchronizes the device; the next lease's stream waits for the work this
// lease queued with the handle.
struct BlasLease {
    cublasHandle_t h = nullptr;
    cudaEvent_t ev = nullptr;
    cudaStream_t st = nullptr;
    int dev = -1;
    explicit BlasLease(cudaStream_t st);
    ~BlasLease();
    BlasLease(const BlasLease &) = delete;
    BlasLease &operator=(const BlasLease &) = delete;
};

struct SolverLease {
    cusolverDnHandle_t h = nullptr;
    cudaEvent_t ev = nullptr;
    cudaStream_t st = nullptr;
    int dev = -1;
    explicit SolverLease(cudaStream_t st);
    ~SolverLease();
    SolverLease(const SolverLease &) = delete;
    SolverLease &operator=(const SolverLease &) = delete;
};
