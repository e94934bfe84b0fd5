// devmem.cu -- device memory, pinned host memory and library handles for the
// engines, the batches and the purification objects.
//
// A served stream creates and destroys a molecule's engine every few hundred
// milliseconds while other molecules' kernels keep the GPU busy on other
// streams.  cudaMalloc / cudaFree, cudaFreeHost and the creation and
// destruction of cuBLAS / cuSOLVER handles synchronize the whole device, so
// each of them would wait for every other lane's work in flight.  Here:
//   * device buffers come from the device's stream-ordered memory pool
//     (cudaMallocAsync / cudaFreeAsync on the stream that uses them); a
//     buffer is freed on a stream that orders the free after its last use
//     (its own stream, or any stream once the host has synchronized every
//     stream that used it);
//   * pinned host buffers come from a process-wide free list of blocks that
//     are never returned to the driver;
//   * cuBLAS and cuSOLVER handles are leased from a process-wide pool per
//     device for the duration of one call, and bound to the caller's stream.
#include <cublas_v2.h>
#include <cuda_runtime.h>
#include <cusolverDn.h>

#include <mutex>
#include <vector>

#include "devmem.cuh"
#include "gtf_cuda.h"

namespace {
constexpr int kMaxDev = 64;
std::once_flag g_pool_once[kMaxDev];

// Keep up to 16 GiB of freed blocks in the pool between synchronizations,
// so that the next molecule's buffers are carved from memory already mapped:
// returning many GiB to the driver at a synchronization takes a large
// fraction of a second, which a served stream would otherwise pay at random
// points.  gtf_device_memory counts these cached blocks as free, and
// gtf_device_trim returns them at a quiet moment.
constexpr uint64_t kPoolKeep = 16ull << 30;
void configure_pool(int dev)
{
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, dev) != cudaSuccess) {
        cudaGetLastError();
        return;
    }
    uint64_t thr = kPoolKeep;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
}
}  // namespace

// bytes the current device's pool holds without an allocation in them
extern "C" size_t gtf_pool_cached_bytes(void)
{
    int dev = 0;
    cudaMemPool_t pool;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetDefaultMemPool(&pool, dev) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    uint64_t reserved = 0, used = 0;
    if (cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &reserved) != cudaSuccess ||
        cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemCurrent, &used) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return reserved > used ? (size_t)(reserved - used) : 0;
}

// return the current device's cached pool blocks to the driver, down to
// `keep` bytes (waits for the frees in flight on every stream)
extern "C" int gtf_device_trim(size_t keep)
{
    int dev = 0;
    cudaMemPool_t pool;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetDefaultMemPool(&pool, dev) != cudaSuccess) {
        cudaGetLastError();
        return GTF_ERR_CUDA;
    }
    if (cudaDeviceSynchronize() != cudaSuccess) return GTF_ERR_CUDA;
    return cudaMemPoolTrimTo(pool, keep) == cudaSuccess ? GTF_OK : GTF_ERR_CUDA;
}

extern "C" cudaError_t gtf_dmalloc(void **p, size_t bytes, cudaStream_t st)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev >= 0 && dev < kMaxDev) std::call_once(g_pool_once[dev], configure_pool, dev);
    return cudaMallocAsync(p, bytes ? bytes : 1, st);
}

extern "C" void gtf_dfree(void *p, cudaStream_t st)
{
    if (p) cudaFreeAsync(p, st);
}

// ---------------------------------------------------------------------------
// pinned host blocks: size classes of 2^k bytes (k >= 8), carved from 64 KiB
// (or larger) chunks of cudaMallocHost memory that live until the process ends
// ---------------------------------------------------------------------------
namespace {
struct PinnedPool {
    std::mutex mu;
    std::vector<void *> free_list[48];
};
PinnedPool g_pinned;

int size_class(size_t bytes)
{
    int k = 8;
    while (((size_t)1 << k) < bytes) k++;
    return k;
}
struct PinnedHeader {
    int cls;
    int pad[3];
};
}  // namespace

extern "C" void *gtf_pinned_alloc(size_t bytes)
{
    const int k = size_class(bytes + sizeof(PinnedHeader));
    if (k >= 48) return nullptr;
    const size_t blk = (size_t)1 << k;
    std::lock_guard<std::mutex> lock(g_pinned.mu);
    auto &fl = g_pinned.free_list[k];
    if (fl.empty()) {
        const size_t chunk = blk < (64u << 10) ? (64u << 10) : blk;
        char *c = nullptr;
        if (cudaMallocHost((void **)&c, chunk) != cudaSuccess) {
            cudaGetLastError();
            return nullptr;
        }
        for (size_t o = 0; o + blk <= chunk; o += blk) fl.push_back(c + o);
    }
    PinnedHeader *h = (PinnedHeader *)fl.back();
    fl.pop_back();
    h->cls = k;
    return h + 1;
}

extern "C" void gtf_pinned_free(void *p)
{
    if (!p) return;
    PinnedHeader *h = (PinnedHeader *)p - 1;
    std::lock_guard<std::mutex> lock(g_pinned.mu);
    g_pinned.free_list[h->cls].push_back(h);
}

// ---------------------------------------------------------------------------
// leased library handles.  A handle's workspace may still be in use by work
// queued on the stream of its previous lease, so every lease records an event
// on its stream when it ends, and the next lease makes its own stream wait
// for that event before using the handle.
// ---------------------------------------------------------------------------
namespace {
template <typename H>
struct Pooled {
    H h;
    cudaEvent_t ev;
};
struct HandlePool {
    std::mutex mu;
    std::vector<Pooled<cublasHandle_t>> blas[kMaxDev];
    std::vector<Pooled<cusolverDnHandle_t>> solver[kMaxDev];
};
HandlePool g_handles;

template <typename H>
bool take(std::vector<Pooled<H>> &v, Pooled<H> &out)
{
    std::lock_guard<std::mutex> lock(g_handles.mu);
    if (v.empty()) return false;
    out = v.back();
    v.pop_back();
    return true;
}

template <typename H>
void give(std::vector<Pooled<H>> &v, const Pooled<H> &e)
{
    std::lock_guard<std::mutex> lock(g_handles.mu);
    v.push_back(e);
}
}  // namespace

BlasLease::BlasLease(cudaStream_t s) : st(s)
{
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDev) {
        cudaGetLastError();
        dev = -1;
        return;
    }
    Pooled<cublasHandle_t> e{nullptr, nullptr};
    if (take(g_handles.blas[dev], e)) {
        cudaStreamWaitEvent(st, e.ev, 0);
    } else if (cublasCreate(&e.h) != CUBLAS_STATUS_SUCCESS ||
               cudaEventCreateWithFlags(&e.ev, cudaEventDisableTiming) != cudaSuccess) {
        cudaGetLastError();
        return;
    }
    h = e.h;
    ev = e.ev;
    cublasSetStream(h, st);
}

BlasLease::~BlasLease()
{
    if (!h || dev < 0) return;
    cudaEventRecord(ev, st);
    give(g_handles.blas[dev], Pooled<cublasHandle_t>{h, ev});
}

SolverLease::SolverLease(cudaStream_t s) : st(s)
{
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDev) {
        cudaGetLastError();
        dev = -1;
        return;
    }
    Pooled<cusolverDnHandle_t> e{nullptr, nullptr};
    if (take(g_handles.solver[dev], e)) {
        cudaStreamWaitEvent(st, e.ev, 0);
    } else if (cusolverDnCreate(&e.h) != CUSOLVER_STATUS_SUCCESS ||
               cudaEventCreateWithFlags(&e.ev, cudaEventDisableTiming) != cudaSuccess) {
        cudaGetLastError();
        return;
    }
    h = e.h;
    ev = e.ev;
    cusolverDnSetStream(h, st);
}

SolverLease::~SolverLease()
{
    if (!h || dev < 0) return;
    cudaEventRecord(ev, st);
    give(g_handles.solver[dev], Pooled<cusolverDnHandle_t>{h, ev});
}
