// purif_bf16.cu -- split-precision products for the purification on the
// tensor cores (tcgen05 / TMEM / TMA, through the CUTLASS sm100 GEMM
// templates instantiated here).
//
// A symmetric-product step of canonical purification needs C = A B^T with
// A, B close to idempotent density matrices (|elements| <= 1).  Each FP64
// operand is split into two BF16 matrices, X = X_hi + X_lo with
// X_hi = bf16(X) and X_lo = bf16(X - X_hi), and
//     C ~= A_hi B_hi^T + A_hi B_lo^T + A_lo B_hi^T
// is one batched BF16 GEMM (batch L = 3, one term each) with FP32
// accumulation: A' = [A_hi | A_hi | A_lo], B' = [B_hi | B_lo | B_hi] row by
// row, batch l reading column block l of both; the three FP32 products are
// summed in FP64.  Three batches of (n / 128)^2 output tiles keep the SMs
// busy at n ~ 830 (147 CTAs for 148 SMs, against 49 for one GEMM over the
// stacked K = 3 n).  The dropped A_lo B_lo^T term and the BF16 rounding of
// the low parts leave a relative error near 2^-16 per product, which is why
// the purification finishes with FP64 steps.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cutlass/cutlass.h>
#include <cute/tensor.hpp>
#include <cutlass/epilogue/collective/collective_builder.hpp>
#include <cutlass/gemm/collective/collective_builder.hpp>
#include <cutlass/gemm/device/gemm_universal_adapter.h>
#include <cutlass/gemm/kernel/gemm_universal.hpp>
#include <cutlass/util/packed_stride.hpp>

#include <type_traits>

#include "devmem.cuh"
#include "gtf_cuda.h"

extern "C" void gtf_note_launches(int n);

namespace {
using namespace cute;
using ElementIn = cutlass::bfloat16_t;
using ElementOut = float;
using ElementAcc = float;
using LayoutA = cutlass::layout::RowMajor;      // A'  (m x 3n)
using LayoutB = cutlass::layout::ColumnMajor;   // B'^T stored row by row = B' column-major (3n x n)
using LayoutC = cutlass::layout::RowMajor;
constexpr int kAlignIn = 8, kAlignOut = 4;
using TileShape = Shape<_128, _128, _64>;
using ClusterShape = Shape<_1, _1, _1>;         // one CTA per tile: no cluster multicast
using Epilogue = typename cutlass::epilogue::collective::CollectiveBuilder<
    cutlass::arch::Sm100, cutlass::arch::OpClassTensorOp, TileShape, ClusterShape,
    cutlass::epilogue::collective::EpilogueTileAuto, ElementAcc, ElementAcc, ElementOut, LayoutC, kAlignOut,
    ElementOut, LayoutC, kAlignOut, cutlass::epilogue::collective::EpilogueScheduleAuto>::CollectiveOp;
using Mainloop = typename cutlass::gemm::collective::CollectiveBuilder<
    cutlass::arch::Sm100, cutlass::arch::OpClassTensorOp, ElementIn, LayoutA, kAlignIn, ElementIn, LayoutB,
    kAlignIn, ElementAcc, TileShape, ClusterShape,
    cutlass::gemm::collective::StageCountAutoCarveout<static_cast<int>(sizeof(typename Epilogue::SharedStorage))>,
    cutlass::gemm::collective::KernelScheduleAuto>::CollectiveOp;
using Kernel = cutlass::gemm::kernel::GemmUniversal<Shape<int, int, int, int>, Mainloop, Epilogue, void>;
using Gemm = cutlass::gemm::device::GemmUniversalAdapter<Kernel>;
}  // namespace

// X (n x n FP64, row-major) -> rows of the stacked BF16 operand:
// A role: [hi | hi | lo],  B role: [hi | lo | hi]; ld = 3 * np, np >= n padded to 8
__global__ void k_split_bf16(const double *__restrict__ X, int n, int np, int role, __nv_bfloat16 *__restrict__ out)
{
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = blockIdx.y;
    if (j >= np) return;
    const double x = (j < n) ? X[(size_t)i * n + j] : 0.0;
    const __nv_bfloat16 hi = __double2bfloat16(x);
    const __nv_bfloat16 lo = __double2bfloat16(x - (double)__bfloat162float(hi));
    __nv_bfloat16 *row = out + (size_t)i * 3 * np;
    row[j] = hi;
    row[np + j] = role == 0 ? hi : lo;
    row[2 * np + j] = role == 0 ? lo : hi;
}

// C_0 + C_1 + C_2 (three n x np FP32 batches) -> n x n FP64
__global__ void k_sum3_f64(const float *__restrict__ C, int n, int np, double *__restrict__ out)
{
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = blockIdx.y;
    if (j >= n) return;
    const size_t o = (size_t)i * np + j, b = (size_t)n * np;
    out[(size_t)i * n + j] = (double)C[o] + (double)C[o + b] + (double)C[o + 2 * b];
}

struct gtf_bf16x3 {
    int n, np;
    __nv_bfloat16 *A, *B;
    float *C;
    void *ws;
    size_t ws_bytes;
    cudaStream_t st;   // the buffers' stream (stream-ordered pool, devmem.cu)
};

// The B operand has np rows (rows n..np-1 zero) so that the output's
// contiguous dimension N = np meets the epilogue's 16-byte alignment.
// Buffers on `stream` (the purification object's); the products must run on
// the same stream, and the caller synchronizes it before destroying.
extern "C" int gtf_bf16x3_create(int n, void *stream, gtf_bf16x3_t **out)
{
    *out = nullptr;
    gtf_bf16x3 *g = new gtf_bf16x3();
    g->n = n;
    g->np = (n + 7) / 8 * 8;
    g->st = (cudaStream_t)stream;
    const size_t ab = sizeof(__nv_bfloat16) * (size_t)g->np * 3 * g->np;
    if (gtf_dmalloc((void **)&g->A, ab, g->st) != cudaSuccess || gtf_dmalloc((void **)&g->B, ab, g->st) != cudaSuccess ||
        gtf_dmalloc((void **)&g->C, sizeof(float) * 3 * (size_t)n * g->np, g->st) != cudaSuccess ||
        cudaMemsetAsync(g->B, 0, ab, g->st) != cudaSuccess) {
        gtf_bf16x3_destroy(g);
        return GTF_ERR_ALLOC;
    }
    g->ws = nullptr;
    g->ws_bytes = 0;
    *out = g;
    return GTF_OK;
}

extern "C" void gtf_bf16x3_destroy(gtf_bf16x3_t *g)
{
    if (!g) return;
    gtf_dfree(g->A, g->st);
    gtf_dfree(g->B, g->st);
    gtf_dfree(g->C, g->st);
    gtf_dfree(g->ws, g->st);
    delete g;
}

// C = A B^T (n x n, FP64 in and out) with the split BF16 product
extern "C" int gtf_bf16x3_abt(gtf_bf16x3_t *g, const double *A, const double *B, double *C, void *stream)
{
    cudaStream_t st = (cudaStream_t)stream;
    const int n = g->n, np = g->np;
    dim3 blk(128), grd((np + 127) / 128, n);
    k_split_bf16<<<grd, blk, 0, st>>>(A, n, np, 0, g->A);
    k_split_bf16<<<grd, blk, 0, st>>>(B, n, np, 1, g->B);
    if (cudaGetLastError() != cudaSuccess) return GTF_ERR_CUDA;
    using StrideA = typename Gemm::GemmKernel::StrideA;
    using StrideB = typename Gemm::GemmKernel::StrideB;
    using StrideC = typename Gemm::GemmKernel::StrideC;
    // batch l: columns [l np, (l + 1) np) of the stacked rows (leading
    // dimension 3 np) for A' and B'; its own n x np FP32 output
    const int M = n, N = np, K = np, L = 3;
    StrideA sa = cute::make_stride(int64_t(3 * np), cute::Int<1>{}, int64_t(np));
    StrideB sb = cute::make_stride(int64_t(3 * np), cute::Int<1>{}, int64_t(np));
    StrideC sc = cute::make_stride(int64_t(np), cute::Int<1>{}, int64_t(n) * np);
    static_assert(std::is_same<StrideA, cute::Stride<int64_t, cute::Int<1>, int64_t>>::value, "row-major A");
    static_assert(std::is_same<StrideB, cute::Stride<int64_t, cute::Int<1>, int64_t>>::value, "K-major B");
    static_assert(std::is_same<StrideC, cute::Stride<int64_t, cute::Int<1>, int64_t>>::value, "row-major C");
    typename Gemm::Arguments args{cutlass::gemm::GemmUniversalMode::kBatched,
                                  {M, N, K, L},
                                  {reinterpret_cast<const ElementIn *>(g->A), sa,
                                   reinterpret_cast<const ElementIn *>(g->B), sb},
                                  {{1.0f, 0.0f}, g->C, sc, g->C, sc}};
    Gemm gemm;
    if (gemm.can_implement(args) != cutlass::Status::kSuccess) return GTF_ERR_INVALID;
    const size_t need = Gemm::get_workspace_size(args);
    if (need > g->ws_bytes) {
        gtf_dfree(g->ws, st);   // ordered after the previous products on st
        g->ws = nullptr;
        if (gtf_dmalloc(&g->ws, need, st) != cudaSuccess) return GTF_ERR_ALLOC;
        g->ws_bytes = need;
    }
    if (gemm.initialize(args, g->ws, st) != cutlass::Status::kSuccess) return GTF_ERR_CUDA;
    if (gemm.run(st) != cutlass::Status::kSuccess) return GTF_ERR_CUDA;
    dim3 grd2((n + 127) / 128, n);
    k_sum3_f64<<<grd2, blk, 0, st>>>(g->C, n, np, C);
    if (cudaGetLastError() != cudaSuccess) return GTF_ERR_CUDA;
    gtf_note_launches(4);
    return GTF_OK;
}
