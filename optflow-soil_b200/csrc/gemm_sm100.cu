// gemm_sm100.cu -- BF16 x BF16 -> FP32 GEMMs on the 5th-generation tensor cores, for the learned coarse proposal's
// convolutions (forward, weight gradient, input gradient). Each is a CUTLASS sm100 collective: TMA loads of 128 x 64
// and 64 x 64 operand tiles into shared memory (clusters of one CTA: each CTA loads only its own tiles),
// tcgen05.mma issued by one thread into a TMEM accumulator, and a TMEM -> register -> TMA-store epilogue. All three
// compute
//   C[l] (M x N, row-major, float) = A[l] (M x K) * B[l] (K x N) + beta C[l],   l < batch,
// and differ in which operand dimension is contiguous:
//   GemmKind::ForwardTN   A K-contiguous (im2col rows), B K-contiguous (weights [N][K])      -> conv forward
//   GemmKind::WgradNT     A M-contiguous (dY^T), B N-contiguous (im2col rows)              -> weight gradient
//   GemmKind::DgradNN     A K-contiguous (dY), B N-contiguous (weights [K][N])              -> input gradient
// Contiguous extents must be multiples of 8 elements and every base address 16-byte aligned (TMA).
#include <cute/tensor.hpp>
#include <cutlass/cutlass.h>
#include <cutlass/epilogue/collective/collective_builder.hpp>
#include <cutlass/epilogue/fusion/operations.hpp>
#include <cutlass/epilogue/thread/activation.h>
#include <cutlass/gemm/collective/collective_builder.hpp>
#include <cutlass/gemm/device/gemm_universal_adapter.h>
#include <cutlass/gemm/kernel/gemm_universal.hpp>

#include "common.cuh"
#include "gemm_sm100.cuh"

namespace ofc {
namespace {

using namespace cute;

template <class LayoutA, class LayoutB>
struct Sm100Gemm {
  using MmaTileMNK = Shape<_128, _64, _64>;
  using ClusterMNK = Shape<_1, _1, _1>;
  using Epilogue = typename cutlass::epilogue::collective::CollectiveBuilder<
      cutlass::arch::Sm100, cutlass::arch::OpClassTensorOp, MmaTileMNK, ClusterMNK,
      cutlass::epilogue::collective::EpilogueTileAuto, float, float, float, cutlass::layout::RowMajor, 4, float,
      cutlass::layout::RowMajor, 4, cutlass::epilogue::TmaWarpSpecialized1Sm>::CollectiveOp;
  using Mainloop = typename cutlass::gemm::collective::CollectiveBuilder<
      cutlass::arch::Sm100, cutlass::arch::OpClassTensorOp, cutlass::bfloat16_t, LayoutA, 8, cutlass::bfloat16_t,
      LayoutB, 8, float, MmaTileMNK, ClusterMNK,
      cutlass::gemm::collective::StageCountAutoCarveout<static_cast<int>(sizeof(typename Epilogue::SharedStorage))>,
      cutlass::gemm::KernelTmaWarpSpecialized1SmSm100>::CollectiveOp;
  using Kernel = cutlass::gemm::kernel::GemmUniversal<Shape<int, int, int, int>, Mainloop, Epilogue, void>;
  using Adapter = cutlass::gemm::device::GemmUniversalAdapter<Kernel>;
  using StrideA = typename Kernel::StrideA;
  using StrideB = typename Kernel::StrideB;
  using StrideC = typename Kernel::StrideC;
  using StrideD = typename Kernel::StrideD;
};

// a (rows, cols, batch) stride tuple: the leading stride goes into the mode that is not the unit one
template <class S>
S make_strides(int64_t ld, int64_t batch) {
  S s{};
  if constexpr (cute::is_static_v<cute::remove_cvref_t<decltype(cute::get<0>(s))>>)
    cute::get<1>(s) = ld;
  else
    cute::get<0>(s) = ld;
  cute::get<2>(s) = batch;
  return s;
}

template <class G>
void run_gemm(const GemmArgs& g, void* workspace, size_t workspace_bytes, cudaStream_t st) {
  using Adapter = typename G::Adapter;
  auto sA = make_strides<typename G::StrideA>(g.lda, g.batch_a);
  auto sB = make_strides<typename G::StrideB>(g.ldb, g.batch_b);
  auto sC = make_strides<typename G::StrideC>(g.ldc, g.batch_c);
  auto sD = make_strides<typename G::StrideD>(g.ldc, g.batch_c);
  typename Adapter::Arguments args{cutlass::gemm::GemmUniversalMode::kGemm,
                                   {g.M, g.N, g.K, g.L},
                                   {reinterpret_cast<const cutlass::bfloat16_t*>(g.A), sA,
                                    reinterpret_cast<const cutlass::bfloat16_t*>(g.B), sB},
                                   {{1.0f, g.beta}, g.C, sC, g.C, sD}};
  Adapter op;
  if (op.can_implement(args) != cutlass::Status::kSuccess)
    throw Error(OFC_ERR_ARG, "tensor-core GEMM: unsupported shape or alignment (M " + std::to_string(g.M) + ", N " +
                                 std::to_string(g.N) + ", K " + std::to_string(g.K) + ")");
  if (Adapter::get_workspace_size(args) > workspace_bytes)
    throw Error(OFC_ERR_DEVICE, "tensor-core GEMM: workspace too small");
  if (op.initialize(args, workspace, st) != cutlass::Status::kSuccess)
    throw Error(OFC_ERR_DEVICE, "tensor-core GEMM: initialisation failed");
  void* tok = nullptr;
  if (::ofc::g_profiler) prof_before(g.name ? g.name : "k_gemm_sm100", st, &tok);
  if (op.run(st) != cutlass::Status::kSuccess) throw Error(OFC_ERR_DEVICE, "tensor-core GEMM: launch failed");
  OFC_CUDA(cudaGetLastError());
  if (tok) prof_after(tok, st);
  if (::ofc::g_launch_counter) ++*::ofc::g_launch_counter;
}

// the forward GEMM with its epilogue fused: D (bfloat16, row-major) = act(acc + bias[n]), the per-column bias and the
// activation applied to the TMEM accumulator before the TMA store (no source matrix)
template <template <class> class Act>
struct Sm100GemmFused {
  using MmaTileMNK = Shape<_128, _64, _64>;
  using ClusterMNK = Shape<_1, _1, _1>;
  using Fusion = cutlass::epilogue::fusion::LinCombPerColBiasEltAct<Act, cutlass::bfloat16_t, float, float>;
  using Epilogue = typename cutlass::epilogue::collective::CollectiveBuilder<
      cutlass::arch::Sm100, cutlass::arch::OpClassTensorOp, MmaTileMNK, ClusterMNK,
      cutlass::epilogue::collective::EpilogueTileAuto, float, float, void, cutlass::layout::RowMajor, 8,
      cutlass::bfloat16_t, cutlass::layout::RowMajor, 8, cutlass::epilogue::TmaWarpSpecialized1Sm, Fusion>::CollectiveOp;
  using Mainloop = typename cutlass::gemm::collective::CollectiveBuilder<
      cutlass::arch::Sm100, cutlass::arch::OpClassTensorOp, cutlass::bfloat16_t, cutlass::layout::RowMajor, 8,
      cutlass::bfloat16_t, cutlass::layout::ColumnMajor, 8, float, MmaTileMNK, ClusterMNK,
      cutlass::gemm::collective::StageCountAutoCarveout<static_cast<int>(sizeof(typename Epilogue::SharedStorage))>,
      cutlass::gemm::KernelTmaWarpSpecialized1SmSm100>::CollectiveOp;
  using Kernel = cutlass::gemm::kernel::GemmUniversal<Shape<int, int, int, int>, Mainloop, Epilogue, void>;
  using Adapter = cutlass::gemm::device::GemmUniversalAdapter<Kernel>;
  using StrideA = typename Kernel::StrideA;
  using StrideB = typename Kernel::StrideB;
  using StrideC = typename Kernel::StrideC;
  using StrideD = typename Kernel::StrideD;
};

template <class G>
void run_fused(const FusedArgs& g, void* workspace, size_t workspace_bytes, cudaStream_t st) {
  using Adapter = typename G::Adapter;
  auto sA = make_strides<typename G::StrideA>(g.lda, 0);
  auto sB = make_strides<typename G::StrideB>(g.ldb, 0);
  auto sD = make_strides<typename G::StrideD>(g.ldd, 0);
  typename Adapter::Arguments args{cutlass::gemm::GemmUniversalMode::kGemm,
                                   {g.M, g.N, g.K, 1},
                                   {reinterpret_cast<const cutlass::bfloat16_t*>(g.A), sA,
                                    reinterpret_cast<const cutlass::bfloat16_t*>(g.B), sB},
                                   {{}, nullptr, typename G::StrideC{}, reinterpret_cast<cutlass::bfloat16_t*>(g.D), sD}};
  args.epilogue.thread.alpha = 1.0f;
  args.epilogue.thread.beta = 0.0f;
  args.epilogue.thread.bias_ptr = g.bias;
  Adapter op;
  if (op.can_implement(args) != cutlass::Status::kSuccess)
    throw Error(OFC_ERR_ARG, "tensor-core GEMM (fused epilogue): unsupported shape or alignment (M " +
                                 std::to_string(g.M) + ", N " + std::to_string(g.N) + ", K " + std::to_string(g.K) + ")");
  if (Adapter::get_workspace_size(args) > workspace_bytes)
    throw Error(OFC_ERR_DEVICE, "tensor-core GEMM: workspace too small");
  if (op.initialize(args, workspace, st) != cutlass::Status::kSuccess)
    throw Error(OFC_ERR_DEVICE, "tensor-core GEMM: initialisation failed");
  void* tok = nullptr;
  if (::ofc::g_profiler) prof_before(g.name ? g.name : "k_gemm_sm100_fused", st, &tok);
  if (op.run(st) != cutlass::Status::kSuccess) throw Error(OFC_ERR_DEVICE, "tensor-core GEMM: launch failed");
  OFC_CUDA(cudaGetLastError());
  if (tok) prof_after(tok, st);
  if (::ofc::g_launch_counter) ++*::ofc::g_launch_counter;
}

using GemmTN = Sm100Gemm<cutlass::layout::RowMajor, cutlass::layout::ColumnMajor>;
using GemmNT = Sm100Gemm<cutlass::layout::ColumnMajor, cutlass::layout::RowMajor>;
using GemmNN = Sm100Gemm<cutlass::layout::RowMajor, cutlass::layout::RowMajor>;

}  // namespace

void gemm_bf16_fused(bool relu, const FusedArgs& g, void* workspace, size_t workspace_bytes, cudaStream_t st) {
  if (relu) run_fused<Sm100GemmFused<cutlass::epilogue::thread::ReLu>>(g, workspace, workspace_bytes, st);
  else run_fused<Sm100GemmFused<cutlass::epilogue::thread::Identity>>(g, workspace, workspace_bytes, st);
}

void gemm_bf16(GemmKind kind, const GemmArgs& g, void* workspace, size_t workspace_bytes, cudaStream_t st) {
  switch (kind) {
    case GemmKind::ForwardTN: run_gemm<GemmTN>(g, workspace, workspace_bytes, st); break;
    case GemmKind::WgradNT: run_gemm<GemmNT>(g, workspace, workspace_bytes, st); break;
    case GemmKind::DgradNN: run_gemm<GemmNN>(g, workspace, workspace_bytes, st); break;
  }
}

}  // namespace ofc
