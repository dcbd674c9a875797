// gemm_sm100.cuh -- the tensor-core GEMMs of the learned coarse proposal (gemm_sm100.cu).
#pragma once
#include <cstdint>

#include <cuda_runtime.h>

namespace ofc {

enum class GemmKind { ForwardTN, WgradNT, DgradNN };

// C[l] = A[l] * B[l] + beta C[l] for l < L; A is M x K, B is K x N, C is M x N row-major float. lda / ldb: the stride
// of the operand's non-contiguous dimension (elements); batch_*: the stride between consecutive l.
struct GemmArgs {
  int M, N, K, L;
  const void* A;  // bf16
  int64_t lda, batch_a;
  const void* B;  // bf16
  int64_t ldb, batch_b;
  float* C;
  int64_t ldc, batch_c;
  float beta;
  const char* name;  // kernel name for the profile mode
};

void gemm_bf16(GemmKind kind, const GemmArgs& g, void* workspace, size_t workspace_bytes, cudaStream_t st);

// D (M x N, row-major bfloat16) = act(A B + bias) with act = ReLU or the identity: the forward GEMM's layouts
// (A K-contiguous, B = weights [N][K]) with the bias and the activation applied in the epilogue
struct FusedArgs {
  int M, N, K;
  const void* A;  // bf16
  int64_t lda;
  const void* B;  // bf16
  int64_t ldb;
  void* D;  // bf16
  int64_t ldd;
  const float* bias;  // N floats
  const char* name;
};

void gemm_bf16_fused(bool relu, const FusedArgs& g, void* workspace, size_t workspace_bytes, cudaStream_t st);

}  // namespace ofc
