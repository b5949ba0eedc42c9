// icp_mlp.h -- internal interface of the surrogate's tensor-core kernels (icp_mlp_gemm.cu,
// icp_mlp.cu).
#pragma once
#include <cstdint>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

namespace icp::mlp {

// Fused epilogues of D = A * B^T (one 128-row tile per CTA, warp w owning rows 32w..32w+31):
//   kStoreF32   out_f32[m * ld_out + n] = D
//   kAtomicF32  out_f32[m * ld_out + n] += D            (split-K partial sums)
//   kHidden     z = D + bias; out_z = z (optional); out_h = silu(z)         (BF16, [M x N])
//   kHead       kHidden, and out_y[m] = sum_n silu(z) * head_w[n] + head_b  (the 256 -> 1 head)
//   kBackprop   out_dz = D * silu'(z_prev)                                  (BF16, [M x N])
enum Epi : int { kStoreF32 = 0, kAtomicF32 = 1, kHidden = 2, kHead = 3, kBackprop = 4 };

struct GemmArgs {
    uint32_t M, N, K;       // M % 128 == 0, N in {64, 128, 256}, K % 64 == 0
    uint32_t k_chunks;      // set by gemm(): 64-wide K chunks per CTA
    float* out_f32;
    uint32_t ld_out;
    const float* bias;
    __nv_bfloat16* out_h;
    __nv_bfloat16* out_z;
    const float* head_w;
    float head_b;
    float* out_y;
    const __nv_bfloat16* z_prev;
    __nv_bfloat16* out_dz;
    unsigned* error;        // set to 1 / 2 when a bounded wait expires
};

// Enqueues D = A[M x K] * B[N x K]^T with the given epilogue; split-K (kAtomicF32 only) over
// `splits` CTAs per row tile.  Returns 0 or a negative / CUDA error code.
int gemm(const void* A, const void* B, GemmArgs g, int epi, uint32_t splits, cudaStream_t stream);

} // namespace icp::mlp
