// icp_mlp.h -- internal interface of the surrogate's kernels: the tensor-core GEMM with fused
// layer epilogues (icp_mlp_gemm.cu) and the elementwise / reduction kernels around it
// (icp_mlp.cu).
#pragma once
#include <cstdint>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

namespace icp::mlp {

// Fused epilogues of D = A * B^T (one 128-row tile per CTA, warp w owning rows 32w..32w+31):
//   kStoreF32   out_f32[m * ld_out + n] = D
//   kAtomicF32  out_f32[m * ld_out + n] += D            (split-K partial sums)
//   kHidden     z = D + bias; out_z = z, out_h = silu(z), out_hT[n * ld_t + m] = silu(z)
//               (BF16; every output optional)
//   kHead       kHidden, and y[m] = sum_n silu(z) * head_w[n] + head_b into out_y (FP32) and / or
//               out_mass[m] = exp(y) (FP64)                  (the 256 -> 1 head)
//   kBackprop   dz = D * silu'(z_prev) into out_dz and out_dzT (BF16); out_db[n] += sum_m dz
// kHidden / kHead write only out_h / out_y, out_mass (inference); kHiddenTrain / kHeadTrain also
// out_z and out_hT (a training step keeps them for the backward pass).
enum Epi : int { kStoreF32 = 0, kAtomicF32 = 1, kHidden = 2, kHead = 3, kBackprop = 4, kHiddenTrain = 5, kHeadTrain = 6 };

struct GemmArgs {
    uint32_t M, N, K;       // M % 128 == 0, N in {64, 128, 256}, K % 64 == 0
    uint32_t k_chunks;      // set by gemm(): 64-wide K chunks per CTA
    float* out_f32;
    uint32_t ld_out;
    uint32_t ld_t;          // row count of the transposed outputs (normally M)
    const float* bias;
    __nv_bfloat16* out_h;
    __nv_bfloat16* out_z;
    __nv_bfloat16* out_hT;
    const float* head_w;
    float head_b;
    float* out_y;
    double* out_mass;
    double* out_mass_sum;   // kHead: += sum of out_mass over each record's rows (or null)
    uint32_t record_rows;   // rows per record (a multiple of 128)
    const __nv_bfloat16* z_prev;
    __nv_bfloat16* out_dz;
    __nv_bfloat16* out_dzT;
    float* out_db;
    unsigned* error;        // set to 1 / 2 when a bounded wait expires
    uint32_t wait_limit;    // tries of the split-K kernel's pipeline waits (0: the default); the waits
                            // that drain loads in flight after an abort keep the default
};

// Enqueues D = A[M x K] * B[N x K]^T with the given epilogue; split-K (kAtomicF32 only) over
// `splits` CTAs per row tile.  Returns 0 or a negative / CUDA error code.
int gemm(const void* A, const void* B, GemmArgs g, int epi, uint32_t splits, cudaStream_t stream);

// The whole inference pass of the 3-hidden-layer network in one persistent kernel (the input
// rows and activations of a 128-row tile never leave the SM): the input rows as launch_features
// defines them (K0 in {64, 128}; rec16, recgeo, cellgeo, P as there, record_rows = C), built from
// xcells, the cell table in the row layout ([C x K0], record columns zero), W1 [256 x K0], W2, W3
// [256 x 256] BF16 (row n = output unit, K contiguous), biases and head in FP32.  Writes y and / or
// exp(y) with the per-record sums as the kHead epilogue does.
struct FusedArgs {
    uint32_t M, K0, P;
    const __nv_bfloat16* rec16;
    const __nv_bfloat16* xcells;
    const double* recgeo;
    const double* cellgeo;
    const float *b1, *b2, *b3, *head_w;
    float head_b;
    float* out_y;
    double* out_mass;
    double* out_mass_sum;
    uint32_t record_rows;
    unsigned* error;
};
bool fused_shape(uint32_t K0, uint32_t H);
int forward_fused(const void* W1, const void* W2, const void* W3, const FusedArgs& f, cudaStream_t stream);

// ---------------------------------------------------------------- icp_mlp.cu
// X[m][k] (BF16, [R*C x K0]) and optionally XT[k][m]: record features in columns [0, 16), the
// cell table (C x (K0-16), row-major) after them; record r owns rows [r*C, (r+1)*C).  The last P
// columns (P % 8 == 0) are the axis harmonics T_1..T_P(cos psi), cos psi = -(sa ct) - (ca sts)
// from the record's (sa, ca) = (sin, cos) of its inclination (recgeo[2r..]) and the cell's
// (ct, sts) = (cos theta, sin theta sin phi) (cellgeo[2c..]), in FP64 without contraction.
int launch_features(const __nv_bfloat16* rec16, const __nv_bfloat16* cells, uint32_t records, uint32_t C, uint32_t K0,
                    uint32_t P, const double* recgeo, const double* cellgeo, __nv_bfloat16* X, __nv_bfloat16* XT,
                    cudaStream_t st);
// Per-record softmax of y against target probabilities p: dy = (softmax(y) - p) * scale and
// loss[r] = sum_p>0 p (log p - log softmax(y)).
int launch_softmax_loss(const float* y, const float* p, uint32_t records, uint32_t C, float scale, float* dy,
                        double* loss, cudaStream_t st);
// Head backward: h3 = silu(z3), dz3 = dy * w4 * silu'(z3) (BF16, row- and column-major), and the
// sums dw4 += sum_m dy h3, db3 += sum_m dz3.
int launch_head_backward(const __nv_bfloat16* z3, const float* dy, const float* w4, uint32_t M, uint32_t H,
                         __nv_bfloat16* dz3, __nv_bfloat16* dz3T, float* dw4, float* db3, cudaStream_t st);
// Adam on the FP32 parameters, then the BF16 copies the GEMMs read (W1, W2, W3 and the
// transposes W2T, W3T).
struct AdamArgs {
    float* p;
    const float* g;
    float* m;
    float* v;
    uint32_t n;
    float lr, beta1, beta2, eps, weight_decay, bias1, bias2; // bias1/2 = 1 - beta^t
};
int launch_adam(const AdamArgs& a, cudaStream_t st);
struct WeightViews {
    const float *w1, *w2, *w3;
    __nv_bfloat16 *w1b, *w2b, *w3b, *w2t, *w3t;
    uint32_t H, K0;
};
int launch_weight_copies(const WeightViews& w, cudaStream_t st);
// Analytic diffraction rows of each record in the units of its predicted cell mass:
// rows[r][i] = sums[r] * frac[r][i] (frac = the diffraction power of row i per cell and per
// unit of geometric power, zero for records without diffraction).
int launch_scale_rows(const double* frac, const double* sums, uint32_t records, uint32_t nt, double* rows,
                      cudaStream_t st);
// Cell probabilities from stored CDFs at the histogram resolution: p[r][i * cp + j] =
// (phi[j+1] - phi[j]) * (theta[j][i+1] - theta[j][i]).
int launch_cdf_cells(const double* phi, const double* theta, uint32_t records, uint32_t ct, uint32_t cp, float* p,
                     cudaStream_t st);

} // namespace icp::mlp
