// icp_mlp.cu -- the surrogate's kernels around the tensor-core GEMMs: input rows, the per-record
// softmax loss, the head's backward pass, Adam with the BF16 weight copies, and cell probabilities
// of stored CDF records (the training targets).  All are bandwidth-bound streaming kernels:
// 16-byte loads / stores along the contiguous dimension, one block per 128-1024 rows.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "icp_mlp.h"
#include "icp_mlp_features.cuh"

namespace icp::mlp {

namespace {

// SiLU and its derivative with the fast exponential and division (relative error ~1e-7, far
// below the BF16 rounding of the stored values); large negative z gives 0.
__device__ __forceinline__ float sigmoid_of(float z) { return __fdividef(1.0f, 1.0f + __expf(-fmaxf(z, -80.0f))); }
__device__ __forceinline__ float silu_of(float z) { return z * sigmoid_of(z); }
__device__ __forceinline__ float silu_grad_of(float z)
{
    const float s = sigmoid_of(z);
    return s * (1.0f + z * (1.0f - s));
}

// X rows: thread per 8 BF16 (one uint4) of a row.
__global__ void features_kernel(const uint4* __restrict__ rec16, const uint4* __restrict__ cells, uint32_t C,
                                uint32_t q_row, uint32_t q_axis, uint64_t total, const double* __restrict__ recgeo,
                                const double* __restrict__ cellgeo, uint4* __restrict__ X)
{
    const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= total) return;
    const uint64_t m = t / q_row;
    const uint32_t q = (uint32_t)(t - m * q_row);
    const uint32_t r = (uint32_t)(m / C), c = (uint32_t)(m - (uint64_t)r * C);
    if (q < 2) {
        X[t] = rec16[2u * r + q];
    } else if (q < q_axis) {
        X[t] = cells[(uint64_t)c * (q_row - 2) + (q - 2)];
    } else {
        __align__(16) __nv_bfloat16 h[8];
        axis_harmonics8(cos_psi(recgeo, cellgeo, r, c), 1u + 8u * (q - q_axis), h);
        X[t] = *reinterpret_cast<const uint4*>(h);
    }
}

// XT[k][m]: thread per 8 consecutive rows m of one column k.
__global__ void features_t_kernel(const __nv_bfloat16* __restrict__ rec16, const uint4* __restrict__ cellsT, uint32_t C,
                                  uint32_t K0, uint32_t P, uint32_t records, const double* __restrict__ recgeo,
                                  const double* __restrict__ cellgeo, __nv_bfloat16* __restrict__ XT)
{
    const uint64_t per_k = (uint64_t)records * C / 8u;
    const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= per_k * K0) return;
    const uint32_t k = (uint32_t)(t / per_k);
    const uint64_t m8 = t - (uint64_t)k * per_k;
    const uint64_t m = 8u * m8;
    const uint32_t r = (uint32_t)(m / C), c = (uint32_t)(m - (uint64_t)r * C);
    uint4 v;
    if (k < 16) {
        const __nv_bfloat16 x = rec16[16u * r + k];
        const uint32_t w = (uint32_t)__bfloat16_as_ushort(x) * 0x10001u;
        v = make_uint4(w, w, w, w);
    } else if (k < K0 - P) {
        v = cellsT[((uint64_t)(k - 16) * C + c) / 8u];
    } else {
        // harmonic j of 8 consecutive cells of one record (C is a multiple of 8)
        const uint32_t j = k - (K0 - P) + 1u;
        __align__(16) __nv_bfloat16 h[8];
        for (int i = 0; i < 8; ++i) {
            const double x = cos_psi(recgeo, cellgeo, r, c + (uint32_t)i);
            double tm = 1.0, tt = x;
            for (uint32_t n = 1; n < j; ++n) {
                const double tn = __dsub_rn(__dmul_rn(__dmul_rn(2.0, x), tt), tm);
                tm = tt;
                tt = tn;
            }
            h[i] = __float2bfloat16_rn(__double2float_rn(tt));
        }
        v = *reinterpret_cast<const uint4*>(h);
    }
    reinterpret_cast<uint4*>(XT + (uint64_t)k * records * C)[m8] = v;
}

__device__ __forceinline__ double block_sum(double v, double* sh)
{
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const uint32_t w = threadIdx.x >> 5, l = threadIdx.x & 31u, nw = blockDim.x >> 5;
    __syncthreads();
    if (l == 0) sh[w] = v;
    __syncthreads();
    double s = 0;
    for (uint32_t i = 0; i < nw; ++i) s += sh[i];
    return s;
}
__device__ __forceinline__ float block_max(float v, float* sh)
{
    for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
    const uint32_t w = threadIdx.x >> 5, l = threadIdx.x & 31u, nw = blockDim.x >> 5;
    __syncthreads();
    if (l == 0) sh[w] = v;
    __syncthreads();
    float s = sh[0];
    for (uint32_t i = 1; i < nw; ++i) s = fmaxf(s, sh[i]);
    return s;
}

// One block per record: max, log-sum-exp (FP64 sums), KL loss and dy.
__global__ void __launch_bounds__(1024) softmax_loss_kernel(const float* __restrict__ y, const float* __restrict__ p,
                                                            uint32_t C, float scale, float* __restrict__ dy,
                                                            double* __restrict__ loss)
{
    __shared__ double shd[32];
    __shared__ float shf[32];
    const uint64_t base = (uint64_t)blockIdx.x * C;
    const float4* y4 = reinterpret_cast<const float4*>(y + base);
    const float4* p4 = reinterpret_cast<const float4*>(p + base);
    const uint32_t n4 = C / 4u;
    float mx = -INFINITY;
    for (uint32_t i = threadIdx.x; i < n4; i += blockDim.x) {
        const float4 v = y4[i];
        mx = fmaxf(mx, fmaxf(fmaxf(v.x, v.y), fmaxf(v.z, v.w)));
    }
    mx = block_max(mx, shf);
    double se = 0, py = 0, plp = 0;
    for (uint32_t i = threadIdx.x; i < n4; i += blockDim.x) {
        const float4 v = y4[i], q = p4[i];
        const float ys[4] = {v.x, v.y, v.z, v.w}, ps[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            se += (double)__expf(ys[j] - mx);
            if (ps[j] > 0.0f) {
                py += (double)ps[j] * (double)(ys[j] - mx);
                plp += (double)ps[j] * log((double)ps[j]);
            }
        }
    }
    se = block_sum(se, shd);
    py = block_sum(py, shd);
    plp = block_sum(plp, shd);
    const double lse = log(se); // relative to mx
    if (threadIdx.x == 0) loss[blockIdx.x] = plp - py + lse; // sum p = 1
    const float lsef = (float)lse + mx;
    float4* d4 = reinterpret_cast<float4*>(dy + base);
    for (uint32_t i = threadIdx.x; i < n4; i += blockDim.x) {
        const float4 v = y4[i], q = p4[i];
        d4[i] = make_float4((__expf(v.x - lsef) - q.x) * scale, (__expf(v.y - lsef) - q.y) * scale,
                            (__expf(v.z - lsef) - q.z) * scale, (__expf(v.w - lsef) - q.w) * scale);
    }
}

// One block of 256 threads per tile of kHeadRows = 64 rows x H columns (H <= 256, a multiple of
// 64).  Load: thread t owns the 8 columns 8 (t mod H/8) .. and the rows t / (H/8) + k (256 / (H/8)),
// reading z3 and writing dz3 as 16-byte vectors (coalesced rows); dz3 also goes into a shared
// tile.  Transpose: thread t < H writes the 64 rows of column t of the tile to dz3T as eight
// 16-byte vectors (one contiguous 128-byte run per column).  Column sums of dy h3 (dw4) and of
// dz3 (db3) are reduced in registers and shared memory, one atomic per column per block.
constexpr uint32_t kHeadRows = 64;
__global__ void __launch_bounds__(256) head_backward_kernel(const __nv_bfloat16* __restrict__ z3,
                                                            const float* __restrict__ dy, const float* __restrict__ w4,
                                                            uint32_t M, uint32_t H, __nv_bfloat16* __restrict__ dz3,
                                                            __nv_bfloat16* __restrict__ dz3T, float* __restrict__ dw4,
                                                            float* __restrict__ db3)
{
    // rows are written and columns read contiguously across a warp: no padding needed
    __shared__ __align__(16) __nv_bfloat16 tile[kHeadRows][256];
    // partial column sums of each row group r0 (rstep groups x H columns = 2048 values for every
    // H): written once per thread, summed in order by one thread per column (no atomics)
    __shared__ float pw[2048], pb[2048];
    const uint32_t t = threadIdx.x, groups = H / 8u, rstep = 256u / groups;
    const uint32_t g = t % groups, r0 = t / groups, c = 8u * g;
    const uint64_t m0 = (uint64_t)blockIdx.x * kHeadRows;
    float w[8], aw[8] = {}, ab[8] = {};
#pragma unroll
    for (int k = 0; k < 8; ++k) w[k] = w4[c + k];
    for (uint32_t r = r0; r < kHeadRows; r += rstep) {
        const uint64_t m = m0 + r;
        const float d = dy[m];
        const uint4 u = *reinterpret_cast<const uint4*>(z3 + m * H + c);
        const uint32_t zw[4] = {u.x, u.y, u.z, u.w};
        uint32_t ow[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const float2 z = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&zw[q]));
            const float g0 = d * w[2 * q] * silu_grad_of(z.x), g1 = d * w[2 * q + 1] * silu_grad_of(z.y);
            aw[2 * q] = fmaf(d, silu_of(z.x), aw[2 * q]);
            aw[2 * q + 1] = fmaf(d, silu_of(z.y), aw[2 * q + 1]);
            ab[2 * q] += g0;
            ab[2 * q + 1] += g1;
            const __nv_bfloat162 p = __floats2bfloat162_rn(g0, g1);
            ow[q] = *reinterpret_cast<const uint32_t*>(&p);
        }
        const uint4 o = make_uint4(ow[0], ow[1], ow[2], ow[3]);
        *reinterpret_cast<uint4*>(dz3 + m * H + c) = o;
        *reinterpret_cast<uint4*>(&tile[r][c]) = o;
    }
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        pw[r0 * H + c + k] = aw[k];
        pb[r0 * H + c + k] = ab[k];
    }
    __syncthreads();
    if (t < H) {
        __nv_bfloat16* dst = dz3T + (uint64_t)t * M + m0;
#pragma unroll
        for (uint32_t r8 = 0; r8 < kHeadRows; r8 += 8) {
            __align__(16) __nv_bfloat16 col[8];
#pragma unroll
            for (int k = 0; k < 8; ++k) col[k] = tile[r8 + k][t];
            *reinterpret_cast<uint4*>(dst + r8) = *reinterpret_cast<const uint4*>(col);
        }
        float sw = 0.0f, sb = 0.0f;
        for (uint32_t k = 0; k < rstep; ++k) {
            sw += pw[k * H + t];
            sb += pb[k * H + t];
        }
        atomicAdd(&dw4[t], sw);
        atomicAdd(&db3[t], sb);
    }
}

__global__ void adam_kernel(AdamArgs a)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    const float g = a.g[i];
    const float m = a.beta1 * a.m[i] + (1.0f - a.beta1) * g;
    const float v = a.beta2 * a.v[i] + (1.0f - a.beta2) * g * g;
    a.m[i] = m;
    a.v[i] = v;
    const float mh = m / a.bias1, vh = v / a.bias2;
    a.p[i] -= a.lr * (mh / (sqrtf(vh) + a.eps) + a.weight_decay * a.p[i]);
}

__global__ void weight_copies_kernel(WeightViews w)
{
    const uint32_t H = w.H, K0 = w.K0;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t n1 = H * K0, n2 = H * H;
    if (i < n1) {
        w.w1b[i] = __float2bfloat16_rn(w.w1[i]);
    } else if (i < n1 + n2) {
        const uint32_t j = i - n1, r = j / H, c = j - r * H;
        const __nv_bfloat16 b = __float2bfloat16_rn(w.w2[j]);
        w.w2b[j] = b;
        w.w2t[c * H + r] = b;
    } else if (i < n1 + 2 * n2) {
        const uint32_t j = i - n1 - n2, r = j / H, c = j - r * H;
        const __nv_bfloat16 b = __float2bfloat16_rn(w.w3[j]);
        w.w3b[j] = b;
        w.w3t[c * H + r] = b;
    }
}

__global__ void scale_rows_kernel(const double* __restrict__ frac, const double* __restrict__ sums, uint32_t nt,
                                  uint32_t total, double* __restrict__ rows)
{
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < total) rows[t] = sums[t / nt] * frac[t];
}

__global__ void cdf_cells_kernel(const double* __restrict__ phi, const double* __restrict__ theta, uint32_t ct,
                                 uint32_t cp, uint64_t total, float* __restrict__ p)
{
    const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= total) return;
    const uint64_t cells = (uint64_t)ct * cp;
    const uint32_t r = (uint32_t)(t / cells);
    const uint32_t k = (uint32_t)(t - (uint64_t)r * cells);
    const uint32_t i = k / cp, j = k - i * cp;
    const double* a = phi + (uint64_t)r * (cp + 1);
    const double* T = theta + ((uint64_t)r * cp + j) * (ct + 1);
    p[t] = (float)((a[j + 1] - a[j]) * (T[i + 1] - T[i]));
}

unsigned blocks_of(uint64_t n, unsigned t) { return (unsigned)((n + t - 1) / t); }

} // namespace

int launch_features(const __nv_bfloat16* rec16, const __nv_bfloat16* cells, uint32_t records, uint32_t C, uint32_t K0,
                    uint32_t P, const double* recgeo, const double* cellgeo, __nv_bfloat16* X, __nv_bfloat16* XT,
                    cudaStream_t st)
{
    if (K0 % 64 || C % 128 || !records || P % 8 || P + 16 > K0) return -1;
    const uint32_t q_row = K0 / 8u;
    const uint64_t total = (uint64_t)records * C * q_row;
    features_kernel<<<blocks_of(total, 256), 256, 0, st>>>(reinterpret_cast<const uint4*>(rec16),
                                                           reinterpret_cast<const uint4*>(cells), C, q_row,
                                                           q_row - P / 8u, total, recgeo, cellgeo,
                                                           reinterpret_cast<uint4*>(X));
    if (XT) {
        // the column-major cell table follows the row-major one in the same allocation
        const uint4* cellsT = reinterpret_cast<const uint4*>(cells + (uint64_t)C * (K0 - 16));
        const uint64_t n = (uint64_t)records * C / 8u * K0;
        features_t_kernel<<<blocks_of(n, 256), 256, 0, st>>>(rec16, cellsT, C, K0, P, records, recgeo, cellgeo, XT);
    }
    return (int)cudaGetLastError();
}

int launch_softmax_loss(const float* y, const float* p, uint32_t records, uint32_t C, float scale, float* dy,
                        double* loss, cudaStream_t st)
{
    if (C % 4 || !records) return -1;
    softmax_loss_kernel<<<records, 1024, 0, st>>>(y, p, C, scale, dy, loss);
    return (int)cudaGetLastError();
}

int launch_head_backward(const __nv_bfloat16* z3, const float* dy, const float* w4, uint32_t M, uint32_t H,
                         __nv_bfloat16* dz3, __nv_bfloat16* dz3T, float* dw4, float* db3, cudaStream_t st)
{
    if (M % kHeadRows || H > 256 || H % 64) return -1;
    head_backward_kernel<<<M / kHeadRows, 256, 0, st>>>(z3, dy, w4, M, H, dz3, dz3T, dw4, db3);
    return (int)cudaGetLastError();
}

int launch_adam(const AdamArgs& a, cudaStream_t st)
{
    adam_kernel<<<blocks_of(a.n, 256), 256, 0, st>>>(a);
    return (int)cudaGetLastError();
}

int launch_weight_copies(const WeightViews& w, cudaStream_t st)
{
    const uint64_t n = (uint64_t)w.H * w.K0 + 2ull * w.H * w.H;
    weight_copies_kernel<<<blocks_of(n, 256), 256, 0, st>>>(w);
    return (int)cudaGetLastError();
}

int launch_scale_rows(const double* frac, const double* sums, uint32_t records, uint32_t nt, double* rows,
                      cudaStream_t st)
{
    const uint32_t total = records * nt;
    scale_rows_kernel<<<blocks_of(total, 256), 256, 0, st>>>(frac, sums, nt, total, rows);
    return (int)cudaGetLastError();
}

int launch_cdf_cells(const double* phi, const double* theta, uint32_t records, uint32_t ct, uint32_t cp, float* p,
                     cudaStream_t st)
{
    const uint64_t total = (uint64_t)records * ct * cp;
    cdf_cells_kernel<<<blocks_of(total, 256), 256, 0, st>>>(phi, theta, ct, cp, total, p);
    return (int)cudaGetLastError();
}

} // namespace icp::mlp
