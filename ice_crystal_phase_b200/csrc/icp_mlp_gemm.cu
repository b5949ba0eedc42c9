// icp_mlp_gemm.cu -- BF16 GEMM on the 5th-generation tensor cores (tcgen05, TMEM, TMA) for the
// surrogate's dense layers, with the layer epilogues fused.
//
//   D[M x N] = A[M x K] * B[N x K]^T      A, B: BF16, K-major (row-major with K contiguous)
//
// Three kernels.  Inference of the default network shape runs as one persistent kernel that takes
// each 128-row tile from its input row to y with the activations on chip (mlp_fused_kernel,
// below).  The layer GEMMs of training and of other shapes (K, N = layer widths <= 256, M = the
// rows of a batch) run persistent and warp-specialised (gemm_persistent_kernel).  The weight
// gradients (M, N =
// layer widths, K = rows of a batch) run split-K (gemm_kernel): one CTA of 128 threads computes a
// 128 x N tile (N in {64, 128, 256}) over a range of K chunks of 64: thread 0 streams A and B
// chunks through a STAGES-deep ring with 2-D TMA loads (128-byte swizzle, completion counted on a
// "full" mbarrier per stage) and issues four K=16 tcgen05.mma per chunk into an FP32 accumulator
// in tensor memory; each chunk's MMAs commit to the stage's "empty" mbarrier, which gates the
// refill.  After the last chunk a commit to "done" releases the epilogue: warp w reads TMEM lanes
// 32w..32w+31 (rows) with tcgen05.ld, 32 columns at a time, and applies one of the fused
// epilogues below.  Split-K (grid.y > 1) adds partial tiles with FP32 atomics.  Every mbarrier
// wait is bounded: on expiry the kernel sets the error word, waits (bounded) for its issued loads
// and MMAs, frees its tensor memory and returns.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "icp_internal.h"
#include "icp_mlp.h"
#include "icp_mlp_features.cuh"
#include "icp_umma.cuh"

namespace icp::mlp {

namespace {

constexpr uint32_t kWaitLimit = 1u << 22;
constexpr uint32_t kA = 128u * 128u; // bytes of one A stage: 128 rows x 64 BF16

// split-K kernel: MT row tiles of 128 per CTA share each B chunk (MT = 2 for the weight gradients,
// whose M is 256: B is then read once instead of once per row tile)
template <int N, int MT = 1> __host__ __device__ constexpr int stages() { return N <= 128 ? 4 : 3; }
template <int N, int MT = 1> __host__ __device__ constexpr uint32_t stage_bytes()
{
    return (uint32_t)MT * kA + (uint32_t)N * 128u;
}
// 1024 (alignment) + stages + barriers / TMEM slot (256) + column sums of the bias gradient (1024)
template <int N, int MT = 1> constexpr size_t smem_bytes()
{
    return 1024 + (size_t)stages<N, MT>() * stage_bytes<N, MT>() + 256 + 1024;
}

// Logistic function 1 / (1 + exp(-z)) with the exponential on the special-function unit and
// the reciprocal on the FMA pipe, so that the two pipes share the epilogue's activation work
// (one SiLU per output element is the MLP's largest non-tensor cost).  Reciprocal of d >= 1:
// the integer seed y0 = bits(0x7EF311C0) - bits(d), a line in log2 space whose offset minimises
// the largest relative error over a binade (0.0505, found by a search over the offsets), then
// one Newton step y <- y (1 + e), e = 1 - d y (error squared: 2.6e-3) and one third-order step
// y <- y (1 + e + e^2) (error cubed: 1.7e-8; 1.1e-7 after the binary32 roundings, measured over
// a binade) -- five FMA-pipe operations.  z is clamped at -80 so that d stays finite; the
// result then is below 2e-35.
// 2^x on the special-function unit with subnormal results flushed (one instruction; the
// exponential here is only ever added to 1).
__device__ __forceinline__ float ex2_ftz(float x)
{
    float y;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float logistic(float z)
{
    const float d = 1.0f + ex2_ftz(fmaxf(z, -80.0f) * -1.44269504088896341f);
    float y = __int_as_float(0x7EF311C0 - __float_as_int(d));
    y = fmaf(y, fmaf(-d, y, 1.0f), y);
    const float e = fmaf(-d, y, 1.0f);
    return fmaf(y, fmaf(e, e, e), y);
}
// The training epilogues (more stores per element, MUFU pipe not the limit) use the
// special-function reciprocal instead: both forms agree to ~1e-7 relative.
__device__ __forceinline__ float logistic_mufu(float z) { return __fdividef(1.0f, 1.0f + __expf(-fmaxf(z, -80.0f))); }
template <bool kFmaRcp> __device__ __forceinline__ float silu(float z)
{
    return z * (kFmaRcp ? logistic(z) : logistic_mufu(z));
}
template <bool kFmaRcp> __device__ __forceinline__ float silu_grad(float z)
{
    const float s = kFmaRcp ? logistic(z) : logistic_mufu(z);
    return s * (1.0f + z * (1.0f - s));
}

__device__ __forceinline__ void store_bf16x32(__nv_bfloat16* dst, const float (&v)[32])
{
    uint4* d = reinterpret_cast<uint4*>(dst);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        uint32_t w[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const __nv_bfloat162 p = __floats2bfloat162_rn(v[8 * q + 2 * i], v[8 * q + 2 * i + 1]);
            w[i] = *reinterpret_cast<const uint32_t*>(&p);
        }
        d[q] = make_uint4(w[0], w[1], w[2], w[3]);
    }
}
// Column sums of a warp's 32 x 32 block (lane = row, v[i] = column i): a butterfly
// reduce-scatter in 31 shuffles, after which lane L holds the sum of column L in v[0].
__device__ __forceinline__ float warp_column_sum(float (&v)[32], uint32_t lane)
{
#pragma unroll
    for (int off = 16; off >= 1; off >>= 1) {
        const bool upper = (lane & (uint32_t)off) != 0;
#pragma unroll
        for (int j = 0; j < off; ++j) {
            const float send = upper ? v[j] : v[j + off];
            const float keep = upper ? v[j + off] : v[j];
            v[j] = keep + __shfl_xor_sync(0xffffffffu, send, off);
        }
    }
    return v[0];
}

// Column-major copy of a warp's 32 rows x 32 columns through the warp's shared transpose buffer
// (32 rows of 40 BF16, 80-byte stride): lane L writes its row, then gathers column L and writes
// its 32 rows (64 contiguous bytes) to dst_col0 + L * ld with four 16-byte stores.  dst_col0 is
// the column's first row of this warp (32-row aligned).  Every index is a compile-time constant.
constexpr uint32_t kTStride = 40; // BF16 per transpose-buffer row
__device__ __forceinline__ void store_bf16x32_t(__nv_bfloat16* dst_col0, uint32_t ld, const float (&v)[32],
                                                __nv_bfloat16* tbuf, uint32_t lane)
{
    uint4* row = reinterpret_cast<uint4*>(tbuf + lane * kTStride);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        uint32_t w[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const __nv_bfloat162 p = __floats2bfloat162_rn(v[8 * q + 2 * i], v[8 * q + 2 * i + 1]);
            w[i] = *reinterpret_cast<const uint32_t*>(&p);
        }
        row[q] = make_uint4(w[0], w[1], w[2], w[3]);
    }
    __syncwarp();
    const uint16_t* col = reinterpret_cast<const uint16_t*>(tbuf) + lane;
    uint32_t w[16];
#pragma unroll
    for (int r = 0; r < 16; ++r)
        w[r] = (uint32_t)col[(2 * r) * kTStride] | ((uint32_t)col[(2 * r + 1) * kTStride] << 16);
    uint4* d = reinterpret_cast<uint4*>(dst_col0 + (size_t)lane * ld);
#pragma unroll
    for (int q = 0; q < 4; ++q) d[q] = make_uint4(w[4 * q], w[4 * q + 1], w[4 * q + 2], w[4 * q + 3]);
    __syncwarp();
}

__device__ __forceinline__ void load_bf16x32(const __nv_bfloat16* src, float (&v)[32])
{
    const uint4* s = reinterpret_cast<const uint4*>(src);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const uint4 u = s[q];
        const uint32_t w[4] = {u.x, u.y, u.z, u.w};
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const __nv_bfloat162 p = *reinterpret_cast<const __nv_bfloat162*>(&w[i]);
            const float2 f = __bfloat1622float2(p);
            v[8 * q + 2 * i] = f.x;
            v[8 * q + 2 * i + 1] = f.y;
        }
    }
}

// Columns [c0, c1) of one row of a 128 x N accumulator tile through the fused epilogue: this
// thread's TMEM lane starts at taddr (column 0); m is the output row; bias / head_w point at N
// values (shared or global memory, 16-byte aligned); colsum collects the bias gradient
// (kBackprop).  Returns the partial head sum of these columns (kHead).
template <int N, int EPI>
__device__ __forceinline__ float epilogue_cols(const GemmArgs& g, uint32_t taddr, uint32_t m, uint32_t lane,
                                              uint32_t c0, uint32_t c1, const float* bias, const float* head_w,
                                              float* colsum, __nv_bfloat16* tbuf)
{
    constexpr bool kHeadEpi = EPI == kHead || EPI == kHeadTrain;
    constexpr bool kTrain = EPI == kHiddenTrain || EPI == kHeadTrain;
    constexpr bool kLayer = kHeadEpi || EPI == kHidden || EPI == kHiddenTrain;
    float yacc = 0.0f;
    // columns in pairs of 32: both TMEM loads of a pair are in flight together (one wait per 64
    // columns; c1 - c0 is a multiple of 64)
#pragma unroll 1
    for (uint32_t c2 = c0; c2 < c1; c2 += 64u) {
        float vv[2][32];
        umma::tmem_ld32x2(taddr + c2, vv[0], vv[1]);
#pragma unroll
    for (uint32_t h = 0; h < 2; ++h) { // unrolled: vv[h] stays in registers
        const uint32_t c = c2 + 32u * h;
        float (&v)[32] = vv[h];
        if constexpr (EPI == kStoreF32) {
            float4* d = reinterpret_cast<float4*>(g.out_f32 + (size_t)m * g.ld_out + c);
#pragma unroll
            for (int q = 0; q < 8; ++q) d[q] = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
        } else if constexpr (EPI == kAtomicF32) {
            float* d = g.out_f32 + (size_t)m * g.ld_out + c;
#pragma unroll
            for (int i = 0; i < 32; ++i) atomicAdd(d + i, v[i]);
        } else if constexpr (kLayer) {
            const float4* b4 = reinterpret_cast<const float4*>(bias + c);
#pragma unroll
            for (int q = 0; q < 8; ++q) {
                const float4 b = b4[q];
                v[4 * q] += b.x;
                v[4 * q + 1] += b.y;
                v[4 * q + 2] += b.z;
                v[4 * q + 3] += b.w;
            }
            if constexpr (kTrain)
                if (g.out_z) store_bf16x32(g.out_z + (size_t)m * N + c, v);
#pragma unroll
            for (int i = 0; i < 32; ++i) v[i] = silu<!kTrain>(v[i]);
            if (g.out_h) store_bf16x32(g.out_h + (size_t)m * N + c, v);
            if constexpr (kTrain)
                if (g.out_hT) store_bf16x32_t(g.out_hT + (size_t)c * g.ld_t + (m - lane), g.ld_t, v, tbuf, lane);
            if constexpr (kHeadEpi) {
                const float4* w4 = reinterpret_cast<const float4*>(head_w + c);
#pragma unroll
                for (int q = 0; q < 8; ++q) {
                    const float4 w = w4[q];
                    yacc = fmaf(v[4 * q], w.x, yacc);
                    yacc = fmaf(v[4 * q + 1], w.y, yacc);
                    yacc = fmaf(v[4 * q + 2], w.z, yacc);
                    yacc = fmaf(v[4 * q + 3], w.w, yacc);
                }
            }
        } else if constexpr (EPI == kBackprop) {
            float z[32];
            load_bf16x32(g.z_prev + (size_t)m * N + c, z);
#pragma unroll
            for (int i = 0; i < 32; ++i) v[i] *= silu_grad<false>(z[i]);
            if (g.out_dz) store_bf16x32(g.out_dz + (size_t)m * N + c, v);
            if (g.out_dzT) store_bf16x32_t(g.out_dzT + (size_t)c * g.ld_t + (m - lane), g.ld_t, v, tbuf, lane);
            if (g.out_db) atomicAdd(&colsum[c + lane], warp_column_sum(v, lane));
        }
    }
    }
    return yacc;
}

// The head's output of row m (one lane per row; called by whole warps whose 32 rows belong to
// one record): y, and the cell mass exp(y) with its per-record sum (one atomic per warp).
__device__ __forceinline__ void head_store(const GemmArgs& g, uint32_t m, float yacc)
{
    const float y = yacc + g.head_b;
    if (g.out_y) g.out_y[m] = y;
    if (g.out_mass) {
        double e = exp((double)y);
        g.out_mass[m] = e;
        if (g.out_mass_sum) {
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) e += __shfl_xor_sync(0xffffffffu, e, o);
            if ((threadIdx.x & 31u) == 0) atomicAdd(&g.out_mass_sum[m / g.record_rows], e);
        }
    }
}

// Split-K GEMM (one 128-row tile and one K range per CTA): the weight gradients, whose K (the
// rows of a batch) is long and whose M and N are the layer widths.
template <int N, int EPI, int MT = 1>
__global__ void __launch_bounds__(128, 1)
    gemm_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB, const GemmArgs g)
{
    constexpr int S = stages<N, MT>();
    constexpr uint32_t SB = stage_bytes<N, MT>();
    constexpr uint32_t BOFF = (uint32_t)MT * kA; // B chunk after the MT A tiles of a stage
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + S * SB);
    uint64_t* empty = full + S;
    uint64_t* done = empty + S;
    uint32_t* tslot = reinterpret_cast<uint32_t*>(done + 1);
    volatile int* abort_flag = reinterpret_cast<volatile int*>(tslot + 1);
    float* colsum = reinterpret_cast<float*>(reinterpret_cast<uint8_t*>(full) + 256);
    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
    if constexpr (EPI == kBackprop)
        for (uint32_t i = threadIdx.x; i < (uint32_t)N; i += blockDim.x) colsum[i] = 0.0f;

    if (threadIdx.x == 0) {
        for (int s = 0; s < S; ++s) {
            umma::mbar_init(&full[s], 1);
            umma::mbar_init(&empty[s], 1);
        }
        umma::mbar_init(done, 1);
        *abort_flag = 0;
        umma::mbar_fence_init();
    }
    if (warp == 0) umma::tmem_alloc(tslot, (uint32_t)(MT * N));
    umma::fence_before_sync();
    __syncthreads();
    umma::fence_after_sync();
    const uint32_t tmem = *tslot;
    const uint32_t m0 = blockIdx.x * 128u * MT;
    const uint32_t nk_total = g.K / 64u;
    const uint32_t kc0 = blockIdx.y * g.k_chunks;
    const uint32_t kc1 = min(nk_total, kc0 + g.k_chunks);
    const uint32_t nk = kc1 > kc0 ? kc1 - kc0 : 0u;

    if (threadIdx.x == 0) {
        bool ok = nk > 0;
        const uint32_t idesc = umma::instr_desc_bf16_f32(128, (uint32_t)N);
        auto load = [&](uint32_t s, uint32_t kc) {
            uint8_t* a = smem + s * SB;
            umma::mbar_arrive_expect_tx(&full[s], SB);
#pragma unroll
            for (int mt = 0; mt < MT; ++mt)
                umma::tma_load_2d(a + mt * kA, &tmA, &full[s], (int32_t)((kc0 + kc) * 64u), (int32_t)(m0 + 128u * mt));
            umma::tma_load_2d(a + BOFF, &tmB, &full[s], (int32_t)((kc0 + kc) * 64u), 0);
        };
        uint32_t issued = nk < (uint32_t)S ? nk : (uint32_t)S, consumed = 0;
        const uint32_t limit = g.wait_limit ? g.wait_limit : kWaitLimit;
        for (uint32_t s = 0; s < issued; ++s) load(s, s);
        for (uint32_t kc = 0; kc < nk && ok; ++kc) {
            const uint32_t s = kc % S, par = (kc / S) & 1u;
            if (!umma::mbar_wait(&full[s], par, limit)) {
                ok = false;
                break;
            }
            consumed = kc + 1;
            umma::fence_after_sync();
            const uint32_t a = umma::smem_u32(smem + s * SB), b = a + BOFF;
#pragma unroll
            for (int mt = 0; mt < MT; ++mt)
#pragma unroll
                for (uint32_t k = 0; k < 4; ++k)
                    umma::mma_bf16(tmem + (uint32_t)(mt * N), umma::smem_desc_sw128(a + mt * kA + 32u * k),
                                   umma::smem_desc_sw128(b + 32u * k), idesc, kc > 0 || k > 0);
            umma::mma_commit(&empty[s]);
            if (kc + S < nk) {
                if (!umma::mbar_wait(&empty[s], par, limit)) {
                    ok = false;
                    break;
                }
                load(s, kc + S);
                issued = kc + S + 1;
            }
        }
        if (!ok) {
            *abort_flag = 1;
            if (nk) atomicExch(g.error, 1u);
            __threadfence_block();
            // loads still in flight land before this CTA's shared memory is released
            for (uint32_t j = consumed; j < issued; ++j) umma::mbar_wait(&full[j % S], (j / S) & 1u, kWaitLimit);
        }
        umma::mma_commit(done); // arrives once every MMA issued above has completed
    }
    // every thread: the accumulator (or the abort) is ready; the epilogue's tcgen05.ld is
    // warp-collective, so the decision is made per warp
    const bool mine = umma::mbar_wait(done, 0, kWaitLimit);
    if (!mine) atomicExch(g.error, 2u);
    const bool ready = __all_sync(0xffffffffu, mine && !*abort_flag);
    umma::fence_after_sync();
    if (ready) {
        // the stages are free once every MMA has completed: one transpose buffer per warp there
        __nv_bfloat16* tbuf = reinterpret_cast<__nv_bfloat16*>(smem) + (size_t)warp * 32u * kTStride;
#pragma unroll 1
        for (int mt = 0; mt < MT; ++mt) {
            const uint32_t m = m0 + 128u * mt + 32u * warp + lane;
            const float y = epilogue_cols<N, EPI>(g, tmem + ((32u * warp) << 16) + (uint32_t)(mt * N), m, lane, 0u,
                                                  (uint32_t)N, g.bias, g.head_w, colsum, tbuf);
            if constexpr (EPI == kHead || EPI == kHeadTrain) head_store(g, m, y);
        }
    }
    if constexpr (EPI == kBackprop) {
        __syncthreads();
        if (g.out_db && ready)
            for (uint32_t i = threadIdx.x; i < (uint32_t)N; i += blockDim.x) atomicAdd(&g.out_db[i], colsum[i]);
    }
    umma::fence_before_sync();
    __syncthreads();
    if (warp == 0) umma::tmem_dealloc(tmem, (uint32_t)(MT * N));
}

// ---------------------------------------------------------------- persistent layer GEMM
// D[M x N] = A[M x K] * B[N x K]^T for the layers (M = rows of a batch, K, N = layer widths):
// the whole B (N x K BF16, <= 128 KB) stays in shared memory; one CTA per SM walks the 128-row
// tiles t = blockIdx.x, blockIdx.x + gridDim.x, ...  Warp 0 streams A chunks through a deep ring
// with TMA; warp 1 allocates 2 N TMEM columns and one of its threads issues the MMAs into
// accumulator buffer (tile & 1); the kEpiWarps warps 2.. drain the other buffer through the
// fused epilogue, so a tile's epilogue overlaps the next tile's MMAs.  Epilogue warp w reads
// TMEM lanes 32 (w mod 4) .. (the rows its lane quarter may access) and column slice
// (w - 2) / 4 of kEpiWarps / 4; the head's partial sums of a row meet in shared memory behind
// a named barrier per lane quarter.  Bias and head weights are staged in shared memory.
// Barriers: a_full / a_empty per ring stage, b_full, acc_full / acc_empty per accumulator, and
// drain (all MMAs complete).  Every wait is bounded; a role that gives up raises the abort flag
// and the error word, the others give up at their next wait, in-flight loads and MMAs are
// waited for, and the tensor memory is freed.
constexpr uint32_t kEpiWarps = 8;
constexpr uint32_t kSlices = kEpiWarps / 4;
constexpr uint32_t kPThreads = 64 + 32 * kEpiWarps;
// per-CTA extras after the ring: barriers (1 KB), colsum, bias, head weights (1 KB each), head
// partial sums (kSlices - 1 slices x 128 floats, rounded up to kSlices)
constexpr int kPExtra = 1024 + 3 * 1024 + (int)kSlices * 512 + (int)(kEpiWarps * 32u * kTStride * 2u);
template <int N, int KC> __host__ __device__ constexpr int pstages()
{
    return (232448 - 1024 - N * 128 * KC - kPExtra) / (int)kA > 8 ? 8
                                                                   : (232448 - 1024 - N * 128 * KC - kPExtra) / (int)kA;
}
template <int N, int KC> constexpr size_t psmem_bytes()
{
    return 1024 + (size_t)N * 128 * KC + (size_t)pstages<N, KC>() * kA + kPExtra;
}

__device__ __forceinline__ void named_sync(uint32_t id, uint32_t threads)
{
    asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(threads) : "memory");
}

template <int N, int KC, int EPI>
__global__ void __launch_bounds__(kPThreads, 1)
    gemm_persistent_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                           const GemmArgs g)
{
    constexpr int S = pstages<N, KC>();
    constexpr bool kHeadEpi = EPI == kHead || EPI == kHeadTrain;
    constexpr uint32_t BB = (uint32_t)N * 128u;   // one 64-wide K chunk of B
    constexpr uint32_t W = (uint32_t)N / kSlices; // columns per epilogue warp
    static_assert(S >= 2, "ring too shallow");
    static_assert(W % 64u == 0, "slice width: the epilogue takes columns in pairs of 32");
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    uint8_t* bres = smem;
    uint8_t* ring = smem + KC * BB;
    uint64_t* a_full = reinterpret_cast<uint64_t*>(ring + S * kA);
    uint64_t* a_empty = a_full + S;
    uint64_t* b_full = a_empty + S;
    uint64_t* acc_full = b_full + 1;
    uint64_t* acc_empty = acc_full + 2;
    uint64_t* drain = acc_empty + 2;
    uint32_t* tslot = reinterpret_cast<uint32_t*>(drain + 1);
    volatile int* abort_flag = reinterpret_cast<volatile int*>(tslot + 1);
    float* colsum = reinterpret_cast<float*>(reinterpret_cast<uint8_t*>(a_full) + 1024);
    float* sbias = colsum + 256;
    float* shead = sbias + 256;
    float* ypart = shead + 256; // [kSlices - 1][128]
    __nv_bfloat16* tbufs = reinterpret_cast<__nv_bfloat16*>(ypart + kSlices * 128u); // per epilogue warp
    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
    const uint32_t tiles = g.M / 128u;

    if (threadIdx.x == 0) {
        for (int s = 0; s < S; ++s) {
            umma::mbar_init(&a_full[s], 1);
            umma::mbar_init(&a_empty[s], 1);
        }
        umma::mbar_init(b_full, 1);
        for (int b = 0; b < 2; ++b) {
            umma::mbar_init(&acc_full[b], 1);
            umma::mbar_init(&acc_empty[b], kEpiWarps);
        }
        umma::mbar_init(drain, 1);
        *abort_flag = 0;
        umma::mbar_fence_init();
    }
    for (uint32_t i = threadIdx.x; i < (uint32_t)N; i += blockDim.x) {
        colsum[i] = 0.0f;
        if constexpr (kHeadEpi || EPI == kHidden || EPI == kHiddenTrain) sbias[i] = g.bias[i];
        if constexpr (kHeadEpi) shead[i] = g.head_w[i];
    }
    if (warp == 1) umma::tmem_alloc(tslot, 2u * N);
    umma::fence_before_sync();
    __syncthreads();
    umma::fence_after_sync();
    const uint32_t tmem = *tslot;

    if (warp == 0) {
        if (lane == 0) {
            // producer: B once, then the A chunks of every tile of this CTA
            bool ok = true;
            umma::mbar_arrive_expect_tx(b_full, KC * BB);
            for (int kc = 0; kc < KC; ++kc) umma::tma_load_2d(bres + kc * BB, &tmB, b_full, kc * 64, 0);
            uint32_t it = 0;
#pragma unroll 1
            for (uint32_t t = blockIdx.x; t < tiles && ok; t += gridDim.x) {
                for (int kc = 0; kc < KC; ++kc, ++it) {
                    const uint32_t s = it % S;
                    if (it >= (uint32_t)S && !umma::mbar_wait(&a_empty[s], ((it / S) & 1u) ^ 1u, kWaitLimit)) {
                        ok = false;
                        break;
                    }
                    if (*abort_flag) {
                        ok = false;
                        break;
                    }
                    umma::mbar_arrive_expect_tx(&a_full[s], kA);
                    umma::tma_load_2d(ring + s * kA, &tmA, &a_full[s], kc * 64, (int32_t)(t * 128u));
                }
            }
            if (!ok) {
                *abort_flag = 1;
                atomicExch(g.error, 3u);
            }
            // every issued load lands before the CTA's shared memory is released
            for (uint32_t j = it > (uint32_t)S ? it - S : 0u; j < it; ++j)
                umma::mbar_wait(&a_full[j % S], (j / S) & 1u, kWaitLimit);
            umma::mbar_wait(b_full, 0, kWaitLimit);
        }
    } else if (warp == 1) {
        if (lane == 0) {
            // MMA issuer
            const uint32_t idesc = umma::instr_desc_bf16_f32(128, (uint32_t)N);
            bool ok = umma::mbar_wait(b_full, 0, kWaitLimit);
            uint32_t it = 0, i = 0;
#pragma unroll 1
            for (uint32_t t = blockIdx.x; t < tiles && ok; t += gridDim.x, ++i) {
                const uint32_t b = i & 1u;
                if (i >= 2 && !umma::mbar_wait(&acc_empty[b], ((i >> 1) - 1u) & 1u, kWaitLimit)) {
                    ok = false;
                    break;
                }
                umma::fence_after_sync();
                const uint32_t d = tmem + b * (uint32_t)N;
                for (int kc = 0; kc < KC; ++kc, ++it) {
                    const uint32_t s = it % S;
                    if (!umma::mbar_wait(&a_full[s], (it / S) & 1u, kWaitLimit) || *abort_flag) {
                        ok = false;
                        break;
                    }
                    umma::fence_after_sync();
                    const uint32_t a = umma::smem_u32(ring + s * kA), bb = umma::smem_u32(bres + kc * BB);
#pragma unroll
                    for (uint32_t k = 0; k < 4; ++k)
                        umma::mma_bf16(d, umma::smem_desc_sw128(a + 32u * k), umma::smem_desc_sw128(bb + 32u * k), idesc,
                                       kc > 0 || k > 0);
                    umma::mma_commit(&a_empty[s]);
                }
                if (!ok) break;
                umma::mma_commit(&acc_full[b]);
            }
            if (!ok) {
                *abort_flag = 1;
                atomicExch(g.error, 4u);
            }
            umma::mma_commit(drain);
            if (!umma::mbar_wait(drain, 0, kWaitLimit)) atomicExch(g.error, 6u);
        }
    } else {
        // epilogue warps
        const uint32_t q = warp & 3u, slice = (warp - 2u) >> 2;
        const uint32_t c0 = slice * W;
        const uint32_t row = 32u * q + lane;
        uint32_t i = 0;
        bool live = true;
#pragma unroll 1
        for (uint32_t t = blockIdx.x; t < tiles; t += gridDim.x, ++i) {
            const uint32_t b = i & 1u;
            const bool mine = live && umma::mbar_wait(&acc_full[b], (i >> 1) & 1u, kWaitLimit);
            if (!__all_sync(0xffffffffu, mine && !*abort_flag)) {
                if (lane == 0 && live) {
                    *abort_flag = 1;
                    atomicExch(g.error, 5u);
                }
                live = false;
            }
            float y = 0.0f;
            if (live) {
                umma::fence_after_sync();
                y = epilogue_cols<N, EPI>(g, tmem + ((32u * q) << 16) + b * (uint32_t)N, t * 128u + row, lane, c0,
                                          c0 + W, sbias, shead, colsum, tbufs + (warp - 2u) * 32u * kTStride);
                umma::fence_before_sync();
                __syncwarp();
                if (lane == 0) umma::mbar_arrive(&acc_empty[b]);
            }
            if constexpr (kHeadEpi) {
                // the slices of a lane quarter meet here every tile (also after an abort, so that
                // the named barrier never waits for a warp that has left the loop)
                if (slice) ypart[(slice - 1u) * 128u + row] = y;
                named_sync(1u + q, 32u * kSlices);
                if (slice == 0 && live) {
                    for (uint32_t k = 1; k < kSlices; ++k) y += ypart[(k - 1u) * 128u + row];
                    head_store(g, t * 128u + row, y);
                }
                named_sync(1u + q, 32u * kSlices);
            }
        }
    }
    umma::fence_before_sync();
    __syncthreads();
    if constexpr (EPI == kBackprop) {
        if (g.out_db && !*abort_flag)
            for (uint32_t k = threadIdx.x; k < (uint32_t)N; k += blockDim.x) atomicAdd(&g.out_db[k], colsum[k]);
    }
    if (warp == 1) umma::tmem_dealloc(tmem, 2u * N);
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link-time libcuda).
using EncodeTiled = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                 const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                 CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
EncodeTiled encode_tiled()
{
    static EncodeTiled fn = [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            p = nullptr;
        return reinterpret_cast<EncodeTiled>(p);
    }();
    return fn;
}

// Tensor map of a row-major BF16 matrix [rows x cols] read in boxes of 64 columns x box_rows.
int make_map(CUtensorMap* map, const void* ptr, uint32_t rows, uint32_t cols, uint32_t box_rows)
{
    const EncodeTiled encode = encode_tiled();
    if (!encode) return -5;
    const cuuint64_t dims[2] = {cols, rows};
    const cuuint64_t strides[1] = {(cuuint64_t)cols * 2u};
    const cuuint32_t box[2] = {64u, box_rows};
    const cuuint32_t elem[2] = {1u, 1u};
    const CUresult r = encode(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(ptr), dims,
                                              strides, box, elem, CU_TENSOR_MAP_INTERLEAVE_NONE,
                                              CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                                              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? 0 : (int)r;
}

template <int N, int EPI, int MT = 1>
int launch_n(const void* A, const void* B, const GemmArgs& g, uint32_t splits, cudaStream_t st)
{
    CUtensorMap ta, tb;
    if (make_map(&ta, A, g.M, g.K, 128u) || make_map(&tb, B, (uint32_t)N, g.K, (uint32_t)N)) return -1;
    const size_t smem = smem_bytes<N, MT>();
    cudaError_t e =
        cudaFuncSetAttribute(gemm_kernel<N, EPI, MT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return (int)e;
    gemm_kernel<N, EPI, MT><<<dim3(g.M / (128u * MT), splits), 128, smem, st>>>(ta, tb, g);
    return (int)cudaGetLastError();
}

template <int EPI> int launch_epi(const void* A, const void* B, const GemmArgs& g, uint32_t splits, cudaStream_t st)
{
    if constexpr (EPI == kAtomicF32) {
        // two row tiles per CTA share each B chunk
        if (g.M % 256u == 0) {
            switch (g.N) {
            case 64: return launch_n<64, EPI, 2>(A, B, g, splits, st);
            case 128: return launch_n<128, EPI, 2>(A, B, g, splits, st);
            case 256: return launch_n<256, EPI, 2>(A, B, g, splits, st);
            default: return -2;
            }
        }
    }
    switch (g.N) {
    case 64: return launch_n<64, EPI>(A, B, g, splits, st);
    case 128: return launch_n<128, EPI>(A, B, g, splits, st);
    case 256: return launch_n<256, EPI>(A, B, g, splits, st);
    default: return -2;
    }
}

int sm_count()
{
    static const int n = [] {
        int dev = 0, v = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev);
        return v > 0 ? v : 148;
    }();
    return n;
}

template <int N, int KC, int EPI> int launch_p(const void* A, const void* B, const GemmArgs& g, cudaStream_t st)
{
    CUtensorMap ta, tb;
    if (make_map(&ta, A, g.M, g.K, 128u) || make_map(&tb, B, (uint32_t)N, g.K, (uint32_t)N)) return -1;
    const size_t smem = psmem_bytes<N, KC>();
    cudaError_t e = cudaFuncSetAttribute(gemm_persistent_kernel<N, KC, EPI>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e != cudaSuccess) return (int)e;
    const uint32_t tiles = g.M / 128u;
    const uint32_t grid = tiles < (uint32_t)sm_count() ? tiles : (uint32_t)sm_count();
    gemm_persistent_kernel<N, KC, EPI><<<grid, kPThreads, smem, st>>>(ta, tb, g);
    return (int)cudaGetLastError();
}

template <int EPI> int launch_pe(const void* A, const void* B, const GemmArgs& g, cudaStream_t st)
{
    const uint32_t kc = g.K / 64u;
    if (g.N == 256) {
        if (kc == 1) return launch_p<256, 1, EPI>(A, B, g, st);
        if (kc == 2) return launch_p<256, 2, EPI>(A, B, g, st);
        if (kc == 4) return launch_p<256, 4, EPI>(A, B, g, st);
    } else if (g.N == 128) {
        if (kc == 1) return launch_p<128, 1, EPI>(A, B, g, st);
        if (kc == 2) return launch_p<128, 2, EPI>(A, B, g, st);
        if (kc == 4) return launch_p<128, 4, EPI>(A, B, g, st);
    }
    return -2;
}

bool persistent_shape(const GemmArgs& g)
{
    const uint32_t kc = g.K / 64u;
    return (g.N == 128 || g.N == 256) && (kc == 1 || kc == 2 || kc == 4);
}

// ---------------------------------------------------------------- fused inference pass
// One persistent CTA per SM takes its 128-row tiles (t = blockIdx.x, blockIdx.x + gridDim.x, ...)
// two at a time, in slots 0 and 1, through the three hidden layers and the head without leaving
// the SM.  Each slot owns a TMEM region (its 128 x 256 FP32 accumulator) and an H buffer (its
// activations as BF16, 128 rows x 256 in the K-major 128-byte-swizzled layout a TMA load would
// have written, four 16 KB chunks).  The MMA thread issues (layer, slot) in the order
// (0, 0), (0, 1), (1, 0), (1, 1), (2, 0), (2, 1), so the tensor pipe computes one slot's layer while
// the epilogue warps drain the other slot's previous layer: a tile's own layers are serial (each
// needs the previous one's activations), the two tiles of a pair overlap.
//   * A tile's input rows X (KC1 chunks of 64 columns: record features, the cell table, the axis
//     harmonics, as launch_features defines them) are built in the first chunks of its slot's H
//     buffer once the slot's previous tile has finished its last layer (h_free): the slot's
//     feature warp loads the tile's 128 cells from the row-layout cell table by TMA (x_land),
//     then writes the record and axis-harmonic columns (x_full).  The rows never exist in
//     global memory.
//   * The weights (W1, W2, W3 in 32 KB chunks of 64 input columns x 256 units, read from L2) go
//     through a kFStages-deep ring in the MMA order, once per (layer, slot).
//   * The epilogue (sixteen warps: lane quarter q, 64-column chunk s) writes a layer's activations
//     into the slot's H buffer, fences them for the tensor core's reads and arrives on the slot's
//     acc_empty: the slot's next layer may then overwrite the accumulator and read H.  The head
//     epilogue forms y = silu(z3) . w4 + b as the kHead epilogue does.
// Barriers per slot: x_land, x_full, h_free, acc_full, acc_empty; per ring stage: w_full, w_empty;
// drain.
// Every wait is bounded as in gemm_persistent_kernel.
constexpr uint32_t kFStages = 2;
constexpr uint32_t kFEpiWarps = 16; // four per TMEM lane quarter, one 64-column chunk each
constexpr uint32_t kFThreads = 128 + 32 * kFEpiWarps; // producer, MMA, two feature warps, epilogue
constexpr uint32_t kWChunk = 256u * 128u; // 64 input columns x 256 units, BF16
constexpr uint32_t kHChunk = 128u * 128u; // 128 rows x 64 columns, BF16
constexpr uint32_t kFExtra = 8192;        // barriers, TMEM slot, abort flag, biases, head, partial sums
template <int KC1> constexpr size_t fsmem_bytes()
{
    return 1024 + 2 * 4 * kHChunk + kFStages * kWChunk + kFExtra;
}

__device__ __forceinline__ void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// Packed FP32 pairs (sm_100 add / mul / fma .f32x2: one instruction for two lanes of work).
__device__ __forceinline__ uint64_t pk2(float a, float b)
{
    uint64_t r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a), "f"(b));
    return r;
}
__device__ __forceinline__ void upk2(uint64_t r, float& a, float& b) { asm("mov.b64 {%0, %1}, %2;" : "=f"(a), "=f"(b) : "l"(r)); }
__device__ __forceinline__ uint64_t add2(uint64_t a, uint64_t b)
{
    uint64_t r;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
    return r;
}
__device__ __forceinline__ uint64_t mul2(uint64_t a, uint64_t b)
{
    uint64_t r;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
    return r;
}
__device__ __forceinline__ uint64_t fma2(uint64_t a, uint64_t b, uint64_t c)
{
    uint64_t r;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r) : "l"(a), "l"(b), "l"(c));
    return r;
}
// silu(a + ba), silu(b + bb) with the arithmetic of logistic() done in pairs, bit for bit: the
// negated denominator -d = ex2 * -1 - 1 is exact, its seed 0xFEF311C0 - bits(-d) equals
// 0x7EF311C0 - bits(d), and fma(-d, y, 1) is the same rounding as before.
__device__ __forceinline__ void silu_pair(float& a, float& b, float ba, float bb)
{
    constexpr float kNegLog2e = -1.44269504088896341f;
    float va, vb;
    upk2(add2(pk2(a, b), pk2(ba, bb)), va, vb);
    float xa, xb;
    upk2(mul2(pk2(fmaxf(va, -80.0f), fmaxf(vb, -80.0f)), pk2(kNegLog2e, kNegLog2e)), xa, xb);
    const uint64_t m1 = pk2(-1.0f, -1.0f), one = pk2(1.0f, 1.0f);
    const uint64_t nd = fma2(pk2(ex2_ftz(xa), ex2_ftz(xb)), m1, m1);
    float da, db;
    upk2(nd, da, db);
    uint64_t y = pk2(__int_as_float((int)(0xFEF311C0u - (uint32_t)__float_as_int(da))),
                     __int_as_float((int)(0xFEF311C0u - (uint32_t)__float_as_int(db))));
    y = fma2(y, fma2(nd, y, one), y);
    const uint64_t e = fma2(nd, y, one);
    upk2(mul2(pk2(va, vb), fma2(y, fma2(e, e, e), y)), a, b);
}


// One 64-column chunk of this thread's accumulator row through bias + SiLU into BF16, stored in
// row `row` of a swizzled H chunk: 16-byte piece p of the row at ((p ^ (row & 7)) << 4).
// 32 columns per TMEM load keep the epilogue within the 96 registers that 18 warps per SM allow.
__device__ __forceinline__ void hidden_chunk(uint32_t taddr, const float* bias, uint8_t* hrow, uint32_t row)
{
#pragma unroll
    for (uint32_t h = 0; h < 2; ++h) {
        float v[32];
        umma::tmem_ld32(taddr + 32u * h, v);
#pragma unroll
        for (uint32_t q = 0; q < 4; ++q) {
            const float4 b0 = *reinterpret_cast<const float4*>(bias + 32u * h + 8u * q);
            const float4 b1 = *reinterpret_cast<const float4*>(bias + 32u * h + 8u * q + 4u);
            const float bb[8] = {b0.x, b0.y, b0.z, b0.w, b1.x, b1.y, b1.z, b1.w};
            uint32_t w[4];
#pragma unroll
            for (uint32_t i = 0; i < 4; ++i) {
                float a = v[8 * q + 2 * i], c = v[8 * q + 2 * i + 1];
                silu_pair(a, c, bb[2 * i], bb[2 * i + 1]);
                const __nv_bfloat162 p = __floats2bfloat162_rn(a, c);
                w[i] = *reinterpret_cast<const uint32_t*>(&p);
            }
            const uint32_t piece = 4u * h + q;
            *reinterpret_cast<uint4*>(hrow + ((piece ^ (row & 7u)) << 4)) = make_uint4(w[0], w[1], w[2], w[3]);
        }
    }
}

// Partial head sum of one 64-column chunk: sum silu(acc + bias) * head_w (four interleaved
// partial sums, so that the products do not wait on one another).
__device__ __forceinline__ float head_chunk(uint32_t taddr, const float* bias, const float* head_w, float y)
{
    float y0 = 0.0f, y1 = 0.0f, y2 = 0.0f, y3 = 0.0f;
#pragma unroll
    for (uint32_t h = 0; h < 2; ++h) {
        float vv[32];
        umma::tmem_ld32(taddr + 32u * h, vv);
#pragma unroll
        for (uint32_t q = 0; q < 8; ++q) {
            const float4 b = *reinterpret_cast<const float4*>(bias + 32u * h + 4u * q);
            const float4 w = *reinterpret_cast<const float4*>(head_w + 32u * h + 4u * q);
            float s0 = vv[4 * q], s1 = vv[4 * q + 1], s2 = vv[4 * q + 2], s3 = vv[4 * q + 3];
            silu_pair(s0, s1, b.x, b.y);
            silu_pair(s2, s3, b.z, b.w);
            y0 = fmaf(s0, w.x, y0);
            y1 = fmaf(s1, w.y, y1);
            y2 = fmaf(s2, w.z, y2);
            y3 = fmaf(s3, w.w, y3);
        }
    }
    return y + ((y0 + y1) + (y2 + y3));
}

__device__ __forceinline__ void fused_head_store(const FusedArgs& f, uint32_t m, float yacc)
{
    const float y = yacc + f.head_b;
    if (f.out_y) f.out_y[m] = y;
    if (f.out_mass) {
        double e = exp((double)y);
        f.out_mass[m] = e;
        if (f.out_mass_sum) {
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) e += __shfl_xor_sync(0xffffffffu, e, o);
            if ((threadIdx.x & 31u) == 0) atomicAdd(&f.out_mass_sum[m / f.record_rows], e);
        }
    }
}

template <int KC1>
__global__ void __launch_bounds__(kFThreads, 1)
    mlp_fused_kernel(const __grid_constant__ CUtensorMap tmXC, const __grid_constant__ CUtensorMap tmW1,
                     const __grid_constant__ CUtensorMap tmW2, const __grid_constant__ CUtensorMap tmW3,
                     const FusedArgs f)
{
    constexpr uint32_t S = kFStages;
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    uint8_t* hbuf = smem; // slot s at hbuf + s * 4 kHChunk; its input rows in chunks [0, KC1)
    uint8_t* ring = hbuf + 2 * 4 * kHChunk;
    uint64_t* bars = reinterpret_cast<uint64_t*>(ring + S * kWChunk);
    uint64_t* x_full = bars;         // [2]
    uint64_t* h_free = bars + 2;     // [2]
    uint64_t* acc_full = bars + 4;   // [2]
    uint64_t* acc_empty = bars + 6;  // [2]
    uint64_t* x_land = bars + 8;     // [2]
    uint64_t* w_full = bars + 10;    // [S]
    uint64_t* w_empty = w_full + S;  // [S]
    uint64_t* drain = w_empty + S;
    uint32_t* tslot = reinterpret_cast<uint32_t*>(drain + 1);
    volatile int* abort_flag = reinterpret_cast<volatile int*>(tslot + 1);
    float* sb = reinterpret_cast<float*>(reinterpret_cast<uint8_t*>(bars) + 1024); // b1, b2, b3, head_w
    float* ypart = sb + 4 * 256;                                                     // [3][128]
    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
    const uint32_t tiles = f.M / 128u;
    // this CTA's tiles: t_k = blockIdx.x + k gridDim.x, k < mine; pair p holds k = 2p (slot 0)
    // and k = 2p + 1 (slot 1, absent in a last pair of an odd count)
    const uint32_t mine = blockIdx.x < tiles ? (tiles - blockIdx.x + gridDim.x - 1) / gridDim.x : 0u;
    const uint32_t pairs = (mine + 1u) / 2u;

    if (threadIdx.x == 0) {
        for (int s = 0; s < 2; ++s) {
            umma::mbar_init(&x_full[s], 1);
            umma::mbar_init(&h_free[s], 1);
            umma::mbar_init(&acc_full[s], 1);
            umma::mbar_init(&acc_empty[s], kFEpiWarps);
            umma::mbar_init(&x_land[s], 1);
        }
        for (uint32_t s = 0; s < S; ++s) {
            umma::mbar_init(&w_full[s], 1);
            umma::mbar_init(&w_empty[s], 1);
        }
        umma::mbar_init(drain, 1);
        *abort_flag = 0;
        umma::mbar_fence_init();
    }
    for (uint32_t i = threadIdx.x; i < 256u; i += blockDim.x) {
        sb[i] = f.b1[i];
        sb[256 + i] = f.b2[i];
        sb[512 + i] = f.b3[i];
        sb[768 + i] = f.head_w[i];
    }
    if (warp == 1) umma::tmem_alloc(tslot, 512u);
    umma::fence_before_sync();
    __syncthreads();
    umma::fence_after_sync();
    const uint32_t tmem = *tslot;

    if (warp == 0) {
        if (lane == 0) {
            // producer: the weight chunks of every (layer, slot) in the MMA order
            bool ok = true;
            uint32_t it = 0; // weight chunks issued
#pragma unroll 1
            for (uint32_t p = 0; p < pairs && ok; ++p) {
#pragma unroll 1
                for (uint32_t l = 0; l < 3 && ok; ++l) {
#pragma unroll 1
                    for (uint32_t sl = 0; sl < 2 && ok; ++sl) {
                        const uint32_t k = 2u * p + sl;
                        if (k >= mine) break;
                        const uint32_t n = l == 0 ? (uint32_t)KC1 : 4u;
                        const CUtensorMap* map = l == 0 ? &tmW1 : (l == 1 ? &tmW2 : &tmW3);
                        for (uint32_t kc = 0; kc < n; ++kc, ++it) {
                            const uint32_t s = it % S;
                            if (it >= S && !umma::mbar_wait(&w_empty[s], ((it / S) & 1u) ^ 1u, kWaitLimit)) {
                                ok = false;
                                break;
                            }
                            if (*abort_flag) {
                                ok = false;
                                break;
                            }
                            umma::mbar_arrive_expect_tx(&w_full[s], kWChunk);
                            umma::tma_load_2d(ring + s * kWChunk, map, &w_full[s], (int32_t)(kc * 64u), 0);
                        }
                    }
                }
            }
            if (!ok) {
                *abort_flag = 1;
                atomicExch(f.error, 3u);
            }
            // every issued load lands before the CTA's shared memory is released
            for (uint32_t j = it > S ? it - S : 0u; j < it; ++j) umma::mbar_wait(&w_full[j % S], (j / S) & 1u, kWaitLimit);
        }
    } else if (warp == 1) {
        if (lane == 0) {
            // MMA issuer: (layer, slot) in the order above.  Layer l of a slot's tile n waits for
            // completion 3 n + l - 1 of the slot's acc_empty (its previous layer drained and its
            // activations written; for l = 0 the previous tile's head), and layer 0 for the rows.
            const uint32_t idesc = umma::instr_desc_bf16_f32(128, 256);
            bool ok = true;
            uint32_t it = 0;
#pragma unroll 1
            for (uint32_t p = 0; p < pairs && ok; ++p) {
#pragma unroll 1
                for (uint32_t l = 0; l < 3 && ok; ++l) {
#pragma unroll 1
                    for (uint32_t sl = 0; sl < 2 && ok; ++sl) {
                        const uint32_t k = 2u * p + sl;
                        if (k >= mine) break;
                        const uint32_t c = 3u * p + l; // this layer's index among the slot's layers
                        if (c >= 1 && !umma::mbar_wait(&acc_empty[sl], (c - 1u) & 1u, kWaitLimit)) {
                            ok = false;
                            break;
                        }
                        if (l == 0 && !umma::mbar_wait(&x_full[sl], p & 1u, kWaitLimit)) {
                            ok = false;
                            break;
                        }
                        umma::fence_after_sync();
                        const uint32_t d = tmem + sl * 256u;
                        const uint32_t n = l == 0 ? (uint32_t)KC1 : 4u;
                        for (uint32_t kc = 0; kc < n; ++kc, ++it) {
                            const uint32_t s = it % S;
                            if (!umma::mbar_wait(&w_full[s], (it / S) & 1u, kWaitLimit) || *abort_flag) {
                                ok = false;
                                break;
                            }
                            umma::fence_after_sync();
                            const uint32_t a = umma::smem_u32(hbuf + (sl * 4u + kc) * kHChunk);
                            const uint32_t b = umma::smem_u32(ring + s * kWChunk);
#pragma unroll
                            for (uint32_t q = 0; q < 4; ++q)
                                umma::mma_bf16(d, umma::smem_desc_sw128(a + 32u * q), umma::smem_desc_sw128(b + 32u * q),
                                               idesc, kc > 0 || q > 0);
                            umma::mma_commit(&w_empty[s]);
                        }
                        if (!ok) break;
                        if (l == 2) umma::mma_commit(&h_free[sl]);
                        umma::mma_commit(&acc_full[sl]);
                    }
                }
            }
            if (!ok) {
                *abort_flag = 1;
                atomicExch(f.error, 4u);
            }
            umma::mma_commit(drain);
            if (!umma::mbar_wait(drain, 0, kWaitLimit)) atomicExch(f.error, 6u);
        }
    } else if (warp < 4) {
        // feature warp of slot sl: the input rows of each of the slot's tiles into its H buffer,
        // bit for bit as features_kernel writes them (16-byte pieces: q < 2 the record features,
        // q < qaxis the cell table, then the axis harmonics).  A tile's rows belong to one record
        // (the record's cell count is a multiple of 128) and to 128 consecutive cells.
        const uint32_t sl = warp - 2u;
        const uint32_t qrow = f.K0 / 8u, qaxis = qrow - f.P / 8u, C = f.record_rows;
        const uint4* rec16 = reinterpret_cast<const uint4*>(f.rec16);
        uint8_t* h = hbuf + sl * 4u * kHChunk;
#pragma unroll 1
        for (uint32_t p = 0; p < pairs; ++p) {
            const uint32_t k = 2u * p + sl;
            if (k >= mine) break;
            const bool ready = p == 0 || umma::mbar_wait(&h_free[sl], (p - 1u) & 1u, kWaitLimit);
            if (!__all_sync(0xffffffffu, ready && !*abort_flag)) {
                if (lane == 0) {
                    *abort_flag = 1;
                    atomicExch(f.error, 7u);
                }
                break;
            }
            const uint32_t row0 = (blockIdx.x + k * gridDim.x) * 128u;
            const uint32_t rec = row0 / C, c0 = row0 - rec * C;
            if (lane == 0) {
                umma::mbar_arrive_expect_tx(&x_land[sl], KC1 * kHChunk);
                for (int kc = 0; kc < KC1; ++kc)
                    umma::tma_load_2d(h + kc * kHChunk, &tmXC, &x_land[sl], kc * 64, (int32_t)c0);
            }
            const bool landed = umma::mbar_wait(&x_land[sl], p & 1u, kWaitLimit);
            if (!__all_sync(0xffffffffu, landed)) {
                if (lane == 0) {
                    *abort_flag = 1;
                    atomicExch(f.error, 7u);
                    umma::mbar_wait(&x_land[sl], p & 1u, kWaitLimit); // the load lands before the CTA ends
                }
                break;
            }
            const uint4 ra = rec16[2u * rec], rb = rec16[2u * rec + 1u];
            for (uint32_t r = lane; r < 128u; r += 32u) {
                // record columns: pieces 0 and 1 of chunk 0
                *reinterpret_cast<uint4*>(h + r * 128u + ((0u ^ (r & 7u)) << 4)) = ra;
                *reinterpret_cast<uint4*>(h + r * 128u + ((1u ^ (r & 7u)) << 4)) = rb;
                const double x = cos_psi(f.recgeo, f.cellgeo, rec, c0 + r);
                double tm = 1.0, t = x; // T_0, T_1: the same recurrence as axis_harmonics8
                for (uint32_t q = qaxis; q < qrow; ++q) {
                    __align__(16) __nv_bfloat16 hv[8];
#pragma unroll
                    for (int i = 0; i < 8; ++i) {
                        hv[i] = __float2bfloat16_rn(__double2float_rn(t));
                        const double tn = __dsub_rn(__dmul_rn(__dmul_rn(2.0, x), t), tm);
                        tm = t;
                        t = tn;
                    }
                    *reinterpret_cast<uint4*>(h + (q >> 3) * kHChunk + r * 128u + (((q & 7u) ^ (r & 7u)) << 4)) =
                        *reinterpret_cast<const uint4*>(hv);
                }
            }
            fence_proxy_async_smem();
            __syncwarp();
            if (lane == 0) umma::mbar_arrive(&x_full[sl]);
        }
    } else {
        // epilogue warps: lane quarter q (TMEM lanes 32 q ..), 64-column chunk `slice`
        const uint32_t q = warp & 3u, slice = (warp - 4u) >> 2;
        const uint32_t row = 32u * q + lane, c = 64u * slice;
        bool live = true;
#pragma unroll 1
        for (uint32_t p = 0; p < pairs; ++p) {
#pragma unroll 1
            for (uint32_t l = 0; l < 3; ++l) {
#pragma unroll 1
                for (uint32_t sl = 0; sl < 2; ++sl) {
                    const uint32_t k = 2u * p + sl;
                    if (k >= mine) break;
                    const uint32_t n = 3u * p + l;
                    const bool ready = live && umma::mbar_wait(&acc_full[sl], n & 1u, kWaitLimit);
                    if (!__all_sync(0xffffffffu, ready && !*abort_flag)) {
                        if (lane == 0 && live) {
                            *abort_flag = 1;
                            atomicExch(f.error, 5u);
                        }
                        live = false;
                    }
                    const uint32_t taddr = tmem + ((32u * q) << 16) + sl * 256u + c;
                    float y = 0.0f;
                    if (live) {
                        umma::fence_after_sync();
                        if (l < 2) {
                            hidden_chunk(taddr, sb + 256u * l + c, hbuf + (sl * 4u + slice) * kHChunk + row * 128u, row);
                            fence_proxy_async_smem();
                        } else {
                            y = head_chunk(taddr, sb + 512u + c, sb + 768u + c, y);
                        }
                        umma::fence_before_sync();
                        __syncwarp();
                        if (lane == 0) umma::mbar_arrive(&acc_empty[sl]);
                    }
                    if (l == 2) {
                        // the four slices of a lane quarter meet here every tile (also after an
                        // abort, so that the named barrier never waits for a warp that has left)
                        if (slice) ypart[(slice - 1u) * 128u + row] = y;
                        named_sync(1u + q, 128u);
                        if (slice == 0 && live)
                            fused_head_store(f, (blockIdx.x + k * gridDim.x) * 128u + row,
                                             ((y + ypart[row]) + ypart[128u + row]) + ypart[256u + row]);
                        named_sync(1u + q, 128u);
                    }
                }
            }
        }
    }
    umma::fence_before_sync();
    __syncthreads();
    if (warp == 1) umma::tmem_dealloc(tmem, 512u);
}

template <int KC1>
int launch_fused(const void* W1, const void* W2, const void* W3, const FusedArgs& f, cudaStream_t st)
{
    CUtensorMap tc, t1, t2, t3;
    if (make_map(&tc, f.xcells, f.record_rows, f.K0, 128u) || make_map(&t1, W1, 256u, f.K0, 256u) ||
        make_map(&t2, W2, 256u, 256u, 256u) || make_map(&t3, W3, 256u, 256u, 256u))
        return -1;
    const size_t smem = fsmem_bytes<KC1>();
    cudaError_t e =
        cudaFuncSetAttribute(mlp_fused_kernel<KC1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return (int)e;
    const uint32_t tiles = f.M / 128u;
    const uint32_t grid = tiles < (uint32_t)sm_count() ? tiles : (uint32_t)sm_count();
    mlp_fused_kernel<KC1><<<grid, kFThreads, smem, st>>>(tc, t1, t2, t3, f);
    return (int)cudaGetLastError();
}

} // namespace

int gemm(const void* A, const void* B, GemmArgs g, int epi, uint32_t splits, cudaStream_t st)
{
    if (g.M == 0 || g.M % 128u || g.K == 0 || g.K % 64u || !splits) return -3;
    if (epi != kAtomicF32) splits = 1; // only the atomic epilogue can add partial K ranges
    const uint32_t nk = g.K / 64u;
    g.k_chunks = (nk + splits - 1) / splits;
    splits = (nk + g.k_chunks - 1) / g.k_chunks; // every CTA gets at least one chunk
    if (epi != kAtomicF32 && persistent_shape(g)) {
        switch (epi) {
        case kStoreF32: return launch_pe<kStoreF32>(A, B, g, st);
        case kHidden: return launch_pe<kHidden>(A, B, g, st);
        case kHead: return launch_pe<kHead>(A, B, g, st);
        case kHiddenTrain: return launch_pe<kHiddenTrain>(A, B, g, st);
        case kHeadTrain: return launch_pe<kHeadTrain>(A, B, g, st);
        case kBackprop: return launch_pe<kBackprop>(A, B, g, st);
        default: return -4;
        }
    }
    switch (epi) {
    case kStoreF32: return launch_epi<kStoreF32>(A, B, g, splits, st);
    case kAtomicF32: return launch_epi<kAtomicF32>(A, B, g, splits, st);
    case kHidden: return launch_epi<kHidden>(A, B, g, 1, st);
    case kHead: return launch_epi<kHead>(A, B, g, 1, st);
    case kHiddenTrain: return launch_epi<kHiddenTrain>(A, B, g, 1, st);
    case kHeadTrain: return launch_epi<kHeadTrain>(A, B, g, 1, st);
    case kBackprop: return launch_epi<kBackprop>(A, B, g, 1, st);
    default: return -4;
    }
}

bool fused_shape(uint32_t K0, uint32_t H) { return H == 256u && (K0 == 64u || K0 == 128u); }

int forward_fused(const void* W1, const void* W2, const void* W3, const FusedArgs& f, cudaStream_t st)
{
    if (f.M == 0 || f.M % 128u || !fused_shape(f.K0, 256u) || f.P % 8u || f.P + 16u > f.K0 || !f.record_rows ||
        f.record_rows % 128u)
        return -3;
    return f.K0 == 64u ? launch_fused<1>(W1, W2, W3, f, st) : launch_fused<2>(W1, W2, W3, f, st);
}

} // namespace icp::mlp
