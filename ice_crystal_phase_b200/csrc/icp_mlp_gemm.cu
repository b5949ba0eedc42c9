// icp_mlp_gemm.cu -- BF16 GEMM on the 5th-generation tensor cores (tcgen05, TMEM, TMA) for the
// surrogate's dense layers, with the layer epilogues fused.
//
//   D[M x N] = A[M x K] * B[N x K]^T      A, B: BF16, K-major (row-major with K contiguous)
//
// One CTA of 128 threads computes a 128 x N tile (N in {64, 128, 256}) over a range of K chunks
// of 64: thread 0 streams A and B chunks through a STAGES-deep ring with 2-D TMA loads (128-byte
// swizzle, completion counted on a "full" mbarrier per stage) and issues four K=16
// tcgen05.mma per chunk into an FP32 accumulator in tensor memory; each chunk's MMAs commit to the
// stage's "empty" mbarrier, which gates the refill.  After the last chunk a commit to "done"
// releases the epilogue: warp w reads TMEM lanes 32w..32w+31 (rows) with tcgen05.ld, 32 columns at
// a time, and applies one of the fused epilogues below.  Split-K (grid.y > 1) adds partial tiles
// with FP32 atomics.  Every mbarrier wait is bounded: on expiry the kernel sets the error word,
// waits (bounded) for its issued MMAs, frees its tensor memory and returns.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "icp_internal.h"
#include "icp_mlp.h"
#include "icp_umma.cuh"

namespace icp::mlp {

namespace {

constexpr uint32_t kWaitLimit = 1u << 22;
constexpr uint32_t kA = 128u * 128u; // bytes of one A stage: 128 rows x 64 BF16

template <int N> __host__ __device__ constexpr int stages() { return N <= 128 ? 4 : 3; }
template <int N> __host__ __device__ constexpr uint32_t stage_bytes() { return kA + (uint32_t)N * 128u; }
// 1024 (alignment) + stages + barriers / TMEM slot (256) + column sums of the bias gradient (1024)
template <int N> constexpr size_t smem_bytes() { return 1024 + (size_t)stages<N>() * stage_bytes<N>() + 256 + 1024; }

__device__ __forceinline__ float silu(float z) { return z / (1.0f + __expf(-z)); }
__device__ __forceinline__ float silu_grad(float z)
{
    const float s = 1.0f / (1.0f + __expf(-z));
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

// Column-major copy of a warp's 32 rows x 32 columns: for each column, the 32 lanes write 32
// consecutive rows (64 contiguous bytes).
__device__ __forceinline__ void store_bf16x32_t(__nv_bfloat16* dst, uint32_t ld, const float (&v)[32])
{
#pragma unroll
    for (int i = 0; i < 32; ++i) dst[(size_t)i * ld] = __float2bfloat16_rn(v[i]);
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

template <int N, int EPI>
__global__ void __launch_bounds__(128, 1)
    gemm_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB, const GemmArgs g)
{
    constexpr int S = stages<N>();
    constexpr uint32_t SB = stage_bytes<N>();
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
    if (warp == 0) umma::tmem_alloc(tslot, (uint32_t)N);
    umma::fence_before_sync();
    __syncthreads();
    umma::fence_after_sync();
    const uint32_t tmem = *tslot;
    const uint32_t m0 = blockIdx.x * 128u;
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
            umma::tma_load_2d(a, &tmA, &full[s], (int32_t)((kc0 + kc) * 64u), (int32_t)m0);
            umma::tma_load_2d(a + kA, &tmB, &full[s], (int32_t)((kc0 + kc) * 64u), 0);
        };
        const uint32_t pre = nk < (uint32_t)S ? nk : (uint32_t)S;
        for (uint32_t s = 0; s < pre; ++s) load(s, s);
        for (uint32_t kc = 0; kc < nk && ok; ++kc) {
            const uint32_t s = kc % S, par = (kc / S) & 1u;
            if (!umma::mbar_wait(&full[s], par, kWaitLimit)) {
                ok = false;
                break;
            }
            umma::fence_after_sync();
            const uint32_t a = umma::smem_u32(smem + s * SB), b = a + kA;
#pragma unroll
            for (uint32_t k = 0; k < 4; ++k)
                umma::mma_bf16(tmem, umma::smem_desc_sw128(a + 32u * k), umma::smem_desc_sw128(b + 32u * k), idesc,
                               kc > 0 || k > 0);
            umma::mma_commit(&empty[s]);
            if (kc + S < nk) {
                if (!umma::mbar_wait(&empty[s], par, kWaitLimit)) {
                    ok = false;
                    break;
                }
                load(s, kc + S);
            }
        }
        if (!ok) {
            *abort_flag = 1;
            if (nk) atomicExch(g.error, 1u);
            __threadfence_block();
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
        const uint32_t row = 32u * warp + lane;
        const uint32_t m = m0 + row;
        float yacc = 0.0f;
        for (uint32_t c = 0; c < (uint32_t)N; c += 32u) {
            float v[32];
            umma::tmem_ld32(tmem + ((32u * warp) << 16) + c, v);
            if constexpr (EPI == kStoreF32) {
                float4* d = reinterpret_cast<float4*>(g.out_f32 + (size_t)m * g.ld_out + c);
#pragma unroll
                for (int q = 0; q < 8; ++q) d[q] = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
            } else if constexpr (EPI == kAtomicF32) {
                float* d = g.out_f32 + (size_t)m * g.ld_out + c;
#pragma unroll
                for (int i = 0; i < 32; ++i) atomicAdd(d + i, v[i]);
            } else if constexpr (EPI == kHidden || EPI == kHead) {
#pragma unroll
                for (int i = 0; i < 32; ++i) v[i] += g.bias[c + i];
                if (g.out_z) store_bf16x32(g.out_z + (size_t)m * N + c, v);
#pragma unroll
                for (int i = 0; i < 32; ++i) v[i] = silu(v[i]);
                if (g.out_h) store_bf16x32(g.out_h + (size_t)m * N + c, v);
                if (g.out_hT) store_bf16x32_t(g.out_hT + (size_t)c * g.ld_t + m, g.ld_t, v);
                if constexpr (EPI == kHead) {
#pragma unroll
                    for (int i = 0; i < 32; ++i) yacc = fmaf(v[i], g.head_w[c + i], yacc);
                }
            } else if constexpr (EPI == kBackprop) {
                float z[32];
                load_bf16x32(g.z_prev + (size_t)m * N + c, z);
#pragma unroll
                for (int i = 0; i < 32; ++i) v[i] *= silu_grad(z[i]);
                if (g.out_dz) store_bf16x32(g.out_dz + (size_t)m * N + c, v);
                if (g.out_dzT) store_bf16x32_t(g.out_dzT + (size_t)c * g.ld_t + m, g.ld_t, v);
                if (g.out_db) atomicAdd(&colsum[c + lane], warp_column_sum(v, lane));
            }
        }
        if constexpr (EPI == kHead) {
            const float y = yacc + g.head_b;
            if (g.out_y) g.out_y[m] = y;
            if (g.out_mass) g.out_mass[m] = exp((double)y);
        }
    }
    if constexpr (EPI == kBackprop) {
        __syncthreads();
        if (g.out_db && ready)
            for (uint32_t i = threadIdx.x; i < (uint32_t)N; i += blockDim.x) atomicAdd(&g.out_db[i], colsum[i]);
    }
    umma::fence_before_sync();
    __syncthreads();
    if (warp == 0) umma::tmem_dealloc(tmem, (uint32_t)N);
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

template <int N, int EPI> int launch_n(const void* A, const void* B, const GemmArgs& g, uint32_t splits, cudaStream_t st)
{
    CUtensorMap ta, tb;
    if (make_map(&ta, A, g.M, g.K, 128u) || make_map(&tb, B, (uint32_t)N, g.K, (uint32_t)N)) return -1;
    const size_t smem = smem_bytes<N>();
    cudaError_t e = cudaFuncSetAttribute(gemm_kernel<N, EPI>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return (int)e;
    gemm_kernel<N, EPI><<<dim3(g.M / 128u, splits), 128, smem, st>>>(ta, tb, g);
    return (int)cudaGetLastError();
}

template <int EPI> int launch_epi(const void* A, const void* B, const GemmArgs& g, uint32_t splits, cudaStream_t st)
{
    switch (g.N) {
    case 64: return launch_n<64, EPI>(A, B, g, splits, st);
    case 128: return launch_n<128, EPI>(A, B, g, splits, st);
    case 256: return launch_n<256, EPI>(A, B, g, splits, st);
    default: return -2;
    }
}

} // namespace

int gemm(const void* A, const void* B, GemmArgs g, int epi, uint32_t splits, cudaStream_t st)
{
    if (g.M == 0 || g.M % 128u || g.K == 0 || g.K % 64u || !splits) return -3;
    if (epi != kAtomicF32) splits = 1; // only the atomic epilogue can add partial K ranges
    const uint32_t nk = g.K / 64u;
    g.k_chunks = (nk + splits - 1) / splits;
    splits = (nk + g.k_chunks - 1) / g.k_chunks; // every CTA gets at least one chunk
    switch (epi) {
    case kStoreF32: return launch_epi<kStoreF32>(A, B, g, splits, st);
    case kAtomicF32: return launch_epi<kAtomicF32>(A, B, g, splits, st);
    case kHidden: return launch_epi<kHidden>(A, B, g, 1, st);
    case kHead: return launch_epi<kHead>(A, B, g, 1, st);
    case kBackprop: return launch_epi<kBackprop>(A, B, g, 1, st);
    default: return -4;
    }
}

} // namespace icp::mlp
