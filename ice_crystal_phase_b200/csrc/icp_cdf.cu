// icp_cdf.cu -- stored-CDF builder for the (u,phi) histogram, one cooperative launch (sm_100a).
//
// Replaces the reference's eight host-synchronised stages (check density, reduce, measure,
// coarsen, make weights / transpose, per-phi serial scan, 1-thread marginal, normalise,
// audit, measure CDF: device/phase_cdf.cu:93-339 driven by src/phase_cdf.cpp:275-472) and
// restates the CPU builder's arithmetic (hex_phase/src/phase_table.cpp:111-187).
//
// Each block owns a strip of CW stored phi columns and keeps it in shared memory for the whole
// build: the coarse masses (array A) and the column prefixes (array B).
//   phase A  without coarsening the fine strip arrives by 3-D TMA boxes (cp.async.bulk.tensor,
//            one mbarrier per box; the rows of a box are processed as soon as it lands), else
//            each thread aggregates its coarse cells from global memory (Kahan, row-major fine
//            order).  Pole caps, per-row additions and the density conversion are applied in
//            the same pass, which also publishes the fine / coarse moments and the maximum.
//   barrier 1 (largest coarse mass, stored total)
//   phase B  weights w = coarse / largest for the strip (all threads; the audit's p = coarse /
//            stored total in the same pass), then one thread per column runs the reference's
//            ordered ascending-theta binary64 scan (s += w) over shared memory and publishes its
//            column sum.
//   barrier 2 (all column sums)
//   phase C  warp 0 runs the ordered marginal scan (phi[j+1] = phi[j] + colsum[j]) while the
//            other warps normalise this strip's conditionals and write T (its rows are one
//            contiguous range of the phi-major output, so the stores are coalesced); then every
//            thread audits its cells (L1, lost mass, malformed, stored moments) from shared
//            memory, and the last block to finish reduces the audits in a fixed order and
//            resets the barrier counters for the next launch.
// Grid barriers are counter spins with an iteration limit: on expiry the kernel records
// ICP_ERR_TIMEOUT and returns without writing further output; the host then clears the
// counters.  Where the two strip arrays do not fit in shared memory, phase C re-reads the coarse
// masses from global memory instead of keeping them (`keep` = 0).
#include <algorithm>
#include <cfloat>
#include <cstdint>
#include <cuda.h>
#include <cuda_runtime.h>

#include "icp_internal.h"
#include "icp_umma.cuh"

namespace icp {

namespace {

struct KSum {
    double v, c;
    __device__ __forceinline__ void add(double x)
    {
        const double y = x - c, t = v + y;
        c = (t - v) - y;
        v = t;
    }
};

// Per-block partial results; doubles first (index constants below), then the counters.
enum : uint32_t {
    kFineMass, kFineAxial, kStoredMass, kStoredAxial, kLargest, kTv, kL1, kLost, kMaxErr, kRecovered, kAxial,
    kInvalid, kLostCells, kMalformed, kUnderflow, kPartialWords
};
constexpr uint32_t kPartialDoubles = kInvalid;
struct BlockPartial {
    unsigned long long w[kPartialWords]; // doubles stored by their bits
};
static_assert(sizeof(BlockPartial) == kCdfPartialBytes, "partial slot size");

struct CdfParams {
    const CdfBatchRecord* recs; // batched: block b builds strip b % strips of record b / strips
    uint32_t strips;           // strips per record (0: one record, strips = gridDim.x)
    const double* values;
    const double* edges; // fine edges, nt+1
    double* phi;
    double* theta;
    double* colsum;        // cp
    BlockPartial* partial; // one per strip
    CdfDeviceReport* report;
    unsigned* sync; // [0] barrier arrivals, [1] finished-block ticket; zero at launch, zero again at exit
    uint32_t kind, nt, np, ct, cp, dt, dp, cw;
    uint32_t keep, tma, box_rows, boxes, rows_alloc, z0, spin_limit, pad;
    double fwd_add, bwd_add;
    const double* row_add;
    const unsigned long long* pole_fx;
    double pole_weight;
};

// Additions to the fine histogram: pole caps on the end rows, an optional per-row term.
struct CdfAdds {
    double fwd, bwd;
    const double* row;
};

// Pole caps from fixed-point pole sums: the host's arithmetic (stats_accumulate, then
// weight x pole power, then / np) evaluated on the device.
__device__ __forceinline__ CdfAdds cdf_adds(const CdfParams& P, unsigned long long* bad)
{
    CdfAdds a{P.fwd_add, P.bwd_add, P.row_add};
    if (P.pole_fx) {
        const double f = (ldexp((double)P.pole_fx[1], 64) + (double)P.pole_fx[0]) * 0x1p-44;
        const double b = (ldexp((double)P.pole_fx[3], 64) + (double)P.pole_fx[2]) * 0x1p-44;
        const double fm = P.pole_weight * f, bm = P.pole_weight * b;
        a.fwd = fm / P.np;
        a.bwd = bm / P.np;
        if ((fm > 0 && !(a.fwd > 0)) || (bm > 0 && !(a.bwd > 0))) ++*bad;
    }
    return a;
}

constexpr unsigned kThreads = 512;
constexpr unsigned kWarps = kThreads / 32;
constexpr unsigned kMaxBoxes = 16;
constexpr unsigned kSpinLimit = 1u << 22;
constexpr unsigned kFull = 0xffffffffu;

// Ordered binary64 chains.  The sums must be the reference's sequential ones, so each addition
// waits for the previous; the loads of the next eight operands are issued before the current
// eight are added (plain registers, no arrays), so the chain runs at the latency of the
// additions alone.  x[k * stride], k < n.
__device__ __forceinline__ double chain_sum(const double* __restrict__ x, uint32_t n, uint32_t stride, double a)
{
    uint32_t i = 0;
    if (n >= 8) {
        double c0 = x[0], c1 = x[stride], c2 = x[2 * stride], c3 = x[3 * stride], c4 = x[4 * stride],
               c5 = x[5 * stride], c6 = x[6 * stride], c7 = x[7 * stride];
        for (i = 8; i + 8 <= n; i += 8) {
            const double* y = x + (size_t)i * stride;
            const double d0 = y[0], d1 = y[stride], d2 = y[2 * stride], d3 = y[3 * stride], d4 = y[4 * stride],
                         d5 = y[5 * stride], d6 = y[6 * stride], d7 = y[7 * stride];
            a += c0; a += c1; a += c2; a += c3; a += c4; a += c5; a += c6; a += c7;
            c0 = d0; c1 = d1; c2 = d2; c3 = d3; c4 = d4; c5 = d5; c6 = d6; c7 = d7;
        }
        a += c0; a += c1; a += c2; a += c3; a += c4; a += c5; a += c6; a += c7;
    }
    for (; i < n; ++i) a += x[(size_t)i * stride];
    return a;
}
// The same chain from zero, each prefix written over its operand: x[k] = x[0] + ... + x[k].  The
// eight prefixes of a group are stored after the group's additions, so no store sits between
// two dependent additions.
__device__ __forceinline__ double chain_prefix(double* x, uint32_t n, uint32_t stride)
{
    double a = 0.0;
    uint32_t i = 0;
    if (n >= 8) {
        double c0 = x[0], c1 = x[stride], c2 = x[2 * stride], c3 = x[3 * stride], c4 = x[4 * stride],
               c5 = x[5 * stride], c6 = x[6 * stride], c7 = x[7 * stride];
        for (i = 8; i + 8 <= n; i += 8) {
            double* y = x + (size_t)i * stride;
            const double d0 = y[0], d1 = y[stride], d2 = y[2 * stride], d3 = y[3 * stride], d4 = y[4 * stride],
                         d5 = y[5 * stride], d6 = y[6 * stride], d7 = y[7 * stride];
            const double p0 = a + c0, p1 = p0 + c1, p2 = p1 + c2, p3 = p2 + c3, p4 = p3 + c4, p5 = p4 + c5,
                         p6 = p5 + c6, p7 = p6 + c7;
            double* z = y - (size_t)8 * stride;
            z[0] = p0; z[stride] = p1; z[2 * stride] = p2; z[3 * stride] = p3;
            z[4 * stride] = p4; z[5 * stride] = p5; z[6 * stride] = p6; z[7 * stride] = p7;
            a = p7;
            c0 = d0; c1 = d1; c2 = d2; c3 = d3; c4 = d4; c5 = d5; c6 = d6; c7 = d7;
        }
        const double p0 = a + c0, p1 = p0 + c1, p2 = p1 + c2, p3 = p2 + c3, p4 = p3 + c4, p5 = p4 + c5,
                     p6 = p5 + c6, p7 = p6 + c7;
        double* z = x + (size_t)(i - 8) * stride;
        z[0] = p0; z[stride] = p1; z[2 * stride] = p2; z[3 * stride] = p3;
        z[4 * stride] = p4; z[5 * stride] = p5; z[6 * stride] = p6; z[7 * stride] = p7;
        a = p7;
    }
    for (; i < n; ++i) {
        a += x[(size_t)i * stride];
        x[(size_t)i * stride] = a;
    }
    return a;
}

// Shared-memory layout of one block (the same function sizes the launch on the host).
struct Layout {
    size_t a, b, e, s, phi, bar, total;
};
__host__ __device__ inline size_t take(size_t& off, size_t bytes)
{
    const size_t o = off;
    off = (off + bytes + 127) / 128 * 128;
    return o;
}
__host__ __device__ inline Layout layout_of(uint32_t ct, uint32_t cp, uint32_t cw, uint32_t rows_alloc, uint32_t keep)
{
    Layout L{};
    size_t off = 0;
    L.a = take(off, sizeof(double) * (size_t)rows_alloc * cw);
    // with `keep`, B is column-major with an odd column stride (the chains read a column
    // contiguously, the parallel passes hit distinct banks); otherwise it aliases A, row-major
    L.b = keep ? take(off, sizeof(double) * (size_t)(ct | 1u) * cw) : L.a;
    L.e = take(off, sizeof(double) * (ct + 1));
    L.s = take(off, sizeof(double) * cp);
    L.phi = take(off, sizeof(double) * (cw + 1));
    L.bar = take(off, sizeof(uint64_t) * kMaxBoxes);
    L.total = off;
    return L;
}

__device__ __forceinline__ unsigned ld_acquire(const unsigned* p)
{
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// Grid barrier in two halves, so that independent work can run between arrival and wait.
__device__ __forceinline__ void grid_arrive(unsigned* counter)
{
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        atomicAdd(counter, 1u);
    }
}
__device__ __forceinline__ bool grid_wait(unsigned* counter, unsigned target, unsigned limit, unsigned* timeout_flag)
{
    __shared__ int ok;
    if (threadIdx.x == 0) {
        unsigned spins = 0;
        while (ld_acquire(counter) < target && spins < limit) {
            __nanosleep(32);
            ++spins;
        }
        ok = spins < limit;
        if (!ok) atomicExch(timeout_flag, 1u);
        __threadfence();
    }
    __syncthreads();
    return ok;
}

__device__ __forceinline__ double adjust_fine(const CdfParams& P, const CdfAdds& A, double m, uint32_t i, double du)
{
    if (P.kind == 1) m = m * du;
    if (A.row) m += A.row[i];
    if (i == 0) m += A.fwd;
    if (i + 1 == P.nt) m += A.bwd;
    return m;
}

__device__ __forceinline__ double fine_mass_at(const CdfParams& P, const CdfAdds& A, uint32_t i, uint32_t j)
{
    return adjust_fine(P, A, P.values[(size_t)i * P.np + j], i, P.kind == 1 ? P.edges[i + 1] - P.edges[i] : 0.0);
}

// Conservative aggregate of one coarse cell: Kahan sum in row-major fine order
// (hex_phase/src/phase_table.cpp:122-123).
__device__ __forceinline__ double coarse_at(const CdfParams& P, const CdfAdds& A, uint32_t ci, uint32_t cj)
{
    KSum acc{0, 0};
    for (uint32_t i = ci * P.dt; i < (ci + 1) * P.dt; ++i)
        for (uint32_t j = cj * P.dp; j < (cj + 1) * P.dp; ++j) acc.add(fine_mass_at(P, A, i, j));
    return acc.v;
}

// Block sum (thread 0's result; warps added in order).
template <class T> __device__ T block_sum(T x, T* red)
{
    for (int o = 16; o; o >>= 1) x += __shfl_xor_sync(kFull, x, o);
    __syncthreads();
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = x;
    __syncthreads();
    T s = T(0);
    if (threadIdx.x == 0)
        for (unsigned w = 0; w < kWarps; ++w) s += red[w];
    return s;
}
__device__ double block_max(double x, double* red)
{
    for (int o = 16; o; o >>= 1) x = fmax(x, __shfl_xor_sync(kFull, x, o));
    __syncthreads();
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = x;
    __syncthreads();
    double s = 0.0;
    if (threadIdx.x == 0)
        for (unsigned w = 0; w < kWarps; ++w) s = fmax(s, red[w]);
    return s;
}

// One partial word over all strips, reduced by one warp in a fixed order (lane l adds strips
// l, l + 32, ... in order, then a shuffle tree); the result is lane 0's, broadcast, so every
// block that runs this on the same partials obtains the same bits.
__device__ __forceinline__ double warp_reduce_word(const BlockPartial* part, uint32_t strips, uint32_t word, bool is_max)
{
    const uint32_t lane = threadIdx.x & 31;
    double v = 0.0;
    for (uint32_t k = lane; k < strips; k += 32) {
        const double x = __longlong_as_double((long long)__ldcg(&part[k].w[word]));
        v = is_max ? fmax(v, x) : v + x;
    }
    for (int o = 16; o; o >>= 1) {
        const double y = __shfl_down_sync(kFull, v, o);
        v = is_max ? fmax(v, y) : v + y;
    }
    return __shfl_sync(kFull, v, 0);
}
__device__ __forceinline__ unsigned long long warp_reduce_count(const BlockPartial* part, uint32_t strips, uint32_t word)
{
    const uint32_t lane = threadIdx.x & 31;
    unsigned long long v = 0;
    for (uint32_t k = lane; k < strips; k += 32) v += __ldcg(&part[k].w[word]);
    for (int o = 16; o; o >>= 1) v += __shfl_down_sync(kFull, v, o);
    return __shfl_sync(kFull, v, 0);
}

__device__ __forceinline__ void put(BlockPartial& p, uint32_t word, double x)
{
    p.w[word] = (unsigned long long)__double_as_longlong(x);
}

__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, uint64_t* bar, int32_t x, int32_t y,
                                            int32_t z)
{
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];" ::
            "r"(umma::smem_u32(dst)),
        "l"(map), "r"(x), "r"(y), "r"(z), "r"(umma::smem_u32(bar))
        : "memory");
}

// The ordered chains (column prefixes in phase B, the marginal scan in phase C) are dependent
// FP64 additions on warps 0 .. chain_warps - 1; warps on the same SM sub-partition (warp mod 4)
// that run FP64 divisions meanwhile slow each addition.  The side work of those phases therefore
// goes to the warps of the other sub-partitions (all non-chain warps when the chains occupy all
// four), numbered densely: this thread's index and the number of side threads.
__device__ __forceinline__ bool side_worker(uint32_t warp, uint32_t lane, uint32_t chain_warps, uint32_t& idx,
                                            uint32_t& count)
{
    const uint32_t busy = chain_warps < 4u ? chain_warps : 0u; // sub-partitions 0 .. busy - 1 hold a chain
    uint32_t before = 0, total = 0;
    for (uint32_t u = chain_warps; u < kWarps; ++u)
        if ((u & 3u) >= busy) {
            before += u < warp ? 1u : 0u;
            ++total;
        }
    idx = before * 32u + lane;
    count = total * 32u;
    return warp >= chain_warps && (warp & 3u) >= busy;
}

__global__ void __launch_bounds__(kThreads, 1) cdf_build_kernel(const __grid_constant__ CUtensorMap map,
                                                                 const CdfParams P0)
{
    extern __shared__ unsigned char smem_raw[];
    // TMA box images start 128-byte aligned: align the base (the launch adds 128 bytes of slack)
    unsigned char* smem = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 127) & ~uintptr_t(127));
    __shared__ double red_d[kWarps];
    __shared__ unsigned long long red_u[kWarps];
    __shared__ double s_tot[4]; // fine total, stored total, largest, marginal total
    __shared__ unsigned long long s_fin[kPartialWords];
    __shared__ int s_last;

    const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint32_t strips = P0.strips ? P0.strips : gridDim.x;
    const uint32_t rec = P0.strips ? blockIdx.x / strips : 0u;
    const uint32_t sb = P0.strips ? blockIdx.x % strips : blockIdx.x; // this block's strip of its record
    CdfParams P = P0;
    if (P0.recs) {
        const CdfBatchRecord& R = P0.recs[rec];
        P.values = R.values;
        P.phi = R.phi;
        P.theta = R.theta;
        P.colsum = R.colsum;
        P.partial = reinterpret_cast<BlockPartial*>(R.partial);
        P.report = R.report;
        P.sync = R.sync;
        P.row_add = R.row_add;
        P.pole_fx = R.pole_fx;
        P.pole_weight = R.pole_weight;
        P.fwd_add = R.fwd_add;
        P.bwd_add = R.bwd_add;
    }
    const uint32_t limit = P.spin_limit ? P.spin_limit : kSpinLimit;
    const uint32_t CW = P.cw, ct = P.ct;
    const uint32_t c0 = sb * CW;
    const uint32_t c1 = min(P.cp, c0 + CW);
    const uint32_t w = c1 > c0 ? c1 - c0 : 0u; // columns in this strip
    const Layout Lo = layout_of(ct, P.cp, CW, P.rows_alloc, P.keep);
    double* A = reinterpret_cast<double*>(smem + Lo.a); // coarse masses, then p = coarse / stored total
    double* B = reinterpret_cast<double*>(smem + Lo.b); // weights, prefixes, normalised conditionals
    // element (row i, column cl) of B at i * b_row + cl * b_col
    const uint32_t b_row = P.keep ? 1u : CW, b_col = P.keep ? (ct | 1u) : 1u;
    double* E = reinterpret_cast<double*>(smem + Lo.e); // coarse u edges
    double* S = reinterpret_cast<double*>(smem + Lo.s); // all column sums
    double* sphi = reinterpret_cast<double*>(smem + Lo.phi);
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem + Lo.bar);
    // per-cell passes: thread -> (column my_cl, rows my_r, my_r + rstep, ...)
    const uint32_t rstep = kThreads / CW;
    const uint32_t my_cl = tid % CW, my_r = tid / CW;
    const bool act = my_r < rstep && my_cl < w;

    // ------------------------------------------------------------ phase A
    if (P.tma) {
        if (tid == 0) {
            for (uint32_t k = 0; k < P.boxes; ++k) umma::mbar_init(&bars[k], 1);
            umma::mbar_fence_init();
        }
        __syncthreads();
        if (tid == 0) {
            const uint32_t box_bytes = P.box_rows * CW * (uint32_t)sizeof(double);
            for (uint32_t k = 0; k < P.boxes; ++k) {
                umma::mbar_arrive_expect_tx(&bars[k], box_bytes);
                tma_load_3d(A + (size_t)k * P.box_rows * CW, &map, &bars[k], (int32_t)c0, (int32_t)(k * P.box_rows),
                            (int32_t)(P.z0 + rec));
            }
        }
    }
    for (uint32_t i = tid; i <= ct; i += kThreads) E[i] = P.edges[(size_t)i * P.dt];
    __syncthreads();

    KSum fm{0, 0}, fa{0, 0}, sm{0, 0}, sa{0, 0};
    double largest = 0.0;
    unsigned long long invalid = 0ull, pole_bad = 0ull;
    const CdfAdds adds = cdf_adds(P, &pole_bad);
    if (tid == 0) invalid += pole_bad;
    if (P.tma) {
        // dt = dp = 1: coarse = fine; the stored moments equal the fine ones.  The box waits
        // keep the default limit, so that no copy is still landing when the block leaves.
        bool late = false;
        for (uint32_t k = 0; k < P.boxes; ++k) {
            if (!umma::mbar_wait(&bars[k], 0, kSpinLimit)) late = true;
            const uint32_t r1 = min(ct, (k + 1) * P.box_rows);
            if (act)
                for (uint32_t i = k * P.box_rows + my_r; i < r1; i += rstep) {
                    const double e0 = E[i], e1 = E[i + 1];
                    const double m = adjust_fine(P, adds, A[(size_t)i * CW + my_cl], i, e1 - e0);
                    if (!(m >= 0.0) || !(m <= DBL_MAX)) ++invalid;
                    A[(size_t)i * CW + my_cl] = m;
                    fm.add(m);
                    fa.add(m * (1.0 - e0 - e1));
                    largest = fmax(largest, m);
                }
        }
        if (late) atomicExch(&P.report->timeout, 1u);
    } else if (act) {
        for (uint32_t ci = my_r; ci < ct; ci += rstep) {
            const uint32_t cj = c0 + my_cl;
            KSum acc{0, 0};
            for (uint32_t i = ci * P.dt; i < (ci + 1) * P.dt; ++i) {
                const double mu = 1.0 - P.edges[i] - P.edges[i + 1];
                for (uint32_t j = cj * P.dp; j < (cj + 1) * P.dp; ++j) {
                    const double m = fine_mass_at(P, adds, i, j);
                    if (!(m >= 0.0) || !(m <= DBL_MAX)) ++invalid;
                    acc.add(m);
                    fm.add(m);
                    fa.add(m * mu);
                }
            }
            const double c = acc.v;
            A[(size_t)ci * CW + my_cl] = c;
            sm.add(c);
            sa.add(c * (1.0 - E[ci] - E[ci + 1]));
            largest = fmax(largest, c);
        }
    }
    {
        const double a = block_sum(fm.v + fm.c, red_d);
        const double b = block_sum(fa.v + fa.c, red_d);
        const double c = P.tma ? a : block_sum(sm.v + sm.c, red_d);
        const double d = P.tma ? b : block_sum(sa.v + sa.c, red_d);
        const double e = block_max(largest, red_d);
        const unsigned long long f = block_sum(invalid, red_u);
        if (tid == 0) {
            BlockPartial& bp = P.partial[sb];
            put(bp, kFineMass, a);
            put(bp, kFineAxial, b);
            put(bp, kStoredMass, c);
            put(bp, kStoredAxial, d);
            put(bp, kLargest, e);
            bp.w[kInvalid] = f;
        }
    }
    grid_arrive(&P.sync[0]);
    if (!grid_wait(&P.sync[0], strips, limit, &P.report->timeout)) return;

    // ------------------------------------------------------------ phase B
    if (warp < 3) {
        const double v = warp_reduce_word(P.partial, strips, warp == 0 ? kFineMass : warp == 1 ? kStoredMass : kLargest,
                                          warp == 2);
        if (lane == 0) s_tot[warp] = v;
    }
    __syncthreads();
    const double fine_total = s_tot[0], stored_total = s_tot[1], big = s_tot[2];
    KSum tv{0, 0};
    if (P.dt > 1 || P.dp > 1) {
        const uint32_t fw = w * P.dp;
        for (uint32_t q = tid; q < P.nt * fw; q += kThreads) {
            const uint32_t i = q / fw, j = c0 * P.dp + q % fw;
            const uint32_t ci = i / P.dt, cl = j / P.dp - c0;
            const double fraction = (P.edges[i + 1] - P.edges[i]) / (E[ci + 1] - E[ci]) / P.dp;
            tv.add(fabs(fine_mass_at(P, adds, i, j) / fine_total - A[(size_t)ci * CW + cl] / stored_total * fraction));
        }
        __syncthreads();
    }
    // weights w = coarse / largest for the whole strip in parallel (the ordered chains below then
    // carry only additions)
    unsigned long long underflow = 0ull, malformed = 0ull;
    if (act)
        for (uint32_t i = my_r; i < ct; i += rstep) {
            const double c = A[(size_t)i * CW + my_cl];
            const double x = c / big;
            if (c > 0 && !(x > 0)) ++underflow;
            B[(size_t)i * b_row + (size_t)my_cl * b_col] = x;
        }
    __syncthreads();
    // the warps that hold a column chain (threads tid < w) sit out the audit pass below, and so
    // do the warps that share their sub-partitions
    uint32_t side_b = 0, sides_b = 0;
    const bool side_in_b = side_worker(warp, lane, (w + 31u) >> 5, side_b, sides_b);
    if (tid < w) {
        // ordered ascending-theta scan of one phi column; the unnormalised prefix of row i+1
        // replaces the weight of row i in place (each column belongs to one thread)
        P.colsum[c0 + tid] = chain_prefix(B + (size_t)tid * b_col, ct, b_row);
    } else if (P.keep && side_in_b) {
        // meanwhile the other warps form the audit's p = coarse / stored total in A
        for (uint32_t k = side_b; k < ct * w; k += sides_b) {
            const size_t a = (size_t)(k / w) * CW + k % w;
            const double c = A[a];
            const double pv = c / stored_total;
            if (c > 0 && !(pv > 0)) ++malformed;
            A[a] = pv;
        }
    }
    {
        const double t = block_sum(tv.v + tv.c, red_d);
        const unsigned long long u = block_sum(underflow, red_u);
        if (tid == 0) {
            put(P.partial[sb], kTv, 0.5 * t);
            P.partial[sb].w[kUnderflow] = u;
        }
    }
    grid_arrive(&P.sync[0]);
    if (!grid_wait(&P.sync[0], 2u * strips, limit, &P.report->timeout)) return;

    // ------------------------------------------------------------ phase C
    for (uint32_t j = tid; j < P.cp; j += kThreads) S[j] = __ldcg(P.colsum + j);
    __syncthreads();
    const uint32_t stride = ct + 1;
    uint32_t side_c = 0, sides_c = 0;
    const bool side_in_c = side_worker(warp, lane, 1u, side_c, sides_c);
    if (tid == 0) {
        // ordered marginal scan (phase_table.cpp:154): phi[j+1] = phi[j] + colsum[j]; this
        // strip keeps the running values at its own columns
        const uint32_t j0 = min(c0, P.cp), j1 = min(c1, P.cp);
        double a = chain_sum(S, j0, 1u, 0.0);
        sphi[0] = a;
        for (uint32_t j = j0; j < j1; ++j) {
            a += S[j];
            sphi[j - j0 + 1] = a;
        }
        s_tot[3] = chain_sum(S + j1, P.cp - j1, 1u, a);
    } else if (side_in_c) {
        // meanwhile the normalised conditionals of this strip, written once each: its output
        // rows are the contiguous range theta[c0*(ct+1) .. c1*(ct+1)); element (cl, i) comes from
        // the prefix of row i kept at B(i-1, cl), which keeps the normalised value for the audit
        const uint32_t span = w * stride, step = sides_c;
        uint32_t q = side_c, cl = q / stride, i = q % stride;
        double* out = P.theta + (size_t)c0 * stride;
        for (; q < span; q += step) {
            const double cs = S[c0 + cl];
            double v;
            if (i == 0) v = 0.0;
            else if (i == ct) v = 1.0;
            else v = cs > 0 ? B[(size_t)(i - 1) * b_row + (size_t)cl * b_col] / cs : E[i];
            out[q] = v;
            if (i > 0) B[(size_t)(i - 1) * b_row + (size_t)cl * b_col] = v;
            i += step;
            while (i >= stride) {
                i -= stride;
                ++cl;
            }
        }
    }
    __syncthreads();
    const double total = s_tot[3];
    // normalised marginal for this strip: phi[0] = 0, phi[cp] = 1, interior / total; the boundary
    // value j = c0 > 0 belongs to the previous strip's output
    for (uint32_t cl = tid; cl <= w; cl += kThreads) {
        const uint32_t j = c0 + cl;
        const double v = j == 0 ? 0.0 : (j == P.cp ? 1.0 : sphi[cl] / total);
        sphi[cl] = v;
        if (cl > 0 || c0 == 0) P.phi[j] = v;
    }
    __syncthreads();
    KSum l1{0, 0}, lost{0, 0}, recv{0, 0}, ax{0, 0};
    double max_err = 0.0;
    unsigned long long lost_cells = 0ull;
    if (act) {
        const double a0 = sphi[my_cl], a1 = sphi[my_cl + 1];
        for (uint32_t i = my_r; i < ct; i += rstep) {
            const double b0 = i == 0 ? 0.0 : B[(size_t)(i - 1) * b_row + (size_t)my_cl * b_col];
            const double b1 = B[(size_t)i * b_row + (size_t)my_cl * b_col]; // row ct - 1 holds 1
            const double qv = (a1 - a0) * (b1 - b0);
            double p;
            if (P.keep) {
                p = A[(size_t)i * CW + my_cl];
            } else {
                const double c = coarse_at(P, adds, i, c0 + my_cl);
                p = c / stored_total;
                if (c > 0 && !(p > 0)) ++malformed;
            }
            const bool bad = !(qv >= 0.0) || !(qv <= DBL_MAX) || a1 < a0 || b1 < b0;
            if (bad) ++malformed;
            const double err = fabs(p - qv);
            l1.add(err);
            max_err = fmax(max_err, err);
            if (p > 0 && qv == 0) {
                lost.add(p);
                ++lost_cells;
            }
            recv.add(qv);
            ax.add(qv * (1.0 - E[i] - E[i + 1]));
        }
    }
    {
        const double a = block_sum(l1.v + l1.c, red_d);
        const double b = block_sum(lost.v + lost.c, red_d);
        const double c = block_sum(recv.v + recv.c, red_d);
        const double d = block_sum(ax.v + ax.c, red_d);
        const double e = block_max(max_err, red_d);
        const unsigned long long f = block_sum(lost_cells, red_u);
        const unsigned long long g = block_sum(malformed, red_u);
        if (tid == 0) {
            BlockPartial& bp = P.partial[sb];
            put(bp, kL1, a);
            put(bp, kLost, b);
            put(bp, kRecovered, c);
            put(bp, kAxial, d);
            put(bp, kMaxErr, e);
            bp.w[kLostCells] = f;
            bp.w[kMalformed] = g;
            __threadfence();
            s_last = (atomicAdd(&P.sync[1], 1u) == strips - 1);
        }
    }
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    // last block: warp f reduces partial word f over all strips in a fixed order
    if (warp < kPartialWords) {
        if (warp < kPartialDoubles) {
            const double v = warp_reduce_word(P.partial, strips, warp, warp == kLargest || warp == kMaxErr);
            if (lane == 0) s_fin[warp] = (unsigned long long)__double_as_longlong(v);
        } else {
            const unsigned long long v = warp_reduce_count(P.partial, strips, warp);
            if (lane == 0) s_fin[warp] = v;
        }
    }
    __syncthreads();
    if (tid != 0) return;
    auto d = [&](uint32_t k) { return __longlong_as_double((long long)s_fin[k]); };
    CdfDeviceReport r{};
    r.fine_mass = d(kFineMass);
    r.fine_axial = d(kFineAxial);
    r.stored_mass = d(kStoredMass);
    r.stored_axial = d(kStoredAxial);
    r.tv = d(kTv);
    r.l1 = d(kL1);
    r.lost = d(kLost);
    r.recovered = d(kRecovered);
    r.axial = d(kAxial);
    r.max_err = d(kMaxErr);
    r.largest = d(kLargest);
    r.total = total;
    r.invalid = s_fin[kInvalid];
    r.lost_cells = s_fin[kLostCells];
    r.malformed = s_fin[kMalformed];
    r.underflow = s_fin[kUnderflow];
    r.timeout = *((volatile unsigned*)&P.report->timeout);
    *P.report = r;
    // every block has passed both barriers and taken its ticket: the counters start the next launch at zero
    P.sync[0] = 0u;
    P.sync[1] = 0u;
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

// FP64 histograms [records][nt][np], boxes of cw columns x box_rows rows x 1 record.
int make_values_map(CUtensorMap* map, const double* values, uint32_t nt, uint32_t np, uint32_t records, uint32_t cw,
                    uint32_t box_rows)
{
    const EncodeTiled encode = encode_tiled();
    if (!encode) return (int)cudaErrorNotSupported;
    const cuuint64_t dims[3] = {np, nt, records};
    const cuuint64_t strides[2] = {(cuuint64_t)np * 8u, (cuuint64_t)np * nt * 8u};
    const cuuint32_t box[3] = {cw, box_rows, 1u};
    const cuuint32_t elem[3] = {1u, 1u, 1u};
    const CUresult r = encode(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, const_cast<double*>(values), dims, strides, box,
                              elem, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                              CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? 0 : (int)cudaErrorInvalidValue;
}

CdfParams params_of(const CdfLaunch& L, const CdfShape& s)
{
    CdfParams P{};
    P.values = L.values;
    P.edges = L.edges;
    P.phi = L.phi;
    P.theta = L.theta;
    P.colsum = L.colsum;
    P.partial = reinterpret_cast<BlockPartial*>(L.partial);
    P.report = L.report;
    P.sync = L.sync;
    P.kind = L.kind;
    P.nt = L.nt;
    P.np = L.np;
    P.ct = L.ct;
    P.cp = L.cp;
    P.dt = L.nt / L.ct;
    P.dp = L.np / L.cp;
    P.cw = s.cw;
    P.keep = s.keep;
    P.tma = s.tma;
    P.box_rows = s.box_rows;
    P.boxes = s.boxes;
    P.rows_alloc = s.rows_alloc;
    P.spin_limit = L.spin_limit;
    P.fwd_add = L.fwd_add;
    P.bwd_add = L.bwd_add;
    P.row_add = L.row_add;
    P.pole_fx = L.pole_fx;
    P.pole_weight = L.pole_weight;
    return P;
}

int launch(const CdfParams& P, const CUtensorMap& map, uint32_t blocks, size_t smem, cudaStream_t stream)
{
    cudaError_t e = cudaFuncSetAttribute(cdf_build_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return (int)e;
    void* args[] = {const_cast<CUtensorMap*>(&map), const_cast<CdfParams*>(&P)};
    e = cudaLaunchCooperativeKernel((const void*)cdf_build_kernel, dim3(blocks), dim3(kThreads), args, smem, stream);
    return (int)e;
}

// Rows per TMA box (at most the strip's rows): a box's shared-memory image must start 128-byte
// aligned and at most kMaxBoxes boxes cover the strip; the fewest padded rows win (then the
// larger box).
bool box_rows_for(uint32_t ct, uint32_t cw, uint32_t& box_rows, uint32_t& boxes)
{
    uint32_t best = 0, best_rows = 0xffffffffu;
    for (uint32_t r = std::min(256u, ct); r >= 1; --r) {
        if ((r * cw * 8u) % 128u) continue;
        const uint32_t n = (ct + r - 1) / r;
        if (n > kMaxBoxes) continue;
        if (n * r < best_rows) {
            best_rows = n * r;
            best = r;
        }
    }
    if (!best) return false;
    box_rows = best;
    boxes = (ct + best - 1) / best;
    return true;
}

} // namespace

int cdf_max_coresident_blocks(size_t smem, int device)
{
    int per_sm = 0, sms = 0;
    if (cudaFuncSetAttribute(cdf_build_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, cdf_build_kernel, kThreads, smem) != cudaSuccess) return 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) return 0;
    return per_sm * sms;
}

size_t cdf_partial_bytes() { return sizeof(BlockPartial); }

size_t cdf_smem_bytes(const CdfShape& s, uint32_t ct, uint32_t cp)
{
    return layout_of(ct, cp, s.cw, s.rows_alloc, s.keep).total + 128; // + alignment slack of the base
}

int cdf_choose_shape(int device, int sms, uint32_t nt, uint32_t np, uint32_t ct, uint32_t cp, bool tma_ok,
                     uint32_t min_width, uint32_t max_blocks, CdfShape& out)
{
    int max_smem = 0;
    if (cudaDeviceGetAttribute(&max_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, device) != cudaSuccess) return -1;
    // static shared memory of the kernel (reductions, totals) comes on top of the dynamic part
    const size_t budget = (size_t)max_smem > 2048 ? (size_t)max_smem - 2048 : 0;
    const bool fine = nt == ct && np == cp;
    const uint32_t modes[3][2] = {{1u, 1u}, {1u, 0u}, {0u, 0u}}; // (keep, tma)
    for (const auto& m : modes) {
        const uint32_t keep = m[0], tma = m[1];
        if (tma && !(tma_ok && fine)) continue;
        uint32_t w = std::max<uint32_t>(min_width, (cp + (uint32_t)sms - 1) / (uint32_t)sms);
        for (; w <= cp && w <= kThreads - 32u; ++w) { // at least one warp besides the column chains
            CdfShape s{};
            s.cw = w;
            s.keep = keep;
            s.tma = tma;
            s.rows_alloc = ct;
            if (tma) {
                if (w % 2 || w > 256 || !box_rows_for(ct, w, s.box_rows, s.boxes)) continue;
                s.rows_alloc = s.box_rows * s.boxes;
            }
            s.smem = cdf_smem_bytes(s, ct, cp);
            if (s.smem > budget) break;
            const uint32_t blocks = (cp + w - 1) / w;
            if (blocks <= max_blocks && (int)blocks <= cdf_max_coresident_blocks(s.smem, device)) {
                out = s;
                return 0;
            }
        }
    }
    return 1;
}

int launch_cdf_build(const CdfLaunch& L, const CdfShape& s, cudaStream_t stream)
{
    const CdfParams P = params_of(L, s);
    CUtensorMap map{};
    if (s.tma)
        if (const int e = make_values_map(&map, L.values, L.nt, L.np, 1u, s.cw, s.box_rows)) return e;
    return launch(P, map, (L.cp + s.cw - 1) / s.cw, s.smem, stream);
}

int launch_cdf_build_batch(const CdfLaunch& L, const CdfShape& s, const CdfBatchRecord* d_recs, uint32_t count,
                           cudaStream_t stream)
{
    CdfParams P = params_of(L, s);
    P.recs = d_recs;
    P.strips = (L.cp + s.cw - 1) / s.cw;
    CUtensorMap map{};
    if (s.tma) return (int)cudaErrorInvalidValue; // batched records are read without TMA
    return launch(P, map, P.strips * count, s.smem, stream);
}

} // namespace icp
