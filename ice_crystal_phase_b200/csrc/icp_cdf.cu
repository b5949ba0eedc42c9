// icp_cdf.cu -- stored-CDF builder for the (u,phi) histogram, one cooperative launch (sm_100a).
//
// Replaces the reference's eight host-synchronised stages (check density, reduce, measure,
// coarsen, make weights / transpose, per-phi serial scan, 1-thread marginal, normalise,
// audit, measure CDF: device/phase_cdf.cu:93-339 driven by src/phase_cdf.cpp:275-472) and
// restates the CPU builder's arithmetic (hex_phase/src/phase_table.cpp:111-187):
//   phase A  each block owns a strip of CW coarse phi columns: reads its fine strip once
//            (coalesced), adds the pole caps to the end rows, aggregates conservatively
//            (Kahan, row-major order), keeps the coarse strip in shared memory, and
//            publishes fine / coarse moments and its maximum;
//   barrier
//   phase B  coarsening TV, the weights w = coarse / largest (parallel), then per column an
//            ordered binary64 scan in ascending theta (exact plateaus, monotone prefixes) kept
//            in shared memory, column sums published;
//   barrier
//   phase C  ordered marginal scan over all column sums (every block, identical result),
//            normalisation (empty column -> the stored u edges), the phi marginal, and the
//            L1 / lost-mass / malformed audit and stored moments from the written values;
//   the last block to finish reduces the audits.
// Grid barriers are counter spins with an iteration limit: on expiry the kernel records
// ICP_ERR_TIMEOUT and returns without writing further output.
#include <cooperative_groups.h>
#include <cstdint>
#include <cuda_runtime.h>

#include "icp_internal.h"

namespace icp {

struct KSum {
    double v, c;
    __device__ __forceinline__ void add(double x)
    {
        const double y = x - c, t = v + y;
        c = (t - v) - y;
        v = t;
    }
};

struct BlockPartial {
    double fine_mass, fine_axial, stored_mass, stored_axial, largest;
    double tv, l1, lost, max_err, recovered, axial;
    unsigned long long invalid, lost_cells, malformed, underflow;
};

struct CdfParams {
    const CdfBatchRecord* recs; // batched: block b builds strip b % strips of record b / strips
    uint32_t strips;           // strips per record (0: one record, strips = gridDim.x)
    const double* values;
    const double* edges; // fine edges, nt+1
    double* phi;
    double* theta;
    double* colsum;       // cp
    BlockPartial* partial; // gridDim.x
    CdfDeviceReport* report;
    unsigned* sync;       // [0] barrier arrivals, [1] finished-block ticket
    uint32_t kind, nt, np, ct, cp, dt, dp, cw;
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

constexpr unsigned kThreads = 256;
constexpr unsigned kSpinLimit = 1u << 22;

__device__ __forceinline__ bool grid_wait(unsigned* counter, unsigned target, unsigned* timeout_flag)
{
    __syncthreads();
    __shared__ int ok;
    if (threadIdx.x == 0) {
        __threadfence();
        atomicAdd(counter, 1u);
        unsigned spins = 0;
        while (*((volatile unsigned*)counter) < target && spins < kSpinLimit) {
            __nanosleep(64);
            ++spins;
        }
        ok = spins < kSpinLimit;
        if (!ok) atomicExch(timeout_flag, 1u);
        __threadfence();
    }
    __syncthreads();
    return ok;
}

__device__ __forceinline__ double fine_mass_at(const CdfParams& P, const CdfAdds& A, uint32_t i, uint32_t j)
{
    double m = P.values[(size_t)i * P.np + j];
    if (P.kind == 1) m = m * (P.edges[i + 1] - P.edges[i]);
    if (A.row) m += A.row[i];
    if (i == 0) m += A.fwd;
    if (i + 1 == P.nt) m += A.bwd;
    return m;
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

template <class T> __device__ __forceinline__ T block_sum(T x, T* red)
{
    for (int o = 16; o; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    __syncthreads();
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = x;
    __syncthreads();
    T s = T(0);
    if (threadIdx.x == 0)
        for (unsigned w = 0; w < blockDim.x / 32; ++w) s += red[w];
    return s; // valid in thread 0
}
__device__ __forceinline__ double block_max(double x, double* red)
{
    for (int o = 16; o; o >>= 1) x = fmax(x, __shfl_xor_sync(0xffffffffu, x, o));
    __syncthreads();
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = x;
    __syncthreads();
    double s = 0.0;
    if (threadIdx.x == 0)
        for (unsigned w = 0; w < blockDim.x / 32; ++w) s = fmax(s, red[w]);
    return s;
}

__global__ void __launch_bounds__(kThreads) cdf_build_kernel(const CdfParams P0)
{
    extern __shared__ __align__(16) double strip[]; // ct x CW coarse strip, then phi strip (CW+1)
    __shared__ double red_d[kThreads / 32];
    __shared__ unsigned long long red_u[kThreads / 32];
    __shared__ double s_glob[6];
    __shared__ int s_last;

    const uint32_t strips = P0.strips ? P0.strips : gridDim.x;
    const uint32_t sb = P0.strips ? blockIdx.x % strips : blockIdx.x; // this block's strip of its record
    CdfParams P = P0;
    if (P0.recs) {
        const CdfBatchRecord& R = P0.recs[blockIdx.x / strips];
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
    const uint32_t c0 = sb * P.cw;
    const uint32_t c1 = min(P.cp, c0 + P.cw);
    const uint32_t w = c1 > c0 ? c1 - c0 : 0u; // columns in this strip
    const uint32_t CW = P.cw;
    double* sphi = strip + (size_t)P.ct * CW;

    // ------------------------------------------------------------ phase A
    KSum fm{0, 0}, fa{0, 0}, sm{0, 0}, sa{0, 0};
    double largest = 0.0;
    unsigned long long invalid = 0ull, pole_bad = 0ull;
    const CdfAdds adds = cdf_adds(P, &pole_bad);
    if (threadIdx.x == 0) invalid += pole_bad;
    const uint32_t cells = P.ct * w;
    for (uint32_t q = threadIdx.x; q < cells; q += blockDim.x) {
        const uint32_t ci = q / w, cl = q % w, cj = c0 + cl;
        KSum acc{0, 0};
        for (uint32_t i = ci * P.dt; i < (ci + 1) * P.dt; ++i) {
            const double mu = 1.0 - P.edges[i] - P.edges[i + 1];
            for (uint32_t j = cj * P.dp; j < (cj + 1) * P.dp; ++j) {
                const double m = fine_mass_at(P, adds, i, j);
                if (!(m >= 0.0) || !(m <= 1.7976931348623157e308)) ++invalid;
                acc.add(m);
                fm.add(m);
                fa.add(m * mu);
            }
        }
        const double c = acc.v;
        strip[(size_t)ci * CW + cl] = c;
        const double E0 = P.edges[(size_t)ci * P.dt], E1 = P.edges[(size_t)(ci + 1) * P.dt];
        sm.add(c);
        sa.add(c * (1.0 - E0 - E1));
        largest = fmax(largest, c);
    }
    {
        const double a = block_sum(fm.v + fm.c, red_d);
        const double b = block_sum(fa.v + fa.c, red_d);
        const double c = block_sum(sm.v + sm.c, red_d);
        const double d = block_sum(sa.v + sa.c, red_d);
        const double e = block_max(largest, red_d);
        const unsigned long long f = block_sum(invalid, red_u);
        if (threadIdx.x == 0) {
            BlockPartial& bp = P.partial[sb];
            bp.fine_mass = a;
            bp.fine_axial = b;
            bp.stored_mass = c;
            bp.stored_axial = d;
            bp.largest = e;
            bp.invalid = f;
        }
    }
    if (!grid_wait(&P.sync[0], strips, &P.report->timeout)) return;

    // ------------------------------------------------------------ phase B
    // block partials staged through shared memory (L2 loads in parallel), then summed in
    // block order by one thread so that every block derives identical totals
    double* stage = sphi + CW + 1; // scratch: max(14 * strips, cp) doubles
    for (unsigned k = threadIdx.x; k < strips; k += blockDim.x) {
        const BlockPartial* bp = P.partial + k;
        stage[5 * k + 0] = __ldcg(&bp->fine_mass);
        stage[5 * k + 1] = __ldcg(&bp->fine_axial);
        stage[5 * k + 2] = __ldcg(&bp->stored_mass);
        stage[5 * k + 3] = __ldcg(&bp->stored_axial);
        stage[5 * k + 4] = __ldcg(&bp->largest);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0, b = 0, c = 0, d = 0, e = 0;
        for (unsigned k = 0; k < strips; ++k) {
            a += stage[5 * k + 0];
            b += stage[5 * k + 1];
            c += stage[5 * k + 2];
            d += stage[5 * k + 3];
            e = fmax(e, stage[5 * k + 4]);
        }
        s_glob[0] = a;
        s_glob[1] = b;
        s_glob[2] = c;
        s_glob[3] = d;
        s_glob[4] = e;
    }
    __syncthreads();
    const double fine_total = s_glob[0], stored_total = s_glob[2], big = s_glob[4];
    KSum tv{0, 0};
    if (P.dt > 1 || P.dp > 1) {
        const uint32_t fw = w * P.dp;
        for (uint32_t q = threadIdx.x; q < P.nt * fw; q += blockDim.x) {
            const uint32_t i = q / fw, j = c0 * P.dp + q % fw;
            const uint32_t ci = i / P.dt, cl = j / P.dp - c0;
            const double fraction = (P.edges[i + 1] - P.edges[i]) /
                                    (P.edges[(size_t)(ci + 1) * P.dt] - P.edges[(size_t)ci * P.dt]) / P.dp;
            tv.add(fabs(fine_mass_at(P, adds, i, j) / fine_total - strip[(size_t)ci * CW + cl] / stored_total * fraction));
        }
    }
    // weights w = coarse / largest for the whole strip in parallel (the ordered chains below
    // then carry only additions); the coarse values are recomputed in phase C for the audit
    unsigned long long underflow = 0ull;
    for (uint32_t q = threadIdx.x; q < P.ct * w; q += blockDim.x) {
        const uint32_t i = q / w, cl = q % w;
        const double c = strip[(size_t)i * CW + cl];
        const double x = c / big;
        if (c > 0 && !(x > 0)) ++underflow;
        strip[(size_t)i * CW + cl] = x;
    }
    __syncthreads();
    if (threadIdx.x < w) {
        // ordered ascending-theta scan of one phi column; the unnormalised prefix of row i+1
        // replaces the weight of row i in place (each column belongs to one thread)
        const uint32_t cl = threadIdx.x, j = c0 + cl;
        double s = 0.0;
#pragma unroll 8
        for (uint32_t i = 0; i < P.ct; ++i) {
            s += strip[(size_t)i * CW + cl];
            strip[(size_t)i * CW + cl] = s;
        }
        P.colsum[j] = s;
    }
    {
        const double t = block_sum(tv.v + tv.c, red_d);
        const unsigned long long u = block_sum(underflow, red_u);
        if (threadIdx.x == 0) {
            P.partial[sb].tv = 0.5 * t;
            P.partial[sb].underflow = u;
        }
    }
    if (!grid_wait(&P.sync[0], 2u * strips, &P.report->timeout)) return;

    // ------------------------------------------------------------ phase C
    for (uint32_t j = threadIdx.x; j < P.cp; j += blockDim.x) stage[j] = __ldcg(P.colsum + j);
    __syncthreads();
    if (threadIdx.x == 0) {
        // ordered marginal scan (phase_table.cpp:154): phi[j+1] = phi[j] + colsum[j]
        double a = 0.0;
        for (uint32_t j = 0; j < c0; ++j) a += stage[j];
        sphi[0] = a;
        for (uint32_t cl = 0; cl < w; ++cl) {
            a += stage[c0 + cl];
            sphi[cl + 1] = a;
        }
        for (uint32_t j = c1; j < P.cp; ++j) a += stage[j];
        s_glob[5] = a;
    }
    __syncthreads();
    const double total = s_glob[5];
    // normalised marginal for this strip: phi[0] = 0, phi[cp] = 1, interior / total
    if (threadIdx.x <= w) {
        const uint32_t j = c0 + threadIdx.x;
        if (threadIdx.x > 0 || c0 == 0) {
            double v = sphi[threadIdx.x];
            if (j == 0) v = 0.0;
            else if (j == P.cp) v = 1.0;
            else v = v / total;
            P.phi[j] = v;
        }
    }
    __syncthreads();
    for (uint32_t cl = threadIdx.x; cl <= w; cl += blockDim.x) {
        const uint32_t j = c0 + cl;
        double v = sphi[cl];
        sphi[cl] = (j == 0) ? 0.0 : (j == P.cp ? 1.0 : v / total);
    }
    __syncthreads();
    KSum l1{0, 0}, lost{0, 0}, rec{0, 0}, ax{0, 0};
    double max_err = 0.0;
    unsigned long long lost_cells = 0ull, malformed = 0ull;
    const uint32_t stride = P.ct + 1;
    // this strip's output rows are contiguous: theta[c0*(ct+1) .. c1*(ct+1)); every element is
    // written once, from the prefixes kept in shared memory (prefix of row i at strip[i-1])
    const uint32_t span = w * stride;
#pragma unroll 2
    for (uint32_t q = threadIdx.x; q < span; q += blockDim.x) {
        const uint32_t cl = q / stride, i = q % stride, j = c0 + cl;
        const double cs = stage[j];
        auto norm = [&](uint32_t k) -> double {
            if (k == 0) return 0.0;
            if (k == P.ct) return 1.0;
            return cs > 0 ? strip[(size_t)(k - 1) * CW + cl] / cs : P.edges[(size_t)k * P.dt];
        };
        const double b0 = norm(i);
        if (i < P.ct) {
            const double b1 = norm(i + 1);
            const double a0 = sphi[cl], a1 = sphi[cl + 1];
            const double qv = (a1 - a0) * (b1 - b0);
            const double c = coarse_at(P, adds, i, j);
            const double p = c / stored_total;
            const bool bad = !(qv >= 0.0) || !(qv <= 1.7976931348623157e308) || a1 < a0 || b1 < b0;
            if (bad) ++malformed;
            if (c > 0 && !(p > 0)) ++malformed;
            const double err = fabs(p - qv);
            l1.add(err);
            max_err = fmax(max_err, err);
            if (p > 0 && qv == 0) {
                lost.add(p);
                ++lost_cells;
            }
            rec.add(qv);
            const double E0 = P.edges[(size_t)i * P.dt], E1 = P.edges[(size_t)(i + 1) * P.dt];
            ax.add(qv * (1.0 - E0 - E1));
        }
        P.theta[(size_t)c0 * stride + q] = b0;
    }
    {
        const double a = block_sum(l1.v + l1.c, red_d);
        const double b = block_sum(lost.v + lost.c, red_d);
        const double c = block_sum(rec.v + rec.c, red_d);
        const double d = block_sum(ax.v + ax.c, red_d);
        const double e = block_max(max_err, red_d);
        const unsigned long long f = block_sum(lost_cells, red_u);
        const unsigned long long g = block_sum(malformed, red_u);
        if (threadIdx.x == 0) {
            BlockPartial& bp = P.partial[sb];
            bp.l1 = a;
            bp.lost = b;
            bp.recovered = c;
            bp.axial = d;
            bp.max_err = e;
            bp.lost_cells = f;
            bp.malformed = g;
            __threadfence();
            s_last = (atomicAdd(&P.sync[1], 1u) == strips - 1);
        }
    }
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    // last block: stage every block's audit partials (parallel L2 loads), sum in block order
    constexpr unsigned kF = 14;
    for (unsigned k = threadIdx.x; k < strips; k += blockDim.x) {
        const BlockPartial* bp = P.partial + k;
        double* o = stage + (size_t)kF * k;
        o[0] = __ldcg(&bp->fine_mass);
        o[1] = __ldcg(&bp->fine_axial);
        o[2] = __ldcg(&bp->stored_mass);
        o[3] = __ldcg(&bp->stored_axial);
        o[4] = __ldcg(&bp->tv);
        o[5] = __ldcg(&bp->l1);
        o[6] = __ldcg(&bp->lost);
        o[7] = __ldcg(&bp->recovered);
        o[8] = __ldcg(&bp->axial);
        o[9] = __ldcg(&bp->max_err);
        o[10] = __longlong_as_double((long long)__ldcg(&bp->lost_cells));
        o[13] = __longlong_as_double((long long)__ldcg(&bp->malformed));
        o[11] = __longlong_as_double((long long)__ldcg(&bp->invalid));
        o[12] = __longlong_as_double((long long)__ldcg(&bp->underflow));
    }
    __syncthreads();
    if (threadIdx.x != 0) return;
    CdfDeviceReport r{};
    for (unsigned k = 0; k < strips; ++k) {
        const double* o = stage + (size_t)kF * k;
        r.fine_mass += o[0];
        r.fine_axial += o[1];
        r.stored_mass += o[2];
        r.stored_axial += o[3];
        r.tv += o[4];
        r.l1 += o[5];
        r.lost += o[6];
        r.recovered += o[7];
        r.axial += o[8];
        r.max_err = fmax(r.max_err, o[9]);
        r.invalid += (unsigned long long)__double_as_longlong(o[11]);
        r.underflow += (unsigned long long)__double_as_longlong(o[12]);
        r.lost_cells += (unsigned long long)__double_as_longlong(o[10]);
        r.malformed += (unsigned long long)__double_as_longlong(o[13]);
    }
    r.largest = s_glob[4];
    r.total = total;
    r.timeout = P.report->timeout;
    *P.report = r;
}

// Fine-grid mass with pole caps for an FP64 histogram (used by the report path).
int launch_cdf_build(const CdfLaunch& L, cudaStream_t stream)
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
    P.cw = L.cw;
    P.fwd_add = L.fwd_add;
    P.bwd_add = L.bwd_add;
    P.row_add = L.row_add;
    P.pole_fx = L.pole_fx;
    P.pole_weight = L.pole_weight;
    const unsigned blocks = (L.cp + L.cw - 1) / L.cw;
    const size_t smem = cdf_smem_bytes(L.ct, L.cp, L.cw);
    cudaError_t e = cudaFuncSetAttribute(cdf_build_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return (int)e;
    void* args[] = {&P};
    e = cudaLaunchCooperativeKernel((const void*)cdf_build_kernel, dim3(blocks), dim3(kThreads), args, smem, stream);
    return (int)e;
}

size_t cdf_smem_bytes(uint32_t ct, uint32_t cp, uint32_t cw)
{
    const size_t blocks = (cp + cw - 1) / cw;
    const size_t stage = blocks * 14 > cp ? blocks * 14 : cp;
    return sizeof(double) * ((size_t)ct * cw + cw + 1 + stage);
}

int launch_cdf_build_batch(const CdfLaunch& L, const CdfBatchRecord* d_recs, uint32_t count, cudaStream_t stream)
{
    CdfParams P{};
    P.recs = d_recs;
    P.edges = L.edges;
    P.kind = L.kind;
    P.nt = L.nt;
    P.np = L.np;
    P.ct = L.ct;
    P.cp = L.cp;
    P.dt = L.nt / L.ct;
    P.dp = L.np / L.cp;
    P.cw = L.cw;
    P.strips = (L.cp + L.cw - 1) / L.cw;
    const size_t smem = cdf_smem_bytes(L.ct, L.cp, L.cw);
    cudaError_t e = cudaFuncSetAttribute(cdf_build_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return (int)e;
    void* args[] = {&P};
    e = cudaLaunchCooperativeKernel((const void*)cdf_build_kernel, dim3(P.strips * count), dim3(kThreads), args, smem,
                                    stream);
    return (int)e;
}

int cdf_max_coresident_blocks(size_t smem, int device)
{
    int per_sm = 0, sms = 0;
    cudaFuncSetAttribute(cdf_build_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, cdf_build_kernel, kThreads, smem) != cudaSuccess) return 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) return 0;
    return per_sm * sms;
}

size_t cdf_partial_bytes() { return sizeof(BlockPartial); }

} // namespace icp
