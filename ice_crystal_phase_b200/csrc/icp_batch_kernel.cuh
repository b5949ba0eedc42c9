// icp_batch_kernel.cuh -- one persistent launch over many records (sm_100a).
//
// Replaces one process (and one launch chain) per record with a device work queue: a batch of
// records of one geometry, all on the same (u, phi) grid, is cut into chunks of `chunk_rays`
// consecutive ray ids; chunk c of record r is found from the prefix chunk_begin[] and handed
// out by an atomic counter, one chunk per warp at a time.  A warp caches its record's trace
// parameters in its own shared-memory slot, traces the chunk with the per-lane refill loop of
// the single-record kernel, and adds its counters to that record's DevStats before it takes the
// next chunk -- no block barrier, so uneven ray counts and uneven ray lengths only cost the
// last chunk of each warp.  Exits go straight to each record's FP64 histogram (continuous-
// direction records saturate any shared table; see icp_capi_drop.cu).  Ray ids, and therefore
// results, are those of the single-record kernel, independent of chunking.
#pragma once
#include "icp_hex_kernel.cuh"

namespace icp {

template <class R, class G> struct BatchParams {
    const TraceParams<R, G>* recs;          // one per record (first = 0, count = total = rays)
    const unsigned long long* chunk_begin;  // n_records + 1: first chunk of each record, total last
    unsigned long long* queue;              // next chunk (zeroed before the launch)
    unsigned long long total_chunks;
    uint32_t n_records;
    uint32_t chunk_rays;                    // ray ids per chunk
    uint32_t smem_edges;                    // 1 = stage the shared u edges in shared memory
    uint32_t nt;
    const float* edges_f;
    const double* edges_d;
};

// Dynamic shared memory: per-warp parameter slots, per-warp tallies, the u edges.
template <class R, class G> __host__ __device__ constexpr size_t batch_slot_bytes()
{
    return (sizeof(TraceParams<R, G>) + 15) / 16 * 16;
}
template <class R, class G> size_t batch_smem_bytes(uint32_t threads, uint32_t nt, bool smem_edges)
{
    const uint32_t warps = threads / 32;
    return warps * batch_slot_bytes<R, G>() + warps * kTallyBytes + (smem_edges ? (nt + 1) * sizeof(R) : 0);
}

template <class R, class G>
__global__ void __launch_bounds__(256, (sizeof(R) == 4 ? 4 : 1)) batch_trace_kernel(const BatchParams<R, G> Q)
{
    extern __shared__ __align__(16) unsigned char smem[];
    const unsigned warps = blockDim.x >> 5, wib = threadIdx.x >> 5, lane = threadIdx.x & 31u;
    unsigned char* slots = smem;
    Tally* tallies = reinterpret_cast<Tally*>(slots + warps * batch_slot_bytes<R, G>());
    R* s_edges = reinterpret_cast<R*>(tallies + warps);
    for (unsigned i = threadIdx.x; i < warps * kTallyBytes / 4; i += blockDim.x) reinterpret_cast<unsigned*>(tallies)[i] = 0u;
    const R* gedges;
    if constexpr (sizeof(R) == 4) gedges = Q.edges_f;
    else gedges = Q.edges_d;
    if (Q.smem_edges)
        for (uint32_t i = threadIdx.x; i <= Q.nt; i += blockDim.x) s_edges[i] = gedges[i];
    __syncthreads();

    TraceParams<R, G>& P = *reinterpret_cast<TraceParams<R, G>*>(slots + wib * batch_slot_bytes<R, G>());
    BlockShared<R> B;
    B.H = SmemHist{nullptr, nullptr, 0u};
    B.T = tallies + wib;
    B.edges = Q.smem_edges ? s_edges : gedges;
    uint32_t cur = 0xffffffffu;
    while (true) {
        unsigned long long c = 0ull;
        uint32_t r = 0u;
        if (lane == 0) {
            c = atomicAdd(Q.queue, 1ull);
            if (c < Q.total_chunks) {
                uint32_t lo = 0u, hi = Q.n_records; // largest r with chunk_begin[r] <= c
                while (hi - lo > 1u) {
                    const uint32_t mid = (lo + hi) >> 1;
                    if (Q.chunk_begin[mid] <= c) lo = mid;
                    else hi = mid;
                }
                r = lo;
            }
        }
        c = __shfl_sync(kFull, c, 0);
        r = __shfl_sync(kFull, r, 0);
        if (c >= Q.total_chunks) break;
        if (r != cur) {
            // this warp's parameter slot <- the record's trace parameters
            const uint32_t* src = reinterpret_cast<const uint32_t*>(Q.recs + r);
            uint32_t* dst = reinterpret_cast<uint32_t*>(&P);
            for (unsigned i = lane; i < sizeof(TraceParams<R, G>) / 4; i += 32u) dst[i] = src[i];
            __syncwarp();
            cur = r;
        }
        const uint64_t first = (uint64_t)(c - Q.chunk_begin[r]) * Q.chunk_rays;
        const uint64_t end = min(first + Q.chunk_rays, (uint64_t)P.total);
        LaneAcc<R> A;
        lane_acc_clear(A);
        trace_slice<R, G>(P, B, first, end, A);
        warp_stats_flush<R>(P.stats, A, B.T);
    }
}

} // namespace icp
