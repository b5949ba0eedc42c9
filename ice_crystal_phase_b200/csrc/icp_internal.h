// icp_internal.h -- declarations shared by the CUDA translation units and the C-ABI layer.
#pragma once
#include <cstddef>
#include <cstdint>
#include <vector>
#include <cuda_runtime.h>

#include "../../include/icp_b200.h"

namespace icp {

// Final audit written by the last block of the CDF kernel.
struct CdfDeviceReport {
    double fine_mass, fine_axial, stored_mass, stored_axial, tv, l1, lost, recovered, axial, max_err, largest, total;
    unsigned long long lost_cells, malformed, invalid, underflow;
    unsigned timeout, pad;
};

struct CdfLaunch {
    const double* values;
    const double* edges;
    double* phi;
    double* theta;
    double* colsum;
    void* partial;
    CdfDeviceReport* report;
    unsigned* sync; // two counters: zero before the first launch; every completed launch leaves them zero
    uint32_t kind, nt, np, ct, cp;
    uint32_t spin_limit; // grid-barrier iteration limit (0: the default)
    double fwd_add, bwd_add;
    // optional device-side inputs of a record launched without a host round trip:
    const double* row_add;             // nt values added to every cell of row i (or null)
    const unsigned long long* pole_fx; // fwd[2], bwd[2] fixed-point pole sums (or null: fwd/bwd_add)
    double pole_weight;                // mm^2 per unit of pole power (with pole_fx)
};

// Launch shape of one CDF build: strip width (stored phi columns per block), whether the coarse
// strip stays in shared memory for the audit (keep), whether the fine strip arrives by TMA boxes
// (tma; fine grid = stored grid only), the boxes' rows, and the dynamic shared memory.
struct CdfShape {
    uint32_t cw, keep, tma, box_rows, boxes, rows_alloc;
    size_t smem;
};
// Widest-first search over (keep, tma) modes and the smallest strip width >= max(min_width,
// ceil(cp / sms)) whose grid of ceil(cp / cw) blocks (at most max_blocks) is co-resident.
// Returns 0 on success.
int cdf_choose_shape(int device, int sms, uint32_t nt, uint32_t np, uint32_t ct, uint32_t cp, bool tma_ok,
                     uint32_t min_width, uint32_t max_blocks, CdfShape& out);
int launch_cdf_build(const CdfLaunch& L, const CdfShape& s, cudaStream_t stream);
// One record of a batched CDF build (device array of these; scratch per record: `strips`
// partials, cp column sums, two zeroed barrier counters, a zeroed report).
struct CdfBatchRecord {
    const double* values;
    double* phi;
    double* theta;
    double* colsum;
    void* partial;
    CdfDeviceReport* report;
    unsigned* sync;
    const double* row_add;
    const unsigned long long* pole_fx;
    double pole_weight, fwd_add, bwd_add;
};
// Builds `count` records of one grid shape (L: edges, kind, nt, np, ct, cp; its per-record
// fields unused; s without tma) in one cooperative launch of count x ceil(cp / s.cw) blocks.
int launch_cdf_build_batch(const CdfLaunch& L, const CdfShape& s, const CdfBatchRecord* d_recs, uint32_t count,
                           cudaStream_t stream);
int cdf_max_coresident_blocks(size_t smem, int device);
// Bytes of one block's partial results in the CDF scratch (15 words).
constexpr size_t kCdfPartialBytes = 120;
size_t cdf_smem_bytes(const CdfShape& s, uint32_t ct, uint32_t cp);
size_t cdf_partial_bytes();
// Sets the calling thread's message returned by icp_last_error().
void set_last_error(const char* message);

// Host-side description of one trace+bin launch (double precision inputs; the launcher
// converts to the kernel's arithmetic type).  geometry: 0 = hexagonal prism, 1 = drop.
struct HexLaunch {
    uint32_t geometry;
    // prism (units of the circumradius)
    double half_len;
    double cum[8];
    uint32_t face_mask;
    double area;
    // drop (units of the equal-volume radius)
    double coeff[8];
    double r_out, r_center;
    uint32_t sphere;
    double disk, back;
    double e1[3];
    // common
    double k[3], ke0[3];
    double n_ext, n_int, tail, bal_tol;
    uint64_t seed, total, first, count;
    uint32_t max_hits, batch_size;
    uint32_t* batch_out;
    // grid transforms
    double rot[9];      // column-major body -> ensemble
    double ki[3], e0[3], e1g[3];
    uint32_t nt, np;
    const double* edges_d;
    const float* edges_f;
    double* mass;
    double to_mass;
    void* stats; // DevStats*
    uint32_t hash_slots;
    uint32_t block_threads;
    uint32_t blocks;
};

// Most rays one lane may trace between two flushes of its 32-bit counters (icp_hex_kernel.cuh
// LaneAcc): a ray adds at most max_hits + 1 outputs and encounters and 40 gauge evaluations per
// intersection, so launch pieces (rays per warp) and batch chunks stay at or below this.
inline uint64_t lane_rays_max(uint32_t max_hits)
{
    const uint64_t per_ray = 40ull * ((uint64_t)max_hits + 1ull);
    const uint64_t n = 0xffffffffull / per_ray;
    return n > 65536ull ? 65536ull : (n ? n : 1ull);
}

size_t hex_stats_bytes();
int launch_hex_f32(const HexLaunch& L, cudaStream_t stream);
int launch_hex_f64(const HexLaunch& L, cudaStream_t stream);
int launch_drop_f32(const HexLaunch& L, cudaStream_t stream);
int launch_drop_f64(const HexLaunch& L, cudaStream_t stream);
int hex_blocks_per_sm_f32(uint32_t slots, uint32_t nt, uint32_t threads);
int hex_blocks_per_sm_f64(uint32_t slots, uint32_t nt, uint32_t threads);
int drop_blocks_per_sm_f32(uint32_t slots, uint32_t nt, uint32_t threads);
int drop_blocks_per_sm_f64(uint32_t slots, uint32_t nt, uint32_t threads);
// the drop trace kernels' block size: the default, and the most threads a block may have
uint32_t drop_trace_threads_f32();
uint32_t drop_trace_threads_f64();

// One persistent launch over many drop records (icp_batch_kernel.cuh).  recs[r] describes
// record r exactly as for a single-record launch (first = 0, count = total = its rays, its
// own mass / stats pointers); the launcher writes the per-record parameter table into
// h_staging (pinned, n_records x drop_batch_param_bytes) and copies it to d_table.
struct BatchLaunch {
    const HexLaunch* recs;
    uint32_t n_records;
    void* h_staging;
    void* d_table;
    const unsigned long long* d_chunk_begin; // n_records + 1
    unsigned long long* d_queue;             // zeroed by the caller
    unsigned long long total_chunks;
    uint32_t chunk_rays, threads, blocks, nt;
    const double* edges_d;
    const float* edges_f;
};
size_t drop_batch_param_bytes(uint32_t precision);
int launch_drop_batch_f32(const BatchLaunch& B, cudaStream_t stream);
int launch_drop_batch_f64(const BatchLaunch& B, cudaStream_t stream);
int drop_batch_blocks_per_sm(uint32_t precision, uint32_t threads, uint32_t nt);

// Device buffer that grows on demand and is reused across calls.
struct Scratch {
    void* ptr = nullptr;
    size_t bytes = 0;
    cudaError_t ensure(size_t n)
    {
        if (n <= bytes) return cudaSuccess;
        if (ptr) cudaFree(ptr);
        ptr = nullptr;
        bytes = 0;
        const cudaError_t e = cudaMalloc(&ptr, n);
        if (e == cudaSuccess) bytes = n;
        return e;
    }
    // As ensure; a buffer (re)allocated here is cleared on the stream (counters that kernels
    // leave at zero after every completed launch start from zero this way).
    cudaError_t ensure_zeroed(size_t n, cudaStream_t stream)
    {
        if (n <= bytes) return cudaSuccess;
        const cudaError_t e = ensure(n);
        return e == cudaSuccess ? cudaMemsetAsync(ptr, 0, bytes, stream) : e;
    }
    void release()
    {
        if (ptr) cudaFree(ptr);
        ptr = nullptr;
        bytes = 0;
    }
};

// Launch counter shared by the ABI files (icp_kernel_launches).
void count_launch();

} // namespace icp

struct icp_context;
namespace icp {
// FP32 copy of the u edges in the context scratch (one small kernel).
int ensure_float_edges(icp_context* c, const double* d_edges, uint32_t nt);
// Adds one launch's device statistics (DevStats bytes) into the public stats struct.
void stats_accumulate(const unsigned char* raw, icp_trace_stats* out);
// Launch shape of the cooperative CDF grid for a (nt, np) -> (ct, cp) build (cached per context).
int cdf_shape(icp_context* c, uint32_t nt, uint32_t np, uint32_t ct, uint32_t cp, bool tma_ok, CdfShape& s);
// Clears `records` CDF reports and barrier-counter pairs after a build gave up waiting (a build
// that completes leaves its counters at zero itself), then waits for the stream.
int cdf_clear(icp_context* c, void* d_reports, void* d_sync, uint32_t records);
// Public CDF report and quality gates (build_host_cdf) from the kernel's device report.
int cdf_finish(const CdfDeviceReport& r, const icp_cdf_policy& p, icp_cdf_report* report);
// Enqueues one cooperative CDF build (no host synchronisation); d_sync[2] and d_report are
// zeroed here.  pole_fx / row_add select the device-side additions (CdfLaunch).
int cdf_enqueue(icp_context* c, const double* d_values, uint32_t nt, uint32_t np, uint32_t ct, uint32_t cp,
                const double* d_edges, double fwd_add, double bwd_add, const unsigned long long* pole_fx,
                double pole_weight, const double* row_add, double* d_phi, double* d_theta, CdfDeviceReport* d_report,
                unsigned* d_sync);

// Inputs of one record of a batched CDF build (see cdf_enqueue).
struct CdfBatchInput {
    const double* values;
    double* phi;
    double* theta;
    const double* row_add;
    const unsigned long long* pole_fx;
    double pole_weight, fwd_add, bwd_add;
};
// Enqueues the CDF builds of `count` records of one grid shape as few cooperative launches
// (16 strips per record, as many records per launch as stay co-resident; the records' a / T
// equal those of one cdf_enqueue per record); d_reports[count] and d_sync[2 count] are zeroed
// here.  Not for use inside a stream capture (the record table is copied from pageable memory).
int cdf_enqueue_batch(icp_context* c, const CdfBatchInput* in, uint32_t count, uint32_t nt, uint32_t np, uint32_t ct,
                      uint32_t cp, const double* d_edges, CdfDeviceReport* d_reports, unsigned* d_sync);

// Analytic diffraction rows of one record on the device (icp_drop_device.cu).
struct DiffractionArgs {
    const double* edges;              // nt + 1 fine u edges
    const unsigned long long* rays;   // DevStats::rays of the record (missed follows at +missed_offset)
    double* row_add;                  // out: nt per-cell additions (row power / np)
    double* power;                    // out: total diffraction power (mm^2)
    double weight, wavelength_nm;     // mm^2 per traced ray, vacuum wavelength
    uint32_t nt, np;
    uint32_t missed_offset;           // words from rays to missed in DevStats
    uint32_t pad;
};
int launch_diffraction_rows(const DiffractionArgs* d_args, uint32_t count, uint32_t nt, cudaStream_t stream);
// Drop-record helpers shared by the single-record and batched entries (icp_capi_drop.cu).
namespace dropx {
bool sphere_of(const double c[8]);
void drop_bounds(const double c[8], double& r_center, double& r_out);
int validate_record(const icp_drop_record* r);
int validate_grid(const icp_drop_record* r);
int grid_of(const icp_drop_record* r, icp_grid& g);
int table_slots(const icp_tuning& t, uint32_t& slots);
HexLaunch drop_launch(const icp_drop_record* r, const icp_grid* g, const double* d_edges, const float* edges_f,
                      double* d_mass, void* d_stats, double area_weight, uint32_t slots);
int finish_report(const icp_drop_record* r, const unsigned char* raw_stats, const CdfDeviceReport& cdf, double power,
                  double weight, icp_drop_report* rep);
double projected_area_of(const icp_drop_record* r, int& status);
} // namespace dropx
// Offsets (in 64-bit words) of fields of the trace kernel's DevStats.
uint32_t devstats_rays_word();
uint32_t devstats_missed_word();
uint32_t devstats_fwd_word();
} // namespace icp

namespace icp {
// Page-locked host staging (copies captured into CUDA graphs must not read pageable memory).
struct Pinned {
    void* ptr = nullptr;
    size_t size = 0;
    cudaError_t ensure(size_t bytes)
    {
        if (bytes <= size) return cudaSuccess;
        if (ptr) cudaFreeHost(ptr);
        ptr = nullptr;
        size = 0;
        const cudaError_t e = cudaMallocHost(&ptr, bytes);
        if (e == cudaSuccess) size = bytes;
        return e;
    }
    ~Pinned()
    {
        if (ptr) cudaFreeHost(ptr);
    }
};
// State of the batched-record entries: host staging, the captured graph, tuned launch shapes.
struct BatchState {
    Pinned h_table, h_chunks, h_dargs, h_edges, h_stats, h_reports, h_powers;
    cudaGraphExec_t exec = nullptr;
    struct Tuned {
        uint32_t precision, nt, threads, chunk_rays;
    };
    std::vector<Tuned> tuned;
    ~BatchState()
    {
        if (exec) cudaGraphExecDestroy(exec);
    }
};
} // namespace icp

// One CUDA device, one non-blocking stream, reusable scratch.
struct icp_context {
    int device = 0;
    int sms = 0;
    cudaStream_t stream = nullptr;
    icp::Scratch stats, edges_f, cdf_partial, cdf_report, cdf_sync, cdf_colsum;
    icp::Scratch rec_edges, rec_mass, rec_phi, rec_theta, rec_batch, rows, dargs;
    // batched records
    icp::Scratch b_table, b_chunks, b_queue, b_stats, b_mass, b_rows, b_dargs, b_reports, b_sync, b_phi, b_theta;
    icp::BatchState batch;
    // surrogate
    icp::Scratch mlp_error;
    // batched CDF builds
    icp::Scratch cdfb_partial, cdfb_colsum, cdfb_recs;
    // deterministic atlas: per-node trace scratch, coupling accumulators
    icp::Scratch atlas_trace, atlas_coupling;
    // Table-II rainbow diffraction: packed samples, row marks, counters
    icp::Scratch rainbow;
    // patch build: cell statuses, block counts, histogram
    icp::Scratch patches;
    // patch query: direction bins, scans, per-direction counts; the bins' patch lists
    icp::Scratch query, query_list;
    // wave-stage density audit accumulators
    icp::Scratch stage_audit;
    // lattice trace tallies
    icp::Scratch lattice;
    // folded-patch records: block counts, candidate list, statistics
    icp::Scratch folded;
    // atlas composition: the compacted nonzero coupling shifts
    icp::Scratch atlas_list;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr, ev2 = nullptr;
    // grid-barrier iteration limit handed to the CDF kernels (0: their default)
    uint32_t wait_limit = 0;
    // CDF launch shapes already chosen: (nt, np, ct, cp, tma allowed) -> shape
    struct ShapeEntry {
        uint32_t nt, np, ct, cp, tma_ok;
        icp::CdfShape shape;
    };
    std::vector<ShapeEntry> cdf_shapes;
    // u edges of the last icp_phase_cdf_enqueue grid (uploaded when nt changes)
    icp::Scratch cdf_edges;
    uint32_t cdf_edges_nt = 0;
};
