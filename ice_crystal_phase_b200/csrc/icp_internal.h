// icp_internal.h -- declarations shared by the CUDA translation units and the C-ABI layer.
#pragma once
#include <cstddef>
#include <cstdint>
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
    unsigned* sync; // two counters, zeroed before launch
    uint32_t kind, nt, np, ct, cp, cw;
    double fwd_add, bwd_add;
};

int launch_cdf_build(const CdfLaunch& L, cudaStream_t stream);
int cdf_max_coresident_blocks(size_t smem, int device);
size_t cdf_smem_bytes(uint32_t ct, uint32_t cp, uint32_t cw);
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

size_t hex_stats_bytes();
int launch_hex_f32(const HexLaunch& L, cudaStream_t stream);
int launch_hex_f64(const HexLaunch& L, cudaStream_t stream);
int launch_drop_f32(const HexLaunch& L, cudaStream_t stream);
int launch_drop_f64(const HexLaunch& L, cudaStream_t stream);
int hex_blocks_per_sm_f32(uint32_t slots, uint32_t nt, uint32_t threads);
int hex_blocks_per_sm_f64(uint32_t slots, uint32_t nt, uint32_t threads);
int drop_blocks_per_sm_f32(uint32_t slots, uint32_t nt, uint32_t threads);
int drop_blocks_per_sm_f64(uint32_t slots, uint32_t nt, uint32_t threads);

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
} // namespace icp

// One CUDA device, one non-blocking stream, reusable scratch.
struct icp_context {
    int device = 0;
    int sms = 0;
    cudaStream_t stream = nullptr;
    icp::Scratch stats, edges_f, cdf_partial, cdf_report, cdf_sync, cdf_colsum;
    icp::Scratch rec_edges, rec_mass, rec_phi, rec_theta, rec_batch, rows;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
};
