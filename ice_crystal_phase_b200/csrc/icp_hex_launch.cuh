// icp_hex_launch.cuh -- host launcher for the trace+bin kernel, instantiated once per
// arithmetic type and geometry in icp_hex_f32.cu / icp_hex_f64.cu / icp_drop_f32.cu / icp_drop_f64.cu.
#pragma once
#include <cmath>
#include <vector>

#include "icp_batch_kernel.cuh"
#include "icp_hex_kernel.cuh"
#include "icp_internal.h"

namespace icp {

constexpr uint32_t kEdgeSmemMax = 4097; // stage u edges in shared memory up to this many

template <class R> size_t trace_smem_bytes(uint32_t hash_slots, uint32_t nt)
{
    size_t b = trace_tally_offset(hash_slots) + kTallyWarps * kTallyBytes;
    if (nt + 1 <= kEdgeSmemMax) b += sizeof(R) * (nt + 1);
    return b;
}

template <class R, class G> void fill_common(TraceParams<R, G>& P, const HexLaunch& L)
{
    P.k = v3((R)L.k[0], (R)L.k[1], (R)L.k[2]);
    P.ke0 = v3((R)L.ke0[0], (R)L.ke0[1], (R)L.ke0[2]);
    P.enter = make_media<R>(L.n_ext, L.n_int);
    P.leave = make_media<R>(L.n_int, L.n_ext);
    P.tail = (R)L.tail;
    P.tail_fx = (unsigned long long)std::floor(L.tail * 0x1p44);
    P.bal_tol = (R)L.bal_tol;
    P.seed = L.seed;
    P.total = L.total;
    P.first = L.first;
    P.count = L.count;
    P.max_hits = L.max_hits;
    P.batch_size = L.batch_size;
    P.batch_out = L.batch_out;
    // FP32 fused transform rows: (e0, e1, ki)^T * rotation
    const double* r = L.rot; // column c = r[3c..3c+2]
    const double* rows[3] = {L.e0, L.e1g, L.ki};
    for (int a = 0; a < 3; ++a)
        for (int c = 0; c < 3; ++c)
            P.gf.m[3 * a + c] = (float)(rows[a][0] * r[3 * c] + rows[a][1] * r[3 * c + 1] + rows[a][2] * r[3 * c + 2]);
    P.gf.nt = L.nt;
    P.gf.np = L.np;
    P.gf.np_f = (float)L.np;
    P.gf.theta_scale = (float)((double)L.nt / kPi);
    for (int i = 0; i < 9; ++i) P.gd.rot[i] = L.rot[i];
    for (int i = 0; i < 3; ++i) {
        P.gd.ki[i] = L.ki[i];
        P.gd.e0[i] = L.e0[i];
        P.gd.e1[i] = L.e1g[i];
    }
    P.gd.edges = L.edges_d;
    P.gd.nt = L.nt;
    P.gd.np = L.np;
    P.edges_d = L.edges_d;
    P.edges_f = L.edges_f;
    P.mass = L.mass;
    P.to_mass = L.to_mass;
    P.stats = reinterpret_cast<DevStats*>(L.stats);
    P.hash_slots = L.hash_slots;
    P.smem_edges = (L.nt + 1 <= kEdgeSmemMax) ? 1u : 0u;
}

template <class R> TraceParams<R, HexGeo<R>> make_hex_params(const HexLaunch& L)
{
    TraceParams<R, HexGeo<R>> P;
    fill_common(P, L);
    P.geo.half_len = (R)L.half_len;
    for (int f = 0; f < 8; ++f) P.geo.cum[f] = (R)L.cum[f];
    P.geo.face_mask = L.face_mask;
    P.geo.area = (R)L.area;
    return P;
}

template <class R> TraceParams<R, DropGeo<R>> make_drop_params(const HexLaunch& L)
{
    TraceParams<R, DropGeo<R>> P;
    fill_common(P, L);
    for (int n = 0; n < 8; ++n) P.geo.shape.c[n] = (R)L.coeff[n];
    // monomial form of 1 + sum_n c_n T_n(mu) in binary64 (T_{n+1} = 2 mu T_n - T_{n-1})
    double mono[8] = {1.0 + L.coeff[0], 0, 0, 0, 0, 0, 0, 0};
    double tm1[8] = {1, 0, 0, 0, 0, 0, 0, 0}, tn[8] = {0, 1, 0, 0, 0, 0, 0, 0};
    for (int k = 0; k < 8; ++k) mono[k] += L.coeff[1] * tn[k];
    for (int n = 2; n < 8; ++n) {
        double tp[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        for (int k = 0; k < 8; ++k) {
            if (k > 0) tp[k] += 2 * tn[k - 1];
            tp[k] -= tm1[k];
        }
        for (int k = 0; k < 8; ++k) {
            tm1[k] = tn[k];
            tn[k] = tp[k];
            mono[k] += L.coeff[n] * tn[k];
        }
    }
    for (int k = 0; k < 8; ++k) P.geo.shape.m[k] = (R)mono[k];
    for (int k = 0; k < 7; ++k) P.geo.shape.md[k] = (R)((k + 1) * mono[k + 1]);
    P.geo.shape.r_out = (R)L.r_out;
    P.geo.shape.r_center = (R)L.r_center;
    {
        // enclosing spheroid of the surface r = 1 + sum c_n T_n(mu), y = -mu r: centre and
        // half-axes from the extents, scaled by the largest spheroid gauge over 2049 samples of
        // mu, then inflated by 1e-5 (far above the binary32 rounding of the roots and above the
        // sampling error, which is second order in the 9.8e-4 spacing: below 1e-6)
        const int n = 2048;
        double ymin = 1e300, ymax = -1e300, hmax = 0;
        std::vector<double> ys(n + 1), hs(n + 1);
        for (int i = 0; i <= n; ++i) {
            const double mu = -1.0 + 2.0 * i / n;
            double tm = 1, t = mu, r = 1 + L.coeff[0] + L.coeff[1] * mu;
            for (int k = 2; k < 8; ++k) {
                const double tn = 2 * mu * t - tm;
                r += L.coeff[k] * tn;
                tm = t;
                t = tn;
            }
            ys[i] = -mu * r;
            hs[i] = std::sqrt(std::fmax(0.0, 1 - mu * mu)) * r;
            ymin = std::fmin(ymin, ys[i]);
            ymax = std::fmax(ymax, ys[i]);
            hmax = std::fmax(hmax, hs[i]);
        }
        const double y0 = 0.5 * (ymax + ymin), A = hmax, B = 0.5 * (ymax - ymin);
        double sc = 0;
        for (int i = 0; i <= n; ++i) {
            const double u = hs[i] / A, v = (ys[i] - y0) / B;
            sc = std::fmax(sc, std::sqrt(u * u + v * v));
        }
        const double Ae = A * sc * (1 + 1e-5) + 1e-7, Be = B * sc * (1 + 1e-5) + 1e-7;
        P.geo.shape.ea_inv = (R)(1.0 / Ae);
        P.geo.shape.eb_inv = (R)(1.0 / Be);
        P.geo.shape.ey0 = (R)y0;
    }
    P.geo.shape.sphere = L.sphere != 0;
    P.geo.disk = (R)L.disk;
    P.geo.back = (R)L.back;
    P.geo.e1 = v3((R)L.e1[0], (R)L.e1[1], (R)L.e1[2]);
    return P;
}

template <class R, class G> int launch_trace(const TraceParams<R, G>& P, const HexLaunch& L, cudaStream_t stream)
{
    const size_t smem = trace_smem_bytes<R>(L.hash_slots, L.nt);
    cudaError_t e = cudaFuncSetAttribute(trace_bin_kernel<R, G>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return (int)e;
    trace_bin_kernel<R, G><<<L.blocks, L.block_threads, smem, stream>>>(P);
    return (int)cudaGetLastError();
}

template <class R, class G> int trace_blocks_per_sm(uint32_t hash_slots, uint32_t nt, uint32_t threads)
{
    const size_t smem = trace_smem_bytes<R>(hash_slots, nt);
    cudaFuncSetAttribute(trace_bin_kernel<R, G>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, trace_bin_kernel<R, G>, (int)threads, smem) != cudaSuccess)
        return 0;
    return per_sm;
}

template <class R> int launch_drop_batch(const BatchLaunch& B, cudaStream_t stream)
{
    using P_ = TraceParams<R, DropGeo<R>>;
    P_* table = static_cast<P_*>(B.h_staging);
    for (uint32_t r = 0; r < B.n_records; ++r) table[r] = make_drop_params<R>(B.recs[r]);
    cudaError_t e = cudaMemcpyAsync(B.d_table, table, sizeof(P_) * B.n_records, cudaMemcpyHostToDevice, stream);
    if (e != cudaSuccess) return (int)e;
    BatchParams<R, DropGeo<R>> Q;
    Q.recs = static_cast<const P_*>(B.d_table);
    Q.chunk_begin = B.d_chunk_begin;
    Q.queue = B.d_queue;
    Q.total_chunks = B.total_chunks;
    Q.n_records = B.n_records;
    Q.chunk_rays = B.chunk_rays;
    Q.nt = B.nt;
    Q.smem_edges = (B.nt + 1 <= kEdgeSmemMax) ? 1u : 0u;
    Q.edges_f = B.edges_f;
    Q.edges_d = B.edges_d;
    const size_t smem = batch_smem_bytes<R, DropGeo<R>>(B.threads, B.nt, Q.smem_edges != 0);
    e = cudaFuncSetAttribute(batch_trace_kernel<R, DropGeo<R>>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return (int)e;
    batch_trace_kernel<R, DropGeo<R>><<<B.blocks, B.threads, smem, stream>>>(Q);
    return (int)cudaGetLastError();
}

template <class R> int drop_batch_blocks(uint32_t threads, uint32_t nt)
{
    const size_t smem = batch_smem_bytes<R, DropGeo<R>>(threads, nt, nt + 1 <= kEdgeSmemMax);
    cudaFuncSetAttribute(batch_trace_kernel<R, DropGeo<R>>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, batch_trace_kernel<R, DropGeo<R>>, (int)threads, smem) !=
        cudaSuccess)
        return 0;
    return per_sm;
}

} // namespace icp
