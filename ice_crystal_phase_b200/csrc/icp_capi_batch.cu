// icp_capi_batch.cu -- C ABI of batched drop records (include/icp_b200.h, "batched drop records").
//
// A batch runs as one device sequence: zero the per-record histograms and counters, one
// persistent trace launch over all records fed from the chunk queue, the diffraction rows of
// every record that asks for them (one block per record), and one cooperative CDF build per
// record reading its pole caps and rows on the device.  With use_graph the sequence is
// captured into a CUDA graph; the executable graph of the previous batch is updated in place
// when the shape allows (cudaGraphExecUpdate) and re-instantiated otherwise.  The CPU
// projected-area integrals of all records run on host threads while the device works.
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <future>
#include <thread>
#include <vector>

#include "../../include/icp_b200.h"
#include "../host/icp_drop_host.hpp"
#include "../host/icp_host_math.hpp"
#include "icp_internal.h"

using namespace icp;
using namespace icp::dropx;
namespace H = icp::host;

namespace {

thread_local char g_msg[1024];

int fail(int status, const char* fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_msg, sizeof g_msg, fmt, ap);
    va_end(ap);
    set_last_error(g_msg);
    return status;
}
int ok()
{
    set_last_error("");
    return ICP_OK;
}
#define ICP_CUDA(call)                                                                                  \
    do {                                                                                                \
        const cudaError_t e_ = (call);                                                                  \
        if (e_ != cudaSuccess) return fail(ICP_ERR_DEVICE, "%s failed: %s", #call, cudaGetErrorString(e_)); \
    } while (0)

constexpr uint32_t kDefaultChunk = 8192u;

icp_drop_record record_of(const icp_drop_item& it, const icp_batch_settings& s)
{
    icp_drop_record r{};
    r.radius_mm = it.radius_mm;
    std::memcpy(r.coefficients, it.coefficients, sizeof r.coefficients);
    r.inclination_deg = it.inclination_deg;
    r.exterior_index = s.exterior_index;
    r.interior_index = it.interior_index;
    r.wavelength_nm = it.wavelength_nm;
    r.tail_tolerance = s.tail_tolerance;
    r.balance_tolerance = s.balance_tolerance;
    r.nt = s.nt;
    r.np = s.np;
    r.ct = s.ct;
    r.cp = s.cp;
    r.max_internal_hits = s.max_internal_hits;
    r.precision = s.precision;
    r.rays = it.rays;
    r.seed = it.seed;
    r.diffraction = it.diffraction;
    r.policy = s.policy;
    return r;
}

const BatchState::Tuned* tuned_for(icp_context* c, uint32_t precision, uint32_t nt)
{
    for (const auto& t : c->batch.tuned)
        if (t.precision == precision && t.nt == nt) return &t;
    return nullptr;
}

struct Shape {
    uint32_t threads, chunk, blocks;
};

int launch_shape(icp_context* c, const icp_batch_settings& s, Shape& sh)
{
    const BatchState::Tuned* t = tuned_for(c, s.precision, s.nt);
    sh.threads = s.block_threads ? s.block_threads : (t ? t->threads : 256u);
    sh.chunk = s.chunk_rays ? s.chunk_rays : (t ? t->chunk_rays : kDefaultChunk);
    if (sh.threads < 64 || sh.threads > 256 || sh.threads % 32)
        return fail(ICP_ERR_INVALID_ARGUMENT, "block_threads must be 64..256, multiple of 32");
    if (sh.chunk < 32) return fail(ICP_ERR_INVALID_ARGUMENT, "chunk_rays must be at least 32");
    // a warp flushes its lanes' 32-bit counters once per chunk: keep a chunk within their range
    sh.chunk = (uint32_t)std::max<uint64_t>(32u, std::min<uint64_t>(sh.chunk, lane_rays_max(s.max_internal_hits)));
    int per_sm = drop_batch_blocks_per_sm(s.precision, sh.threads, s.nt);
    if (per_sm <= 0) return fail(ICP_ERR_DEVICE, "batch trace kernel cannot be resident");
    if (s.blocks_per_sm) per_sm = std::min<int>(per_sm, (int)s.blocks_per_sm);
    sh.blocks = (uint32_t)per_sm * (uint32_t)c->sms;
    return ICP_OK;
}

int validate(const icp_drop_item* items, uint32_t count, const icp_batch_settings* s)
{
    if (!items || !count || !s) return fail(ICP_ERR_INVALID_ARGUMENT, "batch: null or empty argument");
    if (s->precision > 1) return fail(ICP_ERR_INVALID_ARGUMENT, "Unknown precision.");
    for (uint32_t i = 0; i < count; ++i) {
        const icp_drop_record r = record_of(items[i], *s);
        if (const int v = validate_record(&r)) return v;
        if (const int v = validate_grid(&r)) return v;
    }
    return ICP_OK;
}

// Enqueues the trace of the whole batch: zeroing, tables, one persistent launch.
int enqueue_trace(icp_context* c, const icp_drop_item* items, uint32_t count, const icp_batch_settings& s,
                  const Shape& sh, std::vector<double>& weights)
{
    const uint64_t cells = (uint64_t)s.nt * s.np;
    const size_t sb = hex_stats_bytes();
    const size_t pb = drop_batch_param_bytes(s.precision);
    BatchState& B = c->batch;
    ICP_CUDA(c->b_mass.ensure(sizeof(double) * cells * count));
    ICP_CUDA(c->b_stats.ensure(sb * count));
    ICP_CUDA(c->b_table.ensure(pb * count));
    ICP_CUDA(c->b_chunks.ensure(sizeof(unsigned long long) * (count + 1)));
    ICP_CUDA(c->b_queue.ensure(sizeof(unsigned long long)));
    ICP_CUDA(c->rec_edges.ensure(sizeof(double) * (s.nt + 1)));
    ICP_CUDA(B.h_table.ensure(pb * count));
    ICP_CUDA(B.h_chunks.ensure(sizeof(unsigned long long) * (count + 1)));
    ICP_CUDA(B.h_edges.ensure(sizeof(double) * (s.nt + 1)));
    std::vector<double> edges;
    if (!H::u_edges(s.nt, edges)) return fail(ICP_ERR_INVALID_ARGUMENT, "Angular cells cannot be represented in binary64.");
    std::memcpy(B.h_edges.ptr, edges.data(), sizeof(double) * (s.nt + 1));
    ICP_CUDA(cudaMemcpyAsync(c->rec_edges.ptr, B.h_edges.ptr, sizeof(double) * (s.nt + 1), cudaMemcpyHostToDevice,
                             c->stream));
    const double* d_edges = (const double*)c->rec_edges.ptr;
    if (s.precision == ICP_FP32)
        if (const int e = ensure_float_edges(c, d_edges, s.nt)) return e;
    auto* chunks = static_cast<unsigned long long*>(B.h_chunks.ptr);
    std::vector<HexLaunch> launches(count);
    weights.assign(count, 0.0);
    chunks[0] = 0;
    for (uint32_t i = 0; i < count; ++i) {
        const icp_drop_record r = record_of(items[i], s);
        icp_grid g;
        grid_of(&r, g);
        double disk = 0;
        if (icp_drop_sampling_area(r.coefficients, r.radius_mm, &disk)) return ICP_ERR_INVALID_ARGUMENT;
        weights[i] = disk / double(r.rays);
        double* mass = (double*)c->b_mass.ptr + cells * i;
        void* stats = (unsigned char*)c->b_stats.ptr + sb * i;
        launches[i] = drop_launch(&r, &g, d_edges, (const float*)c->edges_f.ptr, mass, stats, weights[i], 0u);
        chunks[i + 1] = chunks[i] + (r.rays + sh.chunk - 1) / sh.chunk;
    }
    ICP_CUDA(cudaMemsetAsync(c->b_mass.ptr, 0, sizeof(double) * cells * count, c->stream));
    ICP_CUDA(cudaMemsetAsync(c->b_stats.ptr, 0, sb * count, c->stream));
    ICP_CUDA(cudaMemsetAsync(c->b_queue.ptr, 0, sizeof(unsigned long long), c->stream));
    ICP_CUDA(cudaMemcpyAsync(c->b_chunks.ptr, chunks, sizeof(unsigned long long) * (count + 1), cudaMemcpyHostToDevice,
                             c->stream));
    BatchLaunch L{};
    L.recs = launches.data();
    L.n_records = count;
    L.h_staging = B.h_table.ptr;
    L.d_table = c->b_table.ptr;
    L.d_chunk_begin = (const unsigned long long*)c->b_chunks.ptr;
    L.d_queue = (unsigned long long*)c->b_queue.ptr;
    L.total_chunks = chunks[count];
    L.chunk_rays = sh.chunk;
    L.threads = sh.threads;
    L.blocks = (uint32_t)std::min<unsigned long long>(sh.blocks, std::max<unsigned long long>(1, (chunks[count] + sh.threads / 32 - 1) / (sh.threads / 32)));
    L.nt = s.nt;
    L.edges_d = d_edges;
    L.edges_f = (const float*)c->edges_f.ptr;
    const int e = s.precision == ICP_FP32 ? launch_drop_batch_f32(L, c->stream) : launch_drop_batch_f64(L, c->stream);
    count_launch();
    if (e) return fail(ICP_ERR_DEVICE, "batch trace launch failed: %s", cudaGetErrorString((cudaError_t)e));
    return ICP_OK;
}

// Enqueues everything after the trace: diffraction rows, one CDF per record, read-backs.
int enqueue_finish(icp_context* c, const icp_drop_item* items, uint32_t count, const icp_batch_settings& s,
                   const std::vector<double>& weights, double* d_phi, double* d_theta)
{
    const uint64_t cells = (uint64_t)s.nt * s.np;
    const size_t sb = hex_stats_bytes();
    BatchState& B = c->batch;
    ICP_CUDA(c->b_rows.ensure(sizeof(double) * (s.nt + 1) * count));
    ICP_CUDA(c->b_dargs.ensure(sizeof(DiffractionArgs) * count));
    ICP_CUDA(c->b_reports.ensure_zeroed(sizeof(CdfDeviceReport) * count, c->stream));
    ICP_CUDA(c->b_sync.ensure_zeroed(2 * sizeof(unsigned) * count, c->stream));
    ICP_CUDA(B.h_dargs.ensure(sizeof(DiffractionArgs) * count));
    ICP_CUDA(B.h_stats.ensure(sb * count));
    ICP_CUDA(B.h_reports.ensure(sizeof(CdfDeviceReport) * count));
    ICP_CUDA(B.h_powers.ensure(sizeof(double) * count));
    const double* d_edges = (const double*)c->rec_edges.ptr;
    auto* args = static_cast<DiffractionArgs*>(B.h_dargs.ptr);
    uint32_t nd = 0;
    for (uint32_t i = 0; i < count; ++i) {
        if (!items[i].diffraction) continue;
        DiffractionArgs a{};
        a.edges = d_edges;
        a.rays = (const unsigned long long*)((unsigned char*)c->b_stats.ptr + sb * i) + devstats_rays_word();
        a.missed_offset = devstats_missed_word() - devstats_rays_word();
        a.row_add = (double*)c->b_rows.ptr + (size_t)(s.nt + 1) * i;
        a.power = a.row_add + s.nt;
        a.weight = weights[i];
        a.wavelength_nm = items[i].wavelength_nm;
        a.nt = s.nt;
        a.np = s.np;
        args[nd++] = a;
    }
    if (nd) {
        ICP_CUDA(cudaMemcpyAsync(c->b_dargs.ptr, args, sizeof(DiffractionArgs) * nd, cudaMemcpyHostToDevice, c->stream));
        const int e = launch_diffraction_rows((const DiffractionArgs*)c->b_dargs.ptr, nd, s.nt, c->stream);
        count_launch();
        if (e) return fail(ICP_ERR_DEVICE, "diffraction launch failed: %s", cudaGetErrorString((cudaError_t)e));
    }
    for (uint32_t i = 0; i < count; ++i) {
        const unsigned long long* stats = (const unsigned long long*)((unsigned char*)c->b_stats.ptr + sb * i);
        double* rows = (double*)c->b_rows.ptr + (size_t)(s.nt + 1) * i;
        if (const int e = cdf_enqueue(c, (const double*)c->b_mass.ptr + cells * i, s.nt, s.np, s.ct, s.cp, d_edges, 0.0,
                                      0.0, stats + devstats_fwd_word(), weights[i],
                                      items[i].diffraction ? rows : nullptr, d_phi + (size_t)(s.cp + 1) * i,
                                      d_theta + (size_t)s.cp * (s.ct + 1) * i,
                                      (CdfDeviceReport*)c->b_reports.ptr + i, (unsigned*)c->b_sync.ptr + 2 * i))
            return e;
    }
    ICP_CUDA(cudaMemcpyAsync(B.h_stats.ptr, c->b_stats.ptr, sb * count, cudaMemcpyDeviceToHost, c->stream));
    ICP_CUDA(cudaMemcpyAsync(B.h_reports.ptr, c->b_reports.ptr, sizeof(CdfDeviceReport) * count, cudaMemcpyDeviceToHost,
                             c->stream));
    for (uint32_t i = 0; i < count; ++i)
        if (items[i].diffraction)
            ICP_CUDA(cudaMemcpyAsync(static_cast<double*>(B.h_powers.ptr) + i,
                                     (double*)c->b_rows.ptr + (size_t)(s.nt + 1) * i + s.nt, sizeof(double),
                                     cudaMemcpyDeviceToHost, c->stream));
    return ICP_OK;
}

// Every allocation of a batch, made before any stream capture begins.
int prepare(icp_context* c, uint32_t count, const icp_batch_settings& s)
{
    const uint64_t cells = (uint64_t)s.nt * s.np;
    const size_t sb = hex_stats_bytes();
    const size_t pb = drop_batch_param_bytes(s.precision);
    BatchState& B = c->batch;
    ICP_CUDA(c->b_mass.ensure(sizeof(double) * cells * count));
    ICP_CUDA(c->b_stats.ensure(sb * count));
    ICP_CUDA(c->b_table.ensure(pb * count));
    ICP_CUDA(c->b_chunks.ensure(sizeof(unsigned long long) * (count + 1)));
    ICP_CUDA(c->b_queue.ensure(sizeof(unsigned long long)));
    ICP_CUDA(c->rec_edges.ensure(sizeof(double) * (s.nt + 1)));
    ICP_CUDA(c->edges_f.ensure(sizeof(float) * (s.nt + 1)));
    ICP_CUDA(c->b_rows.ensure(sizeof(double) * (s.nt + 1) * count));
    ICP_CUDA(c->b_dargs.ensure(sizeof(DiffractionArgs) * count));
    ICP_CUDA(c->b_reports.ensure_zeroed(sizeof(CdfDeviceReport) * count, c->stream));
    ICP_CUDA(c->b_sync.ensure_zeroed(2 * sizeof(unsigned) * count, c->stream));
    ICP_CUDA(B.h_table.ensure(pb * count));
    ICP_CUDA(B.h_chunks.ensure(sizeof(unsigned long long) * (count + 1)));
    ICP_CUDA(B.h_edges.ensure(sizeof(double) * (s.nt + 1)));
    ICP_CUDA(B.h_dargs.ensure(sizeof(DiffractionArgs) * count));
    ICP_CUDA(B.h_stats.ensure(sb * count));
    ICP_CUDA(B.h_reports.ensure(sizeof(CdfDeviceReport) * count));
    ICP_CUDA(B.h_powers.ensure(sizeof(double) * count));
    CdfShape sh{};
    const bool tma_ok = s.nt == s.ct && s.np == s.cp && s.np % 2 == 0; // the record histograms are 256-byte aligned
    if (const int e = cdf_shape(c, s.nt, s.np, s.ct, s.cp, tma_ok, sh)) return e;
    ICP_CUDA(c->cdf_partial.ensure(cdf_partial_bytes() * ((s.cp + sh.cw - 1) / sh.cw)));
    ICP_CUDA(c->cdf_colsum.ensure(sizeof(double) * s.cp));
    return ICP_OK;
}

// Runs the enqueued sequence directly or as a (re)captured graph.
template <class F> int run_sequence(icp_context* c, bool graph, F&& enqueue, uint32_t& graph_used)
{
    graph_used = 0;
    if (!graph) return enqueue();
    cudaStreamCaptureMode mode = cudaStreamCaptureModeRelaxed;
    ICP_CUDA(cudaThreadExchangeStreamCaptureMode(&mode));
    cudaError_t e = cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeRelaxed);
    if (e != cudaSuccess) {
        cudaThreadExchangeStreamCaptureMode(&mode);
        return fail(ICP_ERR_DEVICE, "cudaStreamBeginCapture failed: %s", cudaGetErrorString(e));
    }
    const int st = enqueue();
    cudaGraph_t g = nullptr;
    e = cudaStreamEndCapture(c->stream, &g);
    cudaThreadExchangeStreamCaptureMode(&mode);
    if (st) {
        if (g) cudaGraphDestroy(g);
        return st;
    }
    if (e != cudaSuccess || !g) return fail(ICP_ERR_DEVICE, "stream capture failed: %s", cudaGetErrorString(e));
    BatchState& B = c->batch;
    bool updated = false;
    if (B.exec) {
        cudaGraphExecUpdateResultInfo info{};
        updated = cudaGraphExecUpdate(B.exec, g, &info) == cudaSuccess;
        if (!updated) {
            cudaGetLastError();
            cudaGraphExecDestroy(B.exec);
            B.exec = nullptr;
        }
    }
    if (!B.exec) {
        e = cudaGraphInstantiate(&B.exec, g, 0);
        if (e != cudaSuccess) {
            cudaGraphDestroy(g);
            B.exec = nullptr;
            return fail(ICP_ERR_DEVICE, "cudaGraphInstantiate failed: %s", cudaGetErrorString(e));
        }
    }
    cudaGraphDestroy(g);
    e = cudaGraphLaunch(B.exec, c->stream);
    if (e != cudaSuccess) return fail(ICP_ERR_DEVICE, "cudaGraphLaunch failed: %s", cudaGetErrorString(e));
    graph_used = updated ? 2u : 1u;
    return ICP_OK;
}

int batch(icp_context* c, const icp_drop_item* items, uint32_t count, const icp_batch_settings* settings, double* phi,
          double* theta, double* h_u, bool host, icp_drop_report* reports)
{
    if (!c || !reports) return fail(ICP_ERR_INVALID_ARGUMENT, "batch: null argument");
    if (const int v = validate(items, count, settings)) return v;
    const icp_batch_settings& s = *settings;
    ICP_CUDA(cudaSetDevice(c->device));
    Shape sh;
    if (const int e = launch_shape(c, s, sh)) return e;
    double* d_phi = phi;
    double* d_theta = theta;
    if (host) {
        ICP_CUDA(c->b_phi.ensure(sizeof(double) * (s.cp + 1) * count));
        ICP_CUDA(c->b_theta.ensure(sizeof(double) * (size_t)s.cp * (s.ct + 1) * count));
        d_phi = (double*)c->b_phi.ptr;
        d_theta = (double*)c->b_theta.ptr;
    }
    if (const int e = prepare(c, count, s)) return e;
    // the CPU projected areas run while the device works
    std::vector<double> areas(count, 0.0);
    std::vector<int> area_status(count, ICP_OK);
    const unsigned workers = std::max(1u, std::min<unsigned>(count, std::thread::hardware_concurrency()));
    std::vector<std::future<void>> jobs;
    std::vector<double> weights;
    ICP_CUDA(cudaEventRecord(c->ev0, c->stream));
    uint32_t graph_used = 0;
    const int st = run_sequence(
        c, s.use_graph != 0,
        [&]() -> int {
            if (const int e = enqueue_trace(c, items, count, s, sh, weights)) return e;
            return enqueue_finish(c, items, count, s, weights, d_phi, d_theta);
        },
        graph_used);
    if (st) {
        cudaStreamSynchronize(c->stream);
        return st;
    }
    ICP_CUDA(cudaEventRecord(c->ev1, c->stream));
    for (unsigned w = 0; w < workers; ++w)
        jobs.push_back(std::async(std::launch::async, [&, w]() {
            for (uint32_t i = w; i < count; i += workers) {
                const icp_drop_record r = record_of(items[i], s);
                int stt = ICP_OK;
                areas[i] = projected_area_of(&r, stt);
                area_status[i] = stt;
            }
        }));
    for (auto& j : jobs) j.get();
    if (host) {
        ICP_CUDA(cudaMemcpyAsync(phi, d_phi, sizeof(double) * (s.cp + 1) * count, cudaMemcpyDeviceToHost, c->stream));
        ICP_CUDA(cudaMemcpyAsync(theta, d_theta, sizeof(double) * (size_t)s.cp * (s.ct + 1) * count,
                                 cudaMemcpyDeviceToHost, c->stream));
    }
    ICP_CUDA(cudaStreamSynchronize(c->stream));
    float ms = 0;
    cudaEventElapsedTime(&ms, c->ev0, c->ev1);
    if (host) {
        std::vector<double> edges;
        H::u_edges(s.nt, edges);
        const uint32_t dt = s.nt / s.ct;
        for (uint32_t i = 0; i <= s.ct; ++i) h_u[i] = edges[(size_t)i * dt];
    }
    const BatchState& B = c->batch;
    const size_t sb = hex_stats_bytes();
    int first_error = ICP_OK;
    for (uint32_t i = 0; i < count; ++i) {
        icp_drop_report& rep = reports[i];
        std::memset(&rep, 0, sizeof rep);
        const icp_drop_record r = record_of(items[i], s);
        icp_grid g;
        grid_of(&r, g);
        for (int k = 0; k < 3; ++k) {
            rep.ki[k] = g.ki[k];
            rep.e0[k] = g.e0[k];
            rep.e1[k] = g.e1[k];
        }
        double disk = 0;
        icp_drop_sampling_area(r.coefficients, r.radius_mm, &disk);
        rep.sampled_area_mm2 = disk;
        rep.projected_area_mm2 = areas[i];
        rep.seconds_trace = ms * 1e-3; // the whole batch sequence
        const int e = area_status[i] ? area_status[i]
                                     : finish_report(&r, static_cast<const unsigned char*>(B.h_stats.ptr) + sb * i,
                                                     static_cast<const CdfDeviceReport*>(B.h_reports.ptr)[i],
                                                     static_cast<const double*>(B.h_powers.ptr)[i], weights[i], &rep);
        rep.cdf.status = (uint32_t)e;
        if (e && !first_error) first_error = e;
    }
    for (uint32_t i = 0; i < count; ++i)
        if (static_cast<const CdfDeviceReport*>(B.h_reports.ptr)[i].timeout) {
            // a build gave up waiting: its counters stopped mid-way; clear every record's
            if (const int e = cdf_clear(c, c->b_reports.ptr, c->b_sync.ptr, count)) return e;
            break;
        }
    if (first_error) return first_error; // the message of the first failing record stands
    return ok();
}

} // namespace

extern "C" int icp_drop_batch_generate_device(icp_context* c, const icp_drop_item* items, uint32_t count,
                                              const icp_batch_settings* settings, double* d_phi, double* d_theta,
                                              icp_drop_report* reports)
{
    if (!d_phi || !d_theta) return fail(ICP_ERR_INVALID_ARGUMENT, "batch: null output");
    return batch(c, items, count, settings, d_phi, d_theta, nullptr, false, reports);
}

extern "C" int icp_drop_batch_generate(icp_context* c, const icp_drop_item* items, uint32_t count,
                                       const icp_batch_settings* settings, double* h_phi, double* h_theta, double* h_u,
                                       icp_drop_report* reports)
{
    if (!h_phi || !h_theta || !h_u) return fail(ICP_ERR_INVALID_ARGUMENT, "batch: null output");
    return batch(c, items, count, settings, h_phi, h_theta, h_u, true, reports);
}

extern "C" int icp_drop_batch_autotune(icp_context* c, const icp_drop_item* items, uint32_t count,
                                       icp_batch_settings* settings, double* best_rays_per_second)
{
    if (!c || !settings) return fail(ICP_ERR_INVALID_ARGUMENT, "autotune: null argument");
    if (const int v = validate(items, count, settings)) return v;
    ICP_CUDA(cudaSetDevice(c->device));
    // a bounded sample: up to 32 records of the batch, at most 2^21 rays each
    const uint32_t n = std::min<uint32_t>(count, 32u);
    std::vector<icp_drop_item> sample(items, items + n);
    uint64_t rays = 0;
    for (auto& it : sample) {
        it.rays = std::min<uint64_t>(it.rays, 1ull << 21);
        rays += it.rays;
    }
    static const uint32_t kThreads[] = {128u, 256u};
    static const uint32_t kChunks[] = {2048u, 8192u, 32768u};
    double best = 0;
    uint32_t best_t = 256u, best_c = kDefaultChunk;
    for (uint32_t t : kThreads)
        for (uint32_t ch : kChunks) {
            icp_batch_settings s = *settings;
            s.block_threads = t;
            s.chunk_rays = ch;
            Shape sh;
            if (launch_shape(c, s, sh)) continue;
            if (const int e = prepare(c, n, s)) return e;
            std::vector<double> w;
            double secs = 1e30;
            for (int rep = 0; rep < 2; ++rep) { // the second run is timed
                ICP_CUDA(cudaEventRecord(c->ev0, c->stream));
                if (const int e = enqueue_trace(c, sample.data(), n, s, sh, w)) return e;
                ICP_CUDA(cudaEventRecord(c->ev1, c->stream));
                ICP_CUDA(cudaEventSynchronize(c->ev1));
                float ms = 0;
                cudaEventElapsedTime(&ms, c->ev0, c->ev1);
                secs = ms * 1e-3;
            }
            const double rate = double(rays) / secs;
            if (rate > best) {
                best = rate;
                best_t = t;
                best_c = ch;
            }
        }
    auto& tuned = c->batch.tuned;
    tuned.erase(std::remove_if(tuned.begin(), tuned.end(),
                               [&](const BatchState::Tuned& x) { return x.precision == settings->precision && x.nt == settings->nt; }),
                tuned.end());
    tuned.push_back({settings->precision, settings->nt, best_t, best_c});
    settings->block_threads = best_t;
    settings->chunk_rays = best_c;
    if (best_rays_per_second) *best_rays_per_second = best;
    return ok();
}
