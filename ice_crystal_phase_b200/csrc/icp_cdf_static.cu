// icp_cdf_static.cu -- the CDF builder for callers that cannot allocate device memory.
//
// Some hosts of this library own the whole device memory budget themselves: an embedding
// application with its own pool or caching allocator that has already reserved the device,
// or a plugin/callback context in which allocating is forbidden (it would fail, block on
// the owner's allocator, or fragment its pool).  Such callers can still pass their own
// input and output buffers, but the regular builder also needs scratch memory of its own
// (per-block partial sums, column sums, grid-barrier counters, the audit record and the
// u edges), which it obtains with cudaMalloc.  This variant takes that scratch from one
// file-scope device array instead, so it allocates no device memory.
//
// The array holds the u edges of at most ICP_STATIC_MAX_THETA fine rows, the column sums of
// at most ICP_STATIC_MAX_PHI stored columns, the audit record, the two barrier counters and
// the partials of at most ICP_STATIC_MAX_BLOCKS cooperative blocks: ICP_STATIC_SCRATCH_BYTES
// in all (checked below), which every GPU that loads the library keeps until the process
// exits.  All calls share it and it keeps the previous call's contents, so the counters and
// the audit record are cleared at the start of every call, and calls that overlap on the GPU
// (different streams or threads at the same time) race on it.  The host-side name of the
// array is not a device address: its address in the current CUDA context is looked up with
// cudaGetSymbolAddress by the first call in that context (with its device current) and kept
// per context; make that first call before any stream capture begins.  The entry copies the
// u edges from host memory and waits for the stream, so it is not called inside a capture.
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <cuda.h>
#include <mutex>
#include <vector>

#include "../../include/icp_b200.h"
#include "../host/icp_host_math.hpp"
#include "icp_internal.h"

namespace {

namespace H = icp::host;

constexpr size_t kAlign = 256;
constexpr size_t align_up(size_t x) { return (x + kAlign - 1) / kAlign * kAlign; }
constexpr size_t kEdgesOff = 0;
constexpr size_t kColsumOff = align_up(kEdgesOff + sizeof(double) * (ICP_STATIC_MAX_THETA + 1));
constexpr size_t kReportOff = align_up(kColsumOff + sizeof(double) * ICP_STATIC_MAX_PHI);
constexpr size_t kSyncOff = align_up(kReportOff + sizeof(icp::CdfDeviceReport));
constexpr size_t kPartialOff = align_up(kSyncOff + 2 * sizeof(unsigned));
constexpr size_t kScratchBytes = align_up(kPartialOff + icp::kCdfPartialBytes * ICP_STATIC_MAX_BLOCKS);
static_assert(kScratchBytes == ICP_STATIC_SCRATCH_BYTES, "the header states the static scratch size");

static __device__ __align__(256) unsigned char g_cdf_scratch[kScratchBytes];

// Device address of the array per CUDA context (a module is loaded once per context).
struct Known {
    CUcontext ctx;
    unsigned char* ptr;
};
std::mutex g_setup_mutex;
std::vector<Known> g_known;

thread_local char g_msg[512];

// Driver entry points through the runtime (the library does not link libcuda directly).
template <class F> F driver_fn(const char* name)
{
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPoint(name, &p, cudaEnableDefault, &q) != cudaSuccess || q != cudaDriverEntryPointSuccess)
        return nullptr;
    return reinterpret_cast<F>(p);
}
using CtxGetCurrent = CUresult (*)(CUcontext*);
using StreamGetCtx = CUresult (*)(CUstream, CUcontext*);

int fail(int status, const char* fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_msg, sizeof g_msg, fmt, ap);
    va_end(ap);
    icp::set_last_error(g_msg);
    return status;
}

// Address of the static scratch in the current context; the stream must belong to it.
int scratch_address(cudaStream_t stream, unsigned char** out)
{
    int device = 0;
    cudaError_t e = cudaGetDevice(&device);
    if (e != cudaSuccess) return fail(ICP_ERR_DEVICE, "icp_phase_cdf_build_static: %s", cudaGetErrorString(e));
    static const CtxGetCurrent ctx_get_current = driver_fn<CtxGetCurrent>("cuCtxGetCurrent");
    static const StreamGetCtx stream_get_ctx = driver_fn<StreamGetCtx>("cuStreamGetCtx");
    if (!ctx_get_current || !stream_get_ctx)
        return fail(ICP_ERR_DEVICE, "icp_phase_cdf_build_static: CUDA driver entry points unavailable");
    CUcontext ctx = nullptr;
    if (ctx_get_current(&ctx) != CUDA_SUCCESS)
        return fail(ICP_ERR_DEVICE, "icp_phase_cdf_build_static: cuCtxGetCurrent failed");
    if (!ctx) {
        // no context current on this thread yet: the device's primary context (the runtime's)
        e = cudaSetDevice(device);
        if (e != cudaSuccess || ctx_get_current(&ctx) != CUDA_SUCCESS || !ctx)
            return fail(ICP_ERR_DEVICE, "icp_phase_cdf_build_static: no current CUDA context");
    }
    if (stream) {
        CUcontext sctx = nullptr;
        if (stream_get_ctx(reinterpret_cast<CUstream>(stream), &sctx) != CUDA_SUCCESS)
            return fail(ICP_ERR_INVALID_ARGUMENT, "icp_phase_cdf_build_static: the stream is not valid");
        if (sctx != ctx)
            return fail(ICP_ERR_INVALID_ARGUMENT, "icp_phase_cdf_build_static: the stream belongs to another device or "
                        "context than the current one (device %d); make the stream's device current first", device);
    }
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    for (const Known& k : g_known)
        if (k.ctx == ctx) {
            *out = k.ptr;
            return ICP_OK;
        }
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_cdf_scratch);
    if (e != cudaSuccess || !p)
        return fail(ICP_ERR_DEVICE, "cudaGetSymbolAddress(static CDF scratch) failed: %s", cudaGetErrorString(e));
    g_known.push_back({ctx, static_cast<unsigned char*>(p)});
    *out = static_cast<unsigned char*>(p);
    return ICP_OK;
}

} // namespace

extern "C" int icp_phase_cdf_build_static(void* stream_handle, const double* d_values, uint32_t kind, uint32_t nt,
                                          uint32_t np, double fwd, double bwd, uint32_t ct, uint32_t cp,
                                          const icp_cdf_policy* policy, double* d_phi, double* d_theta,
                                          icp_cdf_report* report)
{
    if (!d_values || !d_phi || !d_theta || !report || !policy)
        return fail(ICP_ERR_INVALID_ARGUMENT, "icp_phase_cdf_build_static: null argument");
    std::memset(report, 0, sizeof *report);
    const icp_cdf_policy& p = *policy;
    if (!(H::finite(p.max_l1_error) && p.max_l1_error >= 0 && p.max_l1_error <= 2 && H::finite(p.max_lost_mass) &&
          p.max_lost_mass >= 0 && p.max_lost_mass <= 1 && H::finite(p.max_coarsening_tv) && p.max_coarsening_tv >= 0 &&
          p.max_coarsening_tv <= 1))
        return fail(ICP_ERR_INVALID_ARGUMENT, "Invalid CDF quality policy.");
    if (kind > 1) return fail(ICP_ERR_INVALID_ARGUMENT, "Unknown CDF input kind.");
    if (!nt || !np || (uint64_t)nt * np > 0xffffffffull)
        return fail(ICP_ERR_INVALID_ARGUMENT, "Unsupported phase grid dimensions.");
    if (!ct || !cp || ct > nt || cp > np || nt % ct || np % cp)
        return fail(ICP_ERR_INVALID_ARGUMENT, "Storage dimensions must divide histogram dimensions.");
    if (nt > ICP_STATIC_MAX_THETA || cp > ICP_STATIC_MAX_PHI)
        return fail(ICP_ERR_CAPACITY, "icp_phase_cdf_build_static: %u theta rows / %u phi columns exceed the static scratch "
                    "maximum of %u / %u; use icp_phase_cdf_build", nt, cp, ICP_STATIC_MAX_THETA, ICP_STATIC_MAX_PHI);
    if (!(fwd >= 0) || !(bwd >= 0) || !H::finite(fwd) || !H::finite(bwd))
        return fail(ICP_ERR_INVALID_ARGUMENT, "Invalid pole masses.");
    const double fa = fwd / np, ba = bwd / np;
    if ((fwd > 0 && !(fa > 0)) || (bwd > 0 && !(ba > 0))) return fail(ICP_ERR_AUDIT, "Pole weight underflow.");
    cudaStream_t stream = static_cast<cudaStream_t>(stream_handle);
    unsigned char* base = nullptr;
    if (const int r = scratch_address(stream, &base)) return r;
    int device = 0, sms = 0;
    cudaError_t e = cudaGetDevice(&device);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    if (e != cudaSuccess) return fail(ICP_ERR_DEVICE, "icp_phase_cdf_build_static: %s", cudaGetErrorString(e));

    // launch shape: the regular builder's choice, capped at the static partial slots
    const bool tma_ok = nt == ct && np == cp && np % 2 == 0 && ((uintptr_t)d_values % 16) == 0;
    icp::CdfShape sh{};
    if (icp::cdf_choose_shape(device, sms, nt, np, ct, cp, tma_ok, 1u, ICP_STATIC_MAX_BLOCKS, sh))
        return fail(ICP_ERR_CAPACITY, "CDF strip for %u theta rows does not fit shared memory with a co-resident grid", ct);

    // u edges: the library's helper (make_phase_u_edges), copied into the static scratch
    std::vector<double> edges;
    if (!H::u_edges(nt, edges)) return fail(ICP_ERR_INVALID_ARGUMENT, "Angular cells cannot be represented in binary64.");
    double* d_edges = reinterpret_cast<double*>(base + kEdgesOff);
    auto* d_report = reinterpret_cast<icp::CdfDeviceReport*>(base + kReportOff);
    auto* d_sync = reinterpret_cast<unsigned*>(base + kSyncOff);
    e = cudaMemcpyAsync(d_edges, edges.data(), sizeof(double) * (nt + 1), cudaMemcpyHostToDevice, stream);
    // the previous call's counters and report are still in the array: clear them
    if (e == cudaSuccess) e = cudaMemsetAsync(d_sync, 0, 2 * sizeof(unsigned), stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(d_report, 0, sizeof(icp::CdfDeviceReport), stream);
    if (e != cudaSuccess) return fail(ICP_ERR_DEVICE, "icp_phase_cdf_build_static: %s", cudaGetErrorString(e));

    icp::CdfLaunch L{};
    L.values = d_values;
    L.edges = d_edges;
    L.phi = d_phi;
    L.theta = d_theta;
    L.colsum = reinterpret_cast<double*>(base + kColsumOff);
    L.partial = base + kPartialOff;
    L.report = d_report;
    L.sync = d_sync;
    L.kind = kind;
    L.nt = nt;
    L.np = np;
    L.ct = ct;
    L.cp = cp;
    L.fwd_add = fa;
    L.bwd_add = ba;
    const int le = icp::launch_cdf_build(L, sh, stream);
    if (le) return fail(ICP_ERR_DEVICE, "CDF launch failed: %s", cudaGetErrorString((cudaError_t)le));
    icp::CdfDeviceReport r{};
    e = cudaMemcpyAsync(&r, d_report, sizeof r, cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) return fail(ICP_ERR_DEVICE, "icp_phase_cdf_build_static: %s", cudaGetErrorString(e));
    // the quality gates and report of the regular builder (build_host_cdf's checks)
    return icp::cdf_finish(r, p, report);
}
