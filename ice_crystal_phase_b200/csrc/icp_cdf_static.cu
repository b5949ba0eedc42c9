// icp_cdf_static.cu -- the CDF builder for callers that cannot allocate device memory.
//
// Some hosts of this library own the whole device memory budget themselves: an embedding
// application with its own pool or caching allocator that has already reserved the device,
// or a plugin/callback context in which allocating is forbidden (it would fail, block on
// the owner's allocator, or fragment its pool).  Such callers can still pass their own
// input and output buffers, but the regular builder also needs scratch memory of its own
// (per-block partial sums, column sums, grid-barrier counters, the audit record and the
// u edges), which it obtains with cudaMalloc.  This variant takes that scratch from one
// file-scope device array instead, so it allocates nothing.
//
// The array is sized for at most ICP_STATIC_MAX_THETA fine u rows, ICP_STATIC_MAX_PHI
// stored phi columns and ICP_STATIC_MAX_BLOCKS cooperative blocks; every GPU that loads the
// library keeps it (about 220 KiB) until the process exits.  All calls share it and it keeps
// the previous call's contents, so the counters that must start at zero are cleared at the
// start of every call, and calls that overlap on the GPU (different streams or threads at
// the same time) race on it.  The device address of the array is looked up once per device
// by the first call on that device (with that device current); make that first call before
// any stream capture begins.
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>

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
constexpr size_t kPartialBytesMax = 160; // >= sizeof(BlockPartial) (checked at run time)
constexpr size_t kScratchBytes = align_up(kPartialOff + kPartialBytesMax * ICP_STATIC_MAX_BLOCKS);

static __device__ __align__(256) unsigned char g_cdf_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
unsigned char* g_scratch_ptr[kMaxDevices] = {};

thread_local char g_msg[512];

int fail(int status, const char* fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_msg, sizeof g_msg, fmt, ap);
    va_end(ap);
    icp::set_last_error(g_msg);
    return status;
}

// Device address of the static scratch on the current device (looked up once per device).
int scratch_address(int device, unsigned char** out)
{
    if (device < 0 || device >= kMaxDevices) return fail(ICP_ERR_INVALID_ARGUMENT, "device ordinal %d unsupported", device);
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_scratch_ptr[device]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_cdf_scratch);
        if (e != cudaSuccess || !p)
            return fail(ICP_ERR_DEVICE, "cudaGetSymbolAddress(static CDF scratch) failed: %s", cudaGetErrorString(e));
        g_scratch_ptr[device] = static_cast<unsigned char*>(p);
    }
    *out = g_scratch_ptr[device];
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
    if (icp::cdf_partial_bytes() > kPartialBytesMax)
        return fail(ICP_ERR_STATE, "static scratch partial slot too small");
    if (!(fwd >= 0) || !(bwd >= 0) || !H::finite(fwd) || !H::finite(bwd))
        return fail(ICP_ERR_INVALID_ARGUMENT, "Invalid pole masses.");
    const double fa = fwd / np, ba = bwd / np;
    if ((fwd > 0 && !(fa > 0)) || (bwd > 0 && !(ba > 0))) return fail(ICP_ERR_AUDIT, "Pole weight underflow.");
    cudaStream_t stream = static_cast<cudaStream_t>(stream_handle);
    int device = 0, sms = 0;
    cudaError_t e = cudaGetDevice(&device);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    if (e != cudaSuccess) return fail(ICP_ERR_DEVICE, "icp_phase_cdf_build_static: %s", cudaGetErrorString(e));
    unsigned char* base = nullptr;
    if (const int r = scratch_address(device, &base)) return r;

    // strip width: smallest whose cooperative grid is co-resident (at least ceil(cp / SMs))
    uint32_t cw = 0;
    for (uint32_t w = cp / (uint32_t)sms + (cp % (uint32_t)sms ? 1u : 0u); w && w <= cp; ++w) {
        const size_t smem = icp::cdf_smem_bytes(ct, cp, w);
        if (smem > 200 * 1024) break;
        const uint32_t blocks = (cp + w - 1) / w;
        if (blocks <= ICP_STATIC_MAX_BLOCKS && (int)blocks <= icp::cdf_max_coresident_blocks(smem, device)) {
            cw = w;
            break;
        }
    }
    if (!cw) return fail(ICP_ERR_CAPACITY, "CDF strip for %u theta rows does not fit shared memory with a co-resident grid", ct);

    // u edges computed on the host into a fixed buffer and copied into the static scratch
    static thread_local double edges[ICP_STATIC_MAX_THETA + 1];
    edges[0] = 0;
    edges[nt] = 1;
    for (uint32_t i = 1; i < nt; ++i) {
        const uint32_t k = i < nt - i ? i : nt - i;
        const double s = std::sin((0.5 * H::kPi) * double(k) / double(nt));
        edges[i] = i <= nt / 2u ? s * s : 1.0 - s * s;
    }
    for (uint32_t i = 0; i < nt; ++i)
        if (!(edges[i + 1] > edges[i]))
            return fail(ICP_ERR_INVALID_ARGUMENT, "Angular cells cannot be represented in binary64.");
    double* d_edges = reinterpret_cast<double*>(base + kEdgesOff);
    auto* d_report = reinterpret_cast<icp::CdfDeviceReport*>(base + kReportOff);
    auto* d_sync = reinterpret_cast<unsigned*>(base + kSyncOff);
    e = cudaMemcpyAsync(d_edges, edges, sizeof(double) * (nt + 1), cudaMemcpyHostToDevice, stream);
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
    L.cw = cw;
    L.fwd_add = fa;
    L.bwd_add = ba;
    const int le = icp::launch_cdf_build(L, stream);
    if (le) return fail(ICP_ERR_DEVICE, "CDF launch failed: %s", cudaGetErrorString((cudaError_t)le));
    icp::CdfDeviceReport r{};
    e = cudaMemcpyAsync(&r, d_report, sizeof r, cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) return fail(ICP_ERR_DEVICE, "icp_phase_cdf_build_static: %s", cudaGetErrorString(e));
    if (r.timeout) return fail(ICP_ERR_TIMEOUT, "CDF grid barrier gave up waiting (co-residency violated?)");
    report->fine_mass = r.fine_mass;
    report->fine_axial = r.fine_axial;
    report->g_source = r.fine_axial / r.fine_mass;
    report->aggregation_relative_error = std::fabs(r.stored_mass / r.fine_mass - 1);
    report->coarsening_tv = r.tv;
    report->l1_error = r.l1;
    report->lost_mass = r.lost;
    report->maximum_cell_error = r.max_err;
    report->cdf_mass = r.recovered;
    report->g_stored = r.axial / r.recovered;
    report->lost_cells = r.lost_cells;
    report->malformed = r.malformed;
    int status = ICP_OK;
    if (r.invalid) status = fail(ICP_ERR_INVALID_ARGUMENT, "Negative/nonfinite mass.");
    else if (!(r.fine_mass > 0) || !H::finite(r.fine_mass) || !H::finite(r.fine_axial))
        status = fail(ICP_ERR_AUDIT, "Empty/nonfinite histogram.");
    else if (!H::finite(report->coarsening_tv) || report->coarsening_tv > p.max_coarsening_tv ||
             report->aggregation_relative_error > 1e-12)
        status = fail(ICP_ERR_AUDIT, "Conservative coarsening audit failed.");
    else if (r.underflow) status = fail(ICP_ERR_AUDIT, "CDF weight underflow.");
    else if (!(r.total > 0) || !H::finite(r.total)) status = fail(ICP_ERR_AUDIT, "Invalid CDF total.");
    else if (r.malformed) status = fail(ICP_ERR_AUDIT, "Malformed CDF; refusing repair.");
    else if (report->l1_error > p.max_l1_error || report->lost_mass > p.max_lost_mass ||
             std::fabs(report->cdf_mass - 1) > 1e-10 || !H::finite(report->g_stored) ||
             !(report->g_stored > -1 && report->g_stored < 1))
        status = fail(ICP_ERR_AUDIT, "CDF mass / HG audit failed.");
    report->status = (uint32_t)status;
    if (status == ICP_OK) icp::set_last_error("");
    return status;
}
