// icp_patches.cu -- the drop's outgoing patches from its ray lattice on the device (sm_100a)
// and the C ABI (include/icp_b200.h, "patch build").  Built with -fmad=false: binary32
// products and sums round on their own; the reference's explicit fmaf and nextafterf calls
// are kept, so the arithmetic is its host build's.
//
// A cell of the lattice (four corner rays of one path family) becomes a patch when its four
// rays left the drop (PatchConstruction::make, include/rainbow/patch_geometry.hpp:117-172):
// the outward-rounded interval test certifies one sign of the bilinear map's Jacobian at the
// corners and that the corners lie in their mean direction's hemisphere; certified cells
// whose two-triangle solid angle agrees in sign are regular (positive / negative), the others
// need refinement.  The patches are stored compactly in patch_id order.
//
// Three kernels, none of them with a host round trip (the reference scans its block counts on
// the CPU between its two kernels, device/patch_build.cu:13-77):
//   patch_classify_kernel  one thread per cell: status, a per-block count of patches
//                          (__syncthreads_count) and the status histogram (shared-memory
//                          counters, one global atomic per status per block)
//   patch_scan_kernel      one block: exclusive scan of the block counts, total patch count
//   patch_compact_kernel   one thread per cell: rank inside the block by warp ballots, then
//                          the patch and its padded bounding box written at block offset + rank
//                          (the construction is recomputed rather than staged: ~300 binary32
//                          operations per cell against 56 staged bytes)
#include <cfloat>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>

#include "../../include/icp_b200.h"
#include "icp_internal.h"

using namespace icp;

namespace {

thread_local char g_msg[512];

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

constexpr unsigned kThreads = 256;
constexpr unsigned kScanThreads = 1024;

struct Layout {
    uint32_t width, per_path, cells, cell_count;
    float area;
};

struct F3 {
    float x, y, z;
};
struct Iv {
    float lo, hi;
};
struct Iv3 {
    Iv x, y, z;
};

__device__ __forceinline__ float dot(F3 a, F3 b) { return fmaf(a.x, b.x, fmaf(a.y, b.y, a.z * b.z)); }
__device__ __forceinline__ F3 minus(F3 a, F3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ F3 plus(F3 a, F3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ bool finite32(float x) { return x >= -FLT_MAX && x <= FLT_MAX; }
__device__ __forceinline__ bool finite(F3 a) { return finite32(a.x) && finite32(a.y) && finite32(a.z); }
__device__ __forceinline__ F3 f3(const icp_vec3f& v) { return {v.x, v.y, v.z}; }

// outward-rounded interval arithmetic (one ulp outward after every operation)
__device__ __forceinline__ Iv add(Iv a, Iv b) { return {nextafterf(a.lo + b.lo, -INFINITY), nextafterf(a.hi + b.hi, INFINITY)}; }
__device__ __forceinline__ Iv sub(Iv a, Iv b) { return {nextafterf(a.lo - b.hi, -INFINITY), nextafterf(a.hi - b.lo, INFINITY)}; }
__device__ __forceinline__ Iv mul(Iv a, Iv b)
{
    const float p0 = a.lo * b.lo, p1 = a.lo * b.hi, p2 = a.hi * b.lo, p3 = a.hi * b.hi;
    return {nextafterf(fminf(fminf(p0, p1), fminf(p2, p3)), -INFINITY),
            nextafterf(fmaxf(fmaxf(p0, p1), fmaxf(p2, p3)), INFINITY)};
}
__device__ __forceinline__ Iv3 point(F3 p) { return {{p.x, p.x}, {p.y, p.y}, {p.z, p.z}}; }
__device__ __forceinline__ Iv3 sub(Iv3 a, Iv3 b) { return {sub(a.x, b.x), sub(a.y, b.y), sub(a.z, b.z)}; }
__device__ __forceinline__ Iv3 cross(Iv3 a, Iv3 b)
{
    return {sub(mul(a.y, b.z), mul(a.z, b.y)), sub(mul(a.z, b.x), mul(a.x, b.z)), sub(mul(a.x, b.y), mul(a.y, b.x))};
}
__device__ __forceinline__ Iv dot(Iv3 a, Iv3 b) { return add(add(mul(a.x, b.x), mul(a.y, b.y)), mul(a.z, b.z)); }

// +1 / -1 when the corner Jacobians have one certified sign and every corner lies in the
// hemisphere of the corners' sum; 0 otherwise.
__device__ int certified_orientation(const F3* c)
{
    const Iv3 p0 = point(c[0]), p1 = point(c[1]), p2 = point(c[2]), p3 = point(c[3]);
    const Iv d0 = dot(p0, cross(sub(p1, p0), sub(p2, p0)));
    const Iv d1 = dot(p1, cross(sub(p1, p0), sub(p3, p1)));
    const Iv d2 = dot(p2, cross(sub(p3, p2), sub(p2, p0)));
    const Iv d3 = dot(p3, cross(sub(p3, p2), sub(p3, p1)));
    const bool positive = d0.lo > 0 && d1.lo > 0 && d2.lo > 0 && d3.lo > 0;
    const bool negative = d0.hi < 0 && d1.hi < 0 && d2.hi < 0 && d3.hi < 0;
    if (!positive && !negative) return 0;
    const Iv3 a = point(plus(plus(c[0], c[1]), plus(c[2], c[3])));
    if (!(dot(a, p0).lo > 0 && dot(a, p1).lo > 0 && dot(a, p2).lo > 0 && dot(a, p3).lo > 0)) return 0;
    return positive ? 1 : -1;
}
// x y - z w with the product z w's rounding error added back
__device__ __forceinline__ float difference_of_products(float x, float y, float z, float w)
{
    const float zw = z * w;
    const float residual = fmaf(-z, w, zw);
    return fmaf(x, y, -zw) + residual;
}
__device__ __forceinline__ float determinant(F3 a, F3 b, F3 c)
{
    const F3 u = minus(b, a), v = minus(c, a);
    return fmaf(a.x, difference_of_products(u.y, v.z, u.z, v.y),
                fmaf(a.y, difference_of_products(u.z, v.x, u.x, v.z), a.z * difference_of_products(u.x, v.y, u.y, v.x)));
}
// signed solid angle of a spherical triangle (Van Oosterom & Strackee)
__device__ __forceinline__ float triangle_angle(F3 a, F3 b, F3 c)
{
    const float la = sqrtf(dot(a, a)), lb = sqrtf(dot(b, b)), lc = sqrtf(dot(c, c));
    const float den = fmaf(la, lb * lc, fmaf(dot(a, b), lc, fmaf(dot(b, c), la, dot(c, a) * lb)));
    return 2.0f * atan2f(determinant(a, b, c), den);
}
__device__ __forceinline__ bool usable(const icp_outgoing_vertex& v)
{
    const F3 d = f3(v.direction_drop);
    const float n2 = dot(d, d);
    const icp_field32& f = v.field;
    return finite(f3(v.position_drop)) && finite(d) && finite(f3(v.basis_x)) && fabsf(n2 - 1.0f) <= 0x1p-16f &&
           v.optical_cycles.fraction >= 0.0f && v.optical_cycles.fraction < 1.0f && finite32(f.x.real) &&
           finite32(f.x.imag) && finite32(f.y.real) && finite32(f.y.imag);
}

__device__ void make_patch(const icp_outgoing_vertex* __restrict__ vertices, const Layout& L, uint32_t id,
                           icp_outgoing_patch& patch, icp_patch_aabb& box)
{
    patch = icp_outgoing_patch{};
    box = icp_patch_aabb{};
    patch.patch_id = id;
    patch.incident_area_drop2 = L.area;
    patch.signed_solid_angle_sr = __int_as_float(0x7fc00000);
    const uint32_t family = id / L.cells, cell = id % L.cells;
    const uint32_t ix = cell % (L.width - 1), iy = cell / (L.width - 1);
    const uint32_t first = family * L.per_path + iy * L.width + ix;
    patch.vertex_indices[0] = first;
    patch.vertex_indices[1] = first + 1;
    patch.vertex_indices[2] = first + L.width;
    patch.vertex_indices[3] = first + L.width + 1;
    unsigned valid = 0;
    bool bad_vertex = false, bad_geometry = false;
    F3 corners[4] = {};
    for (unsigned i = 0; i < 4; ++i) {
        const icp_outgoing_vertex& v = vertices[patch.vertex_indices[i]];
        if (v.status == 1u) {
            ++valid;
            bad_geometry |= !usable(v);
            corners[i] = f3(v.direction_drop);
        } else if (v.status != 2u && v.status != 3u) // neither a miss nor total internal reflection
            bad_vertex = true;
    }
    if (bad_vertex) patch.status = 6;
    else if (bad_geometry) patch.status = 7;
    else if (valid == 0) patch.status = 5;
    else if (valid < 4) patch.status = 4;
    else {
        F3 lo = corners[0], hi = corners[0];
        for (unsigned i = 1; i < 4; ++i) {
            lo = {fminf(lo.x, corners[i].x), fminf(lo.y, corners[i].y), fminf(lo.z, corners[i].z)};
            hi = {fmaxf(hi.x, corners[i].x), fmaxf(hi.y, corners[i].y), fmaxf(hi.z, corners[i].z)};
        }
        const float pad = 0x1p-19f;
        box = {nextafterf(lo.x - pad, -INFINITY), nextafterf(lo.y - pad, -INFINITY), nextafterf(lo.z - pad, -INFINITY),
               nextafterf(hi.x + pad, INFINITY), nextafterf(hi.y + pad, INFINITY), nextafterf(hi.z + pad, INFINITY)};
        const int orientation = certified_orientation(corners);
        patch.status = 3; // needs refinement unless certified regular
        if (orientation != 0) {
            const float angle =
                triangle_angle(corners[0], corners[1], corners[3]) + triangle_angle(corners[0], corners[3], corners[2]);
            if (finite32(angle) && angle * float(orientation) > 0.0f) {
                patch.status = orientation > 0 ? 1u : 2u;
                patch.signed_solid_angle_sr = angle;
            }
        }
    }
}
__device__ __forceinline__ bool has_geometry(uint32_t s) { return s >= 1u && s <= 3u; }

__global__ void __launch_bounds__(kThreads) patch_classify_kernel(const icp_outgoing_vertex* __restrict__ vertices,
                                                                  Layout L, uint32_t* __restrict__ statuses,
                                                                  uint32_t* __restrict__ block_counts,
                                                                  unsigned long long* __restrict__ histogram)
{
    __shared__ unsigned counts[8];
    if (threadIdx.x < 8) counts[threadIdx.x] = 0;
    __syncthreads();
    const unsigned long long id = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x;
    bool geometry = false;
    if (id < L.cell_count) {
        icp_outgoing_patch p;
        icp_patch_aabb b;
        make_patch(vertices, L, uint32_t(id), p, b);
        statuses[id] = p.status;
        atomicAdd(&counts[p.status & 7u], 1u);
        geometry = has_geometry(p.status);
    }
    const int block_total = __syncthreads_count(geometry);
    if (threadIdx.x == 0) block_counts[blockIdx.x] = uint32_t(block_total);
    if (threadIdx.x < 8 && counts[threadIdx.x]) atomicAdd(&histogram[threadIdx.x], (unsigned long long)counts[threadIdx.x]);
}

// Exclusive scan of n block counts in place; total written to *total.
__global__ void __launch_bounds__(kScanThreads) patch_scan_kernel(uint32_t* __restrict__ counts, uint32_t n,
                                                                  uint32_t* __restrict__ total)
{
    __shared__ uint32_t warp_sums[kScanThreads / 32];
    __shared__ uint32_t carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    const unsigned lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    for (uint32_t base = 0; base < n; base += kScanThreads) {
        const uint32_t i = base + threadIdx.x;
        const uint32_t x = i < n ? counts[i] : 0u;
        uint32_t incl = x;
        for (unsigned d = 1; d < 32; d *= 2) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, incl, d);
            if (lane >= d) incl += y;
        }
        if (lane == 31) warp_sums[warp] = incl;
        __syncthreads();
        if (warp == 0) {
            uint32_t w = warp_sums[lane];
            for (unsigned d = 1; d < 32; d *= 2) {
                const uint32_t y = __shfl_up_sync(0xffffffffu, w, d);
                if (lane >= d) w += y;
            }
            warp_sums[lane] = w; // inclusive over warps
        }
        __syncthreads();
        const uint32_t before = carry + (warp ? warp_sums[warp - 1] : 0u) + incl - x;
        if (i < n) counts[i] = before;
        __syncthreads();
        if (threadIdx.x == kScanThreads - 1) carry += warp_sums[kScanThreads / 32 - 1];
        __syncthreads();
    }
    if (threadIdx.x == 0) *total = carry;
}

__global__ void __launch_bounds__(kThreads) patch_compact_kernel(const icp_outgoing_vertex* __restrict__ vertices,
                                                                 Layout L, const uint32_t* __restrict__ statuses,
                                                                 const uint32_t* __restrict__ offsets,
                                                                 icp_outgoing_patch* __restrict__ patches,
                                                                 icp_patch_aabb* __restrict__ boxes)
{
    __shared__ uint32_t warp_counts[kThreads / 32];
    const unsigned long long id = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x;
    const bool active = id < L.cell_count && has_geometry(statuses[id]);
    const unsigned lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    const unsigned mask = __ballot_sync(0xffffffffu, active);
    if (lane == 0) warp_counts[warp] = __popc(mask);
    __syncthreads();
    if (!active) return;
    uint32_t rank = __popc(mask & ((1u << lane) - 1u));
    for (unsigned w = 0; w < warp; ++w) rank += warp_counts[w];
    icp_outgoing_patch p;
    icp_patch_aabb b;
    make_patch(vertices, L, uint32_t(id), p, b);
    const uint32_t at = offsets[blockIdx.x] + rank;
    patches[at] = p;
    if (boxes) boxes[at] = b;
}

} // namespace

extern "C" int icp_patch_build(icp_context* ctx, const icp_outgoing_vertex* d_vertices, uint32_t grid_width,
                               uint32_t grid_height, float grid_half_extent, icp_outgoing_patch* d_patches,
                               icp_patch_aabb* d_aabbs, uint32_t* d_statuses, uint32_t* patch_count,
                               uint64_t histogram[8])
{
    if (!ctx || !d_vertices || !d_patches || !patch_count)
        return fail(ICP_ERR_INVALID_ARGUMENT, "icp_patch_build: null argument");
    // PatchBuildLayout::try_make (include/rainbow/outgoing_patch.hpp:59-76)
    if (grid_width < 2 || grid_height < 2 || !(grid_half_extent > 0.0f) || !(grid_half_extent <= FLT_MAX))
        return fail(ICP_ERR_INVALID_ARGUMENT, "Invalid patch lattice layout.");
    const uint64_t vertices = uint64_t(grid_width) * grid_height, cells = uint64_t(grid_width - 1) * (grid_height - 1);
    if (vertices > 0xffffffffull / 4u || cells > 0xffffffffull / 4u)
        return fail(ICP_ERR_INVALID_ARGUMENT, "Invalid patch lattice layout.");
    const float du = 2.0f * grid_half_extent / float(grid_width - 1), dv = 2.0f * grid_half_extent / float(grid_height - 1);
    const float area = du * dv;
    if (!(area > 0.0f && area <= FLT_MAX)) return fail(ICP_ERR_INVALID_ARGUMENT, "Invalid patch lattice layout.");
    const Layout L{grid_width, uint32_t(vertices), uint32_t(cells), uint32_t(4 * cells), area};
    const uint32_t blocks = uint32_t((uint64_t(L.cell_count) + kThreads - 1) / kThreads);
    // scratch: statuses (unless given), block counts / offsets, total, histogram
    const size_t status_bytes = d_statuses ? 0 : size_t(L.cell_count) * 4;
    const size_t count_bytes = (size_t(blocks) + 2) * 4;
    const size_t hist_off = (status_bytes + count_bytes + 7) & ~size_t(7);
    ICP_CUDA(cudaSetDevice(ctx->device));
    ICP_CUDA(ctx->patches.ensure(hist_off + 8 * sizeof(unsigned long long)));
    char* base = static_cast<char*>(ctx->patches.ptr);
    uint32_t* statuses = d_statuses ? d_statuses : reinterpret_cast<uint32_t*>(base);
    uint32_t* counts = reinterpret_cast<uint32_t*>(base + status_bytes);
    uint32_t* total = counts + blocks;
    auto* hist = reinterpret_cast<unsigned long long*>(base + hist_off);
    ICP_CUDA(cudaMemsetAsync(hist, 0, 8 * sizeof(unsigned long long), ctx->stream));
    patch_classify_kernel<<<blocks, kThreads, 0, ctx->stream>>>(d_vertices, L, statuses, counts, hist);
    ICP_CUDA(cudaGetLastError());
    count_launch();
    patch_scan_kernel<<<1, kScanThreads, 0, ctx->stream>>>(counts, blocks, total);
    ICP_CUDA(cudaGetLastError());
    count_launch();
    patch_compact_kernel<<<blocks, kThreads, 0, ctx->stream>>>(d_vertices, L, statuses, counts, d_patches, d_aabbs);
    ICP_CUDA(cudaGetLastError());
    count_launch();
    unsigned long long h[8];
    ICP_CUDA(cudaMemcpyAsync(patch_count, total, 4, cudaMemcpyDeviceToHost, ctx->stream));
    ICP_CUDA(cudaMemcpyAsync(h, hist, sizeof h, cudaMemcpyDeviceToHost, ctx->stream));
    ICP_CUDA(cudaStreamSynchronize(ctx->stream));
    if (histogram)
        for (unsigned k = 0; k < 8; ++k) histogram[k] = h[k];
    return ok();
}
