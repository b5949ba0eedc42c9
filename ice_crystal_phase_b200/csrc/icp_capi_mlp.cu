// icp_capi_mlp.cu -- C ABI of the learned surrogate (include/icp_b200.h, "surrogate"): the
// record / cell feature rows (host, FP64 rounded to FP32 then BF16), the parameter store
// (FP32 master copy, BF16 copies for the tensor cores, Adam moments), and the device sequences
// of one training step, a prediction and a generated record.
//
// Training step over R records (M = R * nt * np rows, H hidden units, K0 input width):
//   X, XT                          feature rows (row- and column-major)
//   L1  X  W1^T  (kHidden)         z1, h1, h1T
//   L2  h1 W2^T  (kHidden)         z2, h2, h2T
//   L3  h2 W3^T  (kHead)           z3, y = silu(z3) . w4 + head bias
//   softmax per record             dy = (softmax(y) - p) / R, KL loss
//   head backward                  dz3, dz3T, dw4, db3
//   dW3 = dz3T h2T^T (split-K)     dz2 = (dz3 W3) silu'(z2)  -> dz2, dz2T, db2     (kBackprop)
//   dW2 = dz2T h1T^T (split-K)     dz1 = (dz2 W2) silu'(z1)  -> dz1T, db1           (kBackprop)
//   dW1 = dz1T XT^T  (split-K)     Adam, BF16 copies of W1, W2, W3, W2^T, W3^T
// A generated record: L1, L2, L3 with the head writing exp(y) as the FP64 cell mass, then the
// cooperative CDF build of each record.
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
#include "icp_mlp.h"

using namespace icp;
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
#define ICP_TRY(expr)                                                                                   \
    do {                                                                                                \
        const int r_ = (expr);                                                                          \
        if (r_) return r_;                                                                              \
    } while (0)

// Runs the enqueued kernels, then reads the error word the bounded waits set.
int finish(icp_context* c, const char* what)
{
    unsigned err = 0;
    ICP_CUDA(cudaMemcpyAsync(&err, c->mlp_error.ptr, sizeof err, cudaMemcpyDeviceToHost, c->stream));
    ICP_CUDA(cudaStreamSynchronize(c->stream));
    if (err) return fail(ICP_ERR_TIMEOUT, "%s: a tensor-core pipeline wait gave up (code %u)", what, err);
    return ok();
}

// Round to nearest even, FP32 -> BF16 bits.
uint16_t bf16_bits(float f)
{
    uint32_t u;
    std::memcpy(&u, &f, 4);
    if ((u & 0x7fffffffu) > 0x7f800000u) return 0x7fc0u;
    u += 0x7fffu + ((u >> 16) & 1u);
    return (uint16_t)(u >> 16);
}
uint16_t feature(double x) { return bf16_bits((float)x); }
double unit(double x, const double r[2]) { return 2.0 * (x - r[0]) / (r[1] - r[0]) - 1.0; }

bool config_valid(const icp_surrogate_config* g)
{
    if (!g || !g->nt || !g->np || ((uint64_t)g->nt * g->np) % 256u || (uint64_t)g->nt * g->np > (1u << 24)) return false;
    if (g->hidden != 128 && g->hidden != 256) return false;
    if (g->input_width != 64 && g->input_width != 128) return false;
    if (g->axis_harmonics % 8u) return false;
    if (4u + 2u * g->theta_frequencies + g->phi_frequencies + g->axis_harmonics > g->input_width - 16u) return false;
    if (!g->max_records || g->max_records > 256) return false;
    // the rows of a call (records x cells) are 32-bit GEMM sizes and signed 32-bit TMA coordinates
    if ((uint64_t)g->max_records * g->nt * g->np > (1ull << 31)) return false;
    const double* r[3] = {g->log_radius_mm, g->wavelength_nm, g->log_wavelength_over_radius};
    for (auto* x : r)
        if (!(std::isfinite(x[0]) && std::isfinite(x[1]) && x[1] > x[0])) return false;
    if (!(std::isfinite(g->index_center) && g->index_scale > 0 && std::isfinite(g->index_scale))) return false;
    for (double s : g->coefficient_scale)
        if (!std::isfinite(s)) return false;
    return true;
}

bool item_valid(const icp_drop_item& it)
{
    return std::isfinite(it.radius_mm) && it.radius_mm > 0 && std::isfinite(it.wavelength_nm) && it.wavelength_nm > 0 &&
           std::isfinite(it.inclination_deg) && std::isfinite(it.interior_index);
}

void record_row(const icp_surrogate_config& g, const icp_drop_item& it, uint16_t* out)
{
    const double deg = it.inclination_deg * (H::kPi / 180.0);
    double f[16] = {};
    f[0] = unit(std::log(it.radius_mm), g.log_radius_mm);
    f[1] = unit(it.wavelength_nm, g.wavelength_nm);
    f[2] = it.inclination_deg / 90.0;
    f[3] = std::sin(deg);
    f[4] = std::cos(deg);
    f[5] = unit(std::log(it.wavelength_nm * 1e-6 / it.radius_mm), g.log_wavelength_over_radius);
    f[6] = (it.interior_index - g.index_center) / g.index_scale;
    for (int n = 0; n < 8; ++n) f[7 + n] = it.coefficients[n] * g.coefficient_scale[n];
    for (int k = 0; k < 16; ++k) out[k] = feature(f[k]);
}

// Page-locked host staging: copies from it are asynchronous, so a call enqueues its work after
// the forward pass without waiting for it.
struct PinnedHost {
    void* ptr = nullptr;
    size_t bytes = 0;
    cudaError_t ensure(size_t n)
    {
        if (n <= bytes) return cudaSuccess;
        release();
        const cudaError_t e = cudaHostAlloc(&ptr, n, cudaHostAllocDefault);
        if (e == cudaSuccess) bytes = n;
        else ptr = nullptr;
        return e;
    }
    void release()
    {
        if (ptr) cudaFreeHost(ptr);
        ptr = nullptr;
        bytes = 0;
    }
};

} // namespace

struct icp_surrogate {
    icp_context* c = nullptr;
    icp_surrogate_config cfg{};
    uint32_t H = 0, K0 = 0, C = 0, R = 0;
    uint64_t n_params = 0;
    float head_b = 0.0f;
    uint32_t o_w1 = 0, o_b1 = 0, o_w2 = 0, o_b2 = 0, o_w3 = 0, o_b3 = 0, o_w4 = 0, o_hb = 0;
    Scratch params, grads, adam_m, adam_v, wbf, cells, edges, rec16, loss;
    Scratch X, XT, z1, h1, h1T, z2, h2, h2T, z3, y, dy, dz3, dz3T, dz2, dz2T, dz1T, mass, reports, sync;
    Scratch mass_sum, dfrac, drows, cellgeo, recgeo, xcells;
    std::vector<double> h_edges;
    std::vector<uint16_t> h_rec;
    std::vector<double> h_recgeo;
    PinnedHost h_frac, h_reports; // diffraction fractions and CDF reports of a generate call
    ~icp_surrogate()
    {
        h_frac.release();
        h_reports.release();
        Scratch* all[] = {&params, &grads, &adam_m, &adam_v, &wbf, &cells, &edges, &rec16, &loss, &X, &XT, &z1, &h1,
                          &h1T, &z2, &h2, &h2T, &z3, &y, &dy, &dz3, &dz3T, &dz2, &dz2T, &dz1T, &mass, &reports, &sync,
                          &mass_sum, &dfrac, &drows, &cellgeo, &recgeo, &xcells};
        for (Scratch* s : all) s->release();
    }
    float* P(uint32_t o) const { return (float*)params.ptr + o; }
    float* G(uint32_t o) const { return (float*)grads.ptr + o; }
    __nv_bfloat16* w1b() const { return (__nv_bfloat16*)wbf.ptr; }
    __nv_bfloat16* w2b() const { return w1b() + (size_t)H * K0; }
    __nv_bfloat16* w3b() const { return w2b() + (size_t)H * H; }
    __nv_bfloat16* w2t() const { return w3b() + (size_t)H * H; }
    __nv_bfloat16* w3t() const { return w2t() + (size_t)H * H; }
};

namespace {

template <class T> T* as(const Scratch& s) { return static_cast<T*>(s.ptr); }

int check_call(icp_surrogate* s, const icp_drop_item* items, uint32_t count)
{
    if (!s || !items) return fail(ICP_ERR_INVALID_ARGUMENT, "surrogate: null argument");
    if (!count || count > s->R) return fail(ICP_ERR_INVALID_ARGUMENT, "surrogate: 1 to %u records per call", s->R);
    for (uint32_t i = 0; i < count; ++i)
        if (!item_valid(items[i])) return fail(ICP_ERR_INVALID_ARGUMENT, "surrogate: record %u has invalid parameters", i);
    return ICP_OK;
}

// Inference runs as one fused kernel that builds its own input rows (mlp::forward_fused).
bool fused_inference(const icp_surrogate* s) { return mlp::fused_shape(s->K0, s->H); }

// Record feature rows to the device and the feature matrix (XT too when training; no matrix
// when `rows` is false: the fused inference pass builds the rows itself).
int enqueue_features(icp_surrogate* s, const icp_drop_item* items, uint32_t count, bool training, bool rows = true)
{
    icp_context* c = s->c;
    s->h_rec.resize((size_t)16 * count);
    s->h_recgeo.resize((size_t)2 * count);
    for (uint32_t i = 0; i < count; ++i) {
        record_row(s->cfg, items[i], s->h_rec.data() + 16 * i);
        const double deg = items[i].inclination_deg * (H::kPi / 180.0);
        s->h_recgeo[2 * i] = std::sin(deg);
        s->h_recgeo[2 * i + 1] = std::cos(deg);
    }
    const uint64_t M = (uint64_t)count * s->C;
    ICP_CUDA(s->rec16.ensure(32u * s->R));
    ICP_CUDA(s->recgeo.ensure(16u * s->R));
    ICP_CUDA(cudaMemcpyAsync(s->rec16.ptr, s->h_rec.data(), 32u * count, cudaMemcpyHostToDevice, c->stream));
    ICP_CUDA(cudaMemcpyAsync(s->recgeo.ptr, s->h_recgeo.data(), 16u * count, cudaMemcpyHostToDevice, c->stream));
    if (!rows) return ICP_OK;
    ICP_CUDA(s->X.ensure(2 * M * s->K0));
    if (training) ICP_CUDA(s->XT.ensure(2 * M * s->K0));
    const int e = mlp::launch_features(as<__nv_bfloat16>(s->rec16), as<__nv_bfloat16>(s->cells), count, s->C, s->K0,
                                       s->cfg.axis_harmonics, as<double>(s->recgeo), as<double>(s->cellgeo),
                                       as<__nv_bfloat16>(s->X), training ? as<__nv_bfloat16>(s->XT) : nullptr,
                                       c->stream);
    count_launch();
    if (training) count_launch();
    if (e) return fail(ICP_ERR_DEVICE, "feature launch failed (%d)", e);
    return ICP_OK;
}

int run_gemm(icp_surrogate* s, const void* A, const void* B, mlp::GemmArgs g, int epi, uint32_t splits)
{
    g.error = (unsigned*)s->c->mlp_error.ptr;
    const int e = mlp::gemm(A, B, g, epi, splits, s->c->stream);
    count_launch();
    if (e) return fail(ICP_ERR_DEVICE, "surrogate GEMM launch failed (%d)", e);
    return ICP_OK;
}

mlp::GemmArgs layer(uint64_t M, uint32_t N, uint32_t K)
{
    mlp::GemmArgs g{};
    g.M = (uint32_t)M;
    g.N = N;
    g.K = K;
    g.ld_t = (uint32_t)M;
    return g;
}

// Forward pass.  training: keep z1, z2, z3 and the column-major activations; else the head
// writes y (logits) or exp(y) (mass).
int enqueue_forward(icp_surrogate* s, uint32_t count, bool training, float* y_out, double* mass_out,
                    double* mass_sum = nullptr)
{
    const uint64_t M = (uint64_t)count * s->C;
    const uint32_t Hn = s->H;
    if (!training && fused_inference(s)) {
        // inference: input rows, the three layers and the head in one kernel, all kept on chip
        mlp::FusedArgs f{};
        f.M = (uint32_t)M;
        f.K0 = s->K0;
        f.P = s->cfg.axis_harmonics;
        f.rec16 = as<__nv_bfloat16>(s->rec16);
        f.xcells = as<__nv_bfloat16>(s->xcells);
        f.recgeo = as<double>(s->recgeo);
        f.cellgeo = as<double>(s->cellgeo);
        f.b1 = s->P(s->o_b1);
        f.b2 = s->P(s->o_b2);
        f.b3 = s->P(s->o_b3);
        f.head_w = s->P(s->o_w4);
        f.head_b = s->head_b;
        f.out_y = y_out;
        f.out_mass = mass_out;
        f.out_mass_sum = mass_sum;
        f.record_rows = s->C;
        f.error = (unsigned*)s->c->mlp_error.ptr;
        const int e = mlp::forward_fused(s->w1b(), s->w2b(), s->w3b(), f, s->c->stream);
        count_launch();
        if (e) return fail(ICP_ERR_DEVICE, "surrogate forward launch failed (%d)", e);
        return ICP_OK;
    }
    const size_t act = 2 * M * Hn;
    ICP_CUDA(s->h1.ensure(act));
    ICP_CUDA(s->h2.ensure(act));
    if (training) {
        Scratch* t[] = {&s->z1, &s->h1T, &s->z2, &s->h2T, &s->z3};
        for (Scratch* x : t) ICP_CUDA(x->ensure(act));
    }
    mlp::GemmArgs g = layer(M, Hn, s->K0);
    g.bias = s->P(s->o_b1);
    g.out_h = as<__nv_bfloat16>(s->h1);
    if (training) {
        g.out_z = as<__nv_bfloat16>(s->z1);
        g.out_hT = as<__nv_bfloat16>(s->h1T);
    }
    const int hid = training ? mlp::kHiddenTrain : mlp::kHidden;
    ICP_TRY(run_gemm(s, s->X.ptr, s->w1b(), g, hid, 1));
    g = layer(M, Hn, Hn);
    g.bias = s->P(s->o_b2);
    g.out_h = as<__nv_bfloat16>(s->h2);
    if (training) {
        g.out_z = as<__nv_bfloat16>(s->z2);
        g.out_hT = as<__nv_bfloat16>(s->h2T);
    }
    ICP_TRY(run_gemm(s, s->h1.ptr, s->w2b(), g, hid, 1));
    g = layer(M, Hn, Hn);
    g.bias = s->P(s->o_b3);
    g.head_w = s->P(s->o_w4);
    g.head_b = s->head_b;
    if (training) g.out_z = as<__nv_bfloat16>(s->z3);
    g.out_y = y_out;
    g.out_mass = mass_out;
    g.out_mass_sum = mass_sum;
    g.record_rows = s->C;
    return run_gemm(s, s->h2.ptr, s->w3b(), g, training ? mlp::kHeadTrain : mlp::kHead, 1);
}

int enqueue_loss(icp_surrogate* s, uint32_t count, const float* d_target)
{
    const uint64_t M = (uint64_t)count * s->C;
    ICP_CUDA(s->dy.ensure(4 * M));
    const int e = mlp::launch_softmax_loss(as<float>(s->y), d_target, count, s->C, 1.0f / (float)count, as<float>(s->dy),
                                           as<double>(s->loss), s->c->stream);
    count_launch();
    if (e) return fail(ICP_ERR_DEVICE, "softmax launch failed (%d)", e);
    return ICP_OK;
}

int enqueue_backward(icp_surrogate* s, uint32_t count)
{
    icp_context* c = s->c;
    const uint64_t M = (uint64_t)count * s->C;
    const uint32_t Hn = s->H;
    const size_t act = 2 * M * Hn;
    Scratch* t[] = {&s->dz3, &s->dz3T, &s->dz2, &s->dz2T, &s->dz1T};
    for (Scratch* x : t) ICP_CUDA(x->ensure(act));
    ICP_CUDA(cudaMemsetAsync(s->grads.ptr, 0, 4 * s->n_params, c->stream));
    int e = mlp::launch_head_backward(as<__nv_bfloat16>(s->z3), as<float>(s->dy), s->P(s->o_w4), (uint32_t)M, Hn,
                                      as<__nv_bfloat16>(s->dz3), as<__nv_bfloat16>(s->dz3T), s->G(s->o_w4),
                                      s->G(s->o_b3), c->stream);
    count_launch();
    if (e) return fail(ICP_ERR_DEVICE, "head backward launch failed (%d)", e);
    // the weight-gradient GEMMs have M = H <= 256 rows, which one CTA covers (two row tiles share
    // each B chunk): one CTA per SM, each over an equal share of the batch's rows
    const uint32_t splits = std::max<uint32_t>(1u, (uint32_t)c->sms);
    // dW3 = dz3^T h2
    mlp::GemmArgs g = layer(Hn, Hn, (uint32_t)M);
    g.out_f32 = s->G(s->o_w3);
    g.ld_out = Hn;
    ICP_TRY(run_gemm(s, s->dz3T.ptr, s->h2T.ptr, g, mlp::kAtomicF32, splits));
    // dz2 = (dz3 W3) * silu'(z2), db2
    g = layer(M, Hn, Hn);
    g.z_prev = as<__nv_bfloat16>(s->z2);
    g.out_dz = as<__nv_bfloat16>(s->dz2);
    g.out_dzT = as<__nv_bfloat16>(s->dz2T);
    g.out_db = s->G(s->o_b2);
    ICP_TRY(run_gemm(s, s->dz3.ptr, s->w3t(), g, mlp::kBackprop, 1));
    // dW2 = dz2^T h1
    g = layer(Hn, Hn, (uint32_t)M);
    g.out_f32 = s->G(s->o_w2);
    g.ld_out = Hn;
    ICP_TRY(run_gemm(s, s->dz2T.ptr, s->h1T.ptr, g, mlp::kAtomicF32, splits));
    // dz1 = (dz2 W2) * silu'(z1), db1 (only the column-major copy is read afterwards)
    g = layer(M, Hn, Hn);
    g.z_prev = as<__nv_bfloat16>(s->z1);
    g.out_dzT = as<__nv_bfloat16>(s->dz1T);
    g.out_db = s->G(s->o_b1);
    ICP_TRY(run_gemm(s, s->dz2.ptr, s->w2t(), g, mlp::kBackprop, 1));
    // dW1 = dz1^T X
    g = layer(Hn, s->K0, (uint32_t)M);
    g.out_f32 = s->G(s->o_w1);
    g.ld_out = s->K0;
    return run_gemm(s, s->dz1T.ptr, s->XT.ptr, g, mlp::kAtomicF32, splits);
}

int refresh_weights(icp_surrogate* s)
{
    mlp::WeightViews w{};
    w.w1 = s->P(s->o_w1);
    w.w2 = s->P(s->o_w2);
    w.w3 = s->P(s->o_w3);
    w.w1b = s->w1b();
    w.w2b = s->w2b();
    w.w3b = s->w3b();
    w.w2t = s->w2t();
    w.w3t = s->w3t();
    w.H = s->H;
    w.K0 = s->K0;
    const int e = mlp::launch_weight_copies(w, s->c->stream);
    count_launch();
    if (e) return fail(ICP_ERR_DEVICE, "weight copy launch failed (%d)", e);
    return ICP_OK;
}

int begin(icp_surrogate* s)
{
    ICP_CUDA(cudaSetDevice(s->c->device));
    ICP_CUDA(s->c->mlp_error.ensure(sizeof(unsigned)));
    ICP_CUDA(cudaMemsetAsync(s->c->mlp_error.ptr, 0, sizeof(unsigned), s->c->stream));
    return ICP_OK;
}

// Forward, loss and backward of one batch of records (the gradient left in s->grads).
int gradient_pass(icp_surrogate* s, const icp_drop_item* items, uint32_t count, const float* d_target)
{
    ICP_TRY(begin(s));
    ICP_CUDA(s->y.ensure(4 * (uint64_t)count * s->C));
    ICP_TRY(enqueue_features(s, items, count, true));
    ICP_TRY(enqueue_forward(s, count, true, as<float>(s->y), nullptr));
    ICP_TRY(enqueue_loss(s, count, d_target));
    return enqueue_backward(s, count);
}

int read_loss(icp_surrogate* s, uint32_t count, double* loss)
{
    std::vector<double> l(count);
    ICP_CUDA(cudaMemcpyAsync(l.data(), s->loss.ptr, sizeof(double) * count, cudaMemcpyDeviceToHost, s->c->stream));
    ICP_TRY(finish(s->c, "surrogate"));
    double sum = 0;
    for (double v : l) sum += v;
    if (loss) *loss = sum / count;
    if (!std::isfinite(sum)) return fail(ICP_ERR_AUDIT, "surrogate: non-finite loss");
    return ok();
}

// Per-cell diffraction fractions of one record: rows[i] / (np * A) for the Fraunhofer rows of
// the circle of the record's projected area A (CPU FP64), so that the diffraction adds as much
// power as the geometric part carries; zero without diffraction.
int diffraction_fractions(const icp_surrogate* s, const icp_drop_item& it, double* out)
{
    const uint32_t nt = s->cfg.nt;
    std::fill(out, out + nt, 0.0);
    if (!it.diffraction) return ICP_OK;
    double k[3], e0[3], e1[3], area = 0;
    if (const int st = icp_drop_frame(it.inclination_deg, k, e0, e1)) return st;
    if (const int st = icp_drop_projected_area(it.coefficients, it.radius_mm, k, &area)) return st;
    if (!(it.wavelength_nm > 0)) return fail(ICP_ERR_INVALID_ARGUMENT, "Diffraction needs a positive wavelength.");
    const std::vector<double> rows = H::diffraction_rows(s->h_edges, area, it.wavelength_nm);
    const double scale = 1.0 / ((double)s->cfg.np * area);
    for (uint32_t i = 0; i < nt; ++i) out[i] = rows[i] * scale;
    return ICP_OK;
}

} // namespace

extern "C" {

int icp_surrogate_default_config(icp_surrogate_config* g)
{
    if (!g) return fail(ICP_ERR_INVALID_ARGUMENT, "icp_surrogate_default_config: null argument");
    std::memset(g, 0, sizeof *g);
    g->nt = 256;
    g->np = 512;
    g->hidden = 256;
    g->input_width = 128;
    g->theta_frequencies = 40;
    g->phi_frequencies = 12;
    g->axis_harmonics = 16;
    g->max_records = 16;
    g->log_radius_mm[0] = std::log(0.1);
    g->log_radius_mm[1] = std::log(3.0);
    g->wavelength_nm[0] = 400.0;
    g->wavelength_nm[1] = 700.0;
    g->log_wavelength_over_radius[0] = std::log(400e-6 / 3.0);
    g->log_wavelength_over_radius[1] = std::log(700e-6 / 0.1);
    g->index_center = 1.337;
    g->index_scale = 0.0065;
    const double scale[8] = {12, 20, 5, 40, 33, 60, 400, 140};
    std::memcpy(g->coefficient_scale, scale, sizeof scale);
    return ok();
}

uint64_t icp_surrogate_parameter_count(const icp_surrogate_config* g)
{
    if (!config_valid(g)) return 0;
    const uint64_t h = g->hidden;
    return h * g->input_width + 2 * h * h + 4 * h + 1;
}

int icp_surrogate_record_features(const icp_surrogate_config* g, const icp_drop_item* items, uint32_t count, uint16_t* out)
{
    if (!config_valid(g)) return fail(ICP_ERR_INVALID_ARGUMENT, "Invalid surrogate configuration.");
    if (!items || !out) return fail(ICP_ERR_INVALID_ARGUMENT, "icp_surrogate_record_features: null argument");
    for (uint32_t i = 0; i < count; ++i) {
        if (!item_valid(items[i])) return fail(ICP_ERR_INVALID_ARGUMENT, "surrogate: record %u has invalid parameters", i);
        record_row(*g, items[i], out + 16 * (size_t)i);
    }
    return ok();
}

int icp_surrogate_cell_features(const icp_surrogate_config* g, uint16_t* out)
{
    if (!config_valid(g)) return fail(ICP_ERR_INVALID_ARGUMENT, "Invalid surrogate configuration.");
    if (!out) return fail(ICP_ERR_INVALID_ARGUMENT, "icp_surrogate_cell_features: null argument");
    const uint32_t kc = g->input_width - 16u, F = g->theta_frequencies, Gf = g->phi_frequencies;
    std::vector<double> f(kc);
    for (uint32_t i = 0; i < g->nt; ++i)
        for (uint32_t j = 0; j < g->np; ++j) {
            std::fill(f.begin(), f.end(), 0.0);
            const double th = H::kPi * (i + 0.5) / g->nt, ph = 2.0 * H::kPi * (j + 0.5) / g->np;
            f[0] = 2.0 * (i + 0.5) / g->nt - 1.0;
            f[1] = std::cos(th);
            f[2] = i == 0 ? 1.0 : 0.0;
            f[3] = i + 1 == g->nt ? 1.0 : 0.0;
            for (uint32_t k = 1; k <= F; ++k) {
                f[4 + 2 * (k - 1)] = std::sin(k * th);
                f[5 + 2 * (k - 1)] = std::cos(k * th);
            }
            // the pattern of a drop whose axis lies in the plane of ki and e1 is even about
            // phi = pi/2 (the mirror z -> -z maps phi to pi - phi): only cos(l (phi - pi/2))
            for (uint32_t l = 1; l <= Gf; ++l) f[4 + 2 * F + (l - 1)] = std::cos(l * (ph - 0.5 * H::kPi));
            uint16_t* row = out + ((size_t)i * g->np + j) * kc;
            for (uint32_t k = 0; k < kc; ++k) row[k] = feature(f[k]);
        }
    return ok();
}

int icp_surrogate_create(icp_context* c, const icp_surrogate_config* g, icp_surrogate** out)
{
    if (!c || !out) return fail(ICP_ERR_INVALID_ARGUMENT, "icp_surrogate_create: null argument");
    *out = nullptr;
    if (!config_valid(g)) return fail(ICP_ERR_INVALID_ARGUMENT, "Invalid surrogate configuration.");
    ICP_CUDA(cudaSetDevice(c->device));
    auto* s = new icp_surrogate();
    s->c = c;
    s->cfg = *g;
    s->H = g->hidden;
    s->K0 = g->input_width;
    s->C = g->nt * g->np;
    s->R = g->max_records;
    s->n_params = icp_surrogate_parameter_count(g);
    const uint32_t Hn = s->H;
    s->o_w1 = 0;
    s->o_b1 = Hn * s->K0;
    s->o_w2 = s->o_b1 + Hn;
    s->o_b2 = s->o_w2 + Hn * Hn;
    s->o_w3 = s->o_b2 + Hn;
    s->o_b3 = s->o_w3 + Hn * Hn;
    s->o_w4 = s->o_b3 + Hn;
    s->o_hb = s->o_w4 + Hn;
    const size_t kc = s->K0 - 16u;
    std::vector<uint16_t> cells((size_t)s->C * kc);
    std::vector<double> edges;
    int st = icp_surrogate_cell_features(g, cells.data());
    if (!st && !H::u_edges(g->nt, edges)) st = fail(ICP_ERR_INVALID_ARGUMENT, "Angular cells cannot be represented in binary64.");
    if (st) {
        delete s;
        return st;
    }
    // the column-major copy of the cell table follows the row-major one
    std::vector<uint16_t> both(2 * cells.size());
    std::memcpy(both.data(), cells.data(), 2 * cells.size());
    for (size_t m = 0; m < s->C; ++m)
        for (size_t k = 0; k < kc; ++k) both[cells.size() + k * s->C + m] = cells[m * kc + k];
    const size_t np4 = 4 * s->n_params;
    cudaError_t e = cudaSuccess;
    Scratch* p4[] = {&s->params, &s->grads, &s->adam_m, &s->adam_v};
    for (Scratch* x : p4)
        if (e == cudaSuccess) e = x->ensure(np4);
    if (e == cudaSuccess) e = s->wbf.ensure(2 * ((size_t)Hn * s->K0 + 4ull * Hn * Hn));
    if (e == cudaSuccess) e = s->cells.ensure(2 * both.size());
    if (e == cudaSuccess) e = s->edges.ensure(sizeof(double) * edges.size());
    if (e == cudaSuccess) e = s->loss.ensure(sizeof(double) * s->R);
    if (e == cudaSuccess) e = cudaMemcpy(s->cells.ptr, both.data(), 2 * both.size(), cudaMemcpyHostToDevice);
    if (e == cudaSuccess && mlp::fused_shape(s->K0, Hn)) {
        // the cell table in the layout of the input rows (record columns zero), which the fused
        // inference pass loads by TMA before it writes each row's record and axis columns
        std::vector<uint16_t> rows((size_t)s->C * s->K0, 0);
        for (size_t m = 0; m < s->C; ++m) std::memcpy(&rows[m * s->K0 + 16], &cells[m * kc], 2 * kc);
        e = s->xcells.ensure(2 * rows.size());
        if (e == cudaSuccess) e = cudaMemcpy(s->xcells.ptr, rows.data(), 2 * rows.size(), cudaMemcpyHostToDevice);
    }
    if (e == cudaSuccess) e = cudaMemcpy(s->edges.ptr, edges.data(), sizeof(double) * edges.size(), cudaMemcpyHostToDevice);
    s->h_edges = edges;
    // cell geometry of the axis harmonics: cos(theta) and sin(theta) sin(phi), phi the column's
    // azimuth in [-pi, pi)
    std::vector<double> geo(2 * (size_t)s->C);
    for (uint32_t i = 0; i < g->nt; ++i)
        for (uint32_t j = 0; j < g->np; ++j) {
            const double th = H::kPi * (i + 0.5) / g->nt, ph = -H::kPi + 2.0 * H::kPi * (j + 0.5) / g->np;
            geo[2 * ((size_t)i * g->np + j)] = std::cos(th);
            geo[2 * ((size_t)i * g->np + j) + 1] = std::sin(th) * std::sin(ph);
        }
    if (e == cudaSuccess) e = s->cellgeo.ensure(sizeof(double) * geo.size());
    if (e == cudaSuccess) e = cudaMemcpy(s->cellgeo.ptr, geo.data(), sizeof(double) * geo.size(), cudaMemcpyHostToDevice);
    for (Scratch* x : p4)
        if (e == cudaSuccess) e = cudaMemset(x->ptr, 0, np4);
    if (e == cudaSuccess) e = cudaMemset(s->wbf.ptr, 0, s->wbf.bytes);
    if (e != cudaSuccess) {
        delete s;
        return fail(ICP_ERR_DEVICE, "surrogate allocation failed: %s", cudaGetErrorString(e));
    }
    *out = s;
    return ok();
}

void icp_surrogate_destroy(icp_surrogate* s)
{
    if (!s) return;
    cudaSetDevice(s->c->device);
    cudaStreamSynchronize(s->c->stream);
    delete s;
}

int icp_surrogate_set_parameters(icp_surrogate* s, const float* h, uint64_t count)
{
    if (!s || !h) return fail(ICP_ERR_INVALID_ARGUMENT, "icp_surrogate_set_parameters: null argument");
    if (count != s->n_params) return fail(ICP_ERR_INVALID_ARGUMENT, "surrogate: %llu parameters expected",
                                          (unsigned long long)s->n_params);
    for (uint64_t i = 0; i < count; ++i)
        if (!std::isfinite(h[i])) return fail(ICP_ERR_INVALID_ARGUMENT, "surrogate: non-finite parameter %llu",
                                              (unsigned long long)i);
    ICP_TRY(begin(s));
    icp_context* c = s->c;
    ICP_CUDA(cudaMemcpyAsync(s->params.ptr, h, 4 * count, cudaMemcpyHostToDevice, c->stream));
    ICP_CUDA(cudaMemsetAsync(s->adam_m.ptr, 0, 4 * count, c->stream));
    ICP_CUDA(cudaMemsetAsync(s->adam_v.ptr, 0, 4 * count, c->stream));
    s->head_b = h[s->o_hb];
    ICP_TRY(refresh_weights(s));
    return finish(c, "icp_surrogate_set_parameters");
}

int icp_surrogate_get_parameters(icp_surrogate* s, float* h, uint64_t count)
{
    if (!s || !h) return fail(ICP_ERR_INVALID_ARGUMENT, "icp_surrogate_get_parameters: null argument");
    if (count != s->n_params) return fail(ICP_ERR_INVALID_ARGUMENT, "surrogate: %llu parameters expected",
                                          (unsigned long long)s->n_params);
    ICP_CUDA(cudaSetDevice(s->c->device));
    ICP_CUDA(cudaMemcpyAsync(h, s->params.ptr, 4 * count, cudaMemcpyDeviceToHost, s->c->stream));
    ICP_CUDA(cudaStreamSynchronize(s->c->stream));
    h[s->o_hb] = s->head_b;
    return ok();
}

int icp_surrogate_gradient(icp_surrogate* s, const icp_drop_item* items, uint32_t count, const float* d_target,
                           float* h_grad, double* loss)
{
    ICP_TRY(check_call(s, items, count));
    if (!d_target) return fail(ICP_ERR_INVALID_ARGUMENT, "surrogate: null target");
    ICP_TRY(gradient_pass(s, items, count, d_target));
    if (h_grad)
        ICP_CUDA(cudaMemcpyAsync(h_grad, s->grads.ptr, 4 * s->n_params, cudaMemcpyDeviceToHost, s->c->stream));
    return read_loss(s, count, loss);
}

int icp_surrogate_train_step(icp_surrogate* s, const icp_drop_item* items, uint32_t count, const float* d_target,
                             const icp_adam* opt, double* loss)
{
    ICP_TRY(check_call(s, items, count));
    if (!d_target || !opt) return fail(ICP_ERR_INVALID_ARGUMENT, "surrogate: null target or optimiser");
    if (!(opt->lr > 0) || !(opt->beta1 >= 0 && opt->beta1 < 1) || !(opt->beta2 >= 0 && opt->beta2 < 1) ||
        !(opt->eps > 0) || !(opt->weight_decay >= 0) || !opt->step)
        return fail(ICP_ERR_INVALID_ARGUMENT, "surrogate: invalid Adam settings");
    ICP_TRY(gradient_pass(s, items, count, d_target));
    mlp::AdamArgs a{};
    a.p = as<float>(s->params);
    a.g = as<float>(s->grads);
    a.m = as<float>(s->adam_m);
    a.v = as<float>(s->adam_v);
    a.n = (uint32_t)(s->n_params - 1); // the head bias is not trained (softmax is shift-invariant)
    a.lr = opt->lr;
    a.beta1 = opt->beta1;
    a.beta2 = opt->beta2;
    a.eps = opt->eps;
    a.weight_decay = opt->weight_decay;
    a.bias1 = (float)(1.0 - std::pow((double)opt->beta1, (double)opt->step));
    a.bias2 = (float)(1.0 - std::pow((double)opt->beta2, (double)opt->step));
    int e = mlp::launch_adam(a, s->c->stream);
    count_launch();
    if (e) return fail(ICP_ERR_DEVICE, "Adam launch failed (%d)", e);
    ICP_TRY(refresh_weights(s));
    return read_loss(s, count, loss);
}

int icp_surrogate_predict(icp_surrogate* s, const icp_drop_item* items, uint32_t count, float* d_logits)
{
    ICP_TRY(check_call(s, items, count));
    if (!d_logits) return fail(ICP_ERR_INVALID_ARGUMENT, "surrogate: null output");
    ICP_TRY(begin(s));
    ICP_TRY(enqueue_features(s, items, count, false, !fused_inference(s)));
    ICP_TRY(enqueue_forward(s, count, false, d_logits, nullptr));
    return finish(s->c, "icp_surrogate_predict");
}

int icp_surrogate_generate(icp_surrogate* s, const icp_drop_item* items, uint32_t count, uint32_t ct, uint32_t cp,
                           const icp_cdf_policy* policy, double* d_phi, double* d_theta, icp_cdf_report* reports)
{
    ICP_TRY(check_call(s, items, count));
    if (!policy || !d_phi || !d_theta || !reports) return fail(ICP_ERR_INVALID_ARGUMENT, "surrogate: null argument");
    const icp_surrogate_config& g = s->cfg;
    if (!ct || !cp || ct > g.nt || cp > g.np || g.nt % ct || g.np % cp)
        return fail(ICP_ERR_INVALID_ARGUMENT, "Storage dimensions must divide histogram dimensions.");
    const icp_cdf_policy& p = *policy;
    if (!(H::finite(p.max_l1_error) && p.max_l1_error >= 0 && p.max_l1_error <= 2 && H::finite(p.max_lost_mass) &&
          p.max_lost_mass >= 0 && p.max_lost_mass <= 1 && H::finite(p.max_coarsening_tv) && p.max_coarsening_tv >= 0 &&
          p.max_coarsening_tv <= 1))
        return fail(ICP_ERR_INVALID_ARGUMENT, "Invalid CDF quality policy.");
    icp_context* c = s->c;
    ICP_TRY(begin(s));
    ICP_CUDA(s->mass.ensure(sizeof(double) * (uint64_t)count * s->C));
    ICP_CUDA(s->reports.ensure(sizeof(CdfDeviceReport) * s->R));
    ICP_CUDA(s->sync.ensure(2 * sizeof(unsigned) * s->R));
    ICP_CUDA(s->mass_sum.ensure(sizeof(double) * s->R));
    ICP_CUDA(s->dfrac.ensure(sizeof(double) * s->R * g.nt));
    ICP_CUDA(s->drows.ensure(sizeof(double) * s->R * g.nt));
    ICP_CUDA(cudaMemsetAsync(s->mass_sum.ptr, 0, sizeof(double) * count, c->stream));
    ICP_TRY(enqueue_features(s, items, count, false, !fused_inference(s)));
    ICP_TRY(enqueue_forward(s, count, false, nullptr, as<double>(s->mass), as<double>(s->mass_sum)));
    // the analytic diffraction rows on host threads while the device runs the network, into
    // page-locked staging so that the copy, the row scaling, the CDF build and the reports are
    // all enqueued behind the network without waiting for it
    ICP_CUDA(s->h_frac.ensure(sizeof(double) * (size_t)count * g.nt));
    ICP_CUDA(s->h_reports.ensure(sizeof(CdfDeviceReport) * count));
    double* frac = static_cast<double*>(s->h_frac.ptr);
    std::vector<int> fst(count, ICP_OK);
    {
        const unsigned workers = std::max(1u, std::min<unsigned>(count, std::thread::hardware_concurrency()));
        std::vector<std::future<void>> jobs;
        for (unsigned w = 0; w < workers; ++w)
            jobs.push_back(std::async(std::launch::async, [&, w]() {
                for (uint32_t r = w; r < count; r += workers)
                    fst[r] = diffraction_fractions(s, items[r], frac + (size_t)r * g.nt);
            }));
        for (auto& j : jobs) j.get();
    }
    for (uint32_t r = 0; r < count; ++r)
        if (fst[r]) {
            cudaStreamSynchronize(c->stream);
            return fail(fst[r], "surrogate: record %u: diffraction rows failed", r);
        }
    ICP_CUDA(cudaMemcpyAsync(s->dfrac.ptr, frac, sizeof(double) * (size_t)count * g.nt, cudaMemcpyHostToDevice,
                             c->stream));
    {
        const int e = mlp::launch_scale_rows(as<double>(s->dfrac), as<double>(s->mass_sum), count, g.nt,
                                             as<double>(s->drows), c->stream);
        count_launch();
        if (e) return fail(ICP_ERR_DEVICE, "row launch failed (%d)", e);
    }
    std::vector<CdfBatchInput> in(count);
    for (uint32_t r = 0; r < count; ++r) {
        in[r] = CdfBatchInput{};
        in[r].values = as<double>(s->mass) + (uint64_t)r * s->C;
        in[r].phi = d_phi + (size_t)(cp + 1) * r;
        in[r].theta = d_theta + (size_t)cp * (ct + 1) * r;
        in[r].row_add = items[r].diffraction ? as<double>(s->drows) + (size_t)r * g.nt : nullptr;
    }
    ICP_TRY(cdf_enqueue_batch(c, in.data(), count, g.nt, g.np, ct, cp, as<double>(s->edges),
                              as<CdfDeviceReport>(s->reports), as<unsigned>(s->sync)));
    CdfDeviceReport* dev = static_cast<CdfDeviceReport*>(s->h_reports.ptr);
    ICP_CUDA(cudaMemcpyAsync(dev, s->reports.ptr, sizeof(CdfDeviceReport) * count, cudaMemcpyDeviceToHost,
                             c->stream));
    ICP_TRY(finish(c, "icp_surrogate_generate"));
    int first = ICP_OK;
    for (uint32_t r = 0; r < count; ++r) {
        std::memset(&reports[r], 0, sizeof reports[r]);
        const int e = cdf_finish(dev[r], p, &reports[r]);
        reports[r].status = (uint32_t)e;
        if (e && !first) first = e;
    }
    if (first) return first;
    return ok();
}

int icp_surrogate_inputs(icp_surrogate* s, const icp_drop_item* items, uint32_t count, uint16_t* h_out)
{
    ICP_TRY(check_call(s, items, count));
    if (!h_out) return fail(ICP_ERR_INVALID_ARGUMENT, "surrogate: null output");
    ICP_TRY(begin(s));
    ICP_TRY(enqueue_features(s, items, count, false));
    ICP_CUDA(cudaMemcpyAsync(h_out, s->X.ptr, 2 * (size_t)count * s->C * s->K0, cudaMemcpyDeviceToHost, s->c->stream));
    return finish(s->c, "icp_surrogate_inputs");
}

int icp_surrogate_targets(icp_surrogate* s, const double* d_phi, const double* d_theta, uint32_t count, float* d_target)
{
    if (!s || !d_phi || !d_theta || !d_target) return fail(ICP_ERR_INVALID_ARGUMENT, "surrogate: null argument");
    if (!count) return fail(ICP_ERR_INVALID_ARGUMENT, "surrogate: no records");
    ICP_CUDA(cudaSetDevice(s->c->device));
    const int e = mlp::launch_cdf_cells(d_phi, d_theta, count, s->cfg.nt, s->cfg.np, d_target, s->c->stream);
    count_launch();
    if (e) return fail(ICP_ERR_DEVICE, "target launch failed (%d)", e);
    ICP_CUDA(cudaStreamSynchronize(s->c->stream));
    return ok();
}

int icp_mlp_gemm_bf16(icp_context* c, const void* d_a, const void* d_b, uint32_t m, uint32_t n, uint32_t k,
                      uint32_t split_k, float* d_c, int accumulate)
{
    if (!c || !d_a || !d_b || !d_c) return fail(ICP_ERR_INVALID_ARGUMENT, "icp_mlp_gemm_bf16: null argument");
    if (!m || m % 128 || !k || k % 64 || (n != 64 && n != 128 && n != 256))
        return fail(ICP_ERR_INVALID_ARGUMENT, "GEMM shape: M multiple of 128, N in {64,128,256}, K multiple of 64");
    if (m > (1u << 31) || k > (1u << 31)) // tile coordinates are signed 32-bit
        return fail(ICP_ERR_INVALID_ARGUMENT, "GEMM shape: M and K at most 2^31");
    if ((reinterpret_cast<uintptr_t>(d_a) | reinterpret_cast<uintptr_t>(d_b)) & 15)
        return fail(ICP_ERR_INVALID_ARGUMENT, "GEMM operands must be 16-byte aligned");
    if (!accumulate && split_k > 1) return fail(ICP_ERR_INVALID_ARGUMENT, "split-K needs accumulate");
    ICP_CUDA(cudaSetDevice(c->device));
    ICP_CUDA(c->mlp_error.ensure(sizeof(unsigned)));
    ICP_CUDA(cudaMemsetAsync(c->mlp_error.ptr, 0, sizeof(unsigned), c->stream));
    mlp::GemmArgs g{};
    g.M = m;
    g.N = n;
    g.K = k;
    g.out_f32 = d_c;
    g.ld_out = n;
    g.ld_t = m;
    g.error = (unsigned*)c->mlp_error.ptr;
    g.wait_limit = c->wait_limit;
    const int e = mlp::gemm(d_a, d_b, g, accumulate ? mlp::kAtomicF32 : mlp::kStoreF32, split_k ? split_k : 1,
                            c->stream);
    count_launch();
    if (e) return fail(ICP_ERR_DEVICE, "GEMM launch failed (%d)", e);
    return finish(c, "icp_mlp_gemm_bf16");
}

} // extern "C"
