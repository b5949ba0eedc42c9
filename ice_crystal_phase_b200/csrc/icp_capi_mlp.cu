// icp_capi_mlp.cu -- C ABI of the surrogate's tensor-core kernels (include/icp_b200.h,
// "surrogate").
#include <cstdarg>
#include <cstdio>
#include <cstring>

#include "../../include/icp_b200.h"
#include "icp_internal.h"
#include "icp_mlp.h"

using namespace icp;

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

// Runs the enqueued kernels, then reads the error word the bounded waits set.
int finish(icp_context* c, const char* what)
{
    unsigned err = 0;
    ICP_CUDA(cudaMemcpyAsync(&err, c->mlp_error.ptr, sizeof err, cudaMemcpyDeviceToHost, c->stream));
    ICP_CUDA(cudaStreamSynchronize(c->stream));
    if (err) return fail(ICP_ERR_TIMEOUT, "%s: a tensor-core pipeline wait gave up (code %u)", what, err);
    return ok();
}

} // namespace

extern "C" int icp_mlp_gemm_bf16(icp_context* c, const void* d_a, const void* d_b, uint32_t m, uint32_t n, uint32_t k,
                                 uint32_t split_k, float* d_c, int accumulate)
{
    if (!c || !d_a || !d_b || !d_c) return fail(ICP_ERR_INVALID_ARGUMENT, "icp_mlp_gemm_bf16: null argument");
    if (!m || m % 128 || !k || k % 64 || (n != 64 && n != 128 && n != 256))
        return fail(ICP_ERR_INVALID_ARGUMENT, "GEMM shape: M multiple of 128, N in {64,128,256}, K multiple of 64");
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
    g.error = (unsigned*)c->mlp_error.ptr;
    const int e = mlp::gemm(d_a, d_b, g, accumulate ? mlp::kAtomicF32 : mlp::kStoreF32, split_k ? split_k : 1,
                            c->stream);
    count_launch();
    if (e) return fail(ICP_ERR_DEVICE, "GEMM launch failed (%d)", e);
    return finish(c, "icp_mlp_gemm_bf16");
}
