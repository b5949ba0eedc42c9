// icp_mlp_features.cuh -- the device arithmetic of the surrogate's axis harmonics, shared by the
// feature-row kernel (icp_mlp.cu) and the fused inference pass (icp_mlp_gemm.cu), which builds
// its input rows in shared memory.  Uncontracted FP64 (the host restatement repeats it exactly).
#pragma once
#include <cstdint>
#include <cuda_bf16.h>

namespace icp::mlp {

// cos psi of one (record, cell): psi is the angle between the cell's direction and the drop's
// symmetry axis, from the record's (sin, cos) of its inclination and the cell's
// (cos theta, sin theta sin phi).
__device__ __forceinline__ double cos_psi(const double* recgeo, const double* cellgeo, uint32_t r, uint32_t c)
{
    return __dsub_rn(-__dmul_rn(recgeo[2 * r], cellgeo[2 * c]), __dmul_rn(recgeo[2 * r + 1], cellgeo[2 * c + 1]));
}

// Chebyshev values T_k(x), k = k0 .. k0+7, rounded to FP32 then BF16.
__device__ __forceinline__ void axis_harmonics8(double x, uint32_t k0, __nv_bfloat16 (&out)[8])
{
    double tm = 1.0, t = x; // T_0, T_1
    for (uint32_t k = 1; k < k0; ++k) {
        const double tn = __dsub_rn(__dmul_rn(__dmul_rn(2.0, x), t), tm);
        tm = t;
        t = tn;
    }
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        out[i] = __float2bfloat16_rn(__double2float_rn(t));
        const double tn = __dsub_rn(__dmul_rn(__dmul_rn(2.0, x), t), tm);
        tm = t;
        t = tn;
    }
}

} // namespace icp::mlp
