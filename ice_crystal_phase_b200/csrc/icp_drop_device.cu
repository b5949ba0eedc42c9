// icp_drop_device.cu -- device-side pieces of a drop record that follow the trace:
// the analytic diffraction rows (one block per record) and small layout helpers.
//
// Diffraction: Fraunhofer diffraction of the circle of equal traced area a_eq = sqrt(A/pi),
// A = weight x hit rays.  The power within scattering angle theta is Rayleigh's encircled
// energy L(theta) = 1 - J0(x sin theta)^2 - J1(x sin theta)^2, x = 2 pi a_eq / lambda, taken over
// the forward hemisphere and normalised there; row i receives A (L(u_{i+1}) - L(u_i)) / L(1/2),
// spread uniformly over the np cells of the row.  The arithmetic follows the host restatement
// (host/icp_drop_host.hpp diffraction_rows) operation for operation; J0 and J1 are CUDA's.
#include <cstddef>
#include <cuda_runtime.h>

#include "icp_hex_kernel.cuh"
#include "icp_internal.h"

namespace icp {

int drop_batch_blocks_f32(uint32_t threads, uint32_t nt);
int drop_batch_blocks_f64(uint32_t threads, uint32_t nt);
size_t drop_batch_param_bytes_f32();
size_t drop_batch_param_bytes_f64();

namespace {

constexpr double kPiD = 3.141592653589793238462643383279502884;

__device__ __forceinline__ double encircled(double u, double x)
{
    if (u >= 0.5) u = 0.5;
    const double st = 2 * sqrt(u * (1 - u)); // sin(theta) from u = (1 - cos theta) / 2
    const double z = x * st;
    const double a = j0(z), b = j1(z);
    return 1 - a * a - b * b;
}

__global__ void __launch_bounds__(256) diffraction_rows_kernel(const DiffractionArgs* args)
{
    extern __shared__ double enc[]; // nt + 1
    const DiffractionArgs a = args[blockIdx.x];
    const unsigned long long hits = a.rays[0] - a.rays[a.missed_offset];
    const double area = a.weight * (double)hits;
    const double a_eq = sqrt(area / kPiD);
    const double x = 2 * kPiD * a_eq / (a.wavelength_nm * 1e-6);
    for (uint32_t i = threadIdx.x; i <= a.nt; i += blockDim.x) enc[i] = i == 0 ? 0.0 : encircled(a.edges[i], x);
    __syncthreads();
    const double total = encircled(0.5, x);
    for (uint32_t i = threadIdx.x; i < a.nt; i += blockDim.x) a.row_add[i] = area * (enc[i + 1] - enc[i]) / total / a.np;
    if (threadIdx.x == 0) {
        double p = 0.0;
        for (uint32_t i = 0; i < a.nt; ++i) p += area * (enc[i + 1] - enc[i]) / total;
        *a.power = p;
    }
}

} // namespace

int launch_diffraction_rows(const DiffractionArgs* d_args, uint32_t count, uint32_t nt, cudaStream_t stream)
{
    const size_t smem = sizeof(double) * (nt + 1);
    cudaError_t e = cudaFuncSetAttribute(diffraction_rows_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return (int)e;
    diffraction_rows_kernel<<<count, 256, smem, stream>>>(d_args);
    return (int)cudaGetLastError();
}

uint32_t devstats_rays_word() { return (uint32_t)(offsetof(DevStats, rays) / 8); }
uint32_t devstats_missed_word() { return (uint32_t)(offsetof(DevStats, missed) / 8); }
uint32_t devstats_fwd_word() { return (uint32_t)(offsetof(DevStats, fwd) / 8); }

size_t drop_batch_param_bytes(uint32_t precision)
{
    return precision == ICP_FP32 ? drop_batch_param_bytes_f32() : drop_batch_param_bytes_f64();
}
int drop_batch_blocks_per_sm(uint32_t precision, uint32_t threads, uint32_t nt)
{
    return precision == ICP_FP32 ? drop_batch_blocks_f32(threads, nt) : drop_batch_blocks_f64(threads, nt);
}

} // namespace icp
