// icp_hex_f32.cu -- FP32 instantiation of the trace+bin kernel for the hexagonal prism (fast path).
#include "icp_hex_launch.cuh"

namespace icp {
int launch_hex_f32(const HexLaunch& L, cudaStream_t s) { return launch_trace(make_hex_params<float>(L), L, s); }
size_t hex_stats_bytes() { return sizeof(DevStats); }
int hex_blocks_per_sm_f32(uint32_t slots, uint32_t nt, uint32_t threads)
{
    return trace_blocks_per_sm<float, HexGeo<float>>(slots, nt, threads);
}
} // namespace icp
