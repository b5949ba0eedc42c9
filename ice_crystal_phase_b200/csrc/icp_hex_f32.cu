// icp_hex_f32.cu -- FP32 instantiation of the hex trace+bin kernel (fast path).
#include "icp_hex_launch.cuh"

namespace icp {
int launch_hex_f32(const HexLaunch& L, cudaStream_t stream) { return launch_hex<float>(L, stream); }
size_t hex_stats_bytes() { return sizeof(DevStats); }
int hex_blocks_per_sm_f32(uint32_t slots, uint32_t nt, uint32_t threads) { return hex_blocks_per_sm<float>(slots, nt, threads); }
} // namespace icp
