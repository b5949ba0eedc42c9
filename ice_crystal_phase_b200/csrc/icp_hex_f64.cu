// icp_hex_f64.cu -- FP64 instantiation of the hex trace+bin kernel, built with -fmad=false so
// that direction and binning arithmetic round like the reference's binary64 code.
#include "icp_hex_launch.cuh"

namespace icp {
int launch_hex_f64(const HexLaunch& L, cudaStream_t stream) { return launch_hex<double>(L, stream); }
int hex_blocks_per_sm_f64(uint32_t slots, uint32_t nt, uint32_t threads) { return hex_blocks_per_sm<double>(slots, nt, threads); }
} // namespace icp
