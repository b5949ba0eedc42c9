// icp_hex_f64.cu -- FP64 instantiation of the trace+bin kernel for the hexagonal prism, built
// with -fmad=false so that direction and binning arithmetic round like the reference's code.
#include "icp_hex_launch.cuh"

namespace icp {
int launch_hex_f64(const HexLaunch& L, cudaStream_t s) { return launch_trace(make_hex_params<double>(L), L, s); }
int hex_blocks_per_sm_f64(uint32_t slots, uint32_t nt, uint32_t threads)
{
    return trace_blocks_per_sm<double, HexGeo<double>>(slots, nt, threads);
}
} // namespace icp
