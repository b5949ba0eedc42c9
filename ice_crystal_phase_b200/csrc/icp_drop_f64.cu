// icp_drop_f64.cu -- FP64 instantiation of the trace+bin kernel for the axisymmetric drop.
#include "icp_hex_launch.cuh"

namespace icp {
int launch_drop_f64(const HexLaunch& L, cudaStream_t s) { return launch_trace(make_drop_params<double>(L), L, s); }
int drop_blocks_per_sm_f64(uint32_t slots, uint32_t nt, uint32_t threads)
{
    return trace_blocks_per_sm<double, DropGeo<double>>(slots, nt, threads);
}
uint32_t drop_trace_threads_f64() { return TraceShape<double, DropGeo<double>>::threads; }
int launch_drop_batch_f64(const BatchLaunch& B, cudaStream_t s) { return launch_drop_batch<double>(B, s); }
int drop_batch_blocks_f64(uint32_t threads, uint32_t nt) { return drop_batch_blocks<double>(threads, nt); }
size_t drop_batch_param_bytes_f64() { return sizeof(TraceParams<double, DropGeo<double>>); }
} // namespace icp
