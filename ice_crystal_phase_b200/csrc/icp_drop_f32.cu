// icp_drop_f32.cu -- FP32 instantiation of the trace+bin kernel for the axisymmetric drop.
#include "icp_hex_launch.cuh"

namespace icp {
int launch_drop_f32(const HexLaunch& L, cudaStream_t s) { return launch_trace(make_drop_params<float>(L), L, s); }
int drop_blocks_per_sm_f32(uint32_t slots, uint32_t nt, uint32_t threads)
{
    return trace_blocks_per_sm<float, DropGeo<float>>(slots, nt, threads);
}
uint32_t drop_trace_threads_f32() { return TraceShape<float, DropGeo<float>>::threads; }
int launch_drop_batch_f32(const BatchLaunch& B, cudaStream_t s) { return launch_drop_batch<float>(B, s); }
int drop_batch_blocks_f32(uint32_t threads, uint32_t nt) { return drop_batch_blocks<float>(threads, nt); }
size_t drop_batch_param_bytes_f32() { return sizeof(TraceParams<float, DropGeo<float>>); }
} // namespace icp
