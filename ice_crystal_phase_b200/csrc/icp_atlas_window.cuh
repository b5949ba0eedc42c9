// icp_atlas_window.cuh -- phi-index arithmetic of the cyclic composition (atlas_compose_kernel):
// the cell of row m that output cell p reads at shift s is m = (p - s) mod np, reflected to
// np - 1 - m for the mirrored parity; no integer division in the inner loop.  Host and device
// code alike (the host test compiles it with g++).
#pragma once
#include <cstdint>

#ifdef __CUDACC__
#define ICP_WINDOW_HD __host__ __device__ __forceinline__
#else
#define ICP_WINDOW_HD inline
#endif

namespace icp {

// (pm - s) mod np for pm, s < np
ICP_WINDOW_HD uint32_t phi_sub(uint32_t pm, uint32_t s, uint32_t np) { return pm >= s ? pm - s : pm + np - s; }

// (m + k) mod np for m < np and a small k (at most k / np + 1 subtractions)
ICP_WINDOW_HD uint32_t phi_add(uint32_t m, uint32_t k, uint32_t np)
{
    uint32_t x = m + k;
    while (x >= np) x -= np;
    return x;
}

// (m - 1) mod np for m < np
ICP_WINDOW_HD uint32_t phi_prev(uint32_t m, uint32_t np) { return m ? m - 1 : np - 1; }

// the row cell read for index m: m itself, or its phi reflection np - 1 - m
ICP_WINDOW_HD uint32_t phi_cell(uint32_t m, uint32_t np, int reflect) { return reflect ? np - 1 - m : m; }

} // namespace icp
