// grid.cuh -- cell hashing shared by the grid build and the force kernels.
#pragma once

#include "arp_internal.h"

namespace arp {

// Cell coordinate along one axis, as fill_buckets hashes it
// (neighbor_list.rs:95): floor(clamp((p - min) / dim, 0, 1) * sub).  An axis
// of zero extent maps to cell 0 (the shader divides 0/0 there) and a
// coordinate exactly on the upper face is clamped into the last cell.  Every
// operation is separately rounded so host and device agree bit for bit.
__host__ __device__ inline uint32_t axis_cell(float p, float mn, float d, uint32_t sub) {
    if (d == 0.0f) return 0u;
#ifdef __CUDA_ARCH__
    float t = __fdiv_rn(__fsub_rn(p, mn), d);
    t = fminf(fmaxf(t, 0.0f), 1.0f);
    uint32_t c = (uint32_t)floorf(__fmul_rn(t, (float)sub));
#else
    volatile float diff = p - mn;
    volatile float t = diff / d;
    float tc = t < 0.0f ? 0.0f : (t > 1.0f ? 1.0f : t);
    volatile float sc = tc * (float)sub;
    uint32_t c = (uint32_t)__builtin_floorf(sc);
#endif
    return c >= sub ? sub - 1u : c;
}

__host__ __device__ inline bool finite3(float4 p) {
#ifdef __CUDA_ARCH__
    return isfinite(p.x) && isfinite(p.y) && isfinite(p.z);
#else
    return __builtin_isfinite(p.x) && __builtin_isfinite(p.y) && __builtin_isfinite(p.z);
#endif
}

struct CellCoord {
    int x, y, z;
};

__host__ __device__ inline CellCoord cell_coord(float4 p, const Grid& g) {
    CellCoord c;
    c.x = (int)axis_cell(p.x, g.min[0], g.dim[0], g.sub[0]);
    c.y = (int)axis_cell(p.y, g.min[1], g.dim[1], g.sub[1]);
    c.z = (int)axis_cell(p.z, g.min[2], g.dim[2], g.sub[2]);
    return c;
}

__host__ __device__ inline uint32_t cell_id(const CellCoord& c, const Grid& g) {
    return (uint32_t)c.x + (uint32_t)c.y * g.sub[0] + (uint32_t)c.z * g.sub[0] * g.sub[1];
}

}  // namespace arp
