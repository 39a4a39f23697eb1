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

// ---- search grid -------------------------------------------------------------

// Calls f(c0, c1) for the global search-cell ranges [c0, c1) (one x-row
// each, ascending) around the search cell of x: 2 cells each way along a
// halved axis, 1 along the others.  Every particle within h of x lies in them
// (search cells are at least h/2 wide on halved axes and h wide on the
// others).  The ranges are not clipped per particle: the 32 lanes of a warp
// walk rows of equal length, which a per-particle clip would only make
// uneven without shortening the longest.
template <int DIM, class F>
__device__ __forceinline__ void for_search_rows(float4 x, const SceneP& P, F&& f) {
    const Grid& g = P.sgrid;
    const CellCoord c = cell_coord(x, g);
    const int rx = 1 + (int)P.halved[0], ry = 1 + (int)P.halved[1], rz = 1 + (int)P.halved[2];
    const int x0 = max(c.x - rx, 0), x1 = min(c.x + rx, (int)g.sub[0] - 1);
    const int ylo = max(c.y - ry, 0), yhi = min(c.y + ry, (int)g.sub[1] - 1);
    const int zlo = DIM == 3 ? max(c.z - rz, 0) : c.z, zhi = DIM == 3 ? min(c.z + rz, (int)g.sub[2] - 1) : c.z;
    for (int z = zlo; z <= zhi; ++z)
        for (int y = ylo; y <= yhi; ++y) {
            const uint32_t row = P.cell_base + (uint32_t)y * g.sub[0] + (uint32_t)z * g.sub[0] * g.sub[1];
            f(row + (uint32_t)x0, row + (uint32_t)x1 + 1u);
        }
}

// Calls f(c0, c1) for the global search-cell x-rows covering the 3x3(x3)
// reference cells around the reference cell of x (the shaders' neighbor
// stencil, neighbor_list.rs:121-143), ascending.
template <class F>
__device__ __forceinline__ void for_reference_block_rows(float4 x, const SceneP& P, F&& f) {
    const CellCoord c = cell_coord(x, P.grid);
    const int cc[3] = {c.x, c.y, c.z};
    int lo[3], hi[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        lo[a] = max(cc[a] - 1, 0) << P.halved[a];
        hi[a] = ((min(cc[a] + 1, (int)P.grid.sub[a] - 1) + 1) << P.halved[a]) - 1;
    }
    const Grid& g = P.sgrid;
    for (int z = lo[2]; z <= hi[2]; ++z)
        for (int y = lo[1]; y <= hi[1]; ++y) {
            const uint32_t row = P.cell_base + (uint32_t)y * g.sub[0] + (uint32_t)z * g.sub[0] * g.sub[1];
            f(row + (uint32_t)lo[0], row + (uint32_t)hi[0] + 1u);
        }
}

}  // namespace arp
