// renderer.cu -- headless point-splat rendering of the particle state.
//
// Replaces the recording path of the reference's demo renderer
// (examples/test_mods/renderer.rs:4-137 shaders, :305-478 frame set-up and
// glReadnPixels) with CUDA rasterisation into an 8-bit RGB frame:
//   * k_rp_project: the vertex shader -- view matrix (renderer.rs:338-349),
//     clip test, viewport mapping, density colour ramp (renderer.rs:45-55);
//   * without lighting, sprites are binned by (draw-order chunk, 16x16 tile),
//     each tile's sprites of a chunk are sorted by draw order in shared memory
//     and composited per pixel in that order with the blend the reference sets
//     (ONE_MINUS_DST_ALPHA, ONE_MINUS_SRC_ALPHA, DST_ALPHA, SRC_ALPHA), the
//     fragment alpha weighted by the poly6 kernel across the disc
//     (renderer.rs:121-128), channels rounded to 8 bits after every blend as a
//     RGBA8 target stores them;
//   * with lighting, a depth pass keeps the nearest sprite of each pixel (depth
//     test LESS, the first drawn on ties) and a shading pass lights it as a
//     sphere (renderer.rs:99-119).
// Fragments sit at pixel centres; a sprite covers the centres inside its
// square [c - S/2, c + S/2) and gl_PointCoord has its origin at the upper left.
#include "grid.cuh"

namespace arp {

namespace {

constexpr int kTile = 16;
constexpr int kChunk = 1024;  // sprites per draw-order chunk (and per sorted segment)

inline uint32_t nblk(uint32_t n, int t) { return (n + (uint32_t)t - 1u) / (uint32_t)t; }

__device__ __forceinline__ float mixf(float x, float y, float a) {
    return __fadd_rn(__fmul_rn(x, __fsub_rn(1.0f, a)), __fmul_rn(y, a));
}

// Vertex stage of one particle: window position, clip w ("depth"), window z,
// colour.  Invalid sprites get alpha 0 (discarded).
__device__ void project(float4 pd, float4 vm, const RenderCfg& c, float4& PR, float4& PC, float4& PP) {
    PR = make_float4(0.f, 0.f, 0.f, 0.f);
    PC = make_float4(0.f, 0.f, 0.f, 0.f);
    PP = make_float4(0.f, 0.f, 0.f, 0.f);
    const uint32_t mat = __float_as_uint(vm.w);
    if (mat >= c.nmat || !finite3(pd)) return;
    // pos2 = trans * (pos, 1), trans columns (cos t, 0, sin t, 0), (0, 1, 0, 0), (-sin t, 0, cos t, 0), (tx, ty, tz, 1)
    const float x2 = __fadd_rn(__fadd_rn(__fmul_rn(c.ca, pd.x), __fmul_rn(-c.sa, pd.z)), c.tx);
    const float y2 = __fadd_rn(pd.y, c.ty);
    const float z2 = __fadd_rn(__fadd_rn(__fmul_rn(c.sa, pd.x), __fmul_rn(c.ca, pd.z)), c.tz);
    const float w = __fadd_rn(z2, 1.0f);
    if (!(w > 0.0f) || x2 < -w || x2 > w || y2 < -w || y2 > w || z2 < -w || z2 > w) return;  // point clipping
    const float xn = __fdiv_rn(x2, w), yn = __fdiv_rn(y2, w), zn = __fdiv_rn(z2, w);
    const float half = 0.5f * c.s2;
    const float xw = __fadd_rn(__fmul_rn(__fadd_rn(xn, 1.0f), half), c.vx0);
    const float yw = __fadd_rn(__fmul_rn(__fadd_rn(yn, 1.0f), half), c.vy0);
    const float zw = __fmul_rn(__fadd_rn(zn, 1.0f), 0.5f);
    // density colour ramp (renderer.rs:45-55)
    const float d0 = c.d0[mat];
    const float dd = __fdiv_rn(__fsub_rn(pd.w, d0), d0);
    const float4 base = c.c2[mat];
    const float4 other = dd < 0.0f ? c.c1[mat] : c.c3[mat];
    const float t = dd < 0.0f ? __fdiv_rn(-dd, 5.0f) : __fdiv_rn(dd, 5.0f);
    float4 col = make_float4(mixf(base.x, other.x, t), mixf(base.y, other.y, t), mixf(base.z, other.z, t),
                             mixf(base.w, other.w, t));
    col.w = fminf(1.0f, col.w);
    PR = make_float4(xw, yw, w, zw);
    PC = col;
    PP = make_float4(x2, y2, z2, 0.0f);
}

__global__ void k_rp_project(const float4* __restrict__ pd, const float4* __restrict__ vm,
                             const uint32_t* __restrict__ orig, uint32_t n, uint32_t prim_base, RenderCfg c,
                             float4* __restrict__ PR, float4* __restrict__ PC, float4* __restrict__ PP) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const uint32_t prim = prim_base + orig[k];
    float4 r, col, p;
    project(pd[k], vm[k], c, r, col, p);
    PR[prim] = r;
    PC[prim] = col;
    PP[prim] = p;
}

// Half extent of the pixels a sprite can cover: its square, and the disc
// |d| <= 1 with d = 2 (fragment - centre) / S * 2 w.
__device__ __forceinline__ float sprite_reach(const RenderCfg& c, float w) {
    return fminf(0.5f * c.S, __fdiv_rn(c.S, 4.0f * w)) + 1.0f;
}

// Coverage of the pixel centre (fx, fy) by a sprite; r2 = dot(d, d) when covered.
__device__ __forceinline__ bool covers(const RenderCfg& c, float4 r, float fx, float fy, float& dx, float& dy,
                                       float& r2) {
    const float hs = 0.5f * c.S;
    if (fx < __fsub_rn(r.x, hs) || fx >= __fadd_rn(r.x, hs) || fy < __fsub_rn(r.y, hs) || fy >= __fadd_rn(r.y, hs))
        return false;
    // gl_PointCoord (upper-left origin), p = (pc - 0.5) * 2 with p.y negated, d = p * 2 * depth
    const float s = __fadd_rn(0.5f, __fdiv_rn(__fsub_rn(fx, r.x), c.S));
    const float t = __fsub_rn(0.5f, __fdiv_rn(__fsub_rn(fy, r.y), c.S));
    const float px = __fmul_rn(__fsub_rn(s, 0.5f), 2.0f);
    const float py = -__fmul_rn(__fsub_rn(t, 0.5f), 2.0f);
    dx = __fmul_rn(__fmul_rn(px, 2.0f), r.z);
    dy = __fmul_rn(__fmul_rn(py, 2.0f), r.z);
    r2 = __fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy));
    return r2 <= 1.0f;
}

__device__ __forceinline__ void tile_range(const RenderCfg& c, float4 r, int& tx0, int& tx1, int& ty0, int& ty1) {
    const float R = sprite_reach(c, r.z);
    tx0 = max(0, (int)floorf((r.x - R) / kTile));
    tx1 = min((int)c.tiles_x - 1, (int)floorf((r.x + R) / kTile));
    ty0 = max(0, (int)floorf((r.y - R) / kTile));
    ty1 = min((int)c.tiles_y - 1, (int)floorf((r.y + R) / kTile));
}

// pass 1 of the binning: sprites per (chunk, tile)
__global__ void k_rp_count(const float4* __restrict__ PR, const float4* __restrict__ PC, RenderCfg c,
                           uint32_t* __restrict__ counts, uint32_t* __restrict__ fill) {
    const uint32_t prim = blockIdx.x * blockDim.x + threadIdx.x;
    if (prim >= c.nprims) return;
    const float4 r = PR[prim];
    if (PC[prim].w == 0.0f) return;
    int tx0, tx1, ty0, ty1;
    tile_range(c, r, tx0, tx1, ty0, ty1);
    const size_t base = (size_t)(prim / kChunk) * c.tiles_x * c.tiles_y;
    for (int ty = ty0; ty <= ty1; ++ty)
        for (int tx = tx0; tx <= tx1; ++tx) atomicAdd(&counts[base + (size_t)ty * c.tiles_x + tx], 1u);
    (void)fill;
}

// pass 2: sprite ids into their (chunk, tile) segments (any order inside)
__global__ void k_rp_scatter(const float4* __restrict__ PR, const float4* __restrict__ PC, RenderCfg c,
                             const uint32_t* __restrict__ start, uint32_t* __restrict__ fill,
                             uint32_t* __restrict__ list) {
    const uint32_t prim = blockIdx.x * blockDim.x + threadIdx.x;
    if (prim >= c.nprims) return;
    const float4 r = PR[prim];
    if (PC[prim].w == 0.0f) return;
    int tx0, tx1, ty0, ty1;
    tile_range(c, r, tx0, tx1, ty0, ty1);
    const size_t base = (size_t)(prim / kChunk) * c.tiles_x * c.tiles_y;
    for (int ty = ty0; ty <= ty1; ++ty)
        for (int tx = tx0; tx <= tx1; ++tx) {
            const size_t key = base + (size_t)ty * c.tiles_x + tx;
            list[start[key] + atomicAdd(&fill[key], 1u)] = prim;
        }
}

__device__ __forceinline__ uint8_t to8(float v) {
    v = fminf(fmaxf(v, 0.0f), 1.0f);
    return (uint8_t)__float2uint_rd(__fadd_rn(__fmul_rn(v, 255.0f), 0.5f));
}
__device__ __forceinline__ float from8(uint8_t q) { return __fdiv_rn((float)q, 255.0f); }

// One block per tile, one thread per pixel: for each draw-order chunk, sort
// the tile's sprites of the chunk by draw order and blend them in turn.
__global__ void __launch_bounds__(kTile* kTile) k_rp_composite(const float4* __restrict__ PR,
                                                                const float4* __restrict__ PC, RenderCfg c,
                                                                const uint32_t* __restrict__ start,
                                                                const uint32_t* __restrict__ list,
                                                                uint8_t* __restrict__ rgb) {
    __shared__ uint32_t ids[kChunk];
    __shared__ float4 sr[kChunk], sc[kChunk];
    __shared__ uint32_t seg[2];
    const uint32_t tile = blockIdx.x;
    const uint32_t tx = tile % c.tiles_x, ty = tile / c.tiles_x;
    const int px = (int)(tx * kTile + threadIdx.x % kTile), py = (int)(ty * kTile + threadIdx.x / kTile);
    const float fx = px + 0.5f, fy = py + 0.5f;
    uint8_t q[4] = {255, 255, 255, 0};  // white, alpha 0
    const uint32_t ntiles = c.tiles_x * c.tiles_y;
    const uint32_t nchunks = (c.nprims + kChunk - 1) / kChunk;
    for (uint32_t ch = 0; ch < nchunks; ++ch) {
        if (threadIdx.x == 0) {
            const size_t key = (size_t)ch * ntiles + tile;
            seg[0] = start[key];
            seg[1] = start[key + 1];
        }
        __syncthreads();
        const uint32_t b = seg[0], n = seg[1] - seg[0];
        if (n == 0) {
            __syncthreads();
            continue;
        }
        uint32_t m = 1;
        while (m < n) m <<= 1;
        for (uint32_t i = threadIdx.x; i < m; i += blockDim.x) ids[i] = i < n ? list[b + i] : 0xFFFFFFFFu;
        __syncthreads();
        for (uint32_t k = 2; k <= m; k <<= 1)  // bitonic sort by draw order
            for (uint32_t j = k >> 1; j > 0; j >>= 1) {
                for (uint32_t i = threadIdx.x; i < m; i += blockDim.x) {
                    const uint32_t l = i ^ j;
                    if (l > i) {
                        const uint32_t a = ids[i], d = ids[l];
                        if (((i & k) == 0) == (a > d)) {
                            ids[i] = d;
                            ids[l] = a;
                        }
                    }
                }
                __syncthreads();
            }
        for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
            sr[i] = PR[ids[i]];
            sc[i] = PC[ids[i]];
        }
        __syncthreads();
        if (px < (int)c.W && py < (int)c.H) {
            for (uint32_t i = 0; i < n; ++i) {
                float dx, dy, r2;
                if (!covers(c, sr[i], fx, fy, dx, dy, r2)) continue;
                const float4 col = sc[i];
                const float diff = __fsub_rn(1.0f, r2);
                const float wk = __fmul_rn(__fmul_rn(__fmul_rn(c.kconst, diff), diff), diff);
                const float sa = __fmul_rn(col.w, __fdiv_rn(wk, c.kconst));
                const float da = from8(q[3]);
                const float src[3] = {col.x, col.y, col.z};
#pragma unroll
                for (int ch3 = 0; ch3 < 3; ++ch3)
                    q[ch3] = to8(__fadd_rn(__fmul_rn(src[ch3], __fsub_rn(1.0f, da)),
                                           __fmul_rn(from8(q[ch3]), __fsub_rn(1.0f, sa))));
                q[3] = to8(__fadd_rn(__fmul_rn(sa, da), __fmul_rn(da, sa)));
            }
        }
        __syncthreads();
    }
    if (px < (int)c.W && py < (int)c.H) {
        const size_t o = ((size_t)py * c.W + px) * 3;
        rgb[o] = q[0];
        rgb[o + 1] = q[1];
        rgb[o + 2] = q[2];
    }
}

// Lighting: the nearest covering sprite of each pixel (depth LESS, the first
// drawn on ties): min over (window depth bits, draw order).
__global__ void k_rp_depth(const float4* __restrict__ PR, const float4* __restrict__ PC, RenderCfg c,
                           unsigned long long* __restrict__ zkey) {
    const uint32_t prim = blockIdx.x * blockDim.x + threadIdx.x;
    if (prim >= c.nprims) return;
    const float4 r = PR[prim];
    if (PC[prim].w == 0.0f || !(r.w < 1.0f) || !(r.w >= 0.0f)) return;
    const float R = sprite_reach(c, r.z);
    const int i0 = max(0, (int)floorf(r.x - R)), i1 = min((int)c.W - 1, (int)ceilf(r.x + R));
    const int j0 = max(0, (int)floorf(r.y - R)), j1 = min((int)c.H - 1, (int)ceilf(r.y + R));
    const unsigned long long key = ((unsigned long long)__float_as_uint(r.w) << 32) | prim;
    for (int j = j0; j <= j1; ++j)
        for (int i = i0; i <= i1; ++i) {
            float dx, dy, r2;
            if (covers(c, r, i + 0.5f, j + 0.5f, dx, dy, r2)) atomicMin(&zkey[(size_t)j * c.W + i], key);
        }
}

__global__ void k_rp_shade(const float4* __restrict__ PR, const float4* __restrict__ PC,
                           const float4* __restrict__ PP, RenderCfg c, const unsigned long long* __restrict__ zkey,
                           uint8_t* __restrict__ rgb) {
    const uint32_t pix = blockIdx.x * blockDim.x + threadIdx.x;
    if (pix >= c.W * c.H) return;
    const unsigned long long key = zkey[pix];
    uint8_t out[3] = {255, 255, 255};
    const uint32_t prim = (uint32_t)(key & 0xFFFFFFFFull);
    if (prim != 0xFFFFFFFFu) {
        const float4 r = PR[prim], col = PC[prim], p = PP[prim];
        float dx, dy, r2;
        covers(c, r, (pix % c.W) + 0.5f, (pix / c.W) + 0.5f, dx, dy, r2);
        // normal = d.x e_x + d.y e_y + sqrt(1 - n.x^2 - n.y^2) (-e_z)
        const float nz = -sqrtf(1.0f - dx * dx - dy * dy);
        const float sx = p.x + c.render_h * dx, sy = p.y + c.render_h * dy, sz = p.z + c.render_h * nz;
        float lx = c.light[0] - sx, ly = c.light[1] - sy, lz = c.light[2] - sz;
        const float l = rsqrtf(lx * lx + ly * ly + lz * lz);
        const float l3 = l * l * l;
        lx *= l3;
        ly *= l3;
        lz *= l3;
        const float diffuse = lx * dx + ly * dy + lz * nz;
        const float ndl = dx * lx + dy * ly + nz * lz;
        const float rz = lz - 2.0f * ndl * nz;  // reflect(light, normal).z
        float spec = fmaxf(20.0f * rz, 0.0f);
        spec *= spec * spec;
        const float cc[3] = {col.x, col.y, col.z};
        for (int k = 0; k < 3; ++k)
            out[k] = to8(cc[k] * c.amb + diffuse * c.dif * c.lcol[k] + c.lcol[k] * spec * c.spec);
    }
    rgb[(size_t)pix * 3] = out[0];
    rgb[(size_t)pix * 3 + 1] = out[1];
    rgb[(size_t)pix * 3 + 2] = out[2];
}

}  // namespace

int render_project(const float4* pd, const float4* vm, const uint32_t* orig, uint32_t n, uint32_t prim_base,
                   const RenderCfg& c, float4* PR, float4* PC, float4* PP, cudaStream_t st) {
    if (n == 0) return 0;
    k_rp_project<<<nblk(n, 256), 256, 0, st>>>(pd, vm, orig, n, prim_base, c, PR, PC, PP);
    return 1;
}

uint32_t render_chunk_size() { return kChunk; }
uint32_t render_tile_size() { return kTile; }

int render_bin_count(const float4* PR, const float4* PC, const RenderCfg& c, uint32_t* counts, cudaStream_t st) {
    if (c.nprims == 0) return 0;
    k_rp_count<<<nblk(c.nprims, 256), 256, 0, st>>>(PR, PC, c, counts, nullptr);
    return 1;
}

int render_bin_scatter(const float4* PR, const float4* PC, const RenderCfg& c, const uint32_t* start,
                       uint32_t* fill, uint32_t* list, cudaStream_t st) {
    if (c.nprims == 0) return 0;
    k_rp_scatter<<<nblk(c.nprims, 256), 256, 0, st>>>(PR, PC, c, start, fill, list);
    return 1;
}

int render_composite(const float4* PR, const float4* PC, const RenderCfg& c, const uint32_t* start,
                     const uint32_t* list, uint8_t* rgb, cudaStream_t st) {
    k_rp_composite<<<c.tiles_x * c.tiles_y, kTile * kTile, 0, st>>>(PR, PC, c, start, list, rgb);
    return 1;
}

int render_lit(const float4* PR, const float4* PC, const float4* PP, const RenderCfg& c, unsigned long long* zkey,
               uint8_t* rgb, cudaStream_t st) {
    int launches = 0;
    if (c.nprims) {
        k_rp_depth<<<nblk(c.nprims, 128), 128, 0, st>>>(PR, PC, c, zkey);
        ++launches;
    }
    k_rp_shade<<<nblk(c.W * c.H, 256), 256, 0, st>>>(PR, PC, PP, c, zkey, rgb);
    return launches + 1;
}

}  // namespace arp
