// neighbor.cu -- uniform-grid neighbor build (replaces reset_buckets +
// fill_buckets, src/soft_body/neighbor_list.rs:37-143 and update_contents
// :224-294).
//
// The reference appends each particle into a fixed 128-slot bucket with
// atomics, so slot order is nondeterministic on a GPU and particles past 128
// are dropped.  Here the grid is a counting sort with no capacity limit:
//   1. cell key + histogram (one atomic per particle; the returned value is
//      the particle's arrival rank inside its cell);
//   2. exclusive scan of the histogram (warp-shuffle block scan, block sums,
//      offsets), which also clears the histogram for the next build;
//   3. scatter to perm[start[key] + rank];
//   4. sort each cell's run by slot so the order is deterministic for every
//      run length (short runs by one thread, long runs by the whole block);
//      this also records the largest occupancy and cells over the
//      reference's 128.
// Memory traffic per particle: 16 B position read, 4+4 B key/rank write and
// read, 4 B perm write, 4+4 B perm read/write in the run sort.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <mutex>
#include <string>

#include "grid.cuh"

namespace arp {

namespace {

constexpr int kThreads = 256;
constexpr int kScanThreads = 1024;
constexpr int kScanItems = 4;  // per thread
constexpr int kScanTile = kScanThreads * kScanItems;

__device__ __forceinline__ uint32_t scene_of(const float4* vm, const uint32_t* mat_u32, uint32_t i, const Tables& T) {
    const uint32_t m = vm ? __float_as_uint(vm[i].w) : (mat_u32 ? mat_u32[i] : 0u);
    return T.mats[m].scene;
}

__global__ void k_cell_keys(const float4* __restrict__ pos, const float4* __restrict__ vm,
                            const uint32_t* __restrict__ mat_u32, uint32_t n, Tables T, uint32_t* __restrict__ key,
                            uint32_t* __restrict__ rank, uint32_t* __restrict__ count, uint2* __restrict__ coord,
                            DevStats* stats, StageCounters zero) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < 3 && zero.p[i])
        for (uint32_t q = 0; q < zero.n[i]; ++q) zero.p[i][q] = 0u;
    if (i >= n) return;
    float4 p = pos[i];
    uint32_t k;
    if (!finite3(p)) {
        k = T.ncells;
        if (coord) coord[i] = make_uint2(0xFFFFFFFFu, 0xFFFFFFFFu);
        if (stats) atomicAdd(&stats->nonfinite_positions, 1u);
    } else {
        const SceneP& sp = T.scenes[scene_of(vm, mat_u32, i, T)];
        const Grid& grid = sp.grid;
        const CellCoord fc = cell_coord(p, sp.sgrid);
        k = sp.cell_base + cell_id(fc, sp.sgrid);
        if (coord) {
            // reference cell = search cell >> 1 on halved axes (exact, see SceneP)
            const uint32_t x = (uint32_t)fc.x >> sp.halved[0], y = (uint32_t)fc.y >> sp.halved[1],
                           z = (uint32_t)fc.z >> sp.halved[2];
            coord[i] = make_uint2(x | (y << 16), z);
        }
        if (stats) {
            // a coordinate on the upper face would hash one past the last cell
            bool face = (grid.dim[0] != 0.0f && p.x == grid.min[0] + grid.dim[0]) ||
                        (grid.dim[1] != 0.0f && p.y == grid.min[1] + grid.dim[1]) ||
                        (grid.dim[2] != 0.0f && p.z == grid.min[2] + grid.dim[2]);
            if (face) atomicAdd(&stats->clamped_coordinates, 1u);
        }
    }
    key[i] = k;
    rank[i] = atomicAdd(&count[k], 1u);
}

__device__ __forceinline__ uint32_t warp_incl_scan(uint32_t v) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t t = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += t;
    }
    return v;
}

// Block-wide exclusive scan of one value per thread (blockDim.x a multiple
// of 32, at most 1024).  The block total is excl + v of the last thread.
__device__ __forceinline__ void block_excl_scan(uint32_t v, uint32_t& excl) {
    __shared__ uint32_t warp_tot[kScanThreads / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nwarps = (int)(blockDim.x >> 5);
    uint32_t inc = warp_incl_scan(v);
    if (lane == 31) warp_tot[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = lane < nwarps ? warp_tot[lane] : 0u;
        uint32_t wi = warp_incl_scan(w);
        if (lane < nwarps) warp_tot[lane] = wi - w;
    }
    __syncthreads();
    excl = warp_tot[warp] + inc - v;
}

// `count` and `out` may be the same array (the allocation-free build scans in
// place), so they are not declared __restrict__.
__global__ void k_scan_tiles(uint32_t* count, uint32_t len, uint32_t* out, uint32_t* __restrict__ block_sums) {
    __shared__ uint32_t last_total;
    const uint32_t base = blockIdx.x * kScanTile + threadIdx.x * kScanItems;
    uint32_t v[kScanItems];
    uint32_t s = 0;
#pragma unroll
    for (int j = 0; j < kScanItems; ++j) {
        uint32_t idx = base + j;
        v[j] = idx < len ? count[idx] : 0u;
        if (idx < len) count[idx] = 0u;  // ready for the next histogram
        s += v[j];
    }
    uint32_t excl;
    block_excl_scan(s, excl);
    if (threadIdx.x == blockDim.x - 1) last_total = excl + s;
    uint32_t run = excl;
#pragma unroll
    for (int j = 0; j < kScanItems; ++j) {
        uint32_t idx = base + j;
        if (idx < len) out[idx] = run;
        run += v[j];
    }
    __syncthreads();
    if (threadIdx.x == 0) block_sums[blockIdx.x] = last_total;
}

// Adds to each tile of the scan the sum of the totals of the tiles before it;
// each block (one tile of kScanTile items) sums those totals itself, a block
// reduction over at most a few hundred values, so no separate pass scans them.
__global__ void k_scan_add(uint32_t* out, uint32_t len, const uint32_t* __restrict__ sums) {
    __shared__ uint32_t warp_part[kScanThreads / 32];
    __shared__ uint32_t prefix;
    uint32_t part = 0;
    for (uint32_t t = threadIdx.x; t < blockIdx.x; t += blockDim.x) part += sums[t];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
    if ((threadIdx.x & 31) == 0) warp_part[threadIdx.x >> 5] = part;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t p = 0;
        for (uint32_t w = 0; w < blockDim.x / 32; ++w) p += warp_part[w];
        prefix = p;
    }
    __syncthreads();
    const uint32_t add = prefix;
    if (add == 0u) return;
    const uint32_t base = blockIdx.x * kScanTile;
#pragma unroll
    for (int j = 0; j < kScanItems; ++j) {
        const uint32_t idx = base + (uint32_t)j * blockDim.x + threadIdx.x;
        if (idx < len) out[idx] += add;
    }
}

__global__ void k_scatter(const uint32_t* __restrict__ key, const uint32_t* __restrict__ rank, uint32_t n,
                          const uint32_t* __restrict__ start, uint32_t* __restrict__ perm) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    perm[start[key[i]] + rank[i]] = i;
}

// Occupancy (mobile + boundary) of the reference cell whose first search
// cell is global cell c, or 0 when c is not the first search cell of its
// reference cell.
__device__ __forceinline__ uint32_t reference_cell_occupancy(uint32_t c, const uint32_t* __restrict__ start,
                                                             const uint32_t* __restrict__ bstart, const Tables& T) {
    uint32_t lo = 0, hi = T.nscenes;  // scene with the largest cell_base <= c
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (T.scenes[mid].cell_base <= c) lo = mid;
        else hi = mid;
    }
    const SceneP& P = T.scenes[lo];
    const Grid& g = P.sgrid;
    const uint32_t l = c - P.cell_base;
    if ((P.halved[1] | P.halved[2]) == 0u) {
        // only x halved: sub[0] is even, so x and l have the same parity
        if (l & P.halved[0]) return 0u;
    } else {
        const uint32_t x = l % g.sub[0], y = (l / g.sub[0]) % g.sub[1], z = l / (g.sub[0] * g.sub[1]);
        if (((x & P.halved[0]) | (y & P.halved[1]) | (z & P.halved[2])) != 0u) return 0u;
    }
    uint32_t occ = 0;
    for (uint32_t dz = 0; dz <= P.halved[2]; ++dz)
        for (uint32_t dy = 0; dy <= P.halved[1]; ++dy) {
            const uint32_t r0 = c + dy * g.sub[0] + dz * g.sub[0] * g.sub[1], r1 = r0 + 1u + P.halved[0];
            occ += start[r1] - start[r0];
            if (bstart) occ += bstart[r1] - bstart[r0];
        }
    return occ;
}

constexpr uint32_t kShortRun = 32;    // runs up to this length: insertion sort by their own thread
constexpr uint32_t kWarpRun = 256;    // up to this length: bitonic sort in shared memory by one warp
constexpr uint32_t kBlockRun = 4096;  // up to this length: bitonic sort in shared memory by the block

// Block-wide reductions (blockDim.x == kThreads); every thread gets the result.
template <class Op>
__device__ __forceinline__ uint32_t block_reduce(uint32_t v, Op op) {
    __shared__ uint32_t part[kThreads / 32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = op(v, __shfl_xor_sync(0xffffffffu, v, o));
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = v;
    __syncthreads();
    uint32_t r = part[0];
    for (int w = 1; w < kThreads / 32; ++w) r = op(r, part[w]);
    __syncthreads();  // part[] is reused by the next call
    return r;
}

// Sorts one long run perm[b, e) ascending with the whole block: stable
// one-bit LSD radix passes over (v - min), ping-ponging through tmp[b, e).
// The run's values are distinct slots, and a run of a cell-ordered state
// spans few slots, so log2(max - min + 1) passes suffice.
__device__ void block_sort_run(uint32_t* perm, uint32_t* tmp, uint32_t b, uint32_t e) {
    __shared__ uint32_t chunk_zeros;
    const uint32_t L = e - b;
    uint32_t lo = 0xFFFFFFFFu, hi = 0u;
    for (uint32_t i = threadIdx.x; i < L; i += kThreads) {
        const uint32_t v = perm[b + i];
        lo = min(lo, v);
        hi = max(hi, v);
    }
    lo = block_reduce(lo, [](uint32_t x, uint32_t y) { return min(x, y); });
    hi = block_reduce(hi, [](uint32_t x, uint32_t y) { return max(x, y); });
    const uint32_t span = hi - lo;
    const int bits = span ? 32 - __clz(span) : 0;
    uint32_t* src = perm + b;
    uint32_t* dst = tmp + b;
    for (int bit = 0; bit < bits; ++bit) {
        uint32_t z = 0;
        for (uint32_t i = threadIdx.x; i < L; i += kThreads) z += (((src[i] - lo) >> bit) & 1u) ^ 1u;
        z = block_reduce(z, [](uint32_t x, uint32_t y) { return x + y; });
        uint32_t zbase = 0, obase = z;
        for (uint32_t c0 = 0; c0 < L; c0 += kThreads) {
            const uint32_t i = c0 + threadIdx.x;
            const uint32_t v = i < L ? src[i] : 0u;
            const uint32_t f = i < L ? ((((v - lo) >> bit) & 1u) ^ 1u) : 0u;
            uint32_t excl;
            block_excl_scan(f, excl);
            if (threadIdx.x == kThreads - 1) chunk_zeros = excl + f;
            __syncthreads();
            const uint32_t cz = chunk_zeros;
            if (i < L) dst[f ? zbase + excl : obase + (threadIdx.x - excl)] = v;
            zbase += cz;
            obase += min((uint32_t)kThreads, L - c0) - cz;
            __syncthreads();  // chunk_zeros and the scan's shared totals are reused
        }
        __syncthreads();  // dst complete before the next pass reads it
        uint32_t* t = src;
        src = dst;
        dst = t;
    }
    if (src != perm + b)
        for (uint32_t i = threadIdx.x; i < L; i += kThreads) perm[b + i] = src[i];
    __syncthreads();
}

// Sorts one run perm[b, b + L) (L <= kWarpRun) ascending with one warp: a
// bitonic network over the run padded to a power of two in `buf` (shared
// memory, kWarpRun entries of this warp).  The values are distinct slots.
__device__ void warp_sort_run(uint32_t* perm, uint32_t b, uint32_t L, uint32_t* buf) {
    const uint32_t lane = threadIdx.x & 31u;
    uint32_t P = 32u;
    while (P < L) P <<= 1;
    for (uint32_t i = lane; i < P; i += 32u) buf[i] = i < L ? perm[b + i] : 0xFFFFFFFFu;
    __syncwarp();
    for (uint32_t k = 2u; k <= P; k <<= 1)
        for (uint32_t j = k >> 1; j > 0u; j >>= 1) {
            for (uint32_t i = lane; i < P; i += 32u) {
                const uint32_t ixj = i ^ j;
                if (ixj > i) {
                    const uint32_t x = buf[i], y = buf[ixj];
                    if ((x > y) == ((i & k) == 0u)) {
                        buf[i] = y;
                        buf[ixj] = x;
                    }
                }
            }
            __syncwarp();
        }
    for (uint32_t i = lane; i < L; i += 32u) perm[b + i] = buf[i];
    __syncwarp();
}

// Sorts one run perm[b, b + L) (kWarpRun < L <= kBlockRun) ascending with the
// whole block: a bitonic network in shared memory (`buf`, kBlockRun entries).
__device__ void block_bitonic_run(uint32_t* perm, uint32_t b, uint32_t L, uint32_t* buf) {
    uint32_t P = 2u * kWarpRun;
    while (P < L) P <<= 1;
    for (uint32_t i = threadIdx.x; i < P; i += kThreads) buf[i] = i < L ? perm[b + i] : 0xFFFFFFFFu;
    __syncthreads();
    for (uint32_t k = 2u; k <= P; k <<= 1)
        for (uint32_t j = k >> 1; j > 0u; j >>= 1) {
            for (uint32_t i = threadIdx.x; i < P; i += kThreads) {
                const uint32_t ixj = i ^ j;
                if (ixj > i) {
                    const uint32_t x = buf[i], y = buf[ixj];
                    if ((x > y) == ((i & k) == 0u)) {
                        buf[i] = y;
                        buf[ixj] = x;
                    }
                }
            }
            __syncthreads();
        }
    for (uint32_t i = threadIdx.x; i < L; i += kThreads) perm[b + i] = buf[i];
    __syncthreads();
}

// Sort each cell's run ascending, so the order inside a cell never depends
// on the arrival order of the histogram's atomics: runs of at most kShortRun
// by an insertion sort on their own thread, runs of at most kWarpRun by one
// warp each (warp_sort_run; the block's warps share its runs), runs of at
// most kBlockRun by the whole block in shared memory (block_bitonic_run), and
// longer ones (cells that gather particles outside the box, which are
// clamped into the edge cells) by the whole block through the scratch `tmp`,
// free once the scatter has run (block_sort_run).
// With `stats`, also the occupancy counters of the reference cells.
__global__ void __launch_bounds__(kThreads) k_sort_runs(const uint32_t* __restrict__ start, uint32_t ncells,
                                                        uint32_t* __restrict__ perm, uint32_t* __restrict__ tmp,
                                                        const uint32_t* __restrict__ boundary_start, DevStats* stats,
                                                        Tables T) {
    __shared__ uint32_t long_cells[kThreads], mid_cells[kThreads];
    __shared__ uint32_t nlong, nmid;
    __shared__ uint32_t wbuf[kBlockRun];  // kThreads / 32 warp buffers of kWarpRun, or one block buffer
    if (threadIdx.x == 0) nlong = nmid = 0;
    __syncthreads();
    const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c <= ncells) {  // includes the non-finite bucket at index ncells
        const uint32_t b = start[c], e = start[c + 1];
        const uint32_t len = e - b;
        if (stats && c < ncells) {
            const uint32_t occ = reference_cell_occupancy(c, start, boundary_start, T);
            if (occ > 0) atomicMax(&stats->max_cell_occupancy, occ);
            if (occ > kBucketSlots) atomicAdd(&stats->overflow_cells, 1u);
        }
        if (len > kWarpRun) {
            long_cells[atomicAdd(&nlong, 1u)] = c;
        } else if (len > kShortRun) {
            mid_cells[atomicAdd(&nmid, 1u)] = c;
        } else if (len >= 2) {
            for (uint32_t i = b + 1; i < e; ++i) {
                uint32_t v = perm[i];
                uint32_t j = i;
                while (j > b && perm[j - 1] > v) {
                    perm[j] = perm[j - 1];
                    --j;
                }
                perm[j] = v;
            }
        }
    }
    __syncthreads();
    const uint32_t nm = nmid, warp = threadIdx.x >> 5;
    for (uint32_t q = warp; q < nm; q += kThreads / 32) {
        const uint32_t mc = mid_cells[q];
        warp_sort_run(perm, start[mc], start[mc + 1] - start[mc], wbuf + warp * kWarpRun);
    }
    __syncthreads();  // the warps' buffers are the block buffer below
    const uint32_t cnt = nlong;
    for (uint32_t q = 0; q < cnt; ++q) {
        const uint32_t lc = long_cells[q];
        const uint32_t L = start[lc + 1] - start[lc];
        if (L <= kBlockRun) block_bitonic_run(perm, start[lc], L, wbuf);
        else block_sort_run(perm, tmp, start[lc], start[lc + 1]);
    }
}

__global__ void k_gather(const uint32_t* __restrict__ perm, uint32_t n, const float4* __restrict__ a_in,
                         float4* __restrict__ a_out, const float4* __restrict__ b_in, float4* __restrict__ b_out,
                         const uint32_t* __restrict__ c_in, uint32_t* __restrict__ c_out,
                         const uint32_t* __restrict__ d_in, uint32_t* __restrict__ d_out) {
    uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const uint32_t s = perm[k];
    if (a_out) a_out[k] = a_in[s];
    if (b_out) b_out[k] = b_in[s];
    if (c_out) c_out[k] = c_in[s];
    if (d_out) d_out[k] = d_in[s];
}

__device__ __forceinline__ float eos_pressure(uint32_t eq, float density, float c, float d0) {
    switch (eq) {  // fluid.rs:45-52, x^7 by products
        case ARP_EOS_CONSTANT: return c * c;
        case ARP_EOS_IDEAL_GAS: return c * c * (density - d0);
        case ARP_EOS_TAIT: {
            const float x = density / d0;
            const float x2 = x * x;
            const float x3 = x2 * x;
            const float x6 = x3 * x3;
            return (c * c * d0 / 7.0f) * (x6 * x - 1.0f);
        }
        default: return 0.0f;
    }
}

__global__ void k_gather_state(const uint32_t* __restrict__ perm, uint32_t n, const float4* __restrict__ pd_in,
                               float4* __restrict__ pd_out, const float4* __restrict__ vm_in,
                               float4* __restrict__ vm_out, const uint32_t* __restrict__ a_in,
                               uint32_t* __restrict__ a_out, const uint32_t* __restrict__ b_in,
                               uint32_t* __restrict__ b_out, const uint2* __restrict__ c_in,
                               uint2* __restrict__ c_out, float* __restrict__ ps_out,
                               const DevMat* __restrict__ mats, SolidScatter sol) {
    uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const uint32_t s = perm ? perm[k] : k;
    const float4 pd = pd_in[s];
    const float4 vm = vm_in[s];
    if (pd_out) pd_out[k] = pd;
    if (vm_out) vm_out[k] = vm;
    if (sol.sx) {
        const uint32_t sid = sol.sid_of_slot[s];
        if (sid != kInvalid) {
            sol.sx[sid] = pd;
            sol.sv[sid] = vm;
            sol.sc[sid] = sol.coord_of_slot[s];
            if (sol.slot_of) sol.slot_of[sid] = k;
        }
    }
    if (a_out) a_out[k] = a_in[s];
    if (b_out) b_out[k] = b_in[s];
    if (c_out) c_out[k] = c_in[s];
    if (ps_out) {
        const DevMat& m = mats[__float_as_uint(vm.w)];
        const float p = eos_pressure(m.state_eq, pd.w, m.sound_speed, m.target_den);
        ps_out[k] = p / (pd.w * pd.w);
    }
}

// Particle records (48 B, caller order) -> structure of arrays in caller order.
__global__ void k_records_to_soa(const arp_particle* __restrict__ in, uint32_t n, const uint32_t* __restrict__ sid_of,
                                 const uint32_t* __restrict__ mat_of, float4* __restrict__ pd, float4* __restrict__ vm,
                                 uint32_t* __restrict__ orig, uint32_t* __restrict__ sid) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4* r = reinterpret_cast<const float4*>(in + i);
    const float4 h = r[0], p = r[1], v = r[2];  // (den, mat, solid_id, pad), pos, vel
    pd[i] = make_float4(p.x, p.y, p.z, h.x);
    vm[i] = make_float4(v.x, v.y, v.z, __uint_as_float(mat_of[i]));  // batch-wide material id
    orig[i] = i;
    sid[i] = sid_of[i];
}

// Bit 0: a record's material differs from the handle's; bit 1: a w component
// differs from the handle's common w / zero.
__global__ void k_check_records(const arp_particle* __restrict__ in, uint32_t n, const uint32_t* __restrict__ mat_of,
                                const DevMat* __restrict__ mats, float pos_w, uint32_t* __restrict__ flag) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const arp_particle& r = in[i];
    uint32_t bad = (r.mat != mats[mat_of[i]].local) ? 1u : 0u;
    if (r.pos[3] != pos_w || r.vel[3] != 0.0f) bad |= 2u;
    if (bad) atomicOr(flag, bad);
}

// Cell-ordered structure of arrays -> particle records in caller order.
__global__ void k_soa_to_records(const float4* __restrict__ pd, const float4* __restrict__ vm,
                                 const uint32_t* __restrict__ orig, const uint32_t* __restrict__ sid, uint32_t n,
                                 float pos_w, const DevMat* __restrict__ mats, arp_particle* __restrict__ out) {
    uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const float4 p = pd[k], v = vm[k];
    float4* r = reinterpret_cast<float4*>(out + orig[k]);
    const DevMat& m = mats[__float_as_uint(v.w)];
    const uint32_t sk = sid[k];
    // the scene's own material index and solid id
    r[0] = make_float4(p.w, __uint_as_float(m.local), __uint_as_float(sk == kInvalid ? sk : sk - m.solid_base), 0.0f);
    r[1] = make_float4(p.x, p.y, p.z, pos_w);
    r[2] = make_float4(v.x, v.y, v.z, 0.0f);
}

__device__ __forceinline__ bool within_h_exact(float4 q, float4 p, float h2) {
    const float rx = __fsub_rn(q.x, p.x), ry = __fsub_rn(q.y, p.y), rz = __fsub_rn(q.z, p.z);
    const float d = __fadd_rn(__fadd_rn(__fmul_rn(rx, rx), __fmul_rn(ry, ry)), __fmul_rn(rz, rz));
    return __fsub_rn(h2, d) > 0.0f;
}

__global__ void k_count_neighbors(const float4* __restrict__ xs, const float4* __restrict__ vs,
                                  const uint32_t* __restrict__ start, uint32_t n, const float4* __restrict__ bxs,
                                  const uint32_t* __restrict__ bstart, Tables T, uint32_t* __restrict__ out) {
    uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const float4 p = xs[k];
    uint32_t cnt = 0;
    if (finite3(p)) {
        const SceneP& P = T.scenes[scene_of(vs, nullptr, k, T)];
        // the shader's 3x3(x3) reference cells exactly
        for_reference_block_rows(p, P, [&](uint32_t c0, uint32_t c1) {
            if (bstart)
                for (uint32_t j = bstart[c0]; j < bstart[c1]; ++j) cnt += within_h_exact(bxs[j], p, P.h2);
            for (uint32_t j = start[c0]; j < start[c1]; ++j) cnt += within_h_exact(xs[j], p, P.h2);
        });
    }
    out[k] = cnt;
}

inline uint32_t blocks_for(uint32_t n, int t) { return (n + (uint32_t)t - 1u) / (uint32_t)t; }

// ---- allocation-free grid build ---------------------------------------------
// Scratch of arp_grid_build_noalloc: arrival ranks of up to kNoAllocMaxParticles
// particles, then the scan's tile totals.  The histogram and its scan live in
// the caller's cell_start array, and cell keys are recomputed from the
// positions instead of stored.  4 MiB + 4 KiB per GPU that loads the library.
constexpr uint32_t kNoAllocMaxParticles = 1u << 20;
constexpr uint32_t kNoAllocMaxCells = (1u << 22) - 2;  // cell_start then holds at most 2^22 entries
constexpr uint32_t kNoAllocMaxTiles = (kNoAllocMaxCells + 2 + kScanTile - 1) / kScanTile;
__device__ __align__(256) uint32_t g_noalloc_scratch[kNoAllocMaxParticles + kNoAllocMaxTiles];

__global__ void k_rank_noalloc(const float4* __restrict__ pos, uint32_t n, Grid grid, uint32_t* __restrict__ count,
                               uint32_t* __restrict__ rank) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 p = pos[i];
    const uint32_t k = finite3(p) ? cell_id(cell_coord(p, grid), grid) : grid.ncells;
    rank[i] = atomicAdd(&count[k], 1u);
}

__global__ void k_scatter_noalloc(const float4* __restrict__ pos, uint32_t n, Grid grid,
                                  const uint32_t* __restrict__ start, const uint32_t* __restrict__ rank,
                                  uint32_t* __restrict__ perm) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 p = pos[i];
    const uint32_t k = finite3(p) ? cell_id(cell_coord(p, grid), grid) : grid.ncells;
    perm[start[k] + rank[i]] = i;
}

// Device address of g_noalloc_scratch, looked up once per device with that
// device current (host code may not use the symbol itself as an address).
constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mu;
uint32_t* g_noalloc_ptr[kMaxDevices] = {};

cudaError_t noalloc_scratch(uint32_t** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_ptr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return e;
        g_noalloc_ptr[dev] = static_cast<uint32_t*>(p);
    }
    *out = g_noalloc_ptr[dev];
    return cudaSuccess;
}

}  // namespace

int build_grid(const float4* pos, const float4* vm, const uint32_t* mat_u32, uint32_t n, const Tables& T,
               GridBuffers& gb, DevStats* stats, const uint32_t* boundary_start, cudaStream_t st,
               const StageCounters& zero) {
    int launches = 0;
    if (n > 0) {
        // a single scene needs no material to find the scene: skip that read
        const bool one = T.nscenes == 1;
        k_cell_keys<<<blocks_for(n, kThreads), kThreads, 0, st>>>(pos, one ? nullptr : vm, one ? nullptr : mat_u32, n,
                                                                  T, gb.key, gb.rank, gb.count, gb.coord, stats,
                                                                  zero);
        ++launches;
    }
    // cells, the non-finite bucket, and the total
    launches += exclusive_scan(gb.count, T.ncells + 2, gb.start, gb.block_sums, st);
    if (n > 0) {
        k_scatter<<<blocks_for(n, kThreads), kThreads, 0, st>>>(gb.key, gb.rank, n, gb.start, gb.perm);
        ++launches;
    }
    k_sort_runs<<<blocks_for(T.ncells + 1, kThreads), kThreads, 0, st>>>(gb.start, T.ncells, gb.perm, gb.rank,
                                                                         boundary_start, stats, T);
    ++launches;
    return launches;
}

uint32_t scan_block_sums_needed(uint32_t len) { return blocks_for(len, kScanTile) + 1; }

int exclusive_scan(uint32_t* count, uint32_t len, uint32_t* out, uint32_t* block_sums, cudaStream_t st) {
    const uint32_t tiles = blocks_for(len, kScanTile);
    k_scan_tiles<<<tiles, kScanThreads, 0, st>>>(count, len, out, block_sums);
    k_scan_add<<<tiles, kScanThreads, 0, st>>>(out, len, block_sums);
    return 2;
}

int gather_sorted(const uint32_t* perm, uint32_t n, const float4* a_in, float4* a_out, const float4* b_in,
                  float4* b_out, const uint32_t* c_in, uint32_t* c_out, const uint32_t* d_in, uint32_t* d_out,
                  cudaStream_t st) {
    if (n == 0) return 0;
    k_gather<<<blocks_for(n, kThreads), kThreads, 0, st>>>(perm, n, a_in, a_out, b_in, b_out, c_in, c_out, d_in,
                                                           d_out);
    return 1;
}

int gather_state(const uint32_t* perm, uint32_t n, const float4* pd_in, float4* pd_out, const float4* vm_in,
                 float4* vm_out, const uint32_t* a_in, uint32_t* a_out, const uint32_t* b_in, uint32_t* b_out,
                 const uint2* c_in, uint2* c_out, float* ps_out, const DevMat* mats, cudaStream_t st,
                 const SolidScatter& sol) {
    if (n == 0) return 0;
    k_gather_state<<<blocks_for(n, kThreads), kThreads, 0, st>>>(perm, n, pd_in, pd_out, vm_in, vm_out, a_in, a_out,
                                                                 b_in, b_out, c_in, c_out, ps_out, mats, sol);
    return 1;
}

int records_to_soa(const arp_particle* in, uint32_t n, const uint32_t* sid_of, const uint32_t* mat_of, float4* pd,
                   float4* vm, uint32_t* orig, uint32_t* sid, cudaStream_t st) {
    if (n == 0) return 0;
    k_records_to_soa<<<blocks_for(n, kThreads), kThreads, 0, st>>>(in, n, sid_of, mat_of, pd, vm, orig, sid);
    return 1;
}

int check_records(const arp_particle* in, uint32_t n, const uint32_t* mat_of, const DevMat* mats, float pos_w,
                  uint32_t* flag, cudaStream_t st) {
    if (n == 0) return 0;
    k_check_records<<<blocks_for(n, kThreads), kThreads, 0, st>>>(in, n, mat_of, mats, pos_w, flag);
    return 1;
}

int soa_to_records(const float4* pd, const float4* vm, const uint32_t* orig, const uint32_t* sid, uint32_t n,
                   float pos_w, const DevMat* mats, arp_particle* out, cudaStream_t st) {
    if (n == 0) return 0;
    k_soa_to_records<<<blocks_for(n, kThreads), kThreads, 0, st>>>(pd, vm, orig, sid, n, pos_w, mats, out);
    return 1;
}

int count_neighbors(const float4* xs, const float4* vs, const uint32_t* start, uint32_t n, const float4* bxs,
                    const uint32_t* bstart, const Tables& T, uint32_t* out_sorted, cudaStream_t st) {
    if (n == 0) return 0;
    k_count_neighbors<<<blocks_for(n, kThreads), kThreads, 0, st>>>(xs, vs, start, n, bxs, bstart, T, out_sorted);
    return 1;
}

}  // namespace arp

// ---- C ABI: allocation-free grid build ----------------------------------------
extern "C" arp_status arp_grid_build_noalloc(const void* pos_den, uint32_t n, const arp_aabb* bounds,
                                             float kernel_radius, uint32_t* cell_start,
                                             uint32_t cell_start_capacity, uint32_t* perm, void* stream) {
    using namespace arp;
    if (!bounds) return set_error(ARP_ERR_INVALID_ARG, "bounds is null");
    if (!(kernel_radius > 0.0f)) return set_error(ARP_ERR_INVALID_ARG, "kernel_radius must be positive");
    if (bounds->dim[3] > 0.0f) return set_error(ARP_ERR_UNSUPPORTED, "4-dimensional boxes are not supported");
    if (n > kNoAllocMaxParticles)
        return set_error(ARP_ERR_CAPACITY, "arp_grid_build_noalloc: n exceeds the 1048576-particle maximum");
    if (n > 0 && (!pos_den || !perm)) return set_error(ARP_ERR_INVALID_ARG, "null position or perm pointer");
    if (!cell_start) return set_error(ARP_ERR_INVALID_ARG, "cell_start is null");
    if (reinterpret_cast<uintptr_t>(pos_den) % 16 != 0)
        return set_error(ARP_ERR_INVALID_ARG, "pos_den must be 16-byte aligned (float4 records)");
    Grid g{};
    uint64_t nc = 1;
    for (int a = 0; a < 3; ++a) {
        if (!std::isfinite(bounds->min[a]) || !std::isfinite(bounds->dim[a]) || bounds->dim[a] < 0.0f)
            return set_error(ARP_ERR_INVALID_ARG, "bounds must be finite with non-negative extent");
        g.min[a] = bounds->min[a];
        g.dim[a] = bounds->dim[a];
        // neighbor_list.rs:201-206; the quotient is range-checked in float
        // before the conversion (a huge dim / h would not fit in 32 bits)
        const float q = std::max(1.0f, bounds->dim[a] / kernel_radius);
        if (!(q <= (float)kNoAllocMaxCells))
            return set_error(ARP_ERR_CAPACITY, "arp_grid_build_noalloc: the grid exceeds the 4194302-cell maximum");
        g.sub[a] = (uint32_t)q;
        nc *= g.sub[a];
    }
    if (nc > kNoAllocMaxCells)
        return set_error(ARP_ERR_CAPACITY, "arp_grid_build_noalloc: the grid exceeds the 4194302-cell maximum");
    g.ncells = (uint32_t)nc;
    if ((uint64_t)cell_start_capacity < nc + 2)
        return set_error(ARP_ERR_CAPACITY, "cell_start must hold n_cells + 2 entries (" + std::to_string(nc + 2) +
                                               ")");
    uint32_t* scratch = nullptr;
    cudaError_t e = noalloc_scratch(&scratch);
    if (e != cudaSuccess) return set_error(ARP_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
    uint32_t* rank = scratch;
    uint32_t* tile_sums = scratch + kNoAllocMaxParticles;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const uint32_t len = g.ncells + 2;
    e = cudaMemsetAsync(cell_start, 0, (size_t)len * sizeof(uint32_t), st);
    if (e != cudaSuccess) return set_error(ARP_ERR_CUDA, std::string("cudaMemsetAsync: ") + cudaGetErrorString(e));
    const float4* pos = static_cast<const float4*>(pos_den);
    if (n > 0) k_rank_noalloc<<<blocks_for(n, kThreads), kThreads, 0, st>>>(pos, n, g, cell_start, rank);
    exclusive_scan(cell_start, len, cell_start, tile_sums, st);  // in place: counts become starts
    if (n > 0) k_scatter_noalloc<<<blocks_for(n, kThreads), kThreads, 0, st>>>(pos, n, g, cell_start, rank, perm);
    k_sort_runs<<<blocks_for(g.ncells + 1, kThreads), kThreads, 0, st>>>(cell_start, g.ncells, perm, rank, nullptr,
                                                                         nullptr, Tables{});
    e = cudaGetLastError();
    if (e != cudaSuccess) return set_error(ARP_ERR_CUDA, std::string("grid build launch: ") + cudaGetErrorString(e));
    return ARP_OK;
}
