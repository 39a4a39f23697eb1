// fluid.cu -- fluid forces with the Runge-Kutta stage update fused at the tail.
//
// Replaces the reference's `fluid_forces` shader (src/soft_body/shaders/
// fluid.rs:95-251) and the lin_comb stage arithmetic that follows it
// (src/soft_body/particle_state/particles.rs:8-154).  The shader runs one
// 81-invocation workgroup per particle (27 cells x 3 strided lanes) with a
// shared-memory tree reduction; here one thread owns one particle sorted by
// search cell (the reference cell halved along x) and walks 3 (2D) or 9 (3D)
// contiguous x-rows of 5 half-width cells, so neighbor loads are coalesced
// across a warp (consecutive threads sit in the same or adjacent cells) and
// 5/6 of the candidates of the 3x3x3 reference cells are tested.
//
// Per pair the math is the shader's, term by term: continuity density rate,
// symmetric pressure force with the equation of state evaluated for both
// particles, contact potential (with the shader's argument order) and
// friction, physical viscosity and artificial viscosity.  Every term carries
// grad_w, which is zero for |r| >= h, so pairs outside the kernel radius are
// skipped before any of it is evaluated.
//
// Epilogue: k = (v, drho/dt, F/rho - g y) (+ the solid term for solid
// particles) is combined into the next stage state y0 + sum c_j k_j and the
// b-weighted accumulator with separately rounded products and sums, the same
// order the oracle uses.
#include <algorithm>

#include "grid.cuh"

namespace arp {

namespace {

__device__ __forceinline__ float pow7(float x) {
    const float x2 = x * x;
    const float x3 = x2 * x;
    const float x6 = x3 * x3;
    return x6 * x;
}

// fluid.rs:54-67 (called with radius and strength in the shader's order)
__device__ __forceinline__ float contact_potential(uint32_t eq, float r, float strength, float r0) {
    switch (eq) {
        case ARP_CONTACT_CONSTANT: return r <= r0 ? strength : 0.0f;
        case ARP_CONTACT_LINEAR: return strength * (r0 - r);
        case ARP_CONTACT_TAIT: return (strength * r / 7.0f) * (pow7(r0 / r) - 1.0f);
        case ARP_CONTACT_LENNARD_JONES: {
            float f = r0 / r;
            f *= f * f;
            f *= f;
            return strength * (f * f - 2.0f * f);
        }
        case ARP_CONTACT_HERTZ: return (strength * r0 / 7.0f) * (pow7(r / r0) - 1.0f);
        default: return 0.0f;
    }
}

struct Self {
    float3 x, v;
    float d1, m1, pterm1, f1, bf1;
    uint32_t mat;     // global material id
    bool elastic;
    // material table and interaction row of the particle's scene, indexed by
    // the neighbor's global material id (shared-memory copies for the block's
    // first scene, the global tables otherwise)
    const FluidMat* mt;
    const DevInter* it;
};

struct Acc {
    float den;
    float3 f;
};

// One neighbor pair inside the kernel radius (the caller has tested it).
// `ptj` is p_j / rho_j^2 of the neighbor, precomputed per particle.
// The scene scalars the pair terms read, held in registers.
struct PairK {
    float h2, kconst, eps_hh;
};

template <int DIM, bool BOUNDARY>
__device__ __forceinline__ void pair(const Self& s, float4 xj, float4 vj, float ptj, uint32_t mat2, bool elastic2,
                                     const PairK& P, Acc& acc) {
    const float rx = xj.x - s.x.x, ry = xj.y - s.x.y, rz = DIM == 3 ? xj.z - s.x.z : 0.0f;
    const float r2 = DIM == 3 ? (rx * rx + ry * ry) + rz * rz : rx * rx + ry * ry;
    const float diff = fmaxf(P.h2 - r2, 0.0f);
    const float gws = -6.0f * P.kconst * diff * diff;
    const float gx = gws * rx, gy = gws * ry, gz = gws * rz;
    const float vx = vj.x - s.v.x, vy = vj.y - s.v.y, vz = DIM == 3 ? vj.z - s.v.z : 0.0f;
    const float d2 = xj.w;
    const FluidMat m2 = s.mt[mat2];
    const float vgw = DIM == 3 ? (vx * gx + vy * gy) + vz * gz : vx * gx + vy * gy;
    if (!BOUNDARY) acc.den += m2.mass * vgw;
    const float pf = s.m1 * m2.mass * (s.pterm1 + ptj);
    acc.f.x += pf * gx;
    acc.f.y += pf * gy;
    acc.f.z += pf * gz;
    const DevInter it = s.it[mat2];
    if (it.potential != ARP_CONTACT_ZERO) {
        const float cp = contact_potential(it.potential, sqrtf(r2), it.radius, it.strength);
        if (cp != 0.0f) {
            const float cs = m2.mass * cp / d2;
            const float cx = cs * gx, cy = cs * gy, cz = cs * gz;
            if ((s.elastic || elastic2 || BOUNDARY) && s.mat != mat2) {
                // fluid.rs:192-199: friction along the normalised tangential velocity
                const float ix = rx / r2, iy = ry / r2, iz = rz / r2;
                const float cr = DIM == 3 ? (cx * rx + cy * ry) + cz * rz : cx * rx + cy * ry;
                const float nx = ix * cr, ny = iy * cr, nz = iz * cr;
                const float vr = DIM == 3 ? (vx * rx + vy * ry) + vz * rz : vx * rx + vy * ry;
                float tx = vx - ix * vr, ty = vy - iy * vr, tz = vz - iz * vr;
                float tl = sqrtf(DIM == 3 ? (tx * tx + ty * ty) + tz * tz : tx * tx + ty * ty);
                tx /= tl; ty /= tl; tz /= tl;
                if (isfinite(tx) && isfinite(ty) && isfinite(tz)) {
                    // normalize() applied a second time, as the shader does
                    const float tl2 = sqrtf(DIM == 3 ? (tx * tx + ty * ty) + tz * tz : tx * tx + ty * ty);
                    const float nl = sqrtf(DIM == 3 ? (nx * nx + ny * ny) + nz * nz : nx * nx + ny * ny);
                    const float fr = it.friction * nl;
                    acc.f.x += fr * (tx / tl2);
                    acc.f.y += fr * (ty / tl2);
                    acc.f.z += fr * (tz / tl2);
                }
            }
            acc.f.x += cx;
            acc.f.y += cy;
            acc.f.z += cz;
        }
    }
    if (!BOUNDARY) {
        const float denom = r2 + P.eps_hh;
        if (!s.elastic) {
            const float fsum = s.f1 + m2.visc;
            if (fsum != 0.0f) {
                const float rgw = DIM == 3 ? (rx * gx + ry * gy) + rz * gz : rx * gx + ry * gy;
                const float q = s.m1 * m2.mass * fsum * rgw;
                const float dd = s.d1 * d2 * denom;
                // GLSL division carries 2.5 ulp; the 2-ulp hardware quotient is used here
                acc.f.x -= __fdividef(q * vx, dd);
                acc.f.y -= __fdividef(q * vy, dd);
                acc.f.z -= __fdividef(q * vz, dd);
            }
        }
        const float f_ = s.mat == mat2 ? s.bf1 + m2.bulk : it.dampening;
        if (f_ != 0.0f) {
            const float vr = DIM == 3 ? (vx * rx + vy * ry) + vz * rz : vx * rx + vy * ry;
            const float q = s.m1 * m2.mass * __fdividef(f_ * vr, (s.d1 + d2) * denom);
            acc.f.x -= q * gx;
            acc.f.y -= q * gy;
            acc.f.z -= q * gz;
        }
    }
}

__device__ __forceinline__ float4 comb(float4 y0, float4 t, bool keep_w) {
    float4 r;
    r.x = __fadd_rn(y0.x, t.x);
    r.y = __fadd_rn(y0.y, t.y);
    r.z = __fadd_rn(y0.z, t.z);
    r.w = keep_w ? y0.w : __fadd_rn(y0.w, t.w);
    return r;
}
__device__ __forceinline__ float4 axpy(float c, float4 k, float4 t) {
    return make_float4(__fadd_rn(t.x, __fmul_rn(c, k.x)), __fadd_rn(t.y, __fmul_rn(c, k.y)),
                       __fadd_rn(t.z, __fmul_rn(c, k.z)), __fadd_rn(t.w, __fmul_rn(c, k.w)));
}

constexpr uint32_t kBoundaryBit = 0x80000000u;

// Copy one scene's fluid materials and interaction block into shared memory.
__device__ __forceinline__ void load_scene_tables(const Tables& T, uint32_t scene, FluidMat* sm, DevInter* si) {
    const SceneP& sp = T.scenes[scene];
    for (uint32_t i = threadIdx.x; i < sp.nmat; i += blockDim.x) sm[i] = T.fmats[sp.mat_base + i];
    for (uint32_t i = threadIdx.x; i < sp.nmat * sp.nmat; i += blockDim.x) si[i] = T.inter[sp.inter_base + i];
}

// Pair terms of one hit: a boundary particle (index | kBoundaryBit) or a
// mobile one.
template <int DIM>
__device__ __forceinline__ void eval_hit(uint32_t j, const Self& s, const FluidArgs& a, const PairK& K, Acc& acc) {
    if (j & kBoundaryBit) {
        const uint32_t jb = j & ~kBoundaryBit;
        const float4 xj = a.bxs[jb];
        const float4 vj = a.bvs[jb];
        const uint32_t mat2 = __float_as_uint(vj.w);
        bool elastic2 = false;
        if (a.any_stiff_immobile && s.mt[mat2].stiff) {
            // fluid.rs:141: the boundary index reads the mobile array's solid id
            elastic2 = a.sid_of_boundary_index[a.borig[jb]] != kInvalid;
        }
        pair<DIM, true>(s, xj, vj, a.bps[jb], mat2, elastic2, K, acc);
    } else {
        const float4 xj = a.xs[j];
        const float4 vj = a.vs[j];
        const uint32_t mat2 = __float_as_uint(vj.w);
        pair<DIM, false>(s, xj, vj, a.ps[j], mat2, s.mt[mat2].stiff != 0u, K, acc);
    }
}

// The derivative record of one particle (fluid.rs:243-247, plus the solid
// term when active) and the Runge-Kutta stage epilogue: the store of k, the
// b-weighted accumulator and the next stage state, in storage slot `slot`.
__device__ __forceinline__ void stage_epilogue(const FluidArgs& a, const StageCoefs& c, const StageBuffers& b,
                                               uint32_t slot, uint32_t sid, float4 vi, const Acc& acc, float d1,
                                               float g_acc, bool solid_scene) {
    float4 kpd = make_float4(vi.x, vi.y, vi.z, acc.den);
    float4 kvm = make_float4(__fdiv_rn(acc.f.x, d1), __fadd_rn(__fdiv_rn(acc.f.y, d1), -g_acc),
                             __fdiv_rn(acc.f.z, d1), 0.0f);
    if (a.solid_branch && sid != kInvalid && solid_scene) {
        const float4 ks = a.ksol[sid];
        kpd.x = __fadd_rn(kpd.x, vi.x);
        kpd.y = __fadd_rn(kpd.y, vi.y);
        kpd.z = __fadd_rn(kpd.z, vi.z);
        kvm.x = __fadd_rn(kvm.x, ks.x);
        kvm.y = __fadd_rn(kvm.y, ks.y);
        kvm.z = __fadd_rn(kvm.z, ks.z);
    }

    // Runge-Kutta stage epilogue
    if (b.store_pd) {
        b.store_pd[slot] = kpd;
        b.store_vm[slot] = kvm;
    }
    const float4 y0p = b.y0_pd[slot];
    const float4 y0v = b.y0_vm[slot];
    float4 accp = make_float4(0.f, 0.f, 0.f, 0.f), accv = make_float4(0.f, 0.f, 0.f, 0.f);
    if (c.c_acc != 0.0f) {
        if (!c.acc_first) {
            accp = b.acc_pd[slot];
            accv = b.acc_vm[slot];
        }
        accp = axpy(c.c_acc, kpd, accp);
        accv = axpy(c.c_acc, kvm, accv);
        if (!c.last) {
            b.acc_pd[slot] = accp;
            b.acc_vm[slot] = accv;
        }
    } else if (c.last) {
        accp = b.acc_pd[slot];
        accv = b.acc_vm[slot];
    }
    if (c.last) {
        float4 np = comb(y0p, accp, false);
        if (c.kick) {  // a velocity-Verlet kick moves no particle: positions come from the drift
            np.x = y0p.x;
            np.y = y0p.y;
            np.z = y0p.z;
        }
        b.next_pd[slot] = np;
        b.next_vm[slot] = comb(y0v, accv, true);
    } else {
        float4 tp = make_float4(0.f, 0.f, 0.f, 0.f), tv = make_float4(0.f, 0.f, 0.f, 0.f);
        if (c.c_prev0 != 0.0f) {
            tp = axpy(c.c_prev0, b.prev0_pd[slot], tp);
            tv = axpy(c.c_prev0, b.prev0_vm[slot], tv);
        }
        if (c.c_prev1 != 0.0f) {
            tp = axpy(c.c_prev1, b.prev1_pd[slot], tp);
            tv = axpy(c.c_prev1, b.prev1_vm[slot], tv);
        }
        if (c.c_prev2 != 0.0f) {
            tp = axpy(c.c_prev2, b.prev2_pd[slot], tp);
            tv = axpy(c.c_prev2, b.prev2_vm[slot], tv);
        }
        if (c.c_self != 0.0f) {
            tp = axpy(c.c_self, kpd, tp);
            tv = axpy(c.c_self, kvm, tv);
        }
        b.next_pd[slot] = comb(y0p, tp, false);
        b.next_vm[slot] = comb(y0v, tv, true);
    }
}

// The particle's own fields and table pointers for the pair loop; returns
// its scene.  `sm`/`si` hold the tables of scene `scene0`.
__device__ __forceinline__ const SceneP& init_self(uint32_t k, float4 xi, float4 vi, uint32_t sid, const FluidArgs& a,
                                                   const Tables& T, const FluidMat* sm, const DevInter* si,
                                                   uint32_t scene0, Self& s) {
    s.x = make_float3(xi.x, xi.y, xi.z);
    s.v = make_float3(vi.x, vi.y, vi.z);
    s.mat = __float_as_uint(vi.w);
    const uint32_t scene = T.mats[s.mat].scene;
    const SceneP& P = T.scenes[scene];
    const uint32_t li = s.mat - P.mat_base;
    // pre-offset so that [global id] lands on the scene's entry
    s.mt = (scene == scene0 ? sm : T.fmats + P.mat_base) - P.mat_base;
    s.it = (scene == scene0 ? si : T.inter + P.inter_base) + li * P.nmat - P.mat_base;
    s.d1 = xi.w;
    const FluidMat m1 = s.mt[s.mat];
    s.m1 = m1.mass;
    s.f1 = m1.visc;
    s.bf1 = m1.bulk;
    s.elastic = sid != kInvalid && m1.stiff;
    s.pterm1 = a.ps[k];
    return P;
}

// How fluid_particle collects and evaluates the hits of a particle.  Every
// mode sums the pairs in candidate order, so results do not depend on the
// mode, CAP or the launch shape.
enum FluidMode {
    kTwoPass = 0,  // pass 1 fills the list, pass 2 evaluates it; a full list
                   // queues the particle for kFlush (first overflow queue)
    kFlush = 1,    // the warp agrees before each row whether some lane's list
                   // could fill up in it and then evaluates and empties every
                   // list; a row alone above CAP queues the particle for
                   // kDirect (second overflow queue)
    kDirect = 2,   // every hit evaluated during the scan (a row above even the
                   // second queue's list)
};

// Fluid forces and the stage update of sorted particle k.  `lst` is the
// thread's column of the hit list ([CAP][BLOCK]); `sm`/`si` hold the
// tables of scene `scene0`.  A particle handed to an overflow queue writes
// nothing here.  `wmask` (kFlush): the lanes of this warp that run
// fluid_particle, all of which take part in the per-row vote.  QUEUE false
// (kFlush): a particle whose row holds more than CAP hits is not queued; the
// call returns false, having written nothing, and the caller finishes it.
template <int DIM, int BLOCK, int CAP, int MODE, bool QUEUE = true>
__device__ __forceinline__ bool fluid_particle(uint32_t k, const FluidArgs& a, const Tables& T, const StageCoefs& c,
                                               const StageBuffers& b, uint32_t* lst, const FluidMat* sm,
                                               const DevInter* si, uint32_t scene0, unsigned wmask) {
    const float4 xi = a.xs[k];
    const float4 vi = a.vs[k];
    const uint32_t slot = a.perm ? a.perm[k] : k;
    const uint32_t sid = a.sid[slot];
    Self s;
    const SceneP& P = init_self(k, xi, vi, sid, a, T, sm, si, scene0, s);
    const PairK K{P.h2, P.kconst, P.eps_hh};
    const float g_acc = P.g;

    Acc acc;
    acc.den = 0.0f;
    acc.f = make_float3(0.0f, 0.0f, 0.0f);
    uint32_t* my = lst;
    uint32_t cnt = 0;
    bool full = false;
    // pass 1: candidates of the search rows whose squared distance is inside
    // h^2 (r^2 < h^2 is h^2 - r^2 > 0, grad_w's max(.., 0) test: without
    // flush-to-zero a difference of finite floats is zero only when they are
    // equal).  The particle itself passes the test and is dropped when the
    // hits are evaluated, which keeps the index compare out of this loop.
    auto hit = [&](float4 q) {
        const float rx = q.x - xi.x, ry = q.y - xi.y;
        const float r2 = DIM == 3 ? fmaf(q.z - xi.z, q.z - xi.z, fmaf(ry, ry, rx * rx)) : fmaf(ry, ry, rx * rx);
        return r2 < K.h2;
    };
    constexpr bool DIRECT = MODE == kDirect;
    auto take = [&](uint32_t j) {
        if (DIRECT) {
            if (j != k) eval_hit<DIM>(j, s, a, K, acc);
        } else if (cnt < CAP) {
            my[cnt++ * BLOCK] = j;
        } else {
            full = true;
        }
    };
    // pass 2 over the hits collected so far, in candidate order
    auto flush = [&]() {
        for (uint32_t e = 0; e < cnt; ++e) {
            const uint32_t j = my[e * BLOCK];
            if (j != k) eval_hit<DIM>(j, s, a, K, acc);
        }
        cnt = 0;
    };
    if (MODE == kFlush) {
        // The search rows (x-rows of the search cells within reach, see
        // for_search_rows) in a fixed order and number for every lane, rows
        // outside the grid (and every row of a non-finite particle) empty, so
        // that the warp can vote before each row; the pass after the last row
        // only evaluates what is left (one call site of the pair math keeps
        // the registers down).
        // (y reach: 2 rows for every lane, as dense scenes halve y; a lane
        // whose scene does not skips the outer two as empty)
        constexpr int RY = 2, RZ = 1 + (int)(kSearchHalve >> 2 & 1u);
        constexpr int NY = 2 * RY + 1, NZ = DIM == 3 ? 2 * RZ + 1 : 1;
        const bool fin = finite3(xi);
        const Grid& g = P.sgrid;
        const CellCoord cc = fin ? cell_coord(xi, g) : CellCoord{0, 0, 0};
        const int rx = 1 + (int)P.halved[0], ry = 1 + (int)P.halved[1];
        const int x0 = max(cc.x - rx, 0), x1 = min(cc.x + rx, (int)g.sub[0] - 1);
        for (int r = 0;; ++r) {
            const bool last = r == NY * NZ;
            const int dy = r % NY - RY;
            const int y = cc.y + dy;
            const int z = DIM == 3 ? cc.z - RZ + r / NY : cc.z;
            uint32_t bb = 0, be = 0, jb = 0, je = 0;
            if (!last && fin && abs(dy) <= ry && y >= 0 && y < (int)g.sub[1] && z >= 0 && z < (int)g.sub[2]) {
                const uint32_t row = P.cell_base + (uint32_t)y * g.sub[0] + (uint32_t)z * g.sub[0] * g.sub[1];
                const uint32_t c0 = row + (uint32_t)x0, c1 = row + (uint32_t)x1 + 1u;
                bb = a.bstart[c0];
                be = a.bstart[c1];
                jb = a.start[c0];
                je = a.start[c1];
            }
            const bool fl = last || __any_sync(wmask, !full && cnt + (be - bb) + (je - jb) > (uint32_t)CAP);
            if (fl && !full) flush();
            if (last) break;
            if (full) continue;
            for (uint32_t j = bb; j < be; ++j)
                if (hit(a.bxs[j])) take(j | kBoundaryBit);
            for (uint32_t j = jb; j < je; ++j)
                if (hit(a.xs[j])) take(j);
        }
        if (full) {
            if (!QUEUE) return false;
            a.overflow[a.n + atomicAdd(a.overflow_count + 1, 1u)] = k;
            return true;
        }
    } else if (finite3(xi)) {
        for_search_rows<DIM>(xi, P, [&](uint32_t c0, uint32_t c1) {
            if (full) return;
            const uint32_t bb = a.bstart[c0], be = a.bstart[c1];
            for (uint32_t j = bb; j < be; ++j)
                if (hit(a.bxs[j])) take(j | kBoundaryBit);
            const uint32_t jb = a.start[c0], je = a.start[c1];
            uint32_t j = jb;
            for (; j + 3u < je; j += 4u) {  // four loads in flight
                const float4 q0 = a.xs[j], q1 = a.xs[j + 1u], q2 = a.xs[j + 2u], q3 = a.xs[j + 3u];
                const bool h0 = hit(q0), h1 = hit(q1), h2 = hit(q2), h3 = hit(q3);
                if (h0) take(j);
                if (h1) take(j + 1u);
                if (h2) take(j + 2u);
                if (h3) take(j + 3u);
            }
            for (; j < je; ++j)
                if (hit(a.xs[j])) take(j);
        });
        if (MODE == kTwoPass) {
            if (full) {
                a.overflow[atomicAdd(a.overflow_count, 1u)] = k;
                return true;
            }
            flush();  // pass 2
        }
    }

    stage_epilogue(a, c, b, slot, sid, vi, acc, s.d1, g_acc, P.solid_branch != 0u);
    return true;
}

// The flush form keeps the row loop's state live around the pair math; left
// alone the compiler gives it 92 registers (5 blocks of 128 per SM), and
// holding it to 7 blocks (72 registers, a few spilled) ran the batched
// workload's fluid kernel 7 % faster.  The two-pass form keeps the
// compiler's own choice (72 registers at 128 threads; an explicit minimum of
// one block raises it to 80).
constexpr int kFlushMinBlocks = 7;

// One tile of BLOCK sorted particles per block.
template <int DIM, int BLOCK, int CAP, int MODE>
__device__ __forceinline__ void fluid_tile(const FluidArgs& a, const Tables& T, const StageCoefs& c,
                                           const StageBuffers& b) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    uint32_t* lst = reinterpret_cast<uint32_t*>(smem_raw);
    FluidMat* sm = reinterpret_cast<FluidMat*>(smem_raw + sizeof(uint32_t) * CAP * BLOCK);
    DevInter* si = reinterpret_cast<DevInter*>(reinterpret_cast<unsigned char*>(sm) + sizeof(FluidMat) * T.max_nmat);
    const uint32_t k0 = blockIdx.x * BLOCK;
    const uint32_t scene0 = T.mats[__float_as_uint(a.vs[min(k0, a.n - 1u)].w)].scene;
    load_scene_tables(T, scene0, sm, si);
    __syncthreads();
    const uint32_t k = k0 + threadIdx.x;
    const unsigned wmask = MODE == kFlush ? __ballot_sync(0xFFFFFFFFu, k < a.n) : 0u;  // lanes with a particle
    if (k < a.n) fluid_particle<DIM, BLOCK, CAP, MODE>(k, a, T, c, b, lst + threadIdx.x, sm, si, scene0, wmask);
}

// Persistent form: each block keeps taking the next tile of the cell-sorted,
// scene-concatenated order from an atomic work counter, so scenes of very
// different sizes share the SMs without a tail of idle blocks.  Blocks never
// wait on each other.
template <int DIM, int BLOCK, int CAP, int MODE>
__device__ __forceinline__ void fluid_tiles_persistent(const FluidArgs& a, const Tables& T, const StageCoefs& c,
                                                       const StageBuffers& b, uint32_t* tile_counter) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    uint32_t* lst = reinterpret_cast<uint32_t*>(smem_raw);
    FluidMat* sm = reinterpret_cast<FluidMat*>(smem_raw + sizeof(uint32_t) * CAP * BLOCK);
    DevInter* si = reinterpret_cast<DevInter*>(reinterpret_cast<unsigned char*>(sm) + sizeof(FluidMat) * T.max_nmat);
    __shared__ uint32_t tile_s;
    uint32_t loaded = kInvalid;
    const uint32_t ntiles = (a.n + BLOCK - 1) / BLOCK;
    for (;;) {
        if (threadIdx.x == 0) tile_s = atomicAdd(tile_counter, 1u);
        __syncthreads();
        const uint32_t tile = tile_s;
        if (tile >= ntiles) break;
        const uint32_t k0 = tile * BLOCK;
        const uint32_t scene0 = T.mats[__float_as_uint(a.vs[k0].w)].scene;
        if (scene0 != loaded) {
            load_scene_tables(T, scene0, sm, si);
            loaded = scene0;
        }
        __syncthreads();
        const uint32_t k = k0 + threadIdx.x;
        const unsigned wmask = MODE == kFlush ? __ballot_sync(0xFFFFFFFFu, k < a.n) : 0u;  // lanes with a particle
        if (k < a.n) fluid_particle<DIM, BLOCK, CAP, MODE>(k, a, T, c, b, lst + threadIdx.x, sm, si, scene0, wmask);
        __syncthreads();
    }
}

template <int DIM, int BLOCK, int CAP>
__global__ void __launch_bounds__(BLOCK) k_fluid(FluidArgs a, Tables T, StageCoefs c, StageBuffers b) {
    fluid_tile<DIM, BLOCK, CAP, kTwoPass>(a, T, c, b);
}
template <int DIM, int BLOCK, int CAP>
__global__ void __launch_bounds__(BLOCK) k_fluid_persistent(FluidArgs a, Tables T, StageCoefs c, StageBuffers b,
                                                            uint32_t* tile_counter) {
    fluid_tiles_persistent<DIM, BLOCK, CAP, kTwoPass>(a, T, c, b, tile_counter);
}
template <int DIM, int BLOCK, int CAP>
__global__ void __launch_bounds__(BLOCK, kFlushMinBlocks * 128 / BLOCK)
    k_fluid_flush(FluidArgs a, Tables T, StageCoefs c, StageBuffers b) {
    fluid_tile<DIM, BLOCK, CAP, kFlush>(a, T, c, b);
}
template <int DIM, int BLOCK, int CAP>
__global__ void __launch_bounds__(BLOCK, kFlushMinBlocks * 128 / BLOCK)
    k_fluid_flush_persistent(FluidArgs a, Tables T, StageCoefs c, StageBuffers b, uint32_t* tile_counter) {
    fluid_tiles_persistent<DIM, BLOCK, CAP, kFlush>(a, T, c, b, tile_counter);
}

// The kernels of one launch shape (only the used ones are instantiated).
template <int DIM, int BLOCK, int CAP, int MODE>
struct FluidKernels {
    static constexpr auto tile_kernel() {
        if constexpr (MODE == kFlush) return k_fluid_flush<DIM, BLOCK, CAP>;
        else return k_fluid<DIM, BLOCK, CAP>;
    }
    static constexpr auto persistent_kernel() {
        if constexpr (MODE == kFlush) return k_fluid_flush_persistent<DIM, BLOCK, CAP>;
        else return k_fluid_persistent<DIM, BLOCK, CAP>;
    }
    static constexpr auto tile = tile_kernel();
    static constexpr auto persistent = persistent_kernel();
};

// First overflow queue: particles whose hit list filled up, evaluated with
// list flushes (kFlush), grid-stride over the queue.
constexpr int kFlushCap = 64;
template <int DIM>
__global__ void __launch_bounds__(128, kFlushMinBlocks) k_fluid_overflow_flush(FluidArgs a, Tables T, StageCoefs c,
                                                                                StageBuffers b) {
    __shared__ uint32_t lst[kFlushCap * 128];
    const uint32_t cnt = a.overflow_count[0];
    for (uint32_t i0 = blockIdx.x * 128u; i0 < cnt; i0 += gridDim.x * 128u) {  // uniform per block
        const uint32_t i = i0 + threadIdx.x;
        const unsigned wmask = __ballot_sync(0xFFFFFFFFu, i < cnt);  // lanes with a particle
        if (i < cnt)
            fluid_particle<DIM, 128, kFlushCap, kFlush>(a.overflow[i], a, T, c, b, lst + threadIdx.x, nullptr,
                                                         nullptr, kInvalid, wmask);
    }
}

// Second overflow queue: particles with more hits in one row than the list
// that queued them holds.  The same flushing scan with lists of kWideCap
// entries (64 threads per block, 40 KB of shared memory); a particle with
// even more hits in one row is finished by its own thread evaluating its
// pairs during the scan.
constexpr int kWideCap = 160;
template <int DIM>
__global__ void __launch_bounds__(64) k_fluid_overflow(FluidArgs a, Tables T, StageCoefs c, StageBuffers b) {
    __shared__ uint32_t lst[kWideCap * 64];
    const uint32_t cnt = a.overflow_count[1];
    for (uint32_t i0 = blockIdx.x * 64u; i0 < cnt; i0 += gridDim.x * 64u) {  // uniform per block
        const uint32_t i = i0 + threadIdx.x;
        const unsigned wmask = __ballot_sync(0xFFFFFFFFu, i < cnt);  // lanes with a particle
        if (i < cnt) {
            const uint32_t k = a.overflow[a.n + i];
            if (!fluid_particle<DIM, 64, kWideCap, kFlush, false>(k, a, T, c, b, lst + threadIdx.x, nullptr,
                                                                   nullptr, kInvalid, wmask))
                fluid_particle<DIM, 64, 1, kDirect>(k, a, T, c, b, nullptr, nullptr, nullptr, kInvalid, 0u);
        }
    }
}

// ---- staged form -----------------------------------------------------------
// One tile of BLOCK consecutive cell-sorted particles per block, with the
// candidates of the tile staged in shared memory before the scan.  The tile's
// particles lie in a few x-rows of search cells ("own rows"); for each own row
// the NY x NZ neighbor rows it reaches are windows of contiguous cells, and
// the positions of each window (a contiguous range of the sorted state) are
// copied into shared memory once per block, instead of each thread reading
// every candidate through L1 (a tile's particles share most candidates).
// The scan then reads candidates from shared memory in the order the global
// scan visits them (rows z-major, then y, cells ascending; boundary
// candidates first in each row, read from global memory), so the pairs are
// summed in the same order and the results are the same bits.  A tile with
// more own rows than kMaxOwnRows or more candidates than kStageSlots sends its
// particles to the first overflow queue.
constexpr int kStageSlots = 1536;   // staged positions per block (24 KB)
constexpr int kMaxOwnRows = 4;
constexpr int kStageRY = 2;         // y reach of a dense scene (x-halved scenes use 1)
constexpr int kStageRZ = 1 + (int)(kSearchHalve >> 2 & 1u);
constexpr int kStageNY = 2 * kStageRY + 1;

template <int DIM>
struct StageShape {
    static constexpr int NZ = DIM == 3 ? 2 * kStageRZ + 1 : 1;
    static constexpr int NQ = kStageNY * NZ;   // windows per own row
    static constexpr int NW = kMaxOwnRows * NQ;
};

// Shared-memory bytes of a staged launch.
template <int DIM, int BLOCK, int CAP>
constexpr size_t staged_smem_fixed() {
    return 16 * (size_t)kStageSlots + sizeof(uint32_t) * (size_t)CAP * BLOCK;
}

// Bulk-copy staging (cp.async.bulk, global -> shared, one copy per window,
// completion counted on an mbarrier).  Waits are bounded: a block whose
// copies have not landed after kStageSpins polls sends its tile to the first
// overflow queue (after waiting, again bounded, for the copies in flight), so
// results never depend on the staging.
constexpr uint32_t kStageSpins = 1u << 22;
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void bulk_copy_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0u;
}
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, uint32_t spins) {
    for (uint32_t k = 0; k < spins; ++k)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

template <int DIM, int BLOCK, int CAP, bool BULK>
__global__ void __launch_bounds__(BLOCK) k_fluid_staged(FluidArgs a, Tables T, StageCoefs c, StageBuffers b) {
    using SS = StageShape<DIM>;
    static_assert(BLOCK >= SS::NW && BLOCK % 32 == 0, "one thread per window");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float4* stg = reinterpret_cast<float4*>(smem_raw);
    uint32_t* lst = reinterpret_cast<uint32_t*>(smem_raw + 16 * (size_t)kStageSlots);
    FluidMat* sm = reinterpret_cast<FluidMat*>(lst + CAP * BLOCK);
    DevInter* si = reinterpret_cast<DevInter*>(reinterpret_cast<unsigned char*>(sm) + sizeof(FluidMat) * T.max_nmat);
    __shared__ uint32_t s_row[BLOCK];          // global row id (first cell of the x-row) of each thread, or invalid
    __shared__ uint32_t s_heads[BLOCK / 32];   // own-row heads per warp
    __shared__ uint32_t r_scene[kMaxOwnRows], r_base[kMaxOwnRows], r_xa[kMaxOwnRows], r_xb[kMaxOwnRows];
    __shared__ int r_y[kMaxOwnRows], r_z[kMaxOwnRows];
    __shared__ uint32_t w_gstart[SS::NW], w_off[SS::NW + 1];
    __shared__ uint32_t s_nrows;
    __shared__ __align__(8) uint64_t s_bar;
    __shared__ uint32_t s_landed;

    const uint32_t k0 = blockIdx.x * BLOCK;
    if (BULK && threadIdx.x == 0) mbar_init(&s_bar, 1);  // ordered before its use by the barriers below
    const uint32_t k = k0 + threadIdx.x;
    const uint32_t scene0 = T.mats[__float_as_uint(a.vs[min(k0, a.n - 1u)].w)].scene;
    load_scene_tables(T, scene0, sm, si);

    // own rows: consecutive threads of one x-row of search cells
    const bool valid = k < a.n;
    float4 xi = make_float4(0.f, 0.f, 0.f, 0.f), vi = xi;
    CellCoord cc{0, 0, 0};
    uint32_t row = kInvalid;
    const SceneP* Pp = nullptr;
    if (valid) {
        xi = a.xs[k];
        vi = a.vs[k];
        Pp = &T.scenes[T.mats[__float_as_uint(vi.w)].scene];
        if (finite3(xi)) {
            const Grid& g = Pp->sgrid;
            cc = cell_coord(xi, g);
            row = Pp->cell_base + (uint32_t)cc.y * g.sub[0] + (uint32_t)cc.z * g.sub[0] * g.sub[1];
        }
    }
    s_row[threadIdx.x] = row;
    __syncthreads();
    const bool head = row != kInvalid && (threadIdx.x == 0 || s_row[threadIdx.x - 1] != row);
    const bool tail = row != kInvalid && (threadIdx.x == BLOCK - 1 || s_row[threadIdx.x + 1] != row);
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const unsigned hb = __ballot_sync(0xFFFFFFFFu, head);
    if (lane == 0) s_heads[warp] = __popc(hb);
    __syncthreads();
    uint32_t before = 0, nrows = 0;
    for (uint32_t w = 0; w < BLOCK / 32; ++w) {
        before += w < warp ? s_heads[w] : 0u;
        nrows += s_heads[w];
    }
    // own-row index of this thread (rows are contiguous runs of threads)
    const int rho = row == kInvalid ? -1 : (int)(before + __popc(hb & ((2u << lane) - 1u))) - 1;
    if (head && rho < kMaxOwnRows) {
        r_scene[rho] = T.mats[__float_as_uint(vi.w)].scene;
        r_base[rho] = row;
        r_y[rho] = cc.y;
        r_z[rho] = cc.z;
        r_xa[rho] = (uint32_t)cc.x;
    }
    if (tail && rho < kMaxOwnRows) r_xb[rho] = (uint32_t)cc.x;
    if (threadIdx.x == 0) s_nrows = nrows;
    __syncthreads();

    // windows: own row r, neighbor row q = (dz + RZ) * NY + (dy + RY)
    const uint32_t nwin = min(nrows, (uint32_t)kMaxOwnRows) * SS::NQ;
    if (threadIdx.x < nwin) {
        const uint32_t r = threadIdx.x / SS::NQ, q = threadIdx.x % SS::NQ;
        const SceneP& P = T.scenes[r_scene[r]];
        const Grid& g = P.sgrid;
        const int dy = (int)(q % kStageNY) - kStageRY;
        const int dz = DIM == 3 ? (int)(q / kStageNY) - kStageRZ : 0;
        const int y = r_y[r] + dy, z = r_z[r] + dz;
        const int ry = 1 + (int)P.halved[1], rx = 1 + (int)P.halved[0];
        uint32_t wstart = 0, wlen = 0;
        if (abs(dy) <= ry && y >= 0 && y < (int)g.sub[1] && z >= 0 && z < (int)g.sub[2]) {
            const uint32_t rb = r_base[r] + (uint32_t)(dy * (int)g.sub[0]) + (uint32_t)(dz * (int)(g.sub[0] * g.sub[1]));
            const uint32_t x0 = (uint32_t)max((int)r_xa[r] - rx, 0);
            const uint32_t x1 = (uint32_t)min((int)r_xb[r] + rx, (int)g.sub[0] - 1);
            wstart = a.start[rb + x0];
            wlen = a.start[rb + x1 + 1u] - wstart;
        }
        w_gstart[threadIdx.x] = wstart;
        w_off[threadIdx.x + 1] = wlen;
    }
    __syncthreads();
    if (threadIdx.x == 0) {  // at most NW (<= 60) windows: a serial prefix sum
        uint32_t t = 0;
        w_off[0] = 0;
        for (uint32_t w = 1; w <= nwin; ++w) {
            t += w_off[w];
            w_off[w] = t;
        }
    }
    __syncthreads();
    const uint32_t total = w_off[nwin];
    const bool staged = s_nrows <= (uint32_t)kMaxOwnRows && total <= (uint32_t)kStageSlots;
    if (!staged) {
        // too many rows or candidates for the staging area: the first overflow
        // queue (global-memory scan with list flushes) takes the tile
        if (valid) a.overflow[atomicAdd(a.overflow_count, 1u)] = k;
        return;
    }
    if (BULK) {
        // one elected thread issues a bulk copy per non-empty window (16-byte
        // aligned float4 ranges) and arms the barrier with their bytes
        if (threadIdx.x == 0) {
            mbar_arrive_expect_tx(&s_bar, total * 16u);
            for (uint32_t w = 0; w < nwin; ++w) {
                const uint32_t o = w_off[w], len = w_off[w + 1] - o;
                if (len) bulk_copy_g2s(stg + o, a.xs + w_gstart[w], len * 16u, &s_bar);
            }
        }
        const bool landed = mbar_wait_bounded(&s_bar, 0u, kStageSpins);
        if (threadIdx.x == 0) s_landed = 1u;
        __syncthreads();
        if (!landed) atomicAnd(&s_landed, 0u);
        __syncthreads();
        if (!s_landed) {
            // copies still in flight may write the staging area: wait for them
            // (bounded) before the block leaves, and let the global-memory scan
            // of the first overflow queue take the tile
            mbar_wait_bounded(&s_bar, 0u, kStageSpins);
            if (valid) a.overflow[atomicAdd(a.overflow_count, 1u)] = k;
            return;
        }
    } else {
        for (uint32_t w = 0; w < nwin; ++w) {
            const uint32_t o = w_off[w], len = w_off[w + 1] - o, gs = w_gstart[w];
            for (uint32_t i = threadIdx.x; i < len; i += BLOCK) stg[o + i] = a.xs[gs + i];
        }
        __syncthreads();
    }
    if (!valid) return;

    const uint32_t slot = a.perm ? a.perm[k] : k;
    const uint32_t sid = a.sid[slot];
    Self s;
    const SceneP& P = init_self(k, xi, vi, sid, a, T, sm, si, scene0, s);
    const PairK K{P.h2, P.kconst, P.eps_hh};
    Acc acc;
    acc.den = 0.0f;
    acc.f = make_float3(0.0f, 0.0f, 0.0f);
    uint32_t* my = lst + threadIdx.x;
    uint32_t cnt = 0;
    bool full = false;
    auto hit = [&](float4 q) {
        const float rx = q.x - xi.x, ry = q.y - xi.y;
        const float r2 = DIM == 3 ? fmaf(q.z - xi.z, q.z - xi.z, fmaf(ry, ry, rx * rx)) : fmaf(ry, ry, rx * rx);
        return r2 < K.h2;
    };
    auto take = [&](uint32_t j) {
        if (cnt < CAP) my[cnt++ * BLOCK] = j;
        else full = true;
    };
    if (rho >= 0) {
        const Grid& g = P.sgrid;
        const int rx = 1 + (int)P.halved[0], ry = 1 + (int)P.halved[1];
        const uint32_t x0 = (uint32_t)max(cc.x - rx, 0), x1 = (uint32_t)min(cc.x + rx, (int)g.sub[0] - 1);
        for (int q = 0; q < SS::NQ; ++q) {
            const int dy = q % kStageNY - kStageRY;
            const int dz = DIM == 3 ? q / kStageNY - kStageRZ : 0;
            const int y = cc.y + dy, z = cc.z + dz;
            if (abs(dy) > ry || y < 0 || y >= (int)g.sub[1] || z < 0 || z >= (int)g.sub[2]) continue;
            const uint32_t rb = row + (uint32_t)(dy * (int)g.sub[0]) + (uint32_t)(dz * (int)(g.sub[0] * g.sub[1]));
            const uint32_t c0 = rb + x0, c1 = rb + x1 + 1u;
            const uint32_t bb = a.bstart[c0], be = a.bstart[c1];
            for (uint32_t j = bb; j < be; ++j)
                if (hit(a.bxs[j])) take(j | kBoundaryBit);
            const uint32_t w = (uint32_t)rho * SS::NQ + (uint32_t)q;
            const uint32_t jb = a.start[c0], je = a.start[c1];
            const int shift = (int)w_off[w] - (int)w_gstart[w];  // global index -> staging slot
            uint32_t j = jb;
            for (; j + 3u < je; j += 4u) {  // four shared-memory loads in flight
                const int i0 = (int)j + shift;
                const float4 q0 = stg[i0], q1 = stg[i0 + 1], q2 = stg[i0 + 2], q3 = stg[i0 + 3];
                const bool h0 = hit(q0), h1 = hit(q1), h2 = hit(q2), h3 = hit(q3);
                if (h0) take(j);
                if (h1) take(j + 1u);
                if (h2) take(j + 2u);
                if (h3) take(j + 3u);
            }
            for (; j < je; ++j)
                if (hit(stg[(int)j + shift])) take(j);
        }
    }
    if (full) {
        a.overflow[atomicAdd(a.overflow_count, 1u)] = k;
        return;
    }
    for (uint32_t e = 0; e < cnt; ++e) {
        const uint32_t j = my[e * BLOCK];
        if (j != k) eval_hit<DIM>(j, s, a, K, acc);
    }
    stage_epilogue(a, c, b, slot, sid, vi, acc, s.d1, P.g, P.solid_branch != 0u);
}

template <int DIM, int BLOCK, int CAP, int MODE>
void launch_variant(const FluidArgs& a, const Tables& T, const StageCoefs& c, const StageBuffers& b, bool persistent,
                    uint32_t* tile_counter, cudaStream_t st) {
    const size_t smem = sizeof(uint32_t) * CAP * BLOCK + sizeof(FluidMat) * T.max_nmat +
                        sizeof(DevInter) * T.max_nmat * T.max_nmat;
    if (smem > 48 * 1024) {
        cudaFuncSetAttribute(FluidKernels<DIM, BLOCK, CAP, MODE>::tile, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smem);
        cudaFuncSetAttribute(FluidKernels<DIM, BLOCK, CAP, MODE>::persistent,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    }
    const uint32_t ntiles = (a.n + BLOCK - 1) / BLOCK;
    if (!a.counters_cleared) cudaMemsetAsync(a.overflow_count, 0, 2 * sizeof(uint32_t), st);
    if (!persistent) {
        FluidKernels<DIM, BLOCK, CAP, MODE>::tile<<<ntiles, BLOCK, smem, st>>>(a, T, c, b);
    } else {
        int per_sm = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, FluidKernels<DIM, BLOCK, CAP, MODE>::persistent, BLOCK,
                                                      smem);
        per_sm = per_sm > 0 ? per_sm : 1;
        int sms = 148;
        int dev = 0;
        if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        const uint32_t blocks = std::min<uint32_t>(ntiles, (uint32_t)(sms * per_sm));
        if (!a.counters_cleared) cudaMemsetAsync(tile_counter, 0, sizeof(uint32_t), st);
        FluidKernels<DIM, BLOCK, CAP, MODE>::persistent<<<blocks, BLOCK, smem, st>>>(a, T, c, b, tile_counter);
    }
    // the overflow queues: grids of at most 1184 blocks striding over the
    // queue, which usually is empty
    const uint32_t oblocks = std::min<uint32_t>(ntiles * BLOCK / 128u + 1u, 1184u);
    k_fluid_overflow_flush<DIM><<<oblocks, 128, 0, st>>>(a, T, c, b);
    k_fluid_overflow<DIM><<<2u * oblocks, 64, 0, st>>>(a, T, c, b);
}

// Velocity Verlet, first half of a step (kick, then drift), in storage
// order: v' = v + (dt/2) a, rho' = rho + (dt/2) drho/dt, x' = x + dt v', with
// (a, drho/dt) the derivative record kept from the previous force evaluation
// (its position part is not used).  Each sum is formed as y + (0 + c k), the
// order of the stage epilogue.
__global__ void k_verlet_kick_drift(const float4* __restrict__ pd, const float4* __restrict__ vm,
                                    const float4* __restrict__ fpd, const float4* __restrict__ fvm, uint32_t n,
                                    float half, float full, float4* __restrict__ out_pd, float4* __restrict__ out_vm) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const float4 p = pd[k], v = vm[k], fp = fpd[k], fv = fvm[k];
    const float4 z = make_float4(0.f, 0.f, 0.f, 0.f);
    const float4 vh = comb(v, axpy(half, fv, z), true);  // w holds the material bits
    const float rho = __fadd_rn(p.w, __fadd_rn(0.0f, __fmul_rn(half, fp.w)));
    const float4 dx = axpy(full, make_float4(vh.x, vh.y, vh.z, 0.0f), z);
    out_pd[k] = make_float4(__fadd_rn(p.x, dx.x), __fadd_rn(p.y, dx.y), __fadd_rn(p.z, dx.z), rho);
    out_vm[k] = vh;
}

// The kick of the plastic strain (4 float4 per solid): e' = e + (0 + c k).
__global__ void k_verlet_kick4(const float4* __restrict__ e, const float4* __restrict__ k4, uint32_t count, float half,
                               float4* __restrict__ out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    out[i] = comb(e[i], axpy(half, k4[i], make_float4(0.f, 0.f, 0.f, 0.f)), false);
}

template <int DIM, int BLOCK, int CAP, bool BULK>
int launch_staged(const FluidArgs& a, const Tables& T, const StageCoefs& c, const StageBuffers& b, cudaStream_t st) {
    const size_t smem = staged_smem_fixed<DIM, BLOCK, CAP>() + sizeof(FluidMat) * T.max_nmat +
                        sizeof(DevInter) * T.max_nmat * T.max_nmat;
    if (smem > 48 * 1024)
        cudaFuncSetAttribute(k_fluid_staged<DIM, BLOCK, CAP, BULK>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smem);
    const uint32_t ntiles = (a.n + BLOCK - 1) / BLOCK;
    if (!a.counters_cleared) cudaMemsetAsync(a.overflow_count, 0, 2 * sizeof(uint32_t), st);
    k_fluid_staged<DIM, BLOCK, CAP, BULK><<<ntiles, BLOCK, smem, st>>>(a, T, c, b);
    const uint32_t oblocks = std::min<uint32_t>(ntiles * BLOCK / 128u + 1u, 1184u);
    k_fluid_overflow_flush<DIM><<<oblocks, 128, 0, st>>>(a, T, c, b);
    k_fluid_overflow<DIM><<<2u * oblocks, 64, 0, st>>>(a, T, c, b);
    return 3;
}

}  // namespace

int verlet_kick_drift(const float4* pd, const float4* vm, const float4* fpd, const float4* fvm, uint32_t n, float half,
                      float full, float4* out_pd, float4* out_vm, cudaStream_t st) {
    if (n == 0) return 0;
    k_verlet_kick_drift<<<(n + 255) / 256, 256, 0, st>>>(pd, vm, fpd, fvm, n, half, full, out_pd, out_vm);
    return 1;
}

int verlet_kick4(const float4* e, const float4* k4, uint32_t count, float half, float4* out, cudaStream_t st) {
    if (count == 0) return 0;
    k_verlet_kick4<<<(count + 255) / 256, 256, 0, st>>>(e, k4, count, half, out);
    return 1;
}

const FluidVariant kFluidVariants[kNumFluidVariants] = {
    {128, 48, 0, 0, 0}, {256, 48, 0, 0, 0}, {128, 48, 1, 0, 0}, {256, 48, 1, 0, 0},
    {128, 96, 0, 0, 0}, {256, 96, 0, 0, 0}, {128, 96, 1, 0, 0}, {256, 96, 1, 0, 0},
    {128, 48, 0, 1, 0}, {128, 48, 1, 1, 0},
    {128, 48, 0, 0, 1}, {64, 48, 0, 0, 1}, {128, 48, 0, 0, 2},
    {128, 40, 0, 1, 0}, {128, 32, 0, 1, 0},
};

int launch_fluid(const FluidArgs& a, const Tables& T, int kdim, const StageCoefs& c, const StageBuffers& b,
                 int variant, uint32_t* tile_counter, cudaStream_t st) {
    if (a.n == 0) return 0;
    const FluidVariant v = kFluidVariants[variant < 0 || variant >= kNumFluidVariants ? 0 : variant];
    const bool pers = v.persistent != 0;
    if (v.staged == 1) {  // cooperative loads
        if (kdim == 3 && v.block == 128) return launch_staged<3, 128, 48, false>(a, T, c, b, st);
        if (kdim == 3 && v.block == 64) return launch_staged<3, 64, 48, false>(a, T, c, b, st);
        if (kdim == 2 && v.block == 128) return launch_staged<2, 128, 48, false>(a, T, c, b, st);
        if (kdim == 2 && v.block == 64) return launch_staged<2, 64, 48, false>(a, T, c, b, st);
        return 0;
    }
    if (v.staged == 2) {  // bulk copies
        if (kdim == 3 && v.block == 128) return launch_staged<3, 128, 48, true>(a, T, c, b, st);
        if (kdim == 2 && v.block == 128) return launch_staged<2, 128, 48, true>(a, T, c, b, st);
        return 0;
    }
#define ARP_FLUID(D, B, C, M)                                               \
    if (kdim == D && v.block == B && v.cap == C && v.flush == M && !v.staged) {  \
        launch_variant<D, B, C, M>(a, T, c, b, pers, tile_counter, st);     \
        return 3; /* the tile kernel and the two overflow kernels */       \
    }
    ARP_FLUID(3, 128, 48, 0) ARP_FLUID(3, 256, 48, 0) ARP_FLUID(3, 128, 96, 0) ARP_FLUID(3, 256, 96, 0)
    ARP_FLUID(2, 128, 48, 0) ARP_FLUID(2, 256, 48, 0) ARP_FLUID(2, 128, 96, 0) ARP_FLUID(2, 256, 96, 0)
    ARP_FLUID(3, 128, 48, 1) ARP_FLUID(2, 128, 48, 1)
    ARP_FLUID(3, 128, 40, 1) ARP_FLUID(3, 128, 32, 1) ARP_FLUID(2, 128, 40, 1) ARP_FLUID(2, 128, 32, 1)
#undef ARP_FLUID
    return 0;
}

}  // namespace arp
