// solid.cu -- Total-Lagrangian solid kernels.
//
// Replaces compute_strain (src/soft_body/shaders/strain.rs:71-183),
// solid_forces (src/soft_body/shaders/solid.rs:276-524) and clear_solids
// (solid.rs:5-37).
//
// The reference rebuilds the reference-configuration buckets, the correction
// matrix L = (sum V_j gradW(dX) (x) dX)^-1 and each neighbor's stress for
// every pair of every stage.  Reference positions never change (their time
// derivative is zero), so here:
//   * once per particle set: a CSR list of reference neighbors within h
//     (solid ids, same-material flag, gradW(X_j - X_i), V_j = m_j / rho0_j)
//     and L (k_ref_count / k_ref_fill / k_ref_L);
//   * per stage, one thread per solid: F, Fdot from the list, Seth-Hill
//     strain + Hooke stress (all strain orders, GLSL mat4 semantics),
//     A = sigma L, the Johnson-Cook plastic rate and its stage update
//     (k_solid_stress);
//   * per stage, one thread per solid: elastic force -V_i V_j (A_i + A_j)
//     gradW over the list, then hourglass control and self-contact over the
//     current 3x3x3 cells (k_solid_forces).  A_j is read, not recomputed.
#include "grid.cuh"
#include "mat4.cuh"
#include "warp.cuh"

namespace arp {

namespace {

constexpr int kThreads = 128;
#ifndef ARP_SOLID_LANES
#define ARP_SOLID_LANES 2
#endif
constexpr int kSolidLanes = ARP_SOLID_LANES;  // threads per solid in the stress and force kernels
constexpr uint32_t kSameMat = 0x80000000u;
// The stage kernels recompute gradW(dX) and W(dX) of each reference pair from
// the reference positions (a gather that neighboring solids share in L1/L2)
// instead of streaming per-entry values from HBM: a list entry costs its
// 4-byte index.  The stored gradW and volume (rl.gw) serve L and the reverse
// pass.

inline uint32_t blocks_for(uint32_t n, int t) { return (n + (uint32_t)t - 1u) / (uint32_t)t; }

__device__ __forceinline__ float3 sub3(float4 a, float4 b) { return make_float3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ float dot3(float3 a, float3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }

// unit diagonal on the axes at or above dim (solid.rs:149, :175, :227)
__device__ __forceinline__ void pad_unit(M4& C, uint32_t dim) {
#pragma unroll
    for (uint32_t i = 0; i < 4; ++i)
        if (i >= dim) C.m[i][i] = 1.0f;
}

// Walk the 27 reference cells around solid i (search-cell rows ascending,
// ascending solid id inside a search cell) and call f(j, dX, diff) for each
// other solid with h^2 - |dX|^2 > 0.
template <class F>
__device__ __forceinline__ void for_ref_neighbors(uint32_t i, const float4* __restrict__ ref,
                                                  const uint32_t* __restrict__ start, const uint32_t* __restrict__ perm,
                                                  const SceneP& P, F&& f) {
    const float4 xi = ref[i];
    if (!finite3(xi)) return;
    for_reference_block_rows(xi, P, [&](uint32_t c0, uint32_t c1) {
        for (uint32_t k = start[c0]; k < start[c1]; ++k) {
            const uint32_t j = perm[k];
            if (j == i) continue;
            const float3 dX = sub3(ref[j], xi);
            const float diff = P.h2 - dot3(dX, dX);
            if (diff > 0.0f) f(j, dX, diff);
        }
    });
}

__global__ void k_ref_count(const float4* __restrict__ ref, const uint32_t* __restrict__ mat_of, uint32_t ns,
                            const uint32_t* __restrict__ start, const uint32_t* __restrict__ perm, Tables T,
                            uint32_t* __restrict__ count) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ns) return;
    uint32_t n = 0;
    const SceneP& P = T.scenes[T.mats[mat_of[i]].scene];
    for_ref_neighbors(i, ref, start, perm, P, [&](uint32_t, float3, float) { ++n; });
    count[i] = n;
}

__global__ void k_ref_fill(const float4* __restrict__ ref, const uint32_t* __restrict__ mat_of, uint32_t ns,
                           const uint32_t* __restrict__ start, const uint32_t* __restrict__ perm, Tables T,
                           const uint32_t* __restrict__ off, uint32_t* __restrict__ nbr, float4* __restrict__ gw) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ns) return;
    uint32_t w = off[i];
    const uint32_t mi = mat_of[i];
    const DevMat* mats = T.mats;
    const SceneP& P = T.scenes[mats[mi].scene];
    for_ref_neighbors(i, ref, start, perm, P, [&](uint32_t j, float3 dX, float diff) {
        const float s = -6.0f * P.kconst * diff * diff;
        const uint32_t mj = mat_of[j];
        nbr[w] = j | (mj == mi ? kSameMat : 0u);
        gw[w] = make_float4(s * dX.x, s * dX.y, s * dX.z, mats[mj].vol0);
        ++w;
    });
}

// L = inverse(sum_j V_j gradW (x) dX), unit diagonal on the unused axes
// (strain.rs:107-136).  Stored as three float4 columns.
__global__ void k_ref_L(const float4* __restrict__ ref, const uint32_t* __restrict__ mat_of, uint32_t ns,
                        const uint32_t* __restrict__ off, const uint32_t* __restrict__ nbr,
                        const float4* __restrict__ gw, Tables T, float4* __restrict__ L) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ns) return;
    const SceneP& P = T.scenes[T.mats[mat_of[i]].scene];
    M4 C = m4_zero();
    const float4 xi = ref[i];
    for (uint32_t k = off[i]; k < off[i + 1]; ++k) {
        const uint32_t j = nbr[k] & ~kSameMat;
        const float4 g = gw[k];
        const float3 dX = sub3(ref[j], xi);
        const float d[3] = {dX.x, dX.y, dX.z};
        const float gg[3] = {g.x, g.y, g.z};
#pragma unroll
        for (int c = 0; c < 3; ++c)
#pragma unroll
            for (int r = 0; r < 3; ++r) C.m[c][r] += g.w * (gg[r] * d[c]);
    }
    pad_unit(C, P.dim);
    const M4 Li = m4_inverse(C);
#pragma unroll
    for (int c = 0; c < 3; ++c) L[3 * i + c] = make_float4(Li.m[c][0], Li.m[c][1], Li.m[c][2], Li.m[c][3]);
}

// ---- per-stage strain / stress ----------------------------------------------

__device__ __forceinline__ float trace_dim(const M4& A, uint32_t dim) {
    float t = A.m[0][0];
#pragma unroll
    for (uint32_t i = 1; i < 4; ++i)
        if (i < dim) t += A.m[i][i];
    return t;
}
__device__ inline M4 mat_log5(const M4& A) {  // solid.rs:105-116
    M4 sum = m4_zero();
    M4 term = m4_scale(-1.0f, m4_ident());
    const M4 X = m4_scale(-1.0f, m4_sub(A, m4_ident()));
    for (int i = 1; i <= 5; ++i) {
        term = m4_mul(term, X);
        sum = m4_add(sum, m4_div(term, (float)i));
    }
    return sum;
}
__device__ inline M4 mat_sqrt_db(const M4& Xm) {  // Denman-Beavers, solid.rs:119-133
    M4 Y = Xm, Z = m4_ident();
    for (int i = 0; i < 15; ++i) {
        const M4 Yn = m4_scale(0.5f, m4_add(Y, m4_inverse(Z)));
        const M4 Zn = m4_scale(0.5f, m4_add(Z, m4_inverse(Y)));
        Y = Yn;
        Z = Zn;
    }
    return Y;
}
template <bool ORDER2>
__device__ inline M4 seth_hill(const M4& F, int two_m, uint32_t dim) {  // solid.rs:147-168
    M4 C = m4_mul(m4_transpose(F), F);
    pad_unit(C, dim);
    if (ORDER2) return m4_scale(1.0f / 2.0f, m4_sub(m4_mul(m4_ident(), C), m4_ident()));
    if (two_m == 0) return m4_scale(0.5f, mat_log5(C));
    const int a = two_m < 0 ? -two_m : two_m;
    const int m = a >> 1;
    M4 Cm = m4_ident();
    for (int i = 0; i < m; ++i) Cm = m4_mul(Cm, C);
    if (a & 1) Cm = m4_mul(Cm, mat_sqrt_db(C));
    if (two_m < 0) Cm = m4_inverse(Cm);
    return m4_scale(1.0f / (float)two_m, m4_sub(Cm, m4_ident()));
}
template <bool ORDER2>
__device__ inline M4 seth_hill_rate(const M4& F, const M4& Fd, int two_m, uint32_t dim) {  // solid.rs:170-204
    M4 dC = m4_mul(m4_transpose(Fd), F);
    dC = m4_add(dC, m4_transpose(dC));
    if (ORDER2) return m4_scale(1.0f / 2.0f, m4_mul(m4_ident(), dC));
    M4 C = m4_mul(m4_transpose(F), F);
    pad_unit(C, dim);
    if (two_m == 0) return m4_mul(m4_scale(0.5f, dC), m4_inverse(C));
    const int a = two_m < 0 ? -two_m : two_m;
    const int m = a >> 1;
    M4 rate = m4_zero();
    for (int i = 0; i < m; ++i) {
        M4 term = m4_ident();
        for (int j = 0; j < m; ++j) term = m4_mul(term, j == i ? dC : C);
        rate = m4_add(rate, term);
    }
    rate = m4_scale(1.0f / (float)two_m, rate);
    if (two_m < 0) {
        const M4 iC = m4_inverse(C);
        return m4_mul(m4_mul(m4_scale(-1.0f, iC), rate), iC);
    }
    return rate;
}
__device__ __forceinline__ M4 hooke(const M4& E, float normal, float shear, uint32_t dim) {
    const M4 a = m4_scale(normal * trace_dim(E, dim), m4_ident());
    return m4_add(a, m4_scale(2.0f * shear, E));
}

__device__ __forceinline__ float4 lin4(float c, float4 k, float4 t) {
    return make_float4(__fadd_rn(t.x, __fmul_rn(c, k.x)), __fadd_rn(t.y, __fmul_rn(c, k.y)),
                       __fadd_rn(t.z, __fmul_rn(c, k.z)), __fadd_rn(t.w, __fmul_rn(c, k.w)));
}
__device__ __forceinline__ float4 add4(float4 a, float4 b) {
    return make_float4(__fadd_rn(a.x, b.x), __fadd_rn(a.y, b.y), __fadd_rn(a.z, b.z), __fadd_rn(a.w, b.w));
}

// ORDER2: every solid material uses strain order 2 (Green-Lagrange), so the
// log-series, square-root and inverse paths are compiled out.
// PLASTIC: some solid material is plastic; otherwise the plastic strain is
// zero throughout and its buffers are neither read nor written.
// LANES threads share one solid: they walk its reference list with stride
// LANES and combine their partial sums with shuffles (group_sum: a fixed
// order, so the result is deterministic); lane 0 finishes the particle.

template <bool ORDER2, bool PLASTIC, int LANES>
__global__ void __launch_bounds__(kThreads) k_solid_stress(SolidArgs a, Tables T, StageCoefs c) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t i = t / LANES, lane = t % LANES;
    if (i >= a.ns) return;  // whole groups leave together
    const float4 xi = a.sx[i];
    const float4 vi = a.sv[i];
    const DevMat mm = T.mats[__float_as_uint(vi.w)];
    const SceneP& P = T.scenes[mm.scene];
    if (!P.solid_branch) return;  // a scene with a single solid skips the solid term
    const float4 L0 = a.L[3 * i], L1 = a.L[3 * i + 1], L2 = a.L[3 * i + 2];
    const float4 Xs = a.ref[i];
    // strain.rs:139-160: F = sum V dx (x) (L gradW), Fdot likewise with dv
    float F[3][3] = {{0.f, 0.f, 0.f}, {0.f, 0.f, 0.f}, {0.f, 0.f, 0.f}};
    float Fd[3][3] = {{0.f, 0.f, 0.f}, {0.f, 0.f, 0.f}, {0.f, 0.f, 0.f}};
    for (uint32_t k = a.rl.off[i] + lane; k < a.rl.off[i + 1]; k += LANES) {
        const uint32_t j = a.rl.nbr[k] & ~kSameMat;
        const float4 vj = a.sv[j];
        // gradW(X_j - X_i) as k_ref_fill computes it; V_j rides in ref.w
        const float4 Xj = a.ref[j];
        const float3 dX = sub3(Xj, Xs);
        const float diff = P.h2 - dot3(dX, dX);
        const float sg = -6.0f * P.kconst * diff * diff;
        const float4 g = make_float4(sg * dX.x, sg * dX.y, sg * dX.z, Xj.w);
        const float3 dx = sub3(a.sx[j], xi);
        const float3 dv = sub3(vj, vi);
        const float gr[3] = {(L0.x * g.x + L1.x * g.y) + L2.x * g.z, (L0.y * g.x + L1.y * g.y) + L2.y * g.z,
                             (L0.z * g.x + L1.z * g.y) + L2.z * g.z};
        const float x[3] = {dx.x, dx.y, dx.z}, v[3] = {dv.x, dv.y, dv.z};
#pragma unroll
        for (int cc = 0; cc < 3; ++cc)
#pragma unroll
            for (int r = 0; r < 3; ++r) {
                F[cc][r] += g.w * (x[r] * gr[cc]);
                Fd[cc][r] += g.w * (v[r] * gr[cc]);
            }
    }
    if (LANES > 1) {
#pragma unroll
        for (int cc = 0; cc < 3; ++cc)
#pragma unroll
            for (int r = 0; r < 3; ++r) {
                F[cc][r] = group_sum<LANES>(F[cc][r]);
                Fd[cc][r] = group_sum<LANES>(Fd[cc][r]);
            }
        if (lane != 0) return;
    }
    M4 Fm = m4_zero(), Fdm = m4_zero(), Lm = m4_zero(), EP;
#pragma unroll
    for (int cc = 0; cc < 3; ++cc)
#pragma unroll
        for (int r = 0; r < 3; ++r) {
            Fm.m[cc][r] = F[cc][r];
            Fdm.m[cc][r] = Fd[cc][r];
        }
    const float4 Lc[3] = {L0, L1, L2};
#pragma unroll
    for (int cc = 0; cc < 3; ++cc) {
        Lm.m[cc][0] = Lc[cc].x;
        Lm.m[cc][1] = Lc[cc].y;
        Lm.m[cc][2] = Lc[cc].z;
        Lm.m[cc][3] = Lc[cc].w;
    }
    Lm.m[3][3] = 1.0f;
    if (PLASTIC) {
#pragma unroll
        for (int cc = 0; cc < 4; ++cc) {
            const float4 e = a.ep[4 * i + cc];
            EP.m[cc][0] = e.x;
            EP.m[cc][1] = e.y;
            EP.m[cc][2] = e.z;
            EP.m[cc][3] = e.w;
        }
    } else {
        EP = m4_zero();
    }
    // Bound used to skip the self-contact scan: max |u_i - u_0| over solids
    // (u = x - X) and whether any solid left the box.
    {
        const float4 X0 = a.ref[0];
        const float4 x0 = a.sx[0];
        const float4 Xi = a.ref[i];
        const float ux = (xi.x - Xi.x) - (x0.x - X0.x), uy = (xi.y - Xi.y) - (x0.y - X0.y),
                    uz = (xi.z - Xi.z) - (x0.z - X0.z);
        const float du = sqrtf((ux * ux + uy * uy) + uz * uz);
        bool outside = !finite3(xi) || !(du == du);
        const float pc[3] = {xi.x, xi.y, xi.z};
#pragma unroll
        for (int ax = 0; ax < 3; ++ax) {
            const float d = P.grid.dim[ax];
            if (d != 0.0f) {
                const float t = (pc[ax] - P.grid.min[ax]) / d;
                outside = outside || !(t >= 0.0f && t < 1.0f);
            }
        }
        const uint32_t mx = __reduce_max_sync(__activemask(), outside ? 0x7F800000u : __float_as_uint(du));
        const uint32_t any_out = __reduce_or_sync(__activemask(), outside ? 1u : 0u);
        if ((threadIdx.x & 31) == __ffs(__activemask()) - 1) {
            atomicMax(&a.contact_bound[0], mx);
            if (any_out) atomicOr(&a.contact_bound[1], 1u);
        }
    }
    // solid.rs:334-341
    const M4 strain = PLASTIC ? m4_add(seth_hill<ORDER2>(Fm, mm.strain_order, P.dim), EP)
                              : seth_hill<ORDER2>(Fm, mm.strain_order, P.dim);
    const M4 rate = seth_hill_rate<ORDER2>(Fm, Fdm, mm.strain_order, P.dim);
    const float2 lm = a.stiff ? a.stiff[i] : make_float2(mm.lam, mm.mu);
    const M4 pk2 = m4_add(hooke(strain, lm.x, lm.y, P.dim), hooke(rate, mm.lam_d, mm.mu_d, P.dim));
    const M4 sigma = m4_mul(Fm, m4_transpose(pk2));
    const M4 A = m4_mul(sigma, Lm);
#pragma unroll
    for (int cc = 0; cc < 3; ++cc) {
        a.F[3 * i + cc] = make_float4(Fm.m[cc][0], Fm.m[cc][1], Fm.m[cc][2], Fm.m[cc][3]);
        a.A[3 * i + cc] = make_float4(A.m[cc][0], A.m[cc][1], A.m[cc][2], A.m[cc][3]);
    }
    // solid.rs:499-517: plastic strain rate (relaxation towards the
    // Johnson-Cook yield surface); the equivalent-strain factor is the
    // shader's integer (dim-1)/dim
    if (!PLASTIC) return;
    M4 kep = m4_zero();
    if (mm.plastic) {
        const float tr = trace_dim(EP, P.dim);
        const M4 dev = m4_sub(EP, m4_div(m4_scale(tr, m4_ident()), (float)P.dim));
        const float eq = (float)((int)(P.dim - 1) / (int)P.dim) * m4_dot(dev, dev);
        float sn = m4_dot(pk2, pk2);
        const float y = (mm.yield_strength + mm.work_hardening * powf(eq, mm.work_hardening_exp / 2.0f)) *
                        (1.0f + mm.kinematic_hardening * logf(1.0f));
        if (y * y <= sn) {
            sn = sqrtf(sn);
            kep = m4_scale((sn - y) / mm.relaxation_time, m4_div(pk2, sn));
        }
    }
    // stage update of the plastic strain (same scheme as the fluid epilogue)
    float4 kv[4];
#pragma unroll
    for (int cc = 0; cc < 4; ++cc) kv[cc] = make_float4(kep.m[cc][0], kep.m[cc][1], kep.m[cc][2], kep.m[cc][3]);
#pragma unroll
    for (int cc = 0; cc < 4; ++cc) {
        const uint32_t o = 4 * i + cc;
        if (a.ep_store) a.ep_store[o] = kv[cc];
        const float4 y0 = a.ep0[o];
        float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
        if (c.c_acc != 0.0f) {
            if (!c.acc_first) acc = a.ep_acc[o];
            acc = lin4(c.c_acc, kv[cc], acc);
            if (!c.last) a.ep_acc[o] = acc;
        } else if (c.last) {
            acc = a.ep_acc[o];
        }
        if (c.last) {
            a.ep_next[o] = add4(y0, acc);
        } else {
            float4 t = make_float4(0.f, 0.f, 0.f, 0.f);
            if (c.c_prev0 != 0.0f) t = lin4(c.c_prev0, a.ep_prev0[o], t);
            if (c.c_prev1 != 0.0f) t = lin4(c.c_prev1, a.ep_prev1[o], t);
            if (c.c_prev2 != 0.0f) t = lin4(c.c_prev2, a.ep_prev2[o], t);
            if (c.c_self != 0.0f) t = lin4(c.c_self, kv[cc], t);
            a.ep_next[o] = add4(y0, t);
        }
    }
}

__device__ __forceinline__ bool in_stencil(uint2 a, uint2 b) {
    const int dx = (int)(a.x & 0xFFFFu) - (int)(b.x & 0xFFFFu);
    const int dy = (int)(a.x >> 16) - (int)(b.x >> 16);
    const int dz = (int)a.y - (int)b.y;
    return a.y != 0xFFFFFFFFu && b.y != 0xFFFFFFFFu && dx >= -1 && dx <= 1 && dy >= -1 && dy <= 1 && dz >= -1 &&
           dz <= 1;
}

template <int LANES>
__global__ void __launch_bounds__(kThreads) k_solid_forces(SolidArgs a, Tables T) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t i = t / LANES, lane = t % LANES;
    if (i >= a.ns) return;  // whole groups leave together
    const float4 xi = a.sx[i];
    const uint32_t mat = __float_as_uint(a.sv[i].w);
    const DevMat mm = T.mats[mat];
    const SceneP& P = T.scenes[mm.scene];
    if (!P.solid_branch) return;
    const float m1 = mm.mass, d1 = xi.w;
    const float V1 = m1 / d1;
    const float4 Ai0 = a.A[3 * i], Ai1 = a.A[3 * i + 1], Ai2 = a.A[3 * i + 2];
    const float4 Xi = a.ref[i];
    const float4 Fi0 = a.F[3 * i], Fi1 = a.F[3 * i + 1], Fi2 = a.F[3 * i + 2];
    const uint2 ci = a.sc[i];
    float fx = 0.f, fy = 0.f, fz = 0.f;
    // Reference neighbors of the same material: the elastic force
    // (solid.rs:343-374) and, when the neighbor also sits in the current
    // 3x3x3 cells, hourglass control (solid.rs:430-443; kernel(dX) is
    // non-zero exactly for these pairs).
    for (uint32_t k = a.rl.off[i] + lane; k < a.rl.off[i + 1]; k += LANES) {
        const uint32_t e = a.rl.nbr[k];
        if (!(e & kSameMat)) continue;
        const uint32_t j = e & ~kSameMat;
        // dX = X_j - X_i, gradW(dX) as k_ref_fill computes it
        const float3 dX = sub3(a.ref[j], Xi);
        const float diff = P.h2 - dot3(dX, dX);
        const float sg = -6.0f * P.kconst * diff * diff;
        const float3 g = make_float3(sg * dX.x, sg * dX.y, sg * dX.z);
        const float4 xj = a.sx[j];
        const float d2 = xj.w;
        const float V2 = __fdividef(m1, d2);  // GLSL division carries 2.5 ulp; the 2-ulp hardware quotient is used
        const float s = -V1 * V2;
        const float4 Aj0 = a.A[3 * j], Aj1 = a.A[3 * j + 1], Aj2 = a.A[3 * j + 2];
        const float4 c0 = make_float4(s * (Ai0.x + Aj0.x), s * (Ai0.y + Aj0.y), s * (Ai0.z + Aj0.z), 0.f);
        const float4 c1 = make_float4(s * (Ai1.x + Aj1.x), s * (Ai1.y + Aj1.y), s * (Ai1.z + Aj1.z), 0.f);
        const float4 c2 = make_float4(s * (Ai2.x + Aj2.x), s * (Ai2.y + Aj2.y), s * (Ai2.z + Aj2.z), 0.f);
        // components at or above dim are dropped (solid.rs:370)
        fx += (c0.x * g.x + c1.x * g.y) + c2.x * g.z;
        if (P.dim >= 2) fy += (c0.y * g.x + c1.y * g.y) + c2.y * g.z;
        if (P.dim >= 3) fz += (c0.z * g.x + c1.z * g.y) + c2.z * g.z;
        if (in_stencil(a.sc[j], ci)) {
            const float3 dx = sub3(xj, xi);
            const float l = sqrtf(dot3(dx, dx));
            const float4 Fj0 = a.F[3 * j], Fj1 = a.F[3 * j + 1], Fj2 = a.F[3 * j + 2];
            const float ex = ((0.5f * (Fi0.x + Fj0.x)) * dX.x + (0.5f * (Fi1.x + Fj1.x)) * dX.y) +
                             (0.5f * (Fi2.x + Fj2.x)) * dX.z - dx.x;
            const float ey = ((0.5f * (Fi0.y + Fj0.y)) * dX.x + (0.5f * (Fi1.y + Fj1.y)) * dX.y) +
                             (0.5f * (Fi2.y + Fj2.y)) * dX.z - dx.y;
            const float ez = ((0.5f * (Fi0.z + Fj0.z)) * dX.x + (0.5f * (Fi1.z + Fj1.z)) * dX.y) +
                             (0.5f * (Fi2.z + Fj2.z)) * dX.z - dx.z;
            const float kern = P.kconst * diff * diff * diff;  // W(dX)
            const float sh = ((__fdividef(100000000.0f * m1 * m1, d1 * d2) *
                               __fdividef(0.5f * ((ex * dx.x + ey * dx.y) + ez * dx.z), l + P.hg_h)) *
                              __fdividef(1.0f, l * l + P.eps_hh)) *
                             kern;
            const float den = l + P.eps_h;
            fx -= __fdividef(sh * dx.x, den);
            fy -= __fdividef(sh * dx.y, den);
            fz -= __fdividef(sh * dx.z, den);
        }
    }
    if (LANES > 1) {
        fx = group_sum<LANES>(fx);
        fy = group_sum<LANES>(fy);
        fz = group_sum<LANES>(fz);
        if (lane != 0) return;
    }
    // Self-contact (solid.rs:428,445-450): same-material neighbors in the
    // current cells whose reference distance exceeds r_cut.  Skipped when
    // every solid is inside the box and r_cut - max|dx in stencil| exceeds
    // 2 max|u_k - u_0|, which bounds |dX| below r_cut for all such pairs.
    const float U = __uint_as_float(a.contact_bound[0]);
    const bool maybe = !mm.plastic && (P.contact_slack <= 0.0f || a.contact_bound[1] != 0u || !(2.0f * U < P.contact_slack));
    if (maybe && finite3(xi)) {
        for_reference_block_rows(xi, P, [&](uint32_t c0, uint32_t c1) {
            for (uint32_t k = a.start[c0]; k < a.start[c1]; ++k) {
                if (__float_as_uint(a.vs[k].w) != mat) continue;
                const uint32_t sj = a.sid_sorted[k];
                if (sj == kInvalid) continue;
                const float4 xj = a.xs[k];
                const float3 dx = sub3(xj, xi);
                const float3 dX = sub3(a.ref[sj], Xi);
                const float dXX = dot3(dX, dX), dxx = dot3(dx, dx);
                if (!(dXX > P.rcut2 && dxx < P.rcut2)) continue;
                const float l = sqrtf(dxx);
                const float dr = fmaxf(P.rcut - l, 0.0f);
                const float cs = -5000.0f * sqrtf(dr * P.r_geom);
                fx += (cs * dx.x) / l;
                fy += (cs * dx.y) / l;
                fz += (cs * dx.z) / l;
            }
        });
    }
    // solid.rs:492-494 (den term is zero)
    a.ksol[i] = make_float4(__fdiv_rn(fx, d1), __fadd_rn(__fdiv_rn(fy, d1), -P.g), __fdiv_rn(fz, d1), 0.0f);
}

}  // namespace

int ref_lists_count(const float4* ref, const uint32_t* mat_of, uint32_t ns, const GridBuffers& gb, const Tables& T,
                    uint32_t* count, cudaStream_t st) {
    k_ref_count<<<blocks_for(ns, kThreads), kThreads, 0, st>>>(ref, mat_of, ns, gb.start, gb.perm, T, count);
    return 1;
}

int ref_lists_fill(const float4* ref, const uint32_t* mat_of, uint32_t ns, const GridBuffers& gb, const Tables& T,
                   SolidRefList& rl, float4* L, cudaStream_t st) {
    k_ref_fill<<<blocks_for(ns, kThreads), kThreads, 0, st>>>(ref, mat_of, ns, gb.start, gb.perm, T, rl.off, rl.nbr,
                                                              rl.gw);
    k_ref_L<<<blocks_for(ns, kThreads), kThreads, 0, st>>>(ref, mat_of, ns, rl.off, rl.nbr, rl.gw, T, L);
    return 2;
}

int launch_solid(const SolidArgs& a, const Tables& T, const StageCoefs& c, cudaStream_t st) {
    if (a.ns == 0) return 0;
    if (!a.counters_cleared) cudaMemsetAsync(a.contact_bound, 0, 2 * sizeof(uint32_t), st);
    // a.sx, a.sv, a.sc were written by the stage's gather (gather_state)
    constexpr int L = kSolidLanes;
    const uint32_t blocks = blocks_for(a.ns * L, kThreads);
    if (a.all_order2 && !a.any_plastic) k_solid_stress<true, false, L><<<blocks, kThreads, 0, st>>>(a, T, c);
    else if (a.all_order2) k_solid_stress<true, true, L><<<blocks, kThreads, 0, st>>>(a, T, c);
    else if (!a.any_plastic) k_solid_stress<false, false, L><<<blocks, kThreads, 0, st>>>(a, T, c);
    else k_solid_stress<false, true, L><<<blocks, kThreads, 0, st>>>(a, T, c);
    k_solid_forces<L><<<blocks, kThreads, 0, st>>>(a, T);
    return 2;
}

}  // namespace arp
