// adjoint.cu -- reverse mode of one Runge-Kutta stage of the SPH step.
//
// For a stage state Y and the adjoint mu of its derivative record k = f(Y)
// (one (x, rho) and one (v) float4 per particle), these kernels accumulate
// lam_Y += J_f(Y)^T mu, hand-derived term by term from the forward kernels:
//   * k_adj_solid   elastic force (solid.rs:343-374), hourglass control
//                   (solid.rs:430-443) and the stress chain of any strain order
//                   F, dF/dt -> E, dE/dt -> S (Hooke) -> sigma = F S^T -> A = sigma L
//                   (strain.rs:139-160, solid.rs:147-204,334-341), plus the
//                   gradient of the per-solid (normal, shear) stiffness;
//   * k_adj_strain  F and dF/dt as sums over the reference neighbors;
//   * k_adj_fluid   every fluid pair term (continuity, pressure with the
//                   state equation, contact potential, viscosity, artificial
//                   viscosity, friction; fluid.rs:154-247) and dx/dt = v.
// Neighbor sets (hits within h, reference lists, the current-cell condition
// of the hourglass term) are those of the recorded forward stage and are not
// differentiated.  Each particle gathers the contributions of its own pairs
// and of its neighbors' pairs (pairwise-symmetric gathers): no atomics, each
// thread writes only its own particle.  Not differentiated: self-contact
// (flagged when a pair is active).
#include "grid.cuh"
#include "warp.cuh"

namespace arp {

namespace {

constexpr int kT = 128;
#ifndef ARP_ADJ_SOLID_LANES
#define ARP_ADJ_SOLID_LANES 4
#endif
constexpr int kAdjSolidLanes = ARP_ADJ_SOLID_LANES;  // threads per solid in k_adj_solid
constexpr uint32_t kSameMatBit = 0x80000000u;

inline uint32_t nblocks(uint32_t n, int t) { return (n + (uint32_t)t - 1u) / (uint32_t)t; }

__device__ __forceinline__ float3 f3(float4 a) { return make_float3(a.x, a.y, a.z); }
__device__ __forceinline__ float3 add(float3 a, float3 b) { return make_float3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ float3 sub(float3 a, float3 b) { return make_float3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ float3 mul(float s, float3 a) { return make_float3(s * a.x, s * a.y, s * a.z); }
__device__ __forceinline__ float dot(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ float3 neg(float3 a) { return make_float3(-a.x, -a.y, -a.z); }

// gradW(X_j - X_i) of a reference pair, as the reference-list build computes
// it: recomputed from the reference positions (shared by neighboring solids
// in L1/L2) rather than streamed per list entry.
__device__ __forceinline__ float3 ref_grad(const float4* __restrict__ ref, uint32_t j, float3 Xi, const SceneP& P) {
    const float3 dX = sub(f3(ref[j]), Xi);
    const float diff = P.h2 - ((dX.x * dX.x + dX.y * dX.y) + dX.z * dX.z);
    const float s = -6.0f * P.kconst * diff * diff;
    return make_float3(s * dX.x, s * dX.y, s * dX.z);
}

// 3x3 matrices, row-major: m[r][c]
struct M3 {
    float m[3][3];
};
__device__ __forceinline__ M3 m3_zero() {
    M3 r;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) r.m[i][j] = 0.0f;
    return r;
}
// three float4 columns -> matrix
__device__ __forceinline__ M3 m3_cols(const float4* c) {
    const float4 c0 = c[0], c1 = c[1], c2 = c[2];
    M3 r;
    r.m[0][0] = c0.x; r.m[1][0] = c0.y; r.m[2][0] = c0.z;
    r.m[0][1] = c1.x; r.m[1][1] = c1.y; r.m[2][1] = c1.z;
    r.m[0][2] = c2.x; r.m[1][2] = c2.y; r.m[2][2] = c2.z;
    return r;
}
__device__ __forceinline__ void m3_store_cols(const M3& a, float4* c) {
#pragma unroll
    for (int j = 0; j < 3; ++j) c[j] = make_float4(a.m[0][j], a.m[1][j], a.m[2][j], 0.0f);
}
__device__ __forceinline__ float3 m3_vec(const M3& a, float3 v) {
    return make_float3(a.m[0][0] * v.x + a.m[0][1] * v.y + a.m[0][2] * v.z,
                       a.m[1][0] * v.x + a.m[1][1] * v.y + a.m[1][2] * v.z,
                       a.m[2][0] * v.x + a.m[2][1] * v.y + a.m[2][2] * v.z);
}
__device__ __forceinline__ M3 m3_mul(const M3& a, const M3& b) {
    M3 r;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) r.m[i][j] = a.m[i][0] * b.m[0][j] + a.m[i][1] * b.m[1][j] + a.m[i][2] * b.m[2][j];
    return r;
}
__device__ __forceinline__ M3 m3_t(const M3& a) {
    M3 r;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) r.m[i][j] = a.m[j][i];
    return r;
}
__device__ __forceinline__ void m3_add_outer(M3& a, float s, float3 u, float3 v) {
    const float uu[3] = {u.x, u.y, u.z}, vv[3] = {v.x, v.y, v.z};
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) a.m[i][j] += s * uu[i] * vv[j];
}
__device__ __forceinline__ void m3_acc(M3& a, const M3& b) {
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) a.m[i][j] += b.m[i][j];
}

__device__ __forceinline__ float3 mask_dim(float3 v, uint32_t dim) {
    return make_float3(v.x, dim >= 2 ? v.y : 0.0f, dim >= 3 ? v.z : 0.0f);
}

// p / rho^2 of a state equation (fluid.rs:45-52) and its derivative in rho
__device__ __forceinline__ void eos_pt(uint32_t eq, float rho, float c, float d0, float& pt, float& dpt) {
    float p = 0.0f, dp = 0.0f;
    if (eq == ARP_EOS_CONSTANT) {
        p = c * c;
    } else if (eq == ARP_EOS_IDEAL_GAS) {
        p = c * c * (rho - d0);
        dp = c * c;
    } else if (eq == ARP_EOS_TAIT) {
        const float x = rho / d0;
        const float x2 = x * x, x3 = x2 * x, x6 = x3 * x3;
        p = (c * c * d0 / 7.0f) * (x6 * x - 1.0f);
        dp = c * c * x6;
    }
    const float ir = 1.0f / rho;
    pt = p * ir * ir;
    dpt = dp * ir * ir - 2.0f * p * ir * ir * ir;
}

// contact potential P(r) in the shader's argument order (strength, r0) and dP/dr
__device__ __forceinline__ float cpot(uint32_t eq, float r, float S, float R0, float& d) {
    d = 0.0f;
    switch (eq) {
        case ARP_CONTACT_CONSTANT: return r <= R0 ? S : 0.0f;
        case ARP_CONTACT_LINEAR: d = -S; return S * (R0 - r);
        case ARP_CONTACT_TAIT: {
            const float x = R0 / r, x2 = x * x, x3 = x2 * x, x6 = x3 * x3, x7 = x6 * x;
            d = S / 7.0f * (x7 - 1.0f) - S * x7;
            return (S * r / 7.0f) * (x7 - 1.0f);
        }
        case ARP_CONTACT_LENNARD_JONES: {
            float f = R0 / r;
            f *= f * f;
            f *= f;
            d = -12.0f * S * f * (f - 1.0f) / r;
            return S * (f * f - 2.0f * f);
        }
        case ARP_CONTACT_HERTZ: {
            const float x = r / R0, x2 = x * x, x3 = x2 * x, x6 = x3 * x3;
            d = S * x6;
            return (S * R0 / 7.0f) * (x6 * x - 1.0f);
        }
        default: return 0.0f;
    }
}

struct PairSide {
    float3 x, v;
    float d, inv_d, pt;
    float m, visc, bulk;
    uint32_t mat;
    bool elastic;
};
// What the two orientations of a pair share: r = x_b - x_a, v_b - v_a, gradW,
// the contact potential (the interaction matrix is symmetric).
struct PairGeom {
    float3 r, vv, g;
    float gws, c24, inv_denom;  // c24 = 24 k (h^2 - r.r): d gws / d r = c24 r
    float cp, dcp_over_R;
    bool contact;
};
struct PairGrad {
    float3 F;        // forward force contribution to the self particle
    float3 lr;       // dL/dr, r = x_nbr - x_self
    float3 lvv;      // dL/d(v_nbr - v_self)
    float ld_self, ld_nbr, lpt;
};

template <int DIM>
__device__ __forceinline__ PairGeom make_geom(float3 xa, float3 va, float3 xb, float3 vb, const DevInter& it,
                                              float h2, float kc, float eps_hh) {
    PairGeom G;
    G.r = sub(xb, xa);
    G.vv = sub(vb, va);
    if (DIM == 2) {
        G.r.z = 0.0f;
        G.vv.z = 0.0f;
    }
    const float r2 = dot(G.r, G.r);
    const float diff = fmaxf(h2 - r2, 0.0f);
    G.gws = -6.0f * kc * diff * diff;
    G.c24 = 24.0f * kc * diff;
    G.g = mul(G.gws, G.r);
    G.inv_denom = __fdividef(1.0f, r2 + eps_hh);
    G.cp = 0.0f;
    G.dcp_over_R = 0.0f;
    G.contact = false;
    if (it.potential != ARP_CONTACT_ZERO) {
        const float R = sqrtf(r2);
        float dcp;
        G.cp = cpot(it.potential, R, it.radius, it.strength, dcp);
        G.contact = G.cp != 0.0f;
        G.dcp_over_R = R > 0.0f ? __fdividef(dcp, R) : 0.0f;
    }
    return G;
}
__device__ __forceinline__ PairGeom flipped(const PairGeom& G) {
    PairGeom H = G;
    H.r = neg(G.r);
    H.vv = neg(G.vv);
    H.g = neg(G.g);
    return H;
}

// The fluid pair term of `a` with neighbor `b` (fluid.rs:154-214, as the
// forward kernel evaluates it) and its vector-Jacobian product for weights
// wd (on d rho/dt) and wF (on the force sum), friction (fluid.rs:192-199)
// included.
template <int DIM, bool BOUNDARY>
__device__ __forceinline__ void pair_vjp(const PairGeom& G, const PairSide& a, const PairSide& b, float dampening,
                                         float friction, float wd, float3 wF, PairGrad& o) {
    const float3 r = G.r, vv = G.vv, g = G.g;
    float3 F = make_float3(0.f, 0.f, 0.f), lg = F, lr = F, lvv = F;
    float ld1 = 0.f, ld2 = 0.f;
    if (!BOUNDARY) {
        lvv = mul(wd * b.m, g);
        lg = mul(wd * b.m, vv);
    }
    const float mm = a.m * b.m;
    const float pf = mm * (a.pt + b.pt);
    F = mul(pf, g);
    lg = add(lg, mul(pf, wF));
    const float wg = dot(wF, g);
    const float lpt = mm * wg;
    if (G.contact) {
        const float cs = b.m * G.cp * b.inv_d;
        F = add(F, mul(cs, g));
        lg = add(lg, mul(cs, wF));
        ld2 -= wg * cs * b.inv_d;
        lr = mul(wg * b.m * b.inv_d * G.dcp_over_R, r);
        if (friction != 0.0f && (a.elastic || b.elastic || BOUNDARY) && a.mat != b.mat) {
            // forward: the normal force r (cs g.r) / r.r = cs gws r has length
            // N = |cs gws| R; the tangential velocity u = vv - r (vv.r) / r.r
            // gives t = u / |u|, and the force gains friction N t (the second
            // normalize of the shader leaves t as it is)
            const float r2 = dot(r, r);
            const float sv = dot(vv, r) / r2;
            const float3 u = sub(vv, mul(sv, r));
            const float ul = sqrtf(dot(u, u));
            const float3 t = mul(1.0f / ul, u);
            if (isfinite(t.x) && isfinite(t.y) && isfinite(t.z)) {
                const float R = sqrtf(r2);
                const float acs = fabsf(cs), ags = fabsf(G.gws);
                const float N = acs * ags * R;
                F = add(F, mul(friction * N, t));
                const float wt = dot(wF, t);
                // through t = u / |u| and u = (I - r r^T / r.r) vv
                const float3 lu = mul(friction * N / ul, sub(wF, mul(wt, t)));
                const float lur = dot(lu, r);
                lvv = add(lvv, sub(lu, mul(lur / r2, r)));
                lr = add(lr, sub(mul(-sv, lu), mul(lur / r2, sub(vv, mul(2.0f * sv, r)))));
                // through N: |cs| ~ 1/rho_b; dN/dR from cp(R), gws(R) (d gws/dR = c24 R) and R
                const float lN = friction * wt;
                ld2 -= lN * N * b.inv_d;
                const float dcs = copysignf(b.m * b.inv_d * G.dcp_over_R * R, cs);
                const float dgs = copysignf(G.c24 * R, G.gws);
                const float dN = dcs * ags * R + acs * dgs * R + acs * ags;
                lr = add(lr, mul(lN * dN / R, r));
            }
        }
    }
    if (!BOUNDARY) {
        float ldenom = 0.0f;
        if (!a.elastic) {
            const float fsum = a.visc + b.visc;
            if (fsum != 0.0f) {
                const float rgw = dot(r, g);
                const float idd = a.inv_d * b.inv_d * G.inv_denom;
                const float t = mm * fsum * rgw * idd;
                F = sub(F, mul(t, vv));
                lvv = sub(lvv, mul(t, wF));
                const float lt = -dot(wF, vv);
                const float lrgw = lt * mm * fsum * idd;
                ld1 -= lt * t * a.inv_d;
                ld2 -= lt * t * b.inv_d;
                ldenom -= lt * t * G.inv_denom;
                lr = add(lr, mul(lrgw, g));
                lg = add(lg, mul(lrgw, r));
            }
        }
        const float f_ = a.mat == b.mat ? a.bulk + b.bulk : dampening;
        if (f_ != 0.0f) {
            const float vr = dot(vv, r);
            const float ids = __fdividef(1.0f, a.d + b.d);
            const float q0 = mm * f_ * ids * G.inv_denom;
            const float Q = q0 * vr;
            F = sub(F, mul(Q, g));
            lg = sub(lg, mul(Q, wF));
            const float lQ = -wg;
            const float lvr = lQ * q0;
            ld1 -= lQ * Q * ids;
            ld2 -= lQ * Q * ids;
            ldenom -= lQ * Q * G.inv_denom;
            lvv = add(lvv, mul(lvr, r));
            lr = add(lr, mul(lvr, vv));
        }
        lr = add(lr, mul(2.0f * ldenom, r));
    }
    // g = gws(r) r, gws = -6 k (h^2 - r.r)^2
    lr = add(lr, add(mul(G.gws, lg), mul(G.c24 * dot(lg, r), r)));
    if (DIM == 2) {
        lr.z = 0.0f;
        lvv.z = 0.0f;
    }
    o.F = F;
    o.lr = lr;
    o.lvv = lvv;
    o.ld_self = ld1;
    o.ld_nbr = ld2;
    o.lpt = lpt;
}

// Per particle of the stage: the weights of its derivative record and its
// state-equation terms, read by its own thread and by its neighbors':
// w = (mu_v / rho, mu_rho), e = (p / rho^2, d(p / rho^2)/d rho, 1 / rho);
// and the positions in cell order for the neighbor scan.  Thread k is cell
// position k.
__global__ void k_adj_prep(AdjArgs a, Tables T, float4* __restrict__ w, float4* __restrict__ e) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= a.n) return;
    const uint32_t i = a.st.perm ? a.st.perm[k] : k;
    const float4 xi = a.st.pd[i];
    a.xs[k] = xi;
    const FluidMat fm = T.fmats[__float_as_uint(a.st.vm[i].w)];
    const float ir = 1.0f / xi.w;
    const float4 mv = a.mu_vm[i];
    w[i] = make_float4(mv.x * ir, mv.y * ir, mv.z * ir, a.mu_pd[i].w);
    float pt, dpt;
    eos_pt(fm.eos, xi.w, fm.c, fm.d0, pt, dpt);
    e[i] = make_float4(pt, dpt, ir, 0.0f);
}

constexpr int kAdjCap = 48;                   // hit-list entries per thread of k_adj_fluid
constexpr uint32_t kHitBoundary = 0x80000000u;  // list entry of a boundary particle

template <int DIM>
__global__ void __launch_bounds__(kT) k_adj_fluid(AdjArgs a, Tables T, const float4* __restrict__ W,
                                                  const float4* __restrict__ EQ) {
    __shared__ uint32_t lst[kAdjCap * kT];
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    const float4 xi = a.st.pd[i], vi = a.st.vm[i];
    const uint32_t mat = __float_as_uint(vi.w);
    const DevMat& mm = T.mats[mat];
    const SceneP& P = T.scenes[mm.scene];
    const FluidMat fm = T.fmats[mat];
    const uint32_t sid = a.sid[i];
    const float4 ei = EQ[i], wi = W[i];
    const PairSide si{f3(xi), f3(vi), xi.w, ei.z, ei.x, fm.mass, fm.visc, fm.bulk, mat,
                      sid != kInvalid && fm.stiff != 0u};
    const float dpt_i = ei.y;
    const float wd = wi.w;
    const float3 wF = f3(wi);
    const bool solid_term = a.solid_branch && sid != kInvalid && P.solid_branch;
    float3 lx = make_float3(0.f, 0.f, 0.f);
    float3 lv = mul(solid_term ? 2.0f : 1.0f, f3(a.mu_pd[i]));  // dx/dt = v (twice for solids in the solid branch)
    float lrho = 0.0f;
    float3 Fs = make_float3(0.f, 0.f, 0.f);
    const uint32_t li = mat - P.mat_base;
    const DevInter* row_i = T.inter + P.inter_base + li * P.nmat;
    // Two passes, as in the forward kernel: the scan lists the hits (cell
    // positions; boundary ones flagged) in shared memory, then the pair VJPs
    // run over the list with nearly full warps.  A particle with more hits
    // than the list holds scans again for the next kAdjCap of them (the pair
    // math stays at one call site); the pairs are taken in scan order.
    uint32_t* my = lst + threadIdx.x;
    auto eval = [&](uint32_t h) {
        if (h & kHitBoundary) {
            const uint32_t jb = h & ~kHitBoundary;
            const float4 xb = a.bxs[jb];
            const float4 vb = a.bvs[jb];
            const uint32_t matb = __float_as_uint(vb.w);
            const FluidMat fb = T.fmats[matb];
            const PairSide sb{f3(xb), f3(vb), xb.w, __fdividef(1.0f, xb.w), a.bps[jb], fb.mass, fb.visc,
                              fb.bulk, matb, false};
            const DevInter it = row_i[matb - P.mat_base];
            const PairGeom G = make_geom<DIM>(si.x, si.v, sb.x, sb.v, it, P.h2, P.kconst, P.eps_hh);
            PairGrad o;
            pair_vjp<DIM, true>(G, si, sb, it.dampening, it.friction, wd, wF, o);
            Fs = add(Fs, o.F);
            lx = sub(lx, o.lr);
            lv = sub(lv, o.lvv);
            lrho += o.ld_self + o.lpt * dpt_i;
        } else {
            const uint32_t j = a.st.perm ? a.st.perm[h] : h;
            if (j == i) return;
            const float4 xj = a.st.pd[j];
            const float4 vj = a.st.vm[j];
            const uint32_t matj = __float_as_uint(vj.w);
            const FluidMat fj = T.fmats[matj];
            const uint32_t sidj = a.sid[j];
            const float4 ej = EQ[j], wj = W[j];
            const PairSide sj{f3(xj), f3(vj), xj.w, ej.z, ej.x, fj.mass, fj.visc, fj.bulk, matj,
                              sidj != kInvalid && fj.stiff != 0u};
            const DevInter it = row_i[matj - P.mat_base];  // symmetric: also the neighbor's entry
            const PairGeom G = make_geom<DIM>(si.x, si.v, sj.x, sj.v, it, P.h2, P.kconst, P.eps_hh);
            PairGrad o;
            pair_vjp<DIM, false>(G, si, sj, it.dampening, it.friction, wd, wF, o);
            Fs = add(Fs, o.F);
            lx = sub(lx, o.lr);
            lv = sub(lv, o.lvv);
            lrho += o.ld_self + o.lpt * dpt_i;
            // the neighbor's own pair, in which this particle is the neighbor
            pair_vjp<DIM, false>(flipped(G), sj, si, it.dampening, it.friction, wj.w, f3(wj), o);
            lx = add(lx, o.lr);
            lv = add(lv, o.lvv);
            lrho += o.ld_nbr + o.lpt * dpt_i;
        }
    };
    if (finite3(xi)) {
        for (uint32_t done = 0;;) {
            uint32_t total = 0, cnt = 0;  // hits seen in this scan, hits listed
            auto take = [&](uint32_t h) {
                if (total >= done && cnt < (uint32_t)kAdjCap) my[cnt++ * kT] = h;
                ++total;
            };
            for_search_rows<DIM>(xi, P, [&](uint32_t c0, uint32_t c1) {
                for (uint32_t jb = a.bstart[c0]; jb < a.bstart[c1]; ++jb) {
                    const float4 xb = a.bxs[jb];
                    const float rx = xb.x - xi.x, ry = xb.y - xi.y, rz = DIM == 3 ? xb.z - xi.z : 0.0f;
                    if (P.h2 - (rx * rx + ry * ry + rz * rz) > 0.0f) take(jb | kHitBoundary);
                }
                for (uint32_t k = a.st.start[c0]; k < a.st.start[c1]; ++k) {
                    const float4 xj = a.xs[k];
                    const float rx = xj.x - xi.x, ry = xj.y - xi.y, rz = DIM == 3 ? xj.z - xi.z : 0.0f;
                    if (P.h2 - (rx * rx + ry * ry + rz * rz) > 0.0f) take(k);
                }
            });
            for (uint32_t e = 0; e < cnt; ++e) eval(my[e * kT]);
            done += cnt;
            if (done >= total) break;
        }
    }
    lrho -= dot(wF, Fs) * ei.z;  // k_v = F / rho
    if (DIM == 2) {
        lx.z = 0.0f;
        lv.z = 0.0f;
    }
    float4 lp = a.lam_pd[i], lw = a.lam_vm[i];
    lp.x += lx.x;
    lp.y += lx.y;
    lp.z += lx.z;
    lp.w += lrho;
    lw.x += lv.x;
    lw.y += lv.y;
    lw.z += lv.z;
    a.lam_pd[i] = lp;
    a.lam_vm[i] = lw;
}

// ---- Seth-Hill strain of any order and its VJP (3x3: the padded fourth axis,
// where C = 1, stays out of every matrix function) --------------------------
__device__ __forceinline__ M3 m3_ident() {
    M3 r = m3_zero();
    r.m[0][0] = r.m[1][1] = r.m[2][2] = 1.0f;
    return r;
}
__device__ __forceinline__ M3 m3_scale(float s, const M3& a) {
    M3 r;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) r.m[i][j] = s * a.m[i][j];
    return r;
}
__device__ __forceinline__ M3 m3_add(const M3& a, const M3& b) {
    M3 r = a;
    m3_acc(r, b);
    return r;
}
__device__ __forceinline__ M3 m3_sub(const M3& a, const M3& b) {
    M3 r;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) r.m[i][j] = a.m[i][j] - b.m[i][j];
    return r;
}
__device__ inline M3 m3_inv(const M3& a) {  // adjugate over determinant
    const float (&m)[3][3] = a.m;
    M3 c;
    c.m[0][0] = m[1][1] * m[2][2] - m[1][2] * m[2][1];
    c.m[0][1] = m[0][2] * m[2][1] - m[0][1] * m[2][2];
    c.m[0][2] = m[0][1] * m[1][2] - m[0][2] * m[1][1];
    c.m[1][0] = m[1][2] * m[2][0] - m[1][0] * m[2][2];
    c.m[1][1] = m[0][0] * m[2][2] - m[0][2] * m[2][0];
    c.m[1][2] = m[0][2] * m[1][0] - m[0][0] * m[1][2];
    c.m[2][0] = m[1][0] * m[2][1] - m[1][1] * m[2][0];
    c.m[2][1] = m[0][1] * m[2][0] - m[0][0] * m[2][1];
    c.m[2][2] = m[0][0] * m[1][1] - m[0][1] * m[1][0];
    const float det = m[0][0] * c.m[0][0] + m[0][1] * c.m[1][0] + m[0][2] * c.m[2][0];
    return m3_scale(1.0f / det, c);
}
__device__ inline M3 m3_pow(const M3& c, int m) {
    M3 r = m3_ident();
    for (int i = 0; i < m; ++i) r = m3_mul(r, c);
    return r;
}
// Denman-Beavers square root, the iteration of solid.rs:119-133
__device__ inline M3 m3_sqrt_db(const M3& c) {
    M3 Y = c, Z = m3_ident();
    for (int i = 0; i < 15; ++i) {
        const M3 Yn = m3_scale(0.5f, m3_add(Y, m3_inv(Z)));
        const M3 Zn = m3_scale(0.5f, m3_add(Z, m3_inv(Y)));
        Y = Yn;
        Z = Zn;
    }
    return Y;
}
// X with R X + X R = W (R symmetric): the VJP of the square root, whose
// differential solves R dR + dR R = dC (the operator is self-adjoint for a
// symmetric R).  A 9 x 9 system, Gaussian elimination with partial pivoting.
__device__ inline M3 lyap_solve(const M3& R, const M3& W) {
    float A[9][10];
#pragma unroll
    for (int p = 0; p < 9; ++p)
#pragma unroll
        for (int q = 0; q < 10; ++q) A[p][q] = 0.0f;
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const int p = 3 * r + c;
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                A[p][3 * k + c] += R.m[r][k];
                A[p][3 * r + k] += R.m[k][c];
            }
            A[p][9] = W.m[r][c];
        }
    for (int col = 0; col < 9; ++col) {
        int piv = col;
        for (int p = col + 1; p < 9; ++p)
            if (fabsf(A[p][col]) > fabsf(A[piv][col])) piv = p;
        if (piv != col)
            for (int q = 0; q < 10; ++q) {
                const float t = A[col][q];
                A[col][q] = A[piv][q];
                A[piv][q] = t;
            }
        const float inv = 1.0f / A[col][col];
        for (int p = col + 1; p < 9; ++p) {
            const float f = A[p][col] * inv;
            for (int q = col; q < 10; ++q) A[p][q] -= f * A[col][q];
        }
    }
    float x[9];
    for (int p = 8; p >= 0; --p) {
        float t = A[p][9];
        for (int q = p + 1; q < 9; ++q) t -= A[p][q] * x[q];
        x[p] = t / A[p][p];
    }
    M3 X;
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c) X.m[r][c] = x[3 * r + c];
    return X;
}
// d/dC of C^m against weight W: sum_k C^k W C^(m-1-k) (C symmetric)
__device__ inline M3 m3_pow_vjp(const M3& C, int m, const M3& W) {
    M3 g = m3_zero();
    for (int k = 0; k < m; ++k) m3_acc(g, m3_mul(m3_mul(m3_pow(C, k), W), m3_pow(C, m - 1 - k)));
    return g;
}
// E = seth_hill(C, two_m) (solid.rs:147-168; C padded with ones)
__device__ inline M3 sh_forward(const M3& C, int two_m) {
    if (two_m == 0) {  // 0.5 * the 5-term log series of solid.rs:105-116
        const M3 D = m3_sub(C, m3_ident());
        M3 sum = m3_zero(), Dk = m3_ident();
        for (int i = 1; i <= 5; ++i) {
            Dk = m3_mul(Dk, D);
            m3_acc(sum, m3_scale((i & 1 ? 1.0f : -1.0f) / (float)i, Dk));
        }
        return m3_scale(0.5f, sum);
    }
    const int a = two_m < 0 ? -two_m : two_m;
    M3 M = m3_pow(C, a >> 1);
    if (a & 1) M = m3_mul(M, m3_sqrt_db(C));
    if (two_m < 0) M = m3_inv(M);
    return m3_scale(1.0f / (float)two_m, m3_sub(M, m3_ident()));
}
// dL/dC of E = seth_hill(C, two_m) for the weight W on E
__device__ inline M3 sh_vjp(const M3& C, int two_m, const M3& W) {
    if (two_m == 0) {
        const M3 D = m3_sub(C, m3_ident());
        const M3 hw = m3_scale(0.5f, W);
        M3 g = m3_zero();
        for (int i = 1; i <= 5; ++i) m3_acc(g, m3_scale((i & 1 ? 1.0f : -1.0f) / (float)i, m3_pow_vjp(D, i, hw)));
        return g;
    }
    const int a = two_m < 0 ? -two_m : two_m, m = a >> 1;
    const M3 Pm = m3_pow(C, m);
    const M3 Rt = (a & 1) ? m3_sqrt_db(C) : m3_ident();
    const M3 Q = m3_mul(Pm, Rt);
    M3 lQ = m3_scale(1.0f / (float)two_m, W);
    if (two_m < 0) {  // M = Q^-1: dL/dQ = -Q^-T W' Q^-T
        const M3 Qi = m3_inv(Q);
        lQ = m3_scale(-1.0f, m3_mul(m3_mul(m3_t(Qi), lQ), m3_t(Qi)));
    }
    M3 g = m3_pow_vjp(C, m, m3_mul(lQ, m3_t(Rt)));
    if (a & 1) m3_acc(g, lyap_solve(Rt, m3_mul(m3_t(Pm), lQ)));
    return g;
}
// Ed = seth_hill_rate(C, dC, two_m) (solid.rs:170-204): 0.5 dC C^-1 for order
// 0, else (1/two_m) sum_i C^i dC C^(m-1-i) (the square-root part is not
// differentiated in time there, the shader's TODO), conjugated by -C^-1 for
// negative orders
__device__ inline M3 sh_rate_forward(const M3& C, const M3& dC, int two_m) {
    if (two_m == 0) return m3_mul(m3_scale(0.5f, dC), m3_inv(C));
    const int a = two_m < 0 ? -two_m : two_m, m = a >> 1;
    M3 rate = m3_zero();
    for (int i = 0; i < m; ++i) m3_acc(rate, m3_mul(m3_mul(m3_pow(C, i), dC), m3_pow(C, m - 1 - i)));
    rate = m3_scale(1.0f / (float)two_m, rate);
    if (two_m < 0) {
        const M3 iC = m3_inv(C);
        return m3_scale(-1.0f, m3_mul(m3_mul(iC, rate), iC));
    }
    return rate;
}
__device__ inline void sh_rate_vjp(const M3& C, const M3& dC, int two_m, const M3& W, M3& lC, M3& ldC) {
    if (two_m == 0) {  // 0.5 dC Ci
        const M3 Ci = m3_inv(C);
        ldC = m3_scale(0.5f, m3_mul(W, m3_t(Ci)));
        const M3 lCi = m3_scale(0.5f, m3_mul(m3_t(dC), W));
        lC = m3_scale(-1.0f, m3_mul(m3_mul(m3_t(Ci), lCi), m3_t(Ci)));
        return;
    }
    const int a = two_m < 0 ? -two_m : two_m, m = a >> 1;
    M3 lX = m3_scale(1.0f / (float)two_m, W);
    lC = m3_zero();
    if (two_m < 0) {  // Ed = -Ci X Ci, X = rate / two_m
        const M3 Ci = m3_inv(C);
        M3 X = m3_zero();
        for (int i = 0; i < m; ++i) m3_acc(X, m3_mul(m3_mul(m3_pow(C, i), dC), m3_pow(C, m - 1 - i)));
        X = m3_scale(1.0f / (float)two_m, X);
        const M3 lCi = m3_scale(-1.0f, m3_add(m3_mul(W, m3_t(m3_mul(X, Ci))), m3_mul(m3_t(m3_mul(Ci, X)), W)));
        lC = m3_scale(-1.0f, m3_mul(m3_mul(m3_t(Ci), lCi), m3_t(Ci)));
        lX = m3_scale(-1.0f / (float)two_m, m3_mul(m3_mul(m3_t(Ci), W), m3_t(Ci)));
    }
    ldC = m3_zero();
    for (int i = 0; i < m; ++i) {
        const M3 Pi = m3_pow(C, i), Pj = m3_pow(C, m - 1 - i);
        m3_acc(ldC, m3_mul(m3_mul(m3_t(Pi), lX), m3_t(Pj)));
        m3_acc(lC, m3_pow_vjp(C, i, m3_mul(lX, m3_t(m3_mul(dC, Pj)))));
        m3_acc(lC, m3_pow_vjp(C, m - 1 - i, m3_mul(m3_t(m3_mul(Pi, dC)), lX)));
    }
}

// Hourglass pair term of `self` (solid.rs:430-443 as k_solid_forces evaluates
// it) and its VJP for weight w: forward force f, dL/d(dx) with dx = x_nbr -
// x_self, dL/de (e = 0.5 (F_self + F_nbr) dX - dx), dL/d rho_self, rho_nbr.
struct HgGrad {
    float3 f, ldx, le;
    float lda, ldb;
};
__device__ __forceinline__ void hg_vjp(float3 dx, float3 dX, const M3& Fa, const M3& Fb, float da, float db, float m,
                                       float kern, const SceneP& P, float3 w, HgGrad& o) {
    M3 Fs;
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c) Fs.m[r][c] = 0.5f * (Fa.m[r][c] + Fb.m[r][c]);
    const float3 e = sub(m3_vec(Fs, dX), dx);
    const float l = sqrtf(dot(dx, dx));
    const float ed = dot(e, dx);
    const float a1 = 100000000.0f * m * m / (da * db);
    const float lh = l + P.hg_h;
    const float b1 = 0.5f * ed / lh;
    const float c1 = 1.0f / (l * l + P.eps_hh);
    const float sh = a1 * b1 * c1 * kern;
    const float den = l + P.eps_h;
    const float u = sh / den;
    o.f = mul(-u, dx);
    const float lu = -dot(w, dx);
    float3 ldx = mul(-u, w);
    const float lsh = lu / den;
    const float lden = -lu * u / den;
    const float la1 = lsh * b1 * c1 * kern, lb1 = lsh * a1 * c1 * kern, lc1 = lsh * a1 * b1 * kern;
    o.lda = -la1 * a1 / da;
    o.ldb = -la1 * a1 / db;
    const float led = lb1 * 0.5f / lh;
    float ll = -lb1 * b1 / lh - lc1 * c1 * c1 * 2.0f * l + lden;
    const float3 le = mul(led, dx);
    ldx = add(ldx, mul(led, e));
    ldx = sub(ldx, le);
    if (l > 0.0f) ldx = add(ldx, mul(ll / l, dx));
    o.ldx = ldx;
    o.le = le;
}

__device__ __forceinline__ bool in_stencil2(uint2 a, uint2 b) {
    const int dx = (int)(a.x & 0xFFFFu) - (int)(b.x & 0xFFFFu);
    const int dy = (int)(a.x >> 16) - (int)(b.x >> 16);
    const int dz = (int)a.y - (int)b.y;
    return a.y != 0xFFFFFFFFu && b.y != 0xFFFFFFFFu && dx >= -1 && dx <= 1 && dy >= -1 && dy <= 1 && dz >= -1 &&
           dz <= 1;
}

// LANES threads share one solid: both reference-list loops are split over
// them with stride LANES, their partial sums combined by group_sum; lane 0
// finishes the particle.
// GENERAL: some solid material has a strain order other than 2 (the log
// series, square roots and inverses are compiled out otherwise).  PLASTIC:
// some material is plastic; the plastic strain then enters E and its rate
// (the relaxation towards the Johnson-Cook yield surface, solid.rs:499-517)
// is differentiated, 4 x 4 as the shader holds them.
template <int LANES, bool GENERAL, bool PLASTIC>
__global__ void __launch_bounds__(kT) k_adj_solid(AdjArgs a, Tables T) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t i = t / LANES, lane = t % LANES;
    if (i >= a.ns) return;  // whole groups leave together
    const float4 xi = a.st.sx[i], vi = a.st.sv[i];
    const uint32_t mat = __float_as_uint(vi.w);
    const DevMat mm = T.mats[mat];
    const SceneP& P = T.scenes[mm.scene];
    if (!P.solid_branch) return;
    const uint32_t slot = a.slot_of[i];
    const float d1 = xi.w, m1 = mm.mass, V1 = m1 / d1;
    const float3 w = mul(1.0f / d1, f3(a.mu_vm[slot]));
    const float3 wdm = mask_dim(w, P.dim);
    const M3 Ai = m3_cols(a.st.A + 3 * i), Fi = m3_cols(a.st.F + 3 * i);
    const float3 Xi = f3(a.ref[i]);
    const uint2 ci = a.st.sc[i];
    M3 lA = m3_zero(), lFh = m3_zero();
    float3 lx = make_float3(0.f, 0.f, 0.f), fs = lx;
    float lrho = 0.0f;
    const uint32_t k0 = a.rl.off[i], k1 = a.rl.off[i + 1];
    for (uint32_t k = k0 + lane; k < k1; k += LANES) {
        const uint32_t e = a.rl.nbr[k];
        if (!(e & kSameMatBit)) continue;
        const uint32_t j = e & ~kSameMatBit;
        const float3 g = ref_grad(a.ref, j, Xi, P);
        const float4 xj = a.st.sx[j];
        const float d2 = xj.w;
        const float c = -V1 * (m1 / d2);
        const M3 Aj = m3_cols(a.st.A + 3 * j);
        M3 As;
#pragma unroll
        for (int r = 0; r < 3; ++r)
#pragma unroll
            for (int cc = 0; cc < 3; ++cc) As.m[r][cc] = Ai.m[r][cc] + Aj.m[r][cc];
        const float3 Ag = m3_vec(As, g);
        fs = add(fs, mul(c, mask_dim(Ag, P.dim)));
        m3_add_outer(lA, c, wdm, g);
        lrho += (-c / d1) * dot(wdm, Ag);
        // the neighbor's elastic term: f_j += c (A_j + A_i) grad_w(X_i - X_j), the gradient being -g
        const float3 wj = mul(1.0f / d2, f3(a.mu_vm[a.slot_of[j]]));
        const float3 wjd = mask_dim(wj, P.dim);
        m3_add_outer(lA, -c, wjd, g);
        lrho += (c / d1) * dot(wjd, Ag);
        if (in_stencil2(a.st.sc[j], ci)) {
            const M3 Fj = m3_cols(a.st.F + 3 * j);
            const float3 dx = sub(f3(xj), f3(xi));
            const float3 dX = sub(f3(a.ref[j]), Xi);
            const float diff = P.h2 - dot(dX, dX);
            const float kern = P.kconst * diff * diff * diff;
            HgGrad o;
            hg_vjp(dx, dX, Fi, Fj, d1, d2, m1, kern, P, w, o);
            fs = add(fs, o.f);
            lx = sub(lx, o.ldx);
            m3_add_outer(lFh, 0.5f, o.le, dX);
            lrho += o.lda;
            hg_vjp(neg(dx), neg(dX), Fj, Fi, d2, d1, m1, kern, P, wj, o);
            lx = add(lx, o.ldx);
            m3_add_outer(lFh, -0.5f, o.le, dX);
            lrho += o.ldb;
        }
    }
    // dF/dt of the stage, recomputed from the reference list
    const M3 L = m3_cols(a.L + 3 * i);
    M3 Fd = m3_zero();
    for (uint32_t k = k0 + lane; k < k1; k += LANES) {
        const uint32_t j = a.rl.nbr[k] & ~kSameMatBit;
        const float4 vj = a.st.sv[j];
        const float3 G = m3_vec(L, ref_grad(a.ref, j, Xi, P));
        const float3 dv = sub(f3(vj), f3(vi));
        m3_add_outer(Fd, a.ref[j].w, dv, G);  // ref.w = V_j
    }
    if (LANES > 1) {
#pragma unroll
        for (int r = 0; r < 3; ++r)
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                lA.m[r][c] = group_sum<LANES>(lA.m[r][c]);
                lFh.m[r][c] = group_sum<LANES>(lFh.m[r][c]);
                Fd.m[r][c] = group_sum<LANES>(Fd.m[r][c]);
            }
        lx = make_float3(group_sum<LANES>(lx.x), group_sum<LANES>(lx.y), group_sum<LANES>(lx.z));
        fs = make_float3(group_sum<LANES>(fs.x), group_sum<LANES>(fs.y), group_sum<LANES>(fs.z));
        lrho = group_sum<LANES>(lrho);
        if (lane != 0) return;
    }
    // self-contact (solid.rs:445-450) is not differentiated: flag an active pair
    {
        const float U = __uint_as_float(a.st.contact_bound[0]);
        const bool maybe = !mm.plastic && (P.contact_slack <= 0.0f || a.st.contact_bound[1] != 0u ||
                                          !(2.0f * U < P.contact_slack));
        if (maybe && finite3(xi)) {
            bool active = false;
            for_reference_block_rows(xi, P, [&](uint32_t c0, uint32_t c1) {
                for (uint32_t k = a.st.start[c0]; k < a.st.start[c1] && !active; ++k) {
                    const uint32_t s2 = a.st.perm ? a.st.perm[k] : k;
                    if (__float_as_uint(a.st.vm[s2].w) != mat) continue;
                    const uint32_t sj = a.sid[s2];
                    if (sj == kInvalid) continue;
                    const float3 dx = sub(f3(a.st.pd[s2]), f3(xi));
                    const float3 dX = sub(f3(a.ref[sj]), Xi);
                    if (dot(dX, dX) > P.rcut2 && dot(dx, dx) < P.rcut2) active = true;
                }
            });
            if (active) atomicOr(a.flags, 1u);
        }
    }
    lrho -= dot(w, fs) / d1;  // k_v = f / rho - g
    // stress chain: C = F^T F (padded with ones past dim), dC = dF^T F + F^T dF,
    // E = seth_hill(C), dE/dt = seth_hill_rate(C, dC) (any strain order),
    // S = Hooke(E; n, s) + Hooke(dE/dt; n_d, s_d), sigma = F S^T, A = sigma L
    const uint32_t dim = P.dim;
    const int two_m = mm.strain_order;
    M3 C = m3_mul(m3_t(Fi), Fi);
#pragma unroll
    for (int q = 0; q < 3; ++q)
        if ((uint32_t)q >= dim) C.m[q][q] = 1.0f;
    const M3 Rfd = m3_mul(m3_t(Fd), Fi);
    const M3 dC = m3_add(Rfd, m3_t(Rfd));
    M3 E, Ed;
    if (!GENERAL || two_m == 2) {
        E = m3_scale(0.5f, m3_sub(C, m3_ident()));
        Ed = m3_scale(0.5f, dC);
    } else {
        E = sh_forward(C, two_m);
        Ed = sh_rate_forward(C, dC, two_m);
    }
    const float2 lm = a.stiff ? a.stiff[i] : make_float2(mm.lam, mm.mu);
    // 4 x 4 (row, column) as the shader: E4 = E (+ the plastic strain), S4 =
    // Hooke(E4) + Hooke(dE/dt) with the trace over the first dim axes times the
    // full 4 x 4 identity; sigma reads only S4's upper 3 x 3 block
    float E4[4][4], S4[4][4];
#pragma unroll
    for (int r = 0; r < 4; ++r)
#pragma unroll
        for (int c = 0; c < 4; ++c) E4[r][c] = (r < 3 && c < 3) ? E.m[r][c] : 0.0f;
    if (PLASTIC) {
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            const float4 e = a.st.ep[4 * i + c];  // column c
            E4[0][c] += e.x;
            E4[1][c] += e.y;
            E4[2][c] += e.z;
            E4[3][c] += e.w;
        }
    }
    float trE = 0.f, trEd = 0.f;
#pragma unroll
    for (int q = 0; q < 3; ++q)
        if ((uint32_t)q < dim) {
            trE += E4[q][q];
            trEd += Ed.m[q][q];
        }
#pragma unroll
    for (int r = 0; r < 4; ++r)
#pragma unroll
        for (int c = 0; c < 4; ++c)
            S4[r][c] = 2.0f * lm.y * E4[r][c] + ((r < 3 && c < 3) ? 2.0f * mm.mu_d * Ed.m[r][c] : 0.0f) +
                       (r == c ? lm.x * trE + mm.lam_d * trEd : 0.0f);
    M3 S;
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c) S.m[r][c] = S4[r][c];
    const M3 lsig = m3_mul(lA, m3_t(L));
    M3 lF = m3_mul(lsig, S);
    const M3 lS3 = m3_mul(m3_t(lsig), Fi);
    float lS4[4][4];
#pragma unroll
    for (int r = 0; r < 4; ++r)
#pragma unroll
        for (int c = 0; c < 4; ++c) lS4[r][c] = (r < 3 && c < 3) ? lS3.m[r][c] : 0.0f;
    if (PLASTIC && mm.plastic) {
        // rate = ((|S| - Y) / T) S / |S| when Y^2 <= |S|^2; the yield stress Y
        // is constant (the equivalent strain carries the integer factor
        // (dim-1)/dim = 0, solid.rs:214); its VJP for the weight mu:
        // (1/T) ((1 - Y/|S|) mu + (mu:S) Y S / |S|^3)
        float sn = 0.0f, ms = 0.0f, mu4[4][4];
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            const float4 m = a.mu_ep[4 * i + c];
            mu4[0][c] = m.x;
            mu4[1][c] = m.y;
            mu4[2][c] = m.z;
            mu4[3][c] = m.w;
        }
#pragma unroll
        for (int r = 0; r < 4; ++r)
#pragma unroll
            for (int c = 0; c < 4; ++c) {
                sn += S4[r][c] * S4[r][c];
                ms += mu4[r][c] * S4[r][c];
            }
        const float Y = (mm.yield_strength + mm.work_hardening * powf(0.0f, mm.work_hardening_exp / 2.0f)) *
                        (1.0f + mm.kinematic_hardening * logf(1.0f));
        if (Y * Y <= sn) {
            const float sl = sqrtf(sn);
            const float it = 1.0f / mm.relaxation_time;
            const float c1 = it * (1.0f - Y / sl), c2 = it * ms * Y / (sl * sl * sl);
#pragma unroll
            for (int r = 0; r < 4; ++r)
#pragma unroll
                for (int c = 0; c < 4; ++c) lS4[r][c] += c1 * mu4[r][c] + c2 * S4[r][c];
        }
    }
    float trS = lS4[0][0] + lS4[1][1] + lS4[2][2] + lS4[3][3];
    M3 lE, lEd;
    float gs = 0.0f;
    if (PLASTIC) {
        // E4 = E + plastic strain: its adjoint is the plastic strain's
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            float4 l;
            float* lc = &l.x;
#pragma unroll
            for (int r = 0; r < 4; ++r) lc[r] = 2.0f * lm.y * lS4[r][c] + (r == c && (uint32_t)r < dim ? lm.x * trS : 0.0f);
            float4 acc = a.lam_ep[4 * i + c];
            acc.x += l.x;
            acc.y += l.y;
            acc.z += l.z;
            acc.w += l.w;
            a.lam_ep[4 * i + c] = acc;
        }
    }
#pragma unroll
    for (int r = 0; r < 4; ++r)
#pragma unroll
        for (int c = 0; c < 4; ++c) gs += 2.0f * lS4[r][c] * E4[r][c];
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const bool d = r == c && (uint32_t)r < dim;
            lE.m[r][c] = 2.0f * lm.y * lS4[r][c] + (d ? lm.x * trS : 0.0f);
            lEd.m[r][c] = 2.0f * mm.mu_d * lS4[r][c] + (d ? mm.lam_d * trS : 0.0f);
        }
    const float gn = trE * trS;
    M3 lC, ldC;
    if (!GENERAL || two_m == 2) {
        lC = m3_scale(0.5f, lE);
        ldC = m3_scale(0.5f, lEd);
    } else {
        lC = sh_vjp(C, two_m, lE);
        M3 lC2;
        sh_rate_vjp(C, dC, two_m, lEd, lC2, ldC);
        m3_acc(lC, lC2);
    }
#pragma unroll
    for (int q = 0; q < 3; ++q)
        if ((uint32_t)q >= dim) lC.m[q][q] = 0.0f;  // the padded ones do not depend on F
    // C = F^T F; dC = R + R^T with R = dF^T F
    const M3 lR = m3_add(ldC, m3_t(ldC));
    m3_acc(lF, m3_mul(Fi, m3_add(lC, m3_t(lC))));
    m3_acc(lF, m3_mul(Fd, lR));
    const M3 lFd = m3_mul(Fi, m3_t(lR));
    m3_acc(lF, lFh);
    m3_store_cols(lF, a.lamF + 3 * i);
    m3_store_cols(lFd, a.lamFd + 3 * i);
    // summed over every stage of every step in double: the per-stage terms
    // change sign as the bar oscillates, and a float sum would lose the
    // difference to rounding
    double2 gsum = a.g_stiff[i];
    gsum.x += (double)gn;
    gsum.y += (double)gs;
    a.g_stiff[i] = gsum;
    float4 lp = a.lam_pd[slot];
    lp.x += lx.x;
    lp.y += lx.y;
    lp.z += lx.z;
    lp.w += lrho;
    a.lam_pd[slot] = lp;
}

// F_i = sum_j V_j (x_j - x_i) (x) L_i gradW_ij and dF/dt likewise with v:
// gather the adjoints of F and dF/dt of the particle and of its reference
// neighbors into dL/dx and dL/dv.
__global__ void __launch_bounds__(kT) k_adj_strain(AdjArgs a, Tables T) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.ns) return;
    const uint32_t mat = __float_as_uint(a.st.sv[i].w);
    const DevMat& mm = T.mats[mat];
    const SceneP& P = T.scenes[mm.scene];
    if (!P.solid_branch) return;
    const uint32_t slot = a.slot_of[i];
    const M3 Li = m3_cols(a.L + 3 * i);
    const M3 lFi = m3_cols(a.lamF + 3 * i), lFdi = m3_cols(a.lamFd + 3 * i);
    const float Vri = mm.vol0;
    const float3 Xi = f3(a.ref[i]);
    float3 lx = make_float3(0.f, 0.f, 0.f), lv = lx;
    for (uint32_t k = a.rl.off[i]; k < a.rl.off[i + 1]; ++k) {
        const uint32_t j = a.rl.nbr[k] & ~kSameMatBit;
        const float3 g = ref_grad(a.ref, j, Xi, P);
        const float4 g4 = make_float4(g.x, g.y, g.z, a.ref[j].w);  // ref.w = V_j
        const float3 G = m3_vec(Li, g);
        lx = sub(lx, mul(g4.w, m3_vec(lFi, G)));
        lv = sub(lv, mul(g4.w, m3_vec(lFdi, G)));
        // in F_j this particle enters with V_i and L_j gradW(X_i - X_j) = -L_j g
        const M3 Lj = m3_cols(a.L + 3 * j);
        const float3 Gj = neg(m3_vec(Lj, g));
        lx = add(lx, mul(Vri, m3_vec(m3_cols(a.lamF + 3 * j), Gj)));
        lv = add(lv, mul(Vri, m3_vec(m3_cols(a.lamFd + 3 * j), Gj)));
    }
    float4 lp = a.lam_pd[slot], lw = a.lam_vm[slot];
    lp.x += lx.x;
    lp.y += lx.y;
    lp.z += lx.z;
    lw.x += lv.x;
    lw.y += lv.y;
    lw.z += lv.z;
    a.lam_pd[slot] = lp;
    a.lam_vm[slot] = lw;
}

struct Later {
    const float4* pd[4];
    const float4* vm[4];
    float c[4];
    int n;
};

__device__ __forceinline__ float4 axpy4(float c, float4 x, float4 y) {
    return make_float4(y.x + c * x.x, y.y + c * x.y, y.z + c * x.z, y.w + c * x.w);
}

__global__ void k_adj_weights(uint32_t n, float cb, const float4* __restrict__ lp, const float4* __restrict__ lv,
                              Later L, float4* __restrict__ mp, float4* __restrict__ mv) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const float4 z = make_float4(0.f, 0.f, 0.f, 0.f);
    float4 p = axpy4(cb, lp[k], z), v = axpy4(cb, lv[k], z);
    for (int t = 0; t < L.n; ++t) {
        p = axpy4(L.c[t], L.pd[t][k], p);
        v = axpy4(L.c[t], L.vm[t][k], v);
    }
    v.w = 0.0f;
    mp[k] = p;
    mv[k] = v;
}

__global__ void k_adj_weights_all(uint32_t n, float cb, const float4* __restrict__ l, Later L,
                                  float4* __restrict__ m) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    float4 p = axpy4(cb, l[k], make_float4(0.f, 0.f, 0.f, 0.f));
    for (int t = 0; t < L.n; ++t) p = axpy4(L.c[t], L.pd[t][k], p);
    m[k] = p;
}

__global__ void k_adj_sum_all(uint32_t n, const float4* __restrict__ l, Later L, float4* __restrict__ out) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    float4 p = l[k];
    for (int t = 0; t < L.n; ++t) p = axpy4(1.0f, L.pd[t][k], p);
    out[k] = p;
}

// Velocity Verlet.  The weights of a step's one force evaluation f(y*): the
// closing kick's (dt/2)(lam_rho, lam_v) plus the adjoint of the carried record
// (the next step's kick reads it); positions are not kicked, so no position part.
__global__ void k_verlet_mu(uint32_t n, const float4* __restrict__ lsp, const float4* __restrict__ lsv,
                            const float4* __restrict__ lfp, const float4* __restrict__ lfv, float h,
                            float4* __restrict__ mp, float4* __restrict__ mv) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const float4 a = lsp[k], b = lsv[k], c = lfp[k], d = lfv[k];
    mp[k] = make_float4(0.f, 0.f, 0.f, c.w + h * a.w);
    mv[k] = make_float4(d.x + h * b.x, d.y + h * b.y, d.z + h * b.z, 0.f);
}
// The kick-drift's adjoint, per particle (caller order): from lam of
// y* = (x + dt (v + h a), v + h a, rho + h drho) to lam of (x, v, rho), in
// place, and the adjoint of the record (a, drho) it read, h = dt/2.
__global__ void k_verlet_kd_adj(uint32_t n, float4* __restrict__ lp, float4* __restrict__ lv, float h, float dt,
                                float4* __restrict__ lfp, float4* __restrict__ lfv) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const float4 p = lp[k];
    float4 v = lv[k];
    v.x += dt * p.x;
    v.y += dt * p.y;
    v.z += dt * p.z;
    lv[k] = v;
    lfp[k] = make_float4(0.f, 0.f, 0.f, h * p.w);
    lfv[k] = make_float4(h * v.x, h * v.y, h * v.z, 0.f);
}

__global__ void k_adj_perm(uint32_t n, const uint32_t* __restrict__ orig, const float4* __restrict__ ip,
                           const float4* __restrict__ iv, float4* __restrict__ op, float4* __restrict__ ov,
                           int scatter) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const uint32_t c = orig[k];
    if (scatter) {
        op[c] = ip[k];
        ov[c] = iv[k];
    } else {
        op[k] = ip[c];
        ov[k] = iv[c];
    }
}

}  // namespace

int launch_adjoint_stage(const AdjArgs& a, const Tables& T, int kdim, cudaStream_t st) {
    int launches = 0;
    if (a.solid_branch && a.ns > 0) {
        const uint32_t nb = nblocks(a.ns * kAdjSolidLanes, kT);
        if (a.st.ep) {
            if (a.all_order2) k_adj_solid<kAdjSolidLanes, false, true><<<nb, kT, 0, st>>>(a, T);
            else k_adj_solid<kAdjSolidLanes, true, true><<<nb, kT, 0, st>>>(a, T);
        } else {
            if (a.all_order2) k_adj_solid<kAdjSolidLanes, false, false><<<nb, kT, 0, st>>>(a, T);
            else k_adj_solid<kAdjSolidLanes, true, false><<<nb, kT, 0, st>>>(a, T);
        }
        k_adj_strain<<<nblocks(a.ns, kT), kT, 0, st>>>(a, T);
        launches += 2;
    }
    if (a.n > 0) {
        k_adj_prep<<<nblocks(a.n, 256), 256, 0, st>>>(a, T, a.w, a.eq);
        if (kdim == 2) k_adj_fluid<2><<<nblocks(a.n, kT), kT, 0, st>>>(a, T, a.w, a.eq);
        else k_adj_fluid<3><<<nblocks(a.n, kT), kT, 0, st>>>(a, T, a.w, a.eq);
        launches += 2;
    }
    return launches;
}

int adjoint_stage_weights(uint32_t n, float cb, const float4* lam_pd, const float4* lam_vm, int nlater,
                          const float* ca, const float4* const* lamY_pd, const float4* const* lamY_vm,
                          float4* mu_pd, float4* mu_vm, cudaStream_t st) {
    if (n == 0) return 0;
    Later L{};
    L.n = nlater < 4 ? nlater : 4;
    for (int t = 0; t < L.n; ++t) {
        L.pd[t] = lamY_pd[t];
        L.vm[t] = lamY_vm[t];
        L.c[t] = ca[t];
    }
    k_adj_weights<<<nblocks(n, 256), 256, 0, st>>>(n, cb, lam_pd, lam_vm, L, mu_pd, mu_vm);
    return 1;
}

int adjoint_step_sum(uint32_t n, const float4* lam_pd, const float4* lam_vm, int stages,
                     const float4* const* lamY_pd, const float4* const* lamY_vm, float4* out_pd, float4* out_vm,
                     cudaStream_t st) {
    if (n == 0) return 0;
    Later L{};
    L.n = stages < 4 ? stages : 4;
    for (int t = 0; t < L.n; ++t) {
        L.pd[t] = lamY_pd[t];
        L.vm[t] = lamY_vm[t];
        L.c[t] = 1.0f;
    }
    k_adj_weights<<<nblocks(n, 256), 256, 0, st>>>(n, 1.0f, lam_pd, lam_vm, L, out_pd, out_vm);
    return 1;
}

int adjoint_stage_weights_all(uint32_t n, float cb, const float4* lam, int nlater, const float* ca,
                              const float4* const* lamY, float4* mu, cudaStream_t st) {
    if (n == 0) return 0;
    Later L{};
    L.n = nlater;
    for (int t = 0; t < nlater; ++t) {
        L.pd[t] = lamY[t];
        L.c[t] = ca[t];
    }
    k_adj_weights_all<<<nblocks(n, 256), 256, 0, st>>>(n, cb, lam, L, mu);
    return 1;
}

int adjoint_step_sum_all(uint32_t n, const float4* lam, int stages, const float4* const* lamY, float4* out,
                         cudaStream_t st) {
    if (n == 0) return 0;
    Later L{};
    L.n = stages;
    for (int t = 0; t < stages; ++t) L.pd[t] = lamY[t];
    k_adj_sum_all<<<nblocks(n, 256), 256, 0, st>>>(n, lam, L, out);
    return 1;
}

int verlet_adjoint_weights(uint32_t n, const float4* lsp, const float4* lsv, const float4* lfp, const float4* lfv,
                           float h, float4* mp, float4* mv, cudaStream_t st) {
    if (n == 0) return 0;
    k_verlet_mu<<<nblocks(n, 256), 256, 0, st>>>(n, lsp, lsv, lfp, lfv, h, mp, mv);
    return 1;
}

int verlet_kick_drift_adjoint(uint32_t n, float4* lp, float4* lv, float h, float dt, float4* lfp, float4* lfv,
                              cudaStream_t st) {
    if (n == 0) return 0;
    k_verlet_kd_adj<<<nblocks(n, 256), 256, 0, st>>>(n, lp, lv, h, dt, lfp, lfv);
    return 1;
}

int adjoint_gather(uint32_t n, const uint32_t* orig, const float4* in_pd, const float4* in_vm, float4* out_pd,
                   float4* out_vm, cudaStream_t st) {
    if (n == 0) return 0;
    k_adj_perm<<<nblocks(n, 256), 256, 0, st>>>(n, orig, in_pd, in_vm, out_pd, out_vm, 0);
    return 1;
}

int adjoint_scatter(uint32_t n, const uint32_t* orig, const float4* in_pd, const float4* in_vm, float4* out_pd,
                    float4* out_vm, cudaStream_t st) {
    if (n == 0) return 0;
    k_adj_perm<<<nblocks(n, 256), 256, 0, st>>>(n, orig, in_pd, in_vm, out_pd, out_vm, 1);
    return 1;
}

namespace {
// The C ABI's state gradients are 8 floats per particle (x, y, z, rho, vx,
// vy, vz, unused); on the device they are two float4 arrays.
__global__ void k_adj_unpack(uint32_t n, const float4* __restrict__ in2, float4* __restrict__ p,
                             float4* __restrict__ v) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    p[i] = in2[2 * i];
    const float4 b = in2[2 * i + 1];
    v[i] = make_float4(b.x, b.y, b.z, 0.0f);
}
__global__ void k_adj_pack(uint32_t n, const float4* __restrict__ p, const float4* __restrict__ v,
                           float4* __restrict__ out2) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    out2[2 * i] = p[i];
    const float4 b = v[i];
    out2[2 * i + 1] = make_float4(b.x, b.y, b.z, 0.0f);
}
}  // namespace

int adjoint_unpack(uint32_t n, const float4* in2, float4* p, float4* v, cudaStream_t st) {
    if (n == 0) return 0;
    k_adj_unpack<<<nblocks(n, 256), 256, 0, st>>>(n, in2, p, v);
    return 1;
}

int adjoint_pack(uint32_t n, const float4* p, const float4* v, float4* out2, cudaStream_t st) {
    if (n == 0) return 0;
    k_adj_pack<<<nblocks(n, 256), 256, 0, st>>>(n, p, v, out2);
    return 1;
}

}  // namespace arp
