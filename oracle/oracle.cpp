// oracle.cpp -- CPU restatement of the reference's SPH time step.
//
// TEST INFRASTRUCTURE ONLY.  This file is the parity oracle for the CUDA
// library: only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
// leg load it, and only as the checker or the timed CPU baseline.  The
// product never links it.
//
// PARITY UNPINNED: the reference (jsmith628/ar-physics) ships no tests, no
// golden vectors and no recorded outputs, and its own path (Rust + OpenGL 4.6
// compute shaders) cannot run on these machines.  This restatement is pinned
// only by analytic known-answer tests (tests/test_oracle.py).
//
// It follows the reference's GLSL shaders line by line:
//   - neighbor buckets: src/soft_body/neighbor_list.rs:37-143 (fill_buckets,
//     reset_buckets) and :224-294 (update_contents), run serially so each
//     bucket section lists ids in ascending order;
//   - poly6 kernel: src/soft_body/kernel.rs:54-96 and norm_const :5-11,:60-63;
//   - fluid forces: src/soft_body/shaders/fluid.rs:45-251, including the
//     81-invocation work split (27 cells x 3 strided lanes) and the ternary
//     shared-memory reduction, so float sums happen in the shader's order;
//   - deformation gradient: src/soft_body/shaders/strain.rs:71-183;
//   - solid forces and plasticity: src/soft_body/shaders/solid.rs:5-37,75-524;
//   - force assembly: src/soft_body/shaders/mod.rs:11-86;
//   - stage arithmetic: src/soft_body/particle_state/particles.rs:8-154;
//   - interaction defaults: src/soft_body/mod.rs:93-111 and
//     src/soft_body/material_region/interaction.rs:42-50.
// The Runge-Kutta tableaus are the textbook ones; the reference takes them
// from the un-vendored crate numerical-integration 0.0.1, so the stage
// combination y0 + sum(c_j k_j) is this project's definition.
//
// Instantiated for float (parity target) and double (error reference).
// Build: see oracle/Makefile (-O3 -fopenmp -ffp-contract=off).

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <type_traits>
#include <vector>

#include <omp.h>

#include "../include/arphys.h"
#include "glsl.hpp"

using namespace glsl;

namespace orc {

constexpr uint32_t INVALID = 0xFFFFFFFFu;
constexpr uint32_t MAXB = 128;  // neighbor_list.rs:45, 4*32 slots per bucket

template <class T> struct Particle {
    T den = 0;
    uint32_t mat = 0, solid_id = INVALID;
    vec4<T> pos, vel;
};
template <class T> struct Solid {
    uint32_t part_id = INVALID;
    vec4<T> ref_pos;
    mat4<T> stress;
};
template <class T> struct Mat {
    bool immobile;
    T mass, start_den;
    uint32_t state_eq;
    T sound_speed, target_den, visc, bulk_visc;
    int strain_order;
    T normal_stiffness, shear_stiffness, normal_damp, shear_damp;
    bool plastic;
    T yield_strength, work_hardening, work_hardening_exp, kinematic_hardening, thermal_softening;
    T relaxation_time;
    bool stiff() const { return normal_stiffness != T(0) || shear_stiffness != T(0); }
};
template <class T> struct Inter {
    uint32_t potential;
    T strength, radius, dampening, friction;
};
struct Bucket {
    uint32_t index[4];
    uint32_t count[3];
    uint32_t contents[MAXB];
};
template <class T> struct State {
    std::vector<Particle<T>> p;
    std::vector<Solid<T>> s;
};
template <class T> struct Strain {
    mat4<T> L, F, Fdot;
};

struct Tableau {
    int stages;
    double a[4][4];
    double b[4];
};

// The integrators the reference names (examples/test.rs:165-180), whose
// tableaus live in the un-vendored numerical-integration 0.0.1 crate: the
// textbook explicit Runge-Kutta tableaus, coefficients in double (rounded to
// float where the step multiplies them by dt).
static bool make_tableau(int id, Tableau& t) {
    std::memset(&t, 0, sizeof(t));
    switch (id) {
        case ARP_INT_EULER: t.stages = 1; t.b[0] = 1; return true;
        case ARP_INT_MIDPOINT: t.stages = 2; t.a[1][0] = 0.5; t.b[1] = 1; return true;
        case ARP_INT_VERLET: t.stages = 1; t.b[0] = 0.5; return true;  // see step_verlet
        case ARP_INT_HEUN2: t.stages = 2; t.a[1][0] = 1; t.b[0] = 0.5; t.b[1] = 0.5; return true;
        case ARP_INT_RALSTON:
            t.stages = 2; t.a[1][0] = 2.0 / 3.0; t.b[0] = 0.25; t.b[1] = 0.75; return true;
        case ARP_INT_RK3:
            t.stages = 3; t.a[1][0] = 0.5; t.a[2][0] = -1; t.a[2][1] = 2;
            t.b[0] = 1.0 / 6.0; t.b[1] = 2.0 / 3.0; t.b[2] = 1.0 / 6.0; return true;
        case ARP_INT_HEUN3:
            t.stages = 3; t.a[1][0] = 1.0 / 3.0; t.a[2][1] = 2.0 / 3.0;
            t.b[0] = 0.25; t.b[2] = 0.75; return true;
        case ARP_INT_RK4:
            t.stages = 4; t.a[1][0] = 0.5; t.a[2][1] = 0.5; t.a[3][2] = 1;
            t.b[0] = 1.0 / 6.0; t.b[1] = 1.0 / 3.0; t.b[2] = 1.0 / 3.0; t.b[3] = 1.0 / 6.0;
            return true;
        case ARP_INT_RK_3_8:
            t.stages = 4; t.a[1][0] = 1.0 / 3.0; t.a[2][0] = -1.0 / 3.0; t.a[2][1] = 1;
            t.a[3][0] = 1; t.a[3][1] = -1; t.a[3][2] = 1;
            t.b[0] = 0.125; t.b[1] = 0.375; t.b[2] = 0.375; t.b[3] = 0.125; return true;
        default: return false;
    }
}

// kernel.rs:5-11 (volume_nball) and :60-63 (poly6 norm_const), evaluated
// left to right in T as the Rust code does in f32.
template <class T> static T volume_nball(uint32_t n, T r) {
    if (n == 0) return T(1);
    if (n == 1) return T(2) * r;
    const T pi = T(3.14159265358979323846);
    return T(2) * pi * r * r * volume_nball<T>(n - 2, r) / T(n);
}
template <class T> static T norm_const(uint32_t n, T h) {
    const T pi = T(3.14159265358979323846);
    return (pi * pi * pi) / (T(6) * volume_nball<T>(n + 6, h));
}

// kernel.rs:81-89: poly6 gradient and value, zero from |r| >= h on
template <class T> static inline vec4<T> grad_w(const vec4<T>& r, T h, T k) {
    T diff = std::max(h * h - dot(r, r), T(0));
    return (T(-6) * k * diff * diff) * r;
}
template <class T> static inline T kernel_w(const vec4<T>& r, T h, T k) {
    T diff = std::max(h * h - dot(r, r), T(0));
    return k * diff * diff * diff;
}

// fluid.rs:45-52
template <class T> static inline T pressure(uint32_t eq, T density, T c, T d0) {
    switch (eq) {
        case ARP_EOS_CONSTANT: return c * c;
        case ARP_EOS_IDEAL_GAS: return c * c * (density - d0);
        case ARP_EOS_TAIT: return (c * c * d0 / T(7)) * (pow7(density / d0) - T(1));
        default: return T(0);
    }
}
// fluid.rs:54-67
template <class T> static inline T contact_potential(uint32_t eq, T r, T strength, T r0) {
    switch (eq) {
        case 1: return r <= r0 ? strength : T(0);
        case 2: return strength * (r0 - r);
        case 3: return (strength * r / T(7)) * (pow7(r0 / r) - T(1));
        case 4: {
            T factor = r0 / r;
            factor *= factor * factor;
            factor *= factor;
            return strength * (factor * factor - T(2) * factor);
        }
        case 5: return (strength * r0 / T(7)) * (pow7(r / r0) - T(1));
        default: return T(0);
    }
}

template <class T> class Sim {
public:
    // configuration
    uint32_t dim = 0;
    T h = 0, kconst = 0, g = 0;
    float hf = 0;
    float bmin[4], bdim[4];
    uint32_t sub[4];
    uint32_t ncells = 0;
    std::vector<Mat<T>> mats;
    std::vector<arp_material> raw_mats;  // the f32 records, for sums the reference takes in f32
    std::vector<Inter<T>> inter;
    uint32_t M = 0;
    std::vector<Particle<T>> boundary;
    State<T> st;
    Tableau tab;
    float dt_sub = 0, timestep = 0;
    uint32_t subticks = 1;
    float time = 0;
    bool literal = false;  // evaluate every candidate pair, no cut-off shortcut
    // velocity Verlet: the derivative record of the last force evaluation
    bool verlet = false;
    State<T> fcarry;
    bool fvalid = false;

    // neighbor buckets (neighbor_list.rs:147-160)
    std::vector<Bucket> buckets;
    std::vector<uint32_t> pos_index, ref_index;
    bool boundary_filled = false;
    bool ref_filled = false;

    std::string init(const arp_scene* sc) {
        if (!sc) return "null scene";
        if (sc->n_materials == 0 || !sc->materials) return "no materials";
        if (!make_tableau(sc->integrator, tab)) return "unsupported integrator";
        verlet = sc->integrator == ARP_INT_VERLET;
        M = sc->n_materials;
        for (uint32_t i = 0; i < M; ++i) {
            const arp_material& m = sc->materials[i];
            raw_mats.push_back(m);
            Mat<T> q;
            q.immobile = m.immobile != 0;
            q.mass = m.mass; q.start_den = m.start_den; q.state_eq = m.state_eq;
            q.sound_speed = m.sound_speed; q.target_den = m.target_den; q.visc = m.visc;
            q.bulk_visc = m.bulk_visc; q.strain_order = m.strain_order;
            q.normal_stiffness = m.normal_stiffness; q.shear_stiffness = m.shear_stiffness;
            q.normal_damp = m.normal_damp; q.shear_damp = m.shear_damp; q.plastic = m.plastic != 0;
            q.yield_strength = m.yield_strength; q.work_hardening = m.work_hardening;
            q.work_hardening_exp = m.work_hardening_exp;
            q.kinematic_hardening = m.kinematic_hardening;
            q.thermal_softening = m.thermal_softening; q.relaxation_time = m.relaxation_time;
            mats.push_back(q);
        }
        // mod.rs:93-111 interaction matrix
        inter.assign(size_t(M) * M, Inter<T>{0, 0, 0, 0, 0});
        auto given = [&](uint32_t i, uint32_t j) -> bool {
            if (!sc->interactions) return false;
            if (!sc->interaction_given) return true;
            return sc->interaction_given[size_t(i) * M + j] != 0;
        };
        auto conv = [&](const arp_interaction& a) {
            return Inter<T>{a.potential, T(a.strength), T(a.radius), T(a.dampening), T(a.friction)};
        };
        for (uint32_t i = 0; i < M; ++i)
            for (uint32_t j = i; j < M; ++j) {
                Inter<T> x{0, 0, 0, 0, 0};
                if (given(i, j)) x = conv(sc->interactions[size_t(i) * M + j]);
                else if (given(j, i)) x = conv(sc->interactions[size_t(j) * M + i]);
                else if (i != j) {
                    const arp_material& m1 = sc->materials[i];
                    const arp_material& m2 = sc->materials[j];
                    if (m1.state_eq != 0 && m2.state_eq != 0) x = Inter<T>{0, 0, 0, 0, 0};
                    else x = Inter<T>{2u, T(10000.0f), T(sc->kernel_radius * 2.0f), T(0),
                                      T(m1.visc + m2.visc)};
                }
                inter[size_t(i) * M + j] = x;
                inter[size_t(j) * M + i] = x;
            }
        dim = 0;
        for (int i = 0; i < 4; ++i) {
            bmin[i] = sc->bounds.min[i];
            bdim[i] = sc->bounds.dim[i];
            if (sc->bounds.dim[i] > 0.0f) dim++;
        }
        hf = sc->kernel_radius;
        h = T(hf);
        kconst = norm_const<T>(dim, h);
        g = T(sc->gravity);
        timestep = sc->timestep;
        subticks = sc->subticks ? sc->subticks : 1;
        dt_sub = timestep / float(subticks);
        ncells = 1;
        for (int i = 0; i < 4; ++i) {
            float q = std::max(1.0f, bdim[i] / hf);
            sub[i] = uint32_t(q);
            ncells *= sub[i];
        }
        buckets.assign(ncells, Bucket{});
        for (uint32_t k = 0; k < sub[2]; ++k)
            for (uint32_t j = 0; j < sub[1]; ++j)
                for (uint32_t i = 0; i < sub[0]; ++i) {
                    Bucket& b = buckets[i + j * sub[0] + k * sub[0] * sub[1]];
                    b.index[0] = i; b.index[1] = j; b.index[2] = k; b.index[3] = 0;
                }
        auto conv_p = [&](const arp_particle& a) {
            Particle<T> p;
            p.den = a.den; p.mat = a.mat; p.solid_id = INVALID;
            for (int c = 0; c < 4; ++c) { p.pos[c] = a.pos[c]; p.vel[c] = a.vel[c]; }
            return p;
        };
        for (uint32_t i = 0; i < sc->n_particles; ++i) {
            if (sc->particles[i].mat >= M) return "particle material out of range";
            st.p.push_back(conv_p(sc->particles[i]));
        }
        for (uint32_t i = 0; i < sc->n_boundary; ++i) {
            if (sc->boundary[i].mat >= M) return "boundary material out of range";
            boundary.push_back(conv_p(sc->boundary[i]));
        }
        // particles.rs:488-506 init_solid_particles
        for (uint32_t i = 0; i < st.p.size(); ++i) {
            if (mats[st.p[i].mat].stiff()) {
                st.p[i].solid_id = uint32_t(st.s.size());
                Solid<T> s;
                s.part_id = i;
                s.ref_pos = st.p[i].pos;
                st.s.push_back(s);
            }
        }
        if (st.s.empty()) st.s.push_back(Solid<T>{});  // dummy entry, part_id INVALID
        pos_index.assign(st.p.size(), INVALID);
        ref_index.assign(st.p.size(), INVALID);
        return "";
    }

    // interaction.rs:42-50 MatInteraction::default_between
    Inter<T> default_between(const arp_material& a, const arp_material& b) const {
        if (a.state_eq != 0 && b.state_eq != 0) return Inter<T>{0, 0, 0, 0, 0};
        return Inter<T>{2u, T(10000.0f), T(hf * 2.0f), T(0), T(a.visc + b.visc)};
    }
    static bool same_material(const arp_material& a, const arp_material& b) {  // derived PartialEq
        return a.immobile == b.immobile && a.mass == b.mass && a.start_den == b.start_den &&
               a.state_eq == b.state_eq && a.sound_speed == b.sound_speed && a.target_den == b.target_den &&
               a.visc == b.visc && a.bulk_visc == b.bulk_visc && a.strain_order == b.strain_order &&
               a.normal_stiffness == b.normal_stiffness && a.shear_stiffness == b.shear_stiffness &&
               a.normal_damp == b.normal_damp && a.shear_damp == b.shear_damp && a.plastic == b.plastic &&
               a.yield_strength == b.yield_strength && a.work_hardening == b.work_hardening &&
               a.work_hardening_exp == b.work_hardening_exp && a.kinematic_hardening == b.kinematic_hardening &&
               a.thermal_softening == b.thermal_softening && a.relaxation_time == b.relaxation_time;
    }

    // mod.rs:180-206 FluidSim::add_particles and particles.rs:547-631
    // Particles::add_particles: the particles (already seeded) are shifted by
    // `offset` in f32, take the first equal material (a solid material is
    // always new), and are appended to the current state; new solids get ids
    // after the existing solid entries (the dummy entry included) and their
    // reference position is their position now.  Returns whether a material
    // was appended.  The reference-configuration buckets are refilled at the
    // next step because the particle count grew (neighbor_list.rs:226-235).
    bool add_particles(const arp_particle* in, uint32_t n, const arp_material& m, const float* offset) {
        if (n == 0) return false;
        fvalid = false;  // a new state: velocity Verlet evaluates its forces again
        const bool stiff = m.normal_stiffness != 0.0f || m.shear_stiffness != 0.0f;
        uint32_t id = M;
        if (!stiff)
            for (uint32_t i = 0; i < M; ++i)
                if (same_material(raw_mats[i], m)) {
                    id = i;
                    break;
                }
        const bool added = id == M;
        if (added) {
            Mat<T> q;
            q.immobile = m.immobile != 0;
            q.mass = m.mass; q.start_den = m.start_den; q.state_eq = m.state_eq;
            q.sound_speed = m.sound_speed; q.target_den = m.target_den; q.visc = m.visc;
            q.bulk_visc = m.bulk_visc; q.strain_order = m.strain_order;
            q.normal_stiffness = m.normal_stiffness; q.shear_stiffness = m.shear_stiffness;
            q.normal_damp = m.normal_damp; q.shear_damp = m.shear_damp; q.plastic = m.plastic != 0;
            q.yield_strength = m.yield_strength; q.work_hardening = m.work_hardening;
            q.work_hardening_exp = m.work_hardening_exp;
            q.kinematic_hardening = m.kinematic_hardening;
            q.thermal_softening = m.thermal_softening; q.relaxation_time = m.relaxation_time;
            mats.push_back(q);
            raw_mats.push_back(m);
            const uint32_t old = M;
            std::vector<Inter<T>> ni;
            for (uint32_t i = 0; i < old; ++i) {
                for (uint32_t j = 0; j < old; ++j) ni.push_back(inter[size_t(i) * old + j]);
                ni.push_back(default_between(raw_mats[i], raw_mats[old]));
            }
            for (uint32_t i = 0; i < old; ++i) ni.push_back(default_between(raw_mats[old], raw_mats[i]));
            ni.push_back(stiff ? Inter<T>{0, 0, 0, 0, 0} : default_between(raw_mats[old], raw_mats[old]));
            inter = ni;
            M = old + 1;
        }
        const uint32_t p_offset = uint32_t(st.p.size());
        for (uint32_t k = 0; k < n; ++k) {
            Particle<T> p;
            p.den = in[k].den;
            p.mat = id;
            p.solid_id = INVALID;
            for (int c = 0; c < 4; ++c) {
                float x = in[k].pos[c];
                if (offset) x += offset[c];
                p.pos[c] = x;
                p.vel[c] = in[k].vel[c];
            }
            if (stiff) {
                p.solid_id = uint32_t(st.s.size());
                Solid<T> s;
                s.part_id = p_offset + k;
                s.ref_pos = p.pos;
                st.s.push_back(s);
            }
            st.p.push_back(p);
        }
        pos_index.assign(st.p.size(), INVALID);
        ref_index.assign(st.p.size(), INVALID);
        ref_filled = false;
        return added;
    }

    uint32_t n_solids() const {
        return (st.s.size() == 1 && st.s[0].part_id == INVALID) ? 0u : uint32_t(st.s.size());
    }

    // neighbor_list.rs:95, with an axis of zero extent mapped to cell 0 and a
    // coordinate on the upper face clamped into the last cell.
    uint32_t cell_coord(float p, int a) const {
        if (bdim[a] == 0.0f) return 0;
        float t = (p - bmin[a]) / bdim[a];
        t = std::min(std::max(t, 0.0f), 1.0f);
        uint32_t c = uint32_t(std::floor(t * float(sub[a])));
        if (c >= sub[a]) c = sub[a] - 1;
        return c;
    }
    uint32_t bucket_of(const vec4<T>& pos) const {
        float p[4] = {float(pos[0]), float(pos[1]), float(pos[2]), float(pos[3])};
        return cell_coord(p[0], 0) + cell_coord(p[1], 1) * sub[0] +
               cell_coord(p[2], 2) * sub[0] * sub[1];
    }
    static bool nonfinite(const vec4<T>& v) {
        for (int i = 0; i < 4; ++i)
            if (!std::isfinite(double(v[i]))) return true;
        return false;
    }

    // neighbor_list.rs:115-143 reset_buckets
    void reset_buckets(uint32_t mode) {
        for (auto& b : buckets)
            for (uint32_t i = mode; i < 3; ++i) b.count[i] = 0;
    }
    // neighbor_list.rs:74-111 fill_buckets, serial in id order
    void fill_buckets(uint32_t mode, const std::vector<Particle<T>>& parts,
                      const std::vector<Solid<T>>& solids) {
        for (uint32_t id = 0; id < parts.size(); ++id) {
            uint32_t s_id = parts[id].solid_id;
            if (mode == 1 && s_id == INVALID) { ref_index[id] = INVALID; continue; }
            const vec4<T>& pos = mode == 1 ? solids[s_id].ref_pos : parts[id].pos;
            if (nonfinite(pos)) {
                if (mode == 2) pos_index[id] = INVALID;
                else if (mode == 1) ref_index[id] = INVALID;
                continue;
            }
            uint32_t bucket_id = bucket_of(pos);
            Bucket& b = buckets[bucket_id];
            uint32_t start = 0;
            for (uint32_t i = 0; i < mode; ++i) start += b.count[i];
            uint32_t spot = start + b.count[mode]++;
            if (spot < MAXB) {
                if (mode == 2) pos_index[id] = bucket_id;
                if (mode == 1) ref_index[id] = bucket_id;
                b.contents[spot] = id;
            } else {
                if (mode == 2) pos_index[id] = INVALID;
                if (mode == 1) ref_index[id] = INVALID;
                b.count[mode] = std::min(b.count[mode], MAXB - start);
            }
        }
    }
    // neighbor_list.rs:224-294 update_contents
    void update_contents(const State<T>& y) {
        if (!boundary_filled) {
            reset_buckets(0);
            fill_buckets(0, boundary, y.s);
            boundary_filled = true;
        }
        if (!ref_filled) {
            reset_buckets(1);
            fill_buckets(1, y.p, y.s);
            ref_filled = true;
        } else {
            reset_buckets(2);
        }
        fill_buckets(2, y.p, y.s);
    }

    bool in_bounds(const int b[3]) const {
        return b[0] >= 0 && b[1] >= 0 && b[2] >= 0 && b[0] < int(sub[0]) && b[1] < int(sub[1]) &&
               b[2] < int(sub[2]);
    }
    uint32_t bucket_index(const int b[3]) const {
        return uint32_t(b[0]) + uint32_t(b[1]) * sub[0] + uint32_t(b[2]) * sub[0] * sub[1];
    }
    // local_bucket_pos (fluid.rs:89-93) for invocation gid of a 9x3x3 group
    bool local_bucket(uint32_t bucket, uint32_t gid, int out[3]) const {
        if (bucket == INVALID) return false;
        uint32_t lx = gid % 9, ly = (gid / 9) % 3, lz = gid / 27;
        const Bucket& b = buckets[bucket];
        out[0] = int(b.index[0]) + int(lx % 3) - 1;
        out[1] = int(b.index[1]) + int(ly) - 1;
        out[2] = int(b.index[2]) + int(lz) - 1;
        return in_bounds(out);
    }
    uint32_t mobile_solid_id(uint32_t idx, const std::vector<Particle<T>>& p) const {
        return idx < p.size() ? p[idx].solid_id : INVALID;  // Q2: boundary index read from the mobile array
    }

    // ternary reduction of the 81 shared slots (fluid.rs:226-241)
    template <class V> static V reduce81(std::vector<V>& s) {
        uint32_t shadow = 81;
        while (shadow % 3 == 0) {
            shadow /= 3;
            for (uint32_t gid = 0; gid < shadow; ++gid) s[gid] = s[gid] + (s[gid + shadow] + s[gid + shadow * 2]);
        }
        for (uint32_t i = 1; i < shadow; ++i) s[0] = s[0] + s[i];
        return s[0];
    }

    // fluid.rs:95-251
    void fluid_forces(const State<T>& y, std::vector<Particle<T>>& out) const {
        const auto& P = y.p;
        const T hh_eps = T(0.1f) * h * h;
        out.resize(P.size());
#pragma omp parallel for schedule(dynamic, 64)
        for (long long pl = 0; pl < (long long)P.size(); ++pl) {
            const uint32_t p_id = uint32_t(pl);
            const uint32_t s_id = P[p_id].solid_id;
            const uint32_t mat_id = P[p_id].mat;
            const Mat<T>& m1m = mats[mat_id];
            const T m1 = m1m.mass;
            const T d1 = P[p_id].den;
            const bool elastic = s_id != INVALID && m1m.stiff();
            std::vector<T> sden(81, T(0));
            std::vector<vec4<T>> sforce(81);
            for (uint32_t gid = 0; gid < 81; ++gid) {
                T den = 0;
                vec4<T> force;
                const uint32_t sublocal_id = (gid % 9) / 3;
                int bp[3];
                if (local_bucket(pos_index[p_id], gid, bp)) {
                    const uint32_t state_eq = m1m.state_eq;
                    const T c1 = m1m.sound_speed, f1 = m1m.visc, bf1 = m1m.bulk_visc, d0 = m1m.target_den;
                    const T p1 = pressure(state_eq, d1, c1, d0);
                    const uint32_t bucket_id = bucket_index(bp);
                    const Bucket& B = buckets[bucket_id];
                    const uint32_t bc = B.count[0], ref_count = B.count[1], count = B.count[2];
                    for (uint32_t j = sublocal_id; j < count + ref_count + bc; j += 3) {
                        if (j >= bc && j < ref_count + bc) continue;
                        const uint32_t p_id2 = B.contents[j];
                        const uint32_t s_id2 = mobile_solid_id(p_id2, P);
                        const Particle<T>& q = j < bc ? boundary[p_id2] : P[p_id2];
                        const uint32_t mat_2 = q.mat;
                        const Mat<T>& m2m = mats[mat_2];
                        const T m2 = m2m.mass, f2 = m2m.visc, bf2 = m2m.bulk_visc, c2 = m2m.sound_speed;
                        const vec4<T> r = q.pos - P[p_id].pos;
                        const vec4<T> v = q.vel - P[p_id].vel;
                        const T d2 = q.den;
                        if (!literal && !(h * h - dot(r, r) > T(0))) continue;  // every term carries grad_w == 0
                        const T p2 = pressure(m2m.state_eq, d2, c2, m2m.target_den);
                        const vec4<T> gw = grad_w(r, h, kconst);
                        if (j >= bc) den += m2 * dot(v, gw);
                        vec4<T> contact_force;
                        const bool elastic2 = s_id2 != INVALID && m2m.stiff();
                        const Inter<T>& it = inter[size_t(mat_id) * M + mat_2];
                        const T contact_pressure = contact_potential(it.potential, length(r), it.radius, it.strength);
                        force += (m1 * m2 * (p1 / (d1 * d1) + p2 / (d2 * d2))) * gw;
                        if (contact_pressure != T(0)) {
                            contact_force += (m2 * contact_pressure / d2) * gw;
                            if ((elastic || elastic2 || j < bc) && mat_id != mat_2) {
                                const vec4<T> r_inv = r / dot(r, r);
                                const vec4<T> normal_force = r_inv * dot(contact_force, r);
                                vec4<T> tangent_vel = v - r_inv * dot(v, r);
                                tangent_vel = normalize(tangent_vel);
                                if (!any_nan_or_inf(tangent_vel))
                                    force += (it.friction * length(normal_force)) * normalize(tangent_vel);
                            }
                            force += contact_force;
                        }
                        if (!elastic && j >= bc)
                            force -= ((m1 * m2 * (f1 + f2) * dot(r, gw)) * v) / (d1 * d2 * (dot(r, r) + hh_eps));
                        if (j >= bc) {
                            const T f_ = mat_id == mat_2 ? bf1 + bf2 : it.dampening;
                            force -= (m1 * m2 * ((f_ * dot(v, r)) / ((d1 + d2) * (dot(r, r) + hh_eps)))) * gw;
                        }
                    }
                }
                sden[gid] = den;
                sforce[gid] = force;
            }
            const T den_sum = reduce81(sden);
            const vec4<T> f_sum = reduce81(sforce);
            Particle<T>& o = out[p_id];
            o.mat = mat_id;
            o.solid_id = s_id;
            o.den = den_sum;
            o.vel = f_sum / P[p_id].den + vec4<T>(0, -g, 0, 0);
            o.pos = P[p_id].vel;
        }
    }

    bool is_elastic(uint32_t id, const std::vector<Particle<T>>& P) const { return mats[P[id].mat].stiff(); }

    // strain.rs:71-183
    void compute_strain(const State<T>& y, std::vector<Strain<T>>& strains) const {
        const auto& P = y.p;
        const auto& S = y.s;
        strains.assign(S.size(), Strain<T>{});
#pragma omp parallel for schedule(dynamic, 64)
        for (long long sl = 0; sl < (long long)S.size(); ++sl) {
            const uint32_t s_id = uint32_t(sl);
            const uint32_t p_id = S[s_id].part_id;
            if (p_id == INVALID) continue;
            if (!is_elastic(p_id, P)) continue;
            std::vector<mat4<T>> corr(81), def(81), rate(81);
            for (uint32_t gid = 0; gid < 81; ++gid) {
                const uint32_t sublocal_id = (gid % 9) / 3;
                int bp[3];
                if (local_bucket(ref_index[p_id], gid, bp)) {
                    const Bucket& B = buckets[bucket_index(bp)];
                    const uint32_t start = B.count[0], end = start + B.count[1];
                    for (uint32_t i = start + sublocal_id; i < end; i += 3) {
                        const uint32_t p_id2 = B.contents[i];
                        const uint32_t s_id2 = P[p_id2].solid_id;
                        if (p_id2 == INVALID || s_id2 == INVALID) continue;
                        if (is_elastic(p_id2, P)) {
                            const Mat<T>& m2 = mats[P[p_id2].mat];
                            const T V2 = m2.mass / m2.start_den;
                            const vec4<T> dX = S[s_id2].ref_pos - S[s_id].ref_pos;
                            corr[gid] += V2 * outerProduct(grad_w(dX, h, kconst), dX);
                        }
                    }
                }
            }
            mat4<T> L = reduce81(corr);
            for (uint32_t i = dim; i < 4; ++i) L[i][i] = T(1);
            L = inverse(L);
            for (uint32_t gid = 0; gid < 81; ++gid) {
                const uint32_t sublocal_id = (gid % 9) / 3;
                int bp[3];
                if (local_bucket(ref_index[p_id], gid, bp)) {
                    const Bucket& B = buckets[bucket_index(bp)];
                    const uint32_t start = B.count[0], end = start + B.count[1];
                    for (uint32_t i = start + sublocal_id; i < end; i += 3) {
                        const uint32_t p_id2 = B.contents[i];
                        const uint32_t s_id2 = P[p_id2].solid_id;
                        if (p_id2 == INVALID || s_id2 == INVALID) continue;
                        if (!is_elastic(p_id2, P)) continue;
                        const Mat<T>& m2 = mats[P[p_id2].mat];
                        const T V2 = m2.mass / m2.start_den;
                        const vec4<T> dX = S[s_id2].ref_pos - S[s_id].ref_pos;
                        const vec4<T> dx = P[p_id2].pos - P[p_id].pos;
                        const vec4<T> dv = P[p_id2].vel - P[p_id].vel;
                        const vec4<T> grad = L * grad_w(dX, h, kconst);
                        def[gid] += V2 * outerProduct(dx, grad);
                        rate[gid] += V2 * outerProduct(dv, grad);
                    }
                }
            }
            strains[s_id].L = L;
            strains[s_id].F = reduce81(def);
            strains[s_id].Fdot = reduce81(rate);
        }
    }

    // solid.rs:75-246 helpers
    T trace(const mat4<T>& A) const {
        T t = A[0][0];
        for (uint32_t i = 1; i < dim; ++i) t += A[i][i];
        return t;
    }
    static mat4<T> mat_log(const mat4<T>& A) {
        mat4<T> sum;
        mat4<T> term = -identity<T>();
        for (uint32_t i = 1; i <= 5; ++i) {
            term *= T(-1) * (A - identity<T>());
            sum += term / T(i);
        }
        return sum;
    }
    static void mat_sqrt(const mat4<T>& X, mat4<T>& sq, mat4<T>& inv_sq) {
        mat4<T> Yi = X, Zi = identity<T>();
        for (int i = 0; i < 15; ++i) {
            mat4<T> Y = T(0.5) * (Yi + inverse(Zi));
            mat4<T> Z = T(0.5) * (Zi + inverse(Yi));
            Yi = Y;
            Zi = Z;
        }
        sq = Yi;
        inv_sq = Zi;
    }
    static T mat_dot(const mat4<T>& x, const mat4<T>& y) {
        return ((dot(x[0], y[0]) + dot(x[1], y[1])) + dot(x[2], y[2])) + dot(x[3], y[3]);
    }
    mat4<T> hooke(const mat4<T>& strain, T normal, T shear) const {
        return (normal * trace(strain)) * identity<T>() + (T(2) * shear) * strain;
    }
    mat4<T> seth_hill(const mat4<T>& def, int two_m) const {
        mat4<T> C = transpose(def) * def;
        for (uint32_t i = dim; i < 4; ++i) C[i][i] = T(1);
        if (two_m == 0) return T(0.5) * mat_log(C);
        const uint32_t m = uint32_t(std::abs(two_m)) >> 1;
        mat4<T> C_m = identity<T>();
        for (uint32_t i = 0; i < m; ++i) C_m *= C;
        if ((std::abs(two_m) & 1) == 1) {
            mat4<T> s, inv;
            mat_sqrt(C, s, inv);
            C_m *= s;
        }
        if (two_m < 0) C_m = inverse(C_m);
        return (T(1) / T(two_m)) * (C_m - identity<T>());
    }
    mat4<T> seth_hill_rate(const mat4<T>& def, const mat4<T>& def_rate, int two_m) const {
        mat4<T> dC = transpose(def_rate) * def;
        dC = dC + transpose(dC);
        mat4<T> C = transpose(def) * def;
        for (uint32_t i = dim; i < 4; ++i) C[i][i] = T(1);
        if (two_m == 0) return (T(0.5) * dC) * inverse(C);
        const uint32_t m = uint32_t(std::abs(two_m)) >> 1;
        mat4<T> strain_rate;
        for (uint32_t i = 0; i < m; ++i) {
            mat4<T> term = identity<T>();
            for (uint32_t j = 0; j < m; ++j) term *= (j == i ? dC : C);
            strain_rate += term;
        }
        strain_rate = (T(1) / T(two_m)) * strain_rate;
        if (two_m < 0) {
            mat4<T> inv_C = inverse(C);
            return ((-inv_C) * strain_rate) * inv_C;
        }
        return strain_rate;
    }
    // integer (dim-1)/dim as the shader writes it (solid.rs:212-215)
    T eq_plastic_strain_sq(const mat4<T>& strain) const {
        mat4<T> dev = strain - (trace(strain) * identity<T>()) / T(int(dim));
        return T(int(dim - 1) / int(dim)) * mat_dot(dev, dev);
    }
    // per-solid (normal, shear) stiffness overriding the material's (empty: none)
    std::vector<T> solid_stiff;
    mat4<T> pk2_of(const mat4<T>& def, const mat4<T>& def_rate, const mat4<T>& plastic, const Mat<T>& m,
                   uint32_t s_id) const {
        mat4<T> strain = seth_hill(def, m.strain_order) + plastic;
        mat4<T> rate = seth_hill_rate(def, def_rate, m.strain_order);
        const bool own = 2 * size_t(s_id) + 1 < solid_stiff.size();
        const T n = own ? solid_stiff[2 * s_id] : m.normal_stiffness;
        const T sh = own ? solid_stiff[2 * s_id + 1] : m.shear_stiffness;
        return hooke(strain, n, sh) + hooke(rate, m.normal_damp, m.shear_damp);
    }

    // solid.rs:276-524
    void solid_forces(const State<T>& y, const std::vector<Strain<T>>& strains,
                      std::vector<Particle<T>>& outp, std::vector<Solid<T>>& outs) const {
        const auto& P = y.p;
        const auto& S = y.s;
        const T eps = T(0.1f);
        outp.assign(P.size(), Particle<T>{});
#pragma omp parallel for schedule(dynamic, 64)
        for (long long pl = 0; pl < (long long)P.size(); ++pl) {
            const uint32_t p_id = uint32_t(pl);
            const uint32_t s_id = P[p_id].solid_id;
            const uint32_t mat_id = P[p_id].mat;
            Particle<T>& o = outp[p_id];
            o.mat = mat_id;
            o.solid_id = s_id;
            o.den = 0;
            o.pos = vec4<T>();
            o.vel = vec4<T>();
            if (s_id == INVALID) continue;
            outs[s_id].part_id = p_id;
            outs[s_id].ref_pos = vec4<T>();
            outs[s_id].stress = mat4<T>();
            const Mat<T>& mm = mats[mat_id];
            const T m1 = mm.mass;
            const T d1 = P[p_id].den;
            const bool elastic = mm.stiff();
            if (!elastic) continue;
            const mat4<T>& def = strains[s_id].F;
            const mat4<T> pk2 = pk2_of(def, strains[s_id].Fdot, S[s_id].stress, mm, s_id);
            const mat4<T> stress = def * transpose(pk2);
            std::vector<vec4<T>> sforce(81);
            for (uint32_t gid = 0; gid < 81; ++gid) {
                vec4<T> force;
                const uint32_t sublocal_id = (gid % 9) / 3;
                int bp[3];
                if (local_bucket(ref_index[p_id], gid, bp)) {
                    const mat4<T>& correction = strains[s_id].L;
                    const T V1 = m1 / d1;
                    const Bucket& B = buckets[bucket_index(bp)];
                    const uint32_t start = B.count[0], ref_count = B.count[1];
                    for (uint32_t j = start + sublocal_id; j < start + ref_count; j += 3) {
                        const uint32_t p_id2 = B.contents[j];
                        const uint32_t s_id2 = P[p_id2].solid_id;
                        if (P[p_id2].mat != mat_id) continue;
                        if (p_id2 == INVALID || s_id2 == INVALID) continue;
                        const vec4<T> r = S[s_id2].ref_pos - S[s_id].ref_pos;
                        if (!literal && !(h * h - dot(r, r) > T(0))) continue;  // grad_w == 0
                        const T V2 = m1 / P[p_id2].den;
                        const mat4<T>& def2 = strains[s_id2].F;
                        const mat4<T> pk2b = pk2_of(def2, strains[s_id2].Fdot, S[s_id2].stress, mm, s_id2);
                        const mat4<T> stress2 = def2 * transpose(pk2b);
                        vec4<T> el_force =
                            ((-V1 * V2) * (stress * correction + stress2 * strains[s_id2].L)) * grad_w(r, h, kconst);
                        for (uint32_t k = dim; k < 4; ++k) el_force[k] = T(0);
                        force += el_force;
                    }
                }
                if (local_bucket(pos_index[p_id], gid, bp)) {
                    const Bucket& B = buckets[bucket_index(bp)];
                    const uint32_t bc = B.count[0], ref_count = B.count[1], count = B.count[2];
                    for (uint32_t j = sublocal_id; j < count + ref_count + bc; j += 3) {
                        if (j >= bc && j < ref_count + bc) continue;
                        const uint32_t p_id2 = B.contents[j];
                        const uint32_t s_id2 = mobile_solid_id(p_id2, P);
                        const Particle<T>& q = j < bc ? boundary[p_id2] : P[p_id2];
                        const uint32_t mat_2 = q.mat;
                        if (p_id2 == INVALID || s_id2 == INVALID) continue;
                        const Mat<T>& m2m = mats[mat_2];
                        const T m2 = m2m.mass;
                        const vec4<T> r = q.pos - P[p_id].pos;
                        const T d2 = j < bc ? q.den + d1 : q.den;
                        vec4<T> contact_force;
                        const bool elastic2 = m2m.stiff();
                        const vec4<T> dx = r;
                        const vec4<T> dX = S[s_id2].ref_pos - S[s_id].ref_pos;
                        const T contact = h;
                        const T r_cut = T(8) * contact;
                        const bool in_contact =
                            (!elastic || !elastic2 || dot(dX, dX) > (r_cut * r_cut)) && dot(dx, dx) < r_cut * r_cut;
                        if (mat_id == mat_2 || in_contact) {
                            const T l = length(dx);
                            if (mat_id == mat_2) {
                                const mat4<T>& F1 = strains[s_id].F;
                                const mat4<T>& F2 = strains[s_id2].F;
                                const vec4<T> err = (T(0.5) * (F1 + F2)) * dX - dx;
                                const T s = (((T(100000000) * m1 * m2 / (d1 * d2)) *
                                               (T(0.5) * dot(err, dx) / (l + T(10) * eps * h))) *
                                              (T(1) / (l * l + eps * h * h))) *
                                             kernel_w(dX, h, kconst);
                                force -= (s * dx) / (l + eps * h);
                            }
                            if (mat_id == mat_2 && in_contact && !mm.plastic) {
                                const T r_geom = contact * contact / r_cut;
                                const T dr = std::max(r_cut - l, T(0));
                                contact_force = (T(-5000) * std::sqrt(dr * r_geom)) * r / l;
                                force += contact_force;
                            }
                        }
                        // solid.rs:455-461: friction block with its force line commented out
                    }
                }
                sforce[gid] = force;
            }
            const vec4<T> f_sum = reduce81(sforce);
            o.den = 0;
            o.vel = f_sum / P[p_id].den + vec4<T>(0, -g, 0, 0);
            o.pos = P[p_id].vel;
            if (mm.plastic) {
                const T A = mm.yield_strength, Bh = mm.work_hardening, C = mm.kinematic_hardening;
                const T n = mm.work_hardening_exp, Tr = mm.relaxation_time;
                const T eq_strain = eq_plastic_strain_sq(S[s_id].stress);
                T stress_norm = mat_dot(pk2, pk2);
                const T yield_stress = (A + Bh * std::pow(eq_strain, n / T(2))) * (T(1) + C * std::log(T(1)));
                if (yield_stress * yield_stress <= stress_norm) {
                    stress_norm = std::sqrt(stress_norm);
                    outs[s_id].stress = ((stress_norm - yield_stress) / Tr) * (pk2 / stress_norm);
                }
            }
        }
    }

    // shaders/mod.rs:11-86; the two derivative terms are summed field by field
    void compute_forces(const State<T>& y, State<T>& d) {
        update_contents(y);
        fluid_forces(y, d.p);
        d.s.resize(y.s.size());
        for (size_t i = 0; i < y.s.size(); ++i) {  // solid.rs:26-33 clear_solids
            d.s[i].part_id = y.s[i].part_id;
            d.s[i].ref_pos = vec4<T>();
            d.s[i].stress = mat4<T>();
        }
        if (y.s.size() > 1) {
            std::vector<Strain<T>> strains;
            compute_strain(y, strains);
            std::vector<Particle<T>> p2;
            std::vector<Solid<T>> s2(y.s.size());
            for (size_t i = 0; i < y.s.size(); ++i) s2[i].part_id = y.s[i].part_id;
            solid_forces(y, strains, p2, s2);
            for (size_t i = 0; i < d.p.size(); ++i) {
                d.p[i].den = d.p[i].den + p2[i].den;
                d.p[i].pos = d.p[i].pos + p2[i].pos;
                d.p[i].vel = d.p[i].vel + p2[i].vel;
            }
            for (size_t i = 0; i < d.s.size(); ++i) {
                d.s[i].ref_pos = d.s[i].ref_pos + s2[i].ref_pos;
                d.s[i].stress = d.s[i].stress + s2[i].stress;
            }
        }
    }

    T coef(double a) const {
        if (sizeof(T) == sizeof(float)) return T(float(a * double(dt_sub)));
        return T(a * double(dt_sub));
    }

    // y = y0 + (sum_j c_j k_j), sum in j order
    void combine(const State<T>& y0, const std::vector<State<T>>& ks, const double* a, int n, State<T>& y) const {
        y = y0;
        const size_t np = y0.p.size(), ns = y0.s.size();
        std::vector<T> c(n);
        for (int j = 0; j < n; ++j) c[j] = coef(a[j]);
#pragma omp parallel for schedule(static)
        for (long long i = 0; i < (long long)np; ++i) {
            T den = 0;
            vec4<T> pos, vel;
            for (int j = 0; j < n; ++j) {
                if (a[j] == 0.0) continue;
                den = den + c[j] * ks[j].p[i].den;
                pos = pos + c[j] * ks[j].p[i].pos;
                vel = vel + c[j] * ks[j].p[i].vel;
            }
            y.p[i].den = y0.p[i].den + den;
            y.p[i].pos = y0.p[i].pos + pos;
            y.p[i].vel = y0.p[i].vel + vel;
        }
        for (size_t i = 0; i < ns; ++i) {
            vec4<T> rp;
            mat4<T> sp;
            for (int j = 0; j < n; ++j) {
                if (a[j] == 0.0) continue;
                rp = rp + c[j] * ks[j].s[i].ref_pos;
                sp = sp + c[j] * ks[j].s[i].stress;
            }
            y.s[i].ref_pos = y0.s[i].ref_pos + rp;
            y.s[i].stress = y0.s[i].stress + sp;
        }
    }

    // Velocity Verlet as the textbook kick-drift-kick over the force closure's
    // derivative record f (the velocity closure state.velocity() of
    // src/soft_body/mod.rs:256 moves the positions, so f's position part is
    // not used); f at the initial state comes from the force evaluation of
    // init_with_vel (src/soft_body/mod.rs:213-233).  The scheme inside the
    // un-vendored numerical-integration crate is not observable: this is the
    // stated assumption the library implements too.  Sums are formed as
    // y + (0 + c k), the order combine() uses.
    void step_verlet() {
        time += dt_sub;
        if (!fvalid) {
            compute_forces(st, fcarry);
            fvalid = true;
        }
        const T half = coef(0.5), full = coef(1.0);
        State<T> y = st;
        const size_t np = st.p.size(), ns = st.s.size();
        for (size_t i = 0; i < np; ++i) {
            T z = 0;
            vec4<T> zv;
            y.p[i].den = st.p[i].den + (z + half * fcarry.p[i].den);
            y.p[i].vel = st.p[i].vel + (zv + half * fcarry.p[i].vel);
            y.p[i].pos = st.p[i].pos + (zv + full * y.p[i].vel);
        }
        for (size_t i = 0; i < ns; ++i) {
            mat4<T> zm;
            y.s[i].stress = st.s[i].stress + (zm + half * fcarry.s[i].stress);
        }
        State<T> f;
        compute_forces(y, f);
        for (size_t i = 0; i < np; ++i) {
            T z = 0;
            vec4<T> zv;
            y.p[i].den = y.p[i].den + (z + half * f.p[i].den);
            y.p[i].vel = y.p[i].vel + (zv + half * f.p[i].vel);
        }
        for (size_t i = 0; i < ns; ++i) {
            mat4<T> zm;
            y.s[i].stress = y.s[i].stress + (zm + half * f.s[i].stress);
        }
        st = std::move(y);
        fcarry = std::move(f);
    }

    // One integrator step of y' = f(y) (mod.rs:252-265 through the crate's
    // step_with_vel): stage states y0 + sum_j (a_sj dt) k_j, the result
    // y0 + sum_j (b_j dt) k_j, sums in stage order.
    void step() {
        if (verlet) {
            step_verlet();
            return;
        }
        time += dt_sub;
        std::vector<State<T>> ks(tab.stages);
        State<T> y;
        for (int s = 0; s < tab.stages; ++s) {
            if (s == 0) compute_forces(st, ks[0]);
            else {
                combine(st, ks, tab.a[s], s, y);
                compute_forces(y, ks[s]);
            }
        }
        State<T> ynew;
        combine(st, ks, tab.b, tab.stages, ynew);
        st = std::move(ynew);
    }
};

struct Handle {
    int precision;
    std::unique_ptr<Sim<float>> f;
    std::unique_ptr<Sim<double>> d;
};

}  // namespace orc

using namespace orc;

template <class F> static void dispatch(void* h, F&& f) {
    Handle* H = static_cast<Handle*>(h);
    if (H->precision == 64) f(*H->d);
    else f(*H->f);
}

extern "C" {

void* orc_create(const arp_scene* sc, int precision, int literal, char* err, int errlen) {
    auto h = new Handle();
    h->precision = precision;
    std::string e;
    if (precision == 64) {
        h->d.reset(new Sim<double>());
        h->d->literal = literal != 0;
        e = h->d->init(sc);
    } else {
        h->f.reset(new Sim<float>());
        h->f->literal = literal != 0;
        e = h->f->init(sc);
    }
    if (!e.empty()) {
        if (err && errlen > 0) std::snprintf(err, size_t(errlen), "%s", e.c_str());
        delete h;
        return nullptr;
    }
    return h;
}

void orc_destroy(void* p) { delete static_cast<Handle*>(p); }

void orc_set_threads(int n) { omp_set_num_threads(n > 0 ? n : 1); }
int orc_get_threads(void) { return omp_get_max_threads(); }

int orc_step(void* h, uint32_t n) {
    dispatch(h, [&](auto& S) { for (uint32_t i = 0; i < n; ++i) S.step(); });
    return 0;
}

int orc_update(void* h) {
    dispatch(h, [&](auto& S) { for (uint32_t i = 0; i < S.subticks; ++i) S.step(); });
    return 0;
}

double orc_time(void* h) {
    double t = 0;
    dispatch(h, [&](auto& S) { t = S.time; });
    return t;
}

int orc_counts(void* h, uint32_t* n, uint32_t* nb, uint32_t* ns, uint32_t* ncells, uint32_t* sub4, uint32_t* dim) {
    dispatch(h, [&](auto& S) {
        if (n) *n = uint32_t(S.st.p.size());
        if (nb) *nb = uint32_t(S.boundary.size());
        if (ns) *ns = S.n_solids();
        if (ncells) *ncells = S.ncells;
        if (sub4) for (int i = 0; i < 4; ++i) sub4[i] = S.sub[i];
        if (dim) *dim = S.dim;
    });
    return 0;
}

// Current state as float64 arrays (any pointer may be NULL).
int orc_get_state(void* h, double* den, double* pos, double* vel, uint32_t* mat, uint32_t* solid_id,
                  double* ref_pos, double* plastic) {
    dispatch(h, [&](auto& S) {
        const auto& P = S.st.p;
        for (size_t i = 0; i < P.size(); ++i) {
            if (den) den[i] = double(P[i].den);
            for (int c = 0; c < 4; ++c) {
                if (pos) pos[4 * i + c] = double(P[i].pos[c]);
                if (vel) vel[4 * i + c] = double(P[i].vel[c]);
            }
            if (mat) mat[i] = P[i].mat;
            if (solid_id) solid_id[i] = P[i].solid_id;
        }
        const uint32_t ns = S.n_solids();
        for (uint32_t s = 0; s < ns; ++s) {
            for (int c = 0; c < 4; ++c)
                if (ref_pos) ref_pos[4 * s + c] = double(S.st.s[s].ref_pos[c]);
            for (int c = 0; c < 4; ++c)
                for (int r = 0; r < 4; ++r)
                    if (plastic) plastic[16 * s + 4 * c + r] = double(S.st.s[s].stress[c][r]);
        }
    });
    return 0;
}

int orc_add_particles(void* h, const arp_particle* p, uint32_t n, const arp_material* m, const float* offset,
                      int* material_added) {
    if (!m || (n && !p)) return 1;
    bool added = false;
    dispatch(h, [&](auto& S) { added = S.add_particles(p, n, *m, offset); });
    if (material_added) *material_added = added ? 1 : 0;
    return 0;
}

// Per-solid (normal, shear) stiffness, 2 values per solid id (NULL clears).
int orc_set_solid_stiffness(void* h, const double* normal_shear, uint32_t ns) {
    dispatch(h, [&](auto& S) {
        using TT = std::remove_reference_t<decltype(S.h)>;
        S.solid_stiff.clear();
        if (normal_shear)
            for (uint32_t i = 0; i < 2 * ns; ++i) S.solid_stiff.push_back(TT(normal_shear[i]));
    });
    return 0;
}

int orc_materials(void* h, uint32_t* count, arp_material* out, uint32_t cap) {
    dispatch(h, [&](auto& S) {
        if (count) *count = S.M;
        for (uint32_t i = 0; i < S.M && i < cap && out; ++i) out[i] = S.raw_mats[i];
    });
    return 0;
}

int orc_interactions(void* h, double* out) {  // M x M x (potential, strength, radius, dampening, friction)
    dispatch(h, [&](auto& S) {
        for (size_t i = 0; i < S.inter.size(); ++i) {
            out[5 * i + 0] = double(S.inter[i].potential);
            out[5 * i + 1] = double(S.inter[i].strength);
            out[5 * i + 2] = double(S.inter[i].radius);
            out[5 * i + 3] = double(S.inter[i].dampening);
            out[5 * i + 4] = double(S.inter[i].friction);
        }
    });
    return 0;
}

// Overwrite den/pos/vel (and plastic strain when given) of the current state.
int orc_set_state(void* h, const double* den, const double* pos, const double* vel, const double* plastic) {
    dispatch(h, [&](auto& S) {
        using TT = std::remove_reference_t<decltype(S.st.p[0].den)>;
        auto& P = S.st.p;
        S.fvalid = false;
        for (size_t i = 0; i < P.size(); ++i) {
            if (den) P[i].den = TT(den[i]);
            for (int c = 0; c < 4; ++c) {
                if (pos) P[i].pos[c] = TT(pos[4 * i + c]);
                if (vel) P[i].vel[c] = TT(vel[4 * i + c]);
            }
        }
        const uint32_t ns = S.n_solids();
        if (plastic)
            for (uint32_t s = 0; s < ns; ++s)
                for (int c = 0; c < 4; ++c)
                    for (int r = 0; r < 4; ++r) S.st.s[s].stress[c][r] = TT(plastic[16 * s + 4 * c + r]);
    });
    return 0;
}

// compute_forces of the current state: the summed derivative record.
int orc_derivative(void* h, double* dden, double* dpos, double* dvel, double* dplastic) {
    dispatch(h, [&](auto& S) {
        using St = std::remove_reference_t<decltype(S.st)>;
        St d;
        S.compute_forces(S.st, d);
        for (size_t i = 0; i < d.p.size(); ++i) {
            if (dden) dden[i] = double(d.p[i].den);
            for (int c = 0; c < 4; ++c) {
                if (dpos) dpos[4 * i + c] = double(d.p[i].pos[c]);
                if (dvel) dvel[4 * i + c] = double(d.p[i].vel[c]);
            }
        }
        const uint32_t ns = S.n_solids();
        if (dplastic)
            for (uint32_t s = 0; s < ns; ++s)
                for (int c = 0; c < 4; ++c)
                    for (int r = 0; r < 4; ++r) dplastic[16 * s + 4 * c + r] = double(d.s[s].stress[c][r]);
    });
    return 0;
}

// Deformation data of the current state: per solid L, F, Fdot (3 x 16, column-major).
int orc_strains(void* h, double* out) {
    dispatch(h, [&](auto& S) {
        S.update_contents(S.st);
        std::vector<Strain<std::remove_reference_t<decltype(S.st.p[0].den)>>> strains;
        S.compute_strain(S.st, strains);
        const uint32_t ns = S.n_solids();
        for (uint32_t s = 0; s < ns; ++s)
            for (int c = 0; c < 4; ++c)
                for (int r = 0; r < 4; ++r) {
                    out[48 * s + 4 * c + r] = double(strains[s].L[c][r]);
                    out[48 * s + 16 + 4 * c + r] = double(strains[s].F[c][r]);
                    out[48 * s + 32 + 4 * c + r] = double(strains[s].Fdot[c][r]);
                }
    });
    return 0;
}

// Buckets of the current state after update_contents: counts (ncells x 3),
// contents (ncells x 128), pos_index / ref_index (n), and the number of
// mobile + boundary particles within h of each particle among its 27 cells.
int orc_buckets(void* h, uint32_t* counts, uint32_t* contents, uint32_t* pos_index, uint32_t* ref_index,
                uint32_t* nbr_count) {
    dispatch(h, [&](auto& S) {
        S.update_contents(S.st);
        for (uint32_t c = 0; c < S.ncells; ++c) {
            for (int k = 0; k < 3; ++k)
                if (counts) counts[3 * c + k] = S.buckets[c].count[k];
            if (contents)
                for (uint32_t k = 0; k < MAXB; ++k) contents[size_t(MAXB) * c + k] = S.buckets[c].contents[k];
        }
        const auto& P = S.st.p;
        for (size_t i = 0; i < P.size(); ++i) {
            if (pos_index) pos_index[i] = S.pos_index[i];
            if (ref_index) ref_index[i] = S.ref_index[i];
        }
        if (nbr_count) {
            const float hf = S.hf;
            const float hh = hf * hf;
            for (size_t i = 0; i < P.size(); ++i) {
                uint32_t cnt = 0;
                if (S.pos_index[i] != INVALID) {
                    const uint32_t b = S.pos_index[i];
                    for (int dz = -1; dz <= 1; ++dz)
                        for (int dy = -1; dy <= 1; ++dy)
                            for (int dx = -1; dx <= 1; ++dx) {
                                int bp[3] = {int(S.buckets[b].index[0]) + dx, int(S.buckets[b].index[1]) + dy,
                                             int(S.buckets[b].index[2]) + dz};
                                if (!S.in_bounds(bp)) continue;
                                const Bucket& B = S.buckets[S.bucket_index(bp)];
                                const uint32_t bc = B.count[0], rc = B.count[1], cn = B.count[2];
                                for (uint32_t j = 0; j < bc + rc + cn; ++j) {
                                    if (j >= bc && j < bc + rc) continue;
                                    const auto& q = j < bc ? S.boundary[B.contents[j]] : P[B.contents[j]];
                                    float r[4];
                                    for (int c = 0; c < 4; ++c) r[c] = float(q.pos[c]) - float(P[i].pos[c]);
                                    const float d = ((r[0] * r[0] + r[1] * r[1]) + r[2] * r[2]) + r[3] * r[3];
                                    if (hh - d > 0.0f) cnt++;
                                }
                            }
                }
                nbr_count[i] = cnt;
            }
        }
    });
    return 0;
}

}  // extern "C"

extern "C" {

// poly6 W and grad W (kernel.rs:54-96) for n displacement vectors r (n x 4),
// with the Rust-side normalization constant for `dim`, in double.
int orc_poly6(int dim, double h, const double* r, int n, double* w, double* gw, double* kconst) {
    const double k = orc::norm_const<double>(uint32_t(dim), h);
    if (kconst) *kconst = k;
    for (int i = 0; i < n; ++i) {
        glsl::vec4<double> v(r[4 * i], r[4 * i + 1], r[4 * i + 2], r[4 * i + 3]);
        if (w) w[i] = orc::kernel_w(v, h, k);
        if (gw) {
            auto g = orc::grad_w(v, h, k);
            for (int c = 0; c < 4; ++c) gw[4 * i + c] = g[c];
        }
    }
    return 0;
}

// The f32 normalization constant exactly as the Rust code computes it.
float orc_norm_const_f32(int dim, float h) { return orc::norm_const<float>(uint32_t(dim), h); }

}  // extern "C"
