// sim.cu -- host side of libarphys: the FluidSim equivalent behind the C ABI.
//
// Mirrors src/soft_body/mod.rs (FluidSim::new / init / update / accessors)
// with device state owned by an `arp_sim` handle.  One integrator step:
//   1. grid over y0 positions; y0 (and caller ids, solid ids) gathered into
//      cell order, so stage 0 reads the state in place;
//   2. for each RK stage s: (s > 0) grid over the stage positions and sorted
//      copies; solid kernels when the scene has more than one solid
//      (src/soft_body/shaders/mod.rs:51); fluid kernel with the fused stage
//      update writing y_{s+1} (or y_new) in storage order.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <new>
#include <tuple>
#include <string>
#include <vector>

#include "arp_internal.h"
#include "grid.cuh"
#include "scene_loader.h"

using namespace arp;

namespace {

thread_local std::string g_last_error;

arp_status fail(arp_status code, const std::string& msg) {
    g_last_error = msg;
    return code;
}

#define CUDA_TRY(expr)                                                                          \
    do {                                                                                        \
        cudaError_t e_ = (expr);                                                                \
        if (e_ != cudaSuccess) {                                                                \
            return fail(e_ == cudaErrorMemoryAllocation ? ARP_ERR_OUT_OF_MEMORY : ARP_ERR_CUDA, \
                        std::string(#expr) + ": " + cudaGetErrorString(e_));                    \
        }                                                                                       \
    } while (0)

#define ARP_TRY(expr)                   \
    do {                                \
        arp_status s_ = (expr);         \
        if (s_ != ARP_OK) return s_;    \
    } while (0)

struct Tableau {
    int stages;
    double a[4][4];
    double b[4];
};

bool make_tableau(int id, Tableau& t) {
    std::memset(&t, 0, sizeof(t));
    switch (id) {
        case ARP_INT_EULER: t.stages = 1; t.b[0] = 1; return true;
        case ARP_INT_MIDPOINT: t.stages = 2; t.a[1][0] = 0.5; t.b[1] = 1; return true;
        case ARP_INT_HEUN2: t.stages = 2; t.a[1][0] = 1; t.b[0] = 0.5; t.b[1] = 0.5; return true;
        case ARP_INT_RALSTON: t.stages = 2; t.a[1][0] = 2.0 / 3.0; t.b[0] = 0.25; t.b[1] = 0.75; return true;
        case ARP_INT_RK3:
            t.stages = 3; t.a[1][0] = 0.5; t.a[2][0] = -1; t.a[2][1] = 2;
            t.b[0] = 1.0 / 6.0; t.b[1] = 2.0 / 3.0; t.b[2] = 1.0 / 6.0; return true;
        case ARP_INT_HEUN3:
            t.stages = 3; t.a[1][0] = 1.0 / 3.0; t.a[2][1] = 2.0 / 3.0; t.b[0] = 0.25; t.b[2] = 0.75; return true;
        case ARP_INT_RK4:
            t.stages = 4; t.a[1][0] = 0.5; t.a[2][1] = 0.5; t.a[3][2] = 1;
            t.b[0] = 1.0 / 6.0; t.b[1] = 1.0 / 3.0; t.b[2] = 1.0 / 3.0; t.b[3] = 1.0 / 6.0; return true;
        case ARP_INT_VERLET:  // one force evaluation per step; b[0] = 1/2 is the closing kick
            t.stages = 1; t.b[0] = 0.5; return true;
        case ARP_INT_RK_3_8:
            t.stages = 4; t.a[1][0] = 1.0 / 3.0; t.a[2][0] = -1.0 / 3.0; t.a[2][1] = 1;
            t.a[3][0] = 1; t.a[3][1] = -1; t.a[3][2] = 1;
            t.b[0] = 0.125; t.b[1] = 0.375; t.b[2] = 0.375; t.b[3] = 0.125; return true;
        default: return false;
    }
}

// kernel.rs:5-11 and :60-63, in f32 as the Rust code evaluates them
float volume_nball_f32(uint32_t n, float r) {
    if (n == 0) return 1.0f;
    if (n == 1) return 2.0f * r;
    const float pi = 3.14159265358979323846f;
    volatile float t = 2.0f * pi;
    t = t * r;
    t = t * r;
    t = t * volume_nball_f32(n - 2, r);
    return t / (float)n;
}
float norm_const_f32(uint32_t n, float h) {
    const float pi = 3.14159265358979323846f;
    volatile float p3 = pi * pi;
    p3 = p3 * pi;
    volatile float d = 6.0f * volume_nball_f32(n + 6, h);
    return p3 / d;
}

bool is_stiff(const arp_material& m) { return m.normal_stiffness != 0.0f || m.shear_stiffness != 0.0f; }

// Owning device allocation (move-only).
template <class T>
struct DevBuf {
    T* p = nullptr;
    size_t n = 0;
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    DevBuf(DevBuf&& o) noexcept : p(o.p), n(o.n) {
        o.p = nullptr;
        o.n = 0;
    }
    DevBuf& operator=(DevBuf&& o) noexcept {
        if (this != &o) {
            release();
            p = o.p;
            n = o.n;
            o.p = nullptr;
            o.n = 0;
        }
        return *this;
    }
    ~DevBuf() { release(); }
    cudaError_t alloc(size_t count) {
        release();
        if (count == 0) count = 1;
        cudaError_t e = cudaMalloc(&p, count * sizeof(T));
        if (e == cudaSuccess) n = count;
        else p = nullptr;
        return e;
    }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
};

struct StateBuf {
    DevBuf<float4> pd, vm;
};

// ---- reverse mode: what a recording forward step keeps, and the tape ----------
constexpr int kMaxStages = 4;
struct StepRecord {
    DevBuf<float4> pd[kMaxStages], vm[kMaxStages];      // stage states, storage order
    DevBuf<uint32_t> perm[kMaxStages], start[kMaxStages];
    bool has_perm[kMaxStages] = {false, false, false, false};
    DevBuf<float4> F[kMaxStages], A[kMaxStages], sx[kMaxStages], sv[kMaxStages];
    DevBuf<uint2> sc[kMaxStages];
    DevBuf<uint32_t> cb[kMaxStages];
    DevBuf<float4> ep[kMaxStages];                       // plastic strain of each stage (plastic scenes)
    DevBuf<uint32_t> orig, sid, slot_of;                 // of the step (after its reorder)
};
struct Checkpoint {
    DevBuf<float4> pd, vm;
    DevBuf<float4> ep;  // plastic strain (plastic scenes)
    DevBuf<float4> fpd, fvm, fep;  // velocity Verlet: the carried force record (same storage order as pd)
    bool fvalid = false;
    DevBuf<uint32_t> orig, sid;
    float time = 0.0f;
};
struct Tape {
    uint32_t every = 1;
    uint64_t steps = 0;                 // steps recorded since the tape began
    std::vector<Checkpoint> ckpts;      // state before step c * every
};
// Device memory of the reverse pass, kept by the handle across tapes so that
// repeated taping and backward passes allocate nothing after the first.
struct AdjointPool {
    std::vector<StepRecord> recs;       // one segment of recording steps
    std::vector<Checkpoint> spare;      // checkpoints of ended tapes, reused
    DevBuf<float4> lc_p, lc_v, ls_p, ls_v, out_p, out_v, mu_p, mu_v, w, e, xs;
    DevBuf<float4> io;  // [2n] the caller's 8-float-per-particle gradients, on the device
    DevBuf<float4> lY_p[kMaxStages], lY_v[kMaxStages];
    DevBuf<float4> lamF, lamFd;
    DevBuf<float4> lam_ep, out_ep, mu_ep, lY_ep[kMaxStages];  // adjoint of the plastic strain (solid order)
    DevBuf<double2> gst;
    DevBuf<uint32_t> flags;
    Checkpoint now;
    // velocity Verlet: the adjoint of the carried force record (caller order;
    // solid order for the plastic strain's) and the record of the force
    // evaluation at the tape's start, when the first taped step made one
    DevBuf<float4> lf_p, lf_v, lf_ep;
    StepRecord prime;
    bool prime_recorded = false;
};

}  // namespace

arp_status arp::set_error(arp_status code, const std::string& msg) { return fail(code, msg); }

struct arp_sim {
    // scene
    // One entry per scene of the batch (a single simulation has one).
    struct SceneHost {
        uint32_t p_base, n;       // caller-order particle range
        uint32_t b_base, nb;      // boundary range
        uint32_t mat_base, nmat;  // global material range
        uint32_t inter_base;      // interaction block (nmat x nmat)
        uint32_t s_base;          // first batch-wide solid id
        uint32_t dummy_solid;     // 1 when created without solids: the reference then keeps a
                                  // placeholder solid entry 0 (particles.rs:502), so solids added
                                  // later are numbered from 1 and count one more
        bool flat_z;              // every particle shares one z and moves in the plane
        bool dense = false;       // the search grid halves y as well as x (see scene_params)
        arp_aabb bounds;
        float h, gravity, alpha;
        SceneP sp;
    };
    std::vector<SceneHost> scenes;
    uint32_t n = 0, nb = 0, ns = 0, M = 0;
    uint32_t dim = 0;      // the reference's count of non-zero box axes (scene 0)
    int kdim = 3;          // 2 when every scene is flat in z
    float pos_w = 0.0f;    // common w coordinate of all positions
    bool have_w = false;
    std::vector<arp_material> mats;       // all scenes, scene order
    std::vector<arp_interaction> inter;   // per-scene blocks, scene order
    float h = 0, timestep = 0, dt_sub = 0;
    uint32_t subticks = 1;
    int integrator = 0;
    Tableau tab{};
    float time = 0;
    bool initialized = false;
    bool any_stiff_immobile = false;
    bool all_order2 = true;  // every stiff material uses strain order 2
    bool any_plastic = false;  // some stiff material is plastic
    uint32_t ncells = 0;     // search cells of all scenes
    uint32_t nccells = 0;    // reference cells of all scenes (the C ABI's cell numbering)
    uint32_t max_nmat = 0;
    Tables tables{};
    std::vector<uint32_t> scene_of_material;

    std::vector<arp_particle> host_particles;  // caller order (initial state)
    std::vector<arp_particle> host_boundary;
    std::vector<uint32_t> sid_of_caller;       // caller id -> solid id
    std::vector<uint32_t> part_of_solid;       // solid id -> caller id
    std::vector<float4> host_ref;              // solid id -> reference position (set by init)
    std::vector<float4> host_ep;               // solid id -> plastic strain columns, kept across add_particles
    bool any_solid_branch = false;             // some scene has more than one solid entry

    cudaStream_t own_stream = nullptr, stream = nullptr;
    uint64_t launches = 0;

    // device: scene and material tables
    DevBuf<SceneP> d_scenes;
    DevBuf<DevMat> d_mats;
    DevBuf<FluidMat> d_fmats;
    DevBuf<DevInter> d_inter;
    // mobile state: Y (y0), T (reorder target / y_new), S[2] (stage states)
    StateBuf Y, T, S[2], X, acc, kst[4];
    // velocity Verlet: the derivative record of the last force evaluation
    // (storage order of Y) and its plastic-strain rates (solid-id order);
    // invalid until a force evaluation at the current state has run
    StateBuf vforce;
    DevBuf<float4> ep_force;
    bool vforce_valid = false;
    bool verlet() const { return integrator == ARP_INT_VERLET; }
    DevBuf<uint32_t> orig, orig_r, sid, sid_r, sid_sorted, slot_of;
    DevBuf<float> ps, bps;  // p / rho^2 of sorted particles / boundary particles
    DevBuf<arp_particle> records;      // device copy of caller-order Particle records (state exchange)
    DevBuf<uint32_t> sid_of_caller_d;  // caller id -> solid id
    DevBuf<uint32_t> mat_of_caller_d;  // caller id -> material id
    DevBuf<uint32_t> check_flag;
    // boundary (cell-sorted)
    DevBuf<float4> b_pd, b_vm;
    DevBuf<uint32_t> b_orig, b_start, sid_of_bidx;
    // grid scratch
    GridBuffers gb{};
    DevBuf<uint32_t> g_key, g_rank, g_count, g_start, g_perm, g_bsums;
    DevBuf<uint2> g_coord;  // grid coordinates per slot
    DevBuf<uint32_t> contact_bound;
    DevBuf<uint32_t> tile_counter;  // work queue of the persistent fluid kernel
    DevBuf<uint32_t> overflow, overflow_count;  // the fluid kernel's two overflow queues (2n entries, 2 counts)
    int fluid_variant = 0;
    uint32_t grid_cap = 0;
    // solids
    DevBuf<float4> ref, L, F, A, ksol;
    DevBuf<float4> ep, ep_t, ep_s[2], ep_acc, ep_kst[4];
    DevBuf<float4> sx, sv;  // stage state in solid-id order
    DevBuf<uint2> sc;
    DevBuf<float2> stiff;   // per-solid (normal, shear) stiffness, when set
    bool have_stiff = false;
    // reverse mode
    std::unique_ptr<Tape> tape;
    AdjointPool adj;
    struct RenderBufs {
        DevBuf<float4> PR, PC, PP, c1, c2, c3;
        DevBuf<float> d0;
        DevBuf<uint32_t> counts, start, fill, list, bsums;
        DevBuf<unsigned long long> zkey;
        DevBuf<uint8_t> rgb;
    } rbuf;
    StepRecord* rec = nullptr;  // set while a recording step runs
    StepRecord* rec_prime = nullptr;  // where a recording Verlet step records its force evaluation at y_n
    bool replaying = false;     // steps re-run by the backward pass take no checkpoints
    DevBuf<uint32_t> mat_of_solid, rl_off, rl_nbr;
    DevBuf<float4> rl_gw;
    uint32_t rl_nnz = 0;
    DevBuf<DevStats> d_stats;

    // CUDA graphs of one integrator step.  A step swaps the caller-id and
    // solid-id buffers (and the plastic strain's when it changes), so the
    // steps alternate between two sets of buffer pointers; a graph is kept
    // for each set, keyed by its pointers, and replayed with the step's
    // host-side effects applied by hand.
    struct StepGraph {
        cudaGraph_t g = nullptr;
        cudaGraphExec_t exec = nullptr;
        const void* sig[4] = {nullptr, nullptr, nullptr, nullptr};
        uint64_t launches = 0;  // kernels per replay
    };
    bool use_graph = false;
    StepGraph graphs[2];
    cudaStream_t graph_stream = nullptr;
    void drop_graph() {
        for (auto& x : graphs) {
            if (x.exec) cudaGraphExecDestroy(x.exec);
            if (x.g) cudaGraphDestroy(x.g);
            x = StepGraph{};
        }
        graph_stream = nullptr;
    }

    // profiling: events around the segments of one step in every prof_every
    bool prof_on = false;
    uint32_t prof_every = 1, prof_phase = 0;
    bool profiling = false;  // the current step records events
    std::vector<cudaEvent_t> ev_free;
    struct Mark {
        cudaEvent_t e[4];
    };
    std::vector<Mark> marks;
    double acc_ms[3] = {0, 0, 0};  // neighbor, solid, fluid
    uint64_t prof_steps = 0, prof_stages = 0, prof_launches = 0, prof_l[3] = {0, 0, 0};

    // Asynchronous host exchange (arp_sim_set_particles_async /
    // arp_sim_get_particles_async): records cross PCIe on two copy streams of
    // their own through two device staging slots each way, so that the copy
    // of the next state in, the step on the handle's stream and the copy of
    // the last result out run at the same time.  Events order each slot's
    // reuse; record checks accumulate in a sticky flag that
    // arp_sim_synchronize reports.
    struct HostIO {
        cudaStream_t copy_in = nullptr, copy_out = nullptr;
        DevBuf<arp_particle> in_rec[2], out_rec[2];
        cudaEvent_t in_copied[2] = {}, in_used[2] = {}, out_ready[2] = {}, out_copied[2] = {};
        int in_slot = 0, out_slot = 0;
        uint32_t cap = 0;  // records per staging slot
        DevBuf<uint32_t> flag;
        bool ready = false;
    } io;
    void release_io() {
        if (!io.ready) return;
        if (io.copy_in) cudaStreamSynchronize(io.copy_in);
        if (io.copy_out) cudaStreamSynchronize(io.copy_out);
        for (int q = 0; q < 2; ++q)
            for (cudaEvent_t e : {io.in_copied[q], io.in_used[q], io.out_ready[q], io.out_copied[q]})
                if (e) cudaEventDestroy(e);
        if (io.copy_in) cudaStreamDestroy(io.copy_in);
        if (io.copy_out) cudaStreamDestroy(io.copy_out);
        io.ready = false;
    }

    ~arp_sim() {
        drop_graph();
        if (stream) cudaStreamSynchronize(stream);
        release_io();
        for (auto& m : marks)
            for (auto e : m.e) ev_free.push_back(e);
        for (auto e : ev_free) cudaEventDestroy(e);
        if (own_stream) cudaStreamDestroy(own_stream);
    }

    bool solid_branch() const { return any_solid_branch; }  // shaders/mod.rs:51: solids.len() > 1
};

namespace {

arp_status alloc_state(StateBuf& s, size_t n) {
    CUDA_TRY(s.pd.alloc(n));
    CUDA_TRY(s.vm.alloc(n));
    return ARP_OK;
}

arp_status ensure_grid(arp_sim* S, uint32_t cap) {
    const uint32_t nc = S->ncells;
    if (S->grid_cap >= cap && S->g_start.p) return ARP_OK;
    cap = std::max(cap, 1u);
    CUDA_TRY(S->g_key.alloc(cap));
    CUDA_TRY(S->g_rank.alloc(cap));
    CUDA_TRY(S->g_perm.alloc(cap));
    CUDA_TRY(S->g_coord.alloc(cap));
    if (!S->g_start.p) {
        CUDA_TRY(S->g_count.alloc(size_t(nc) + 2));
        CUDA_TRY(S->g_start.alloc(size_t(nc) + 2));
        CUDA_TRY(cudaMemset(S->g_count.p, 0, (size_t(nc) + 2) * sizeof(uint32_t)));
    }
    const uint32_t bs = std::max(scan_block_sums_needed(nc + 2), scan_block_sums_needed(cap + 1));
    if (S->g_bsums.n < bs) CUDA_TRY(S->g_bsums.alloc(bs));
    S->grid_cap = cap;
    S->gb.key = S->g_key.p;
    S->gb.rank = S->g_rank.p;
    S->gb.count = S->g_count.p;
    S->gb.start = S->g_start.p;
    S->gb.perm = S->g_perm.p;
    S->gb.coord = S->g_coord.p;
    S->gb.block_sums = S->g_bsums.p;
    S->gb.block_sums_cap = (uint32_t)S->g_bsums.n;
    return ARP_OK;
}

arp_status check_launch(const char* what) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(ARP_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
    return ARP_OK;
}

cudaEvent_t take_event(arp_sim* S) {
    if (!S->ev_free.empty()) {
        cudaEvent_t e = S->ev_free.back();
        S->ev_free.pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    cudaEventCreate(&e);
    return e;
}

void harvest_marks(arp_sim* S) {
    if (S->marks.empty()) return;
    cudaEventSynchronize(S->marks.back().e[3]);
    for (auto& m : S->marks) {
        for (int k = 0; k < 3; ++k) {
            float ms = 0;
            if (cudaEventElapsedTime(&ms, m.e[k], m.e[k + 1]) == cudaSuccess) S->acc_ms[k] += ms;
        }
        for (auto e : m.e) S->ev_free.push_back(e);
    }
    S->marks.clear();
}

// Scalars and grid of one scene (neighbor_list.rs:201-206, kernel.rs:60-63,
// the shader constants of fluid.rs / solid.rs).
arp_status scene_params(arp_sim::SceneHost& H, uint32_t dim) {
    SceneP& P = H.sp;
    for (int a = 0; a < 3; ++a) {
        P.grid.min[a] = H.bounds.min[a];
        P.grid.dim[a] = H.bounds.dim[a];
    }
    uint64_t nc = 1;
    for (int a = 0; a < 4; ++a) {
        const float q = std::max(1.0f, H.bounds.dim[a] / H.h);
        // range-checked in float: a quotient past 2^30 would not convert to a
        // meaningful cell count
        if (!(q <= 1073741824.0f)) return fail(ARP_ERR_UNSUPPORTED, "a scene's grid has more than 2^30 cells");
        const uint32_t sub = (uint32_t)q;
        if (a < 3) P.grid.sub[a] = sub;
        nc *= sub;
    }
    if (nc > (1ull << 30)) return fail(ARP_ERR_UNSUPPORTED, "a scene's grid has more than 2^30 cells");
    P.grid.ncells = (uint32_t)nc;
    // search grid: the kSearchHalve axes of non-zero extent halved (the w axis is not hashed)
    P.sgrid = P.grid;
    uint64_t snc = 1;
    for (int a = 0; a < 3; ++a) {
        const bool halve = (kSearchHalve >> a & 1u) || (a == 1 && H.dense);
        P.halved[a] = H.bounds.dim[a] != 0.0f && halve ? 1u : 0u;
        P.sgrid.sub[a] = P.grid.sub[a] << P.halved[a];
        snc *= P.sgrid.sub[a];
    }
    if (snc > (1ull << 30)) return fail(ARP_ERR_UNSUPPORTED, "a scene's search grid has more than 2^30 cells");
    P.sgrid.ncells = (uint32_t)snc;
    P.dim = dim;
    P.h = H.h;
    P.h2 = H.h * H.h;
    P.kconst = norm_const_f32(dim, H.h);
    P.g = H.gravity;
    const float eps = 0.1f;
    volatile float t = eps * H.h;
    P.eps_h = t;
    P.eps_hh = t * H.h;
    volatile float ten_eps = 10.0f * eps;
    P.hg_h = ten_eps * H.h;
    P.rcut = 8.0f * H.h;
    P.rcut2 = P.rcut * P.rcut;
    volatile float hh = H.h * H.h;
    P.r_geom = hh / P.rcut;
    // Largest |dx| between particles inside the box whose cells are within one
    // cell per axis: 2 * |cell diagonal|.  An axis of zero extent contributes
    // nothing only when every particle shares its coordinate (flat z).
    double cs2 = 0.0;
    bool bounded = true;
    for (int a = 0; a < 3; ++a) {
        if (H.bounds.dim[a] > 0.0f) {
            const double cs = (double)H.bounds.dim[a] / (double)P.grid.sub[a];
            cs2 += cs * cs;
        } else if (!(a == 2 && H.flat_z)) {
            bounded = false;
        }
    }
    const double slack = 0.999 * (double)P.rcut - 2.0 * std::sqrt(cs2);
    P.contact_slack = bounded && slack > 0.0 ? (float)slack : 0.0f;
    P.mat_base = H.mat_base;
    P.nmat = H.nmat;
    P.inter_base = H.inter_base;
    return ARP_OK;
}

// Solid data, boundary grid, reference neighbor lists (FluidSim::init).
arp_status do_init(arp_sim* S) {
    cudaStream_t st = S->stream;
    const uint32_t n = S->n, nb = S->nb, ns = S->ns;
    const uint32_t nc = S->ncells;
    ARP_TRY(ensure_grid(S, std::max({n, nb, ns, 1u})));

    // mobile state in caller order
    std::vector<float4> pd(n), vm(n);
    std::vector<uint32_t> orig(n), sid(n);
    for (uint32_t i = 0; i < n; ++i) {
        const arp_particle& p = S->host_particles[i];
        pd[i] = make_float4(p.pos[0], p.pos[1], p.pos[2], p.den);
        uint32_t mbits = p.mat;
        float mf;
        std::memcpy(&mf, &mbits, 4);
        vm[i] = make_float4(p.vel[0], p.vel[1], p.vel[2], mf);
        orig[i] = i;
        sid[i] = S->sid_of_caller[i];
    }
    if (n) {
        CUDA_TRY(cudaMemcpyAsync(S->Y.pd.p, pd.data(), n * sizeof(float4), cudaMemcpyHostToDevice, st));
        CUDA_TRY(cudaMemcpyAsync(S->Y.vm.p, vm.data(), n * sizeof(float4), cudaMemcpyHostToDevice, st));
        CUDA_TRY(cudaMemcpyAsync(S->orig.p, orig.data(), n * sizeof(uint32_t), cudaMemcpyHostToDevice, st));
        CUDA_TRY(cudaMemcpyAsync(S->sid.p, sid.data(), n * sizeof(uint32_t), cudaMemcpyHostToDevice, st));
    }

    // boundary grid: filled once (neighbor_list.rs:247-264)
    {
        std::vector<float4> bpd(nb), bvm(nb);
        std::vector<uint32_t> bo(nb);
        for (uint32_t i = 0; i < nb; ++i) {
            const arp_particle& p = S->host_boundary[i];
            bpd[i] = make_float4(p.pos[0], p.pos[1], p.pos[2], p.den);
            uint32_t mbits = p.mat;
            float mf;
            std::memcpy(&mf, &mbits, 4);
            bvm[i] = make_float4(p.vel[0], p.vel[1], p.vel[2], mf);
            bo[i] = i;
        }
        DevBuf<float4> tmp_pd, tmp_vm;
        DevBuf<uint32_t> tmp_o;
        CUDA_TRY(tmp_pd.alloc(nb));
        CUDA_TRY(tmp_vm.alloc(nb));
        CUDA_TRY(tmp_o.alloc(nb));
        if (nb) {
            CUDA_TRY(cudaMemcpyAsync(tmp_pd.p, bpd.data(), nb * sizeof(float4), cudaMemcpyHostToDevice, st));
            CUDA_TRY(cudaMemcpyAsync(tmp_vm.p, bvm.data(), nb * sizeof(float4), cudaMemcpyHostToDevice, st));
            CUDA_TRY(cudaMemcpyAsync(tmp_o.p, bo.data(), nb * sizeof(uint32_t), cudaMemcpyHostToDevice, st));
        }
        S->launches += build_grid(tmp_pd.p, tmp_vm.p, nullptr, nb, S->tables, S->gb, nullptr, nullptr, st);
        S->launches += gather_state(S->gb.perm, nb, tmp_pd.p, S->b_pd.p, tmp_vm.p, S->b_vm.p, tmp_o.p,
                                    S->b_orig.p, nullptr, nullptr, nullptr, nullptr, S->bps.p, S->d_mats.p, st);
        CUDA_TRY(cudaMemcpyAsync(S->b_start.p, S->gb.start, (size_t(nc) + 2) * sizeof(uint32_t),
                                 cudaMemcpyDeviceToDevice, st));
        CUDA_TRY(cudaStreamSynchronize(st));
        ARP_TRY(check_launch("boundary grid"));
    }
    if (S->any_stiff_immobile) {
        // the scene's boundary index b read as an index into the scene's mobile particles
        std::vector<uint32_t> sb(std::max(nb, 1u), kInvalid);
        for (const auto& H : S->scenes)
            for (uint32_t b = 0; b < H.nb; ++b) sb[H.b_base + b] = b < H.n ? S->sid_of_caller[H.p_base + b] : kInvalid;
        CUDA_TRY(cudaMemcpy(S->sid_of_bidx.p, sb.data(), sb.size() * sizeof(uint32_t), cudaMemcpyHostToDevice));
    }

    // solids: reference positions, plastic strain = 0, neighbor lists, L
    if (ns > 0) {
        // reference positions: the positions at creation, or carried over by
        // add_particles (new solids then start from their position when added)
        const size_t kept = S->host_ref.size() <= ns ? S->host_ref.size() : 0;
        std::vector<uint32_t> mos(ns);
        S->host_ref.resize(ns);
        for (uint32_t s = 0; s < ns; ++s) {
            const arp_particle& p = S->host_particles[S->part_of_solid[s]];
            if (s >= kept) S->host_ref[s] = make_float4(p.pos[0], p.pos[1], p.pos[2], 0.0f);
            mos[s] = p.mat;
        }
        // the device copy carries each solid's rest volume m / rho0 in w, so
        // one gather of a reference neighbor gives dX and V_j
        std::vector<float4> ref_dev(S->host_ref);
        for (uint32_t s = 0; s < ns; ++s) ref_dev[s].w = S->mats[mos[s]].mass / S->mats[mos[s]].start_den;
        CUDA_TRY(cudaMemcpyAsync(S->ref.p, ref_dev.data(), ns * sizeof(float4), cudaMemcpyHostToDevice, st));
        CUDA_TRY(cudaMemcpyAsync(S->mat_of_solid.p, mos.data(), ns * sizeof(uint32_t), cudaMemcpyHostToDevice, st));
        CUDA_TRY(cudaMemsetAsync(S->ep.p, 0, size_t(ns) * 4 * sizeof(float4), st));
        if (!S->host_ep.empty()) {
            const size_t ne = std::min(S->host_ep.size(), size_t(ns) * 4);
            CUDA_TRY(cudaMemcpyAsync(S->ep.p, S->host_ep.data(), ne * sizeof(float4), cudaMemcpyHostToDevice, st));
            CUDA_TRY(cudaStreamSynchronize(st));
            S->host_ep.clear();
        }
        // grid over reference positions (neighbor_list.rs:266-275, mode 1)
        S->launches += build_grid(S->ref.p, nullptr, S->mat_of_solid.p, ns, S->tables, S->gb, nullptr, nullptr, st);
        DevBuf<uint32_t> cnt;
        CUDA_TRY(cnt.alloc(size_t(ns) + 1));
        CUDA_TRY(cudaMemsetAsync(cnt.p, 0, (size_t(ns) + 1) * sizeof(uint32_t), st));
        S->launches += ref_lists_count(S->ref.p, S->mat_of_solid.p, ns, S->gb, S->tables, cnt.p, st);
        CUDA_TRY(S->rl_off.alloc(size_t(ns) + 1));
        S->launches += exclusive_scan(cnt.p, ns + 1, S->rl_off.p, S->gb.block_sums, st);
        uint32_t nnz = 0;
        CUDA_TRY(cudaMemcpyAsync(&nnz, S->rl_off.p + ns, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
        CUDA_TRY(cudaStreamSynchronize(st));
        CUDA_TRY(S->rl_nbr.alloc(std::max(nnz, 1u)));
        CUDA_TRY(S->rl_gw.alloc(std::max(nnz, 1u)));
        S->rl_nnz = nnz;
        SolidRefList rl{S->rl_off.p, S->rl_nbr.p, S->rl_gw.p, nnz};
        S->launches += ref_lists_fill(S->ref.p, S->mat_of_solid.p, ns, S->gb, S->tables, rl, S->L.p, st);
        CUDA_TRY(cudaStreamSynchronize(st));
        ARP_TRY(check_launch("reference neighbor lists"));
    }
    CUDA_TRY(cudaMemsetAsync(S->d_stats.p, 0, sizeof(DevStats), st));
    S->vforce_valid = false;
    S->initialized = true;
    return ARP_OK;
}

arp_status run_autotune(arp_sim* S, bool force);

void mark(arp_sim* S, arp_sim::Mark& m, int k) {
    if (!S->profiling) return;
    m.e[k] = take_event(S);
    cudaEventRecord(m.e[k], S->stream);
}

// Device-to-device copy into a buffer grown to fit.
template <class T>
cudaError_t keep(DevBuf<T>& dst, const T* src, size_t count, cudaStream_t st) {
    if (dst.n < std::max<size_t>(count, 1)) {
        cudaError_t e = dst.alloc(count);
        if (e != cudaSuccess) return e;
    }
    if (count == 0) return cudaSuccess;
    return cudaMemcpyAsync(dst.p, src, count * sizeof(T), cudaMemcpyDeviceToDevice, st);
}

arp_status save_checkpoint(arp_sim* S) {
    Checkpoint c;
    if (!S->adj.spare.empty()) {
        c = std::move(S->adj.spare.back());
        S->adj.spare.pop_back();
    }
    CUDA_TRY(keep(c.pd, (const float4*)S->Y.pd.p, S->n, S->stream));
    CUDA_TRY(keep(c.vm, (const float4*)S->Y.vm.p, S->n, S->stream));
    CUDA_TRY(keep(c.orig, (const uint32_t*)S->orig.p, S->n, S->stream));
    CUDA_TRY(keep(c.sid, (const uint32_t*)S->sid.p, S->n, S->stream));
    if (S->any_plastic) CUDA_TRY(keep(c.ep, (const float4*)S->ep.p, 4 * size_t(S->ns), S->stream));
    c.fvalid = S->verlet() && S->vforce_valid;
    if (c.fvalid) {
        CUDA_TRY(keep(c.fpd, (const float4*)S->vforce.pd.p, S->n, S->stream));
        CUDA_TRY(keep(c.fvm, (const float4*)S->vforce.vm.p, S->n, S->stream));
        if (S->any_plastic) CUDA_TRY(keep(c.fep, (const float4*)S->ep_force.p, 4 * size_t(S->ns), S->stream));
    }
    c.time = S->time;
    S->tape->ckpts.push_back(std::move(c));
    return ARP_OK;
}

arp_status restore_checkpoint(arp_sim* S, const Checkpoint& c) {
    const size_t n = S->n;
    if (n) {
        CUDA_TRY(cudaMemcpyAsync(S->Y.pd.p, c.pd.p, n * sizeof(float4), cudaMemcpyDeviceToDevice, S->stream));
        CUDA_TRY(cudaMemcpyAsync(S->Y.vm.p, c.vm.p, n * sizeof(float4), cudaMemcpyDeviceToDevice, S->stream));
        CUDA_TRY(cudaMemcpyAsync(S->orig.p, c.orig.p, n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, S->stream));
        CUDA_TRY(cudaMemcpyAsync(S->sid.p, c.sid.p, n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, S->stream));
    }
    if (S->any_plastic && S->ns)
        CUDA_TRY(cudaMemcpyAsync(S->ep.p, c.ep.p, 4 * size_t(S->ns) * sizeof(float4), cudaMemcpyDeviceToDevice,
                                 S->stream));
    if (S->verlet()) {
        S->vforce_valid = c.fvalid;
        if (c.fvalid && n) {
            CUDA_TRY(cudaMemcpyAsync(S->vforce.pd.p, c.fpd.p, n * sizeof(float4), cudaMemcpyDeviceToDevice, S->stream));
            CUDA_TRY(cudaMemcpyAsync(S->vforce.vm.p, c.fvm.p, n * sizeof(float4), cudaMemcpyDeviceToDevice, S->stream));
        }
        if (c.fvalid && S->any_plastic && S->ns)
            CUDA_TRY(cudaMemcpyAsync(S->ep_force.p, c.fep.p, 4 * size_t(S->ns) * sizeof(float4),
                                     cudaMemcpyDeviceToDevice, S->stream));
    }
    S->time = c.time;
    return ARP_OK;
}

// One integrator step.  With `prime` (velocity Verlet only) it instead
// evaluates the forces at the current state and keeps their derivative
// record for the next step's kick, the force evaluation of the reference's
// init_with_vel (src/soft_body/mod.rs:213-233): the state is re-sorted into
// cell order but not advanced, and no time passes.
arp_status do_step(arp_sim* S, bool prime = false) {
    cudaStream_t st = S->stream;
    const uint32_t n = S->n, ns = S->ns;
    const Tableau& tab = S->tab;
    const bool sb = S->solid_branch();
    const bool verlet = S->verlet();
    if (S->tape && !S->replaying && !prime) {
        if (S->tape->steps % S->tape->every == 0) ARP_TRY(save_checkpoint(S));
        S->tape->steps++;
    }
    if (verlet && !prime && !S->vforce_valid) {
        // the force evaluation at y_n that the first step after init, a new
        // state or a tape start makes; a recording step records it too
        S->rec_prime = S->rec ? &S->adj.prime : nullptr;
        if (S->rec) S->adj.prime_recorded = true;
        const arp_status ps = do_step(S, true);
        S->rec_prime = nullptr;
        ARP_TRY(ps);
    }
    StepRecord* R = prime ? S->rec_prime : S->rec;
    if (!prime) S->time += S->dt_sub;
    const uint32_t* bstart = S->b_start.p;
    uint64_t l0 = S->launches;
    S->profiling = !prime && S->prof_on && S->prof_phase++ % S->prof_every == 0;
    // velocity Verlet: (dt/2) as the stage epilogue's coefficient b[0] dt
    const float half = (float)(tab.b[0] * (double)S->dt_sub);

    // 1. sort y0 into cell order
    arp_sim::Mark mk{};
    mark(S, mk, 0);
    // each stage's grid build clears the counters the stage's kernels start from
    StageCounters zero;
    zero.p[0] = S->overflow_count.p;
    zero.n[0] = 2;
    zero.p[1] = S->tile_counter.p;
    zero.n[1] = 1;
    if (sb) {
        zero.p[2] = S->contact_bound.p;
        zero.n[2] = 2;
    }
    // velocity Verlet kicks and drifts first (storage order, into X); the grid
    // and the force evaluation then see the drifted state
    const float4* src_pd = S->Y.pd.p;
    const float4* src_vm = S->Y.vm.p;
    if (verlet && !prime) {
        S->launches += verlet_kick_drift(S->Y.pd.p, S->Y.vm.p, S->vforce.pd.p, S->vforce.vm.p, n, half, S->dt_sub,
                                         S->X.pd.p, S->X.vm.p, st);
        src_pd = S->X.pd.p;
        src_vm = S->X.vm.p;
    }
    S->launches += build_grid(src_pd, src_vm, nullptr, n, S->tables, S->gb, S->d_stats.p, bstart, st, zero);
    // the stage-0 solid copies and the solid -> slot map come out of the same gather
    SolidScatter sol0;
    if (ns) {
        sol0.sid_of_slot = S->sid.p;
        sol0.coord_of_slot = S->gb.coord;
        sol0.sx = S->sx.p;
        sol0.sv = S->sv.p;
        sol0.sc = S->sc.p;
        sol0.slot_of = S->slot_of.p;
    }
    S->launches += gather_state(S->gb.perm, n, src_pd, S->T.pd.p, src_vm, S->T.vm.p, S->orig.p, S->orig_r.p,
                                S->sid.p, S->sid_r.p, nullptr, nullptr, S->ps.p, S->d_mats.p, st, sol0);
    std::swap(S->Y, S->T);
    std::swap(S->orig, S->orig_r);
    std::swap(S->sid, S->sid_r);
    if (R) {
        CUDA_TRY(keep(R->orig, (const uint32_t*)S->orig.p, n, st));
        CUDA_TRY(keep(R->sid, (const uint32_t*)S->sid.p, n, st));
        CUDA_TRY(keep(R->slot_of, (const uint32_t*)S->slot_of.p, ns, st));
    }
    uint64_t nl = S->launches - l0;

    StageBuffers B{};
    B.y0_pd = S->Y.pd.p;
    B.y0_vm = S->Y.vm.p;
    B.acc_pd = S->acc.pd.p;
    B.acc_vm = S->acc.vm.p;
    bool acc_started = false;
    const float4* cur_pd = S->Y.pd.p;
    const float4* cur_vm = S->Y.vm.p;
    const float4* cur_ep = S->ep.p;
    const float4* ep_base = S->ep.p;  // the step's y0 of the plastic strain
    if (verlet && !prime && sb && S->any_plastic) {
        S->launches += verlet_kick4(S->ep.p, S->ep_force.p, 4 * ns, half, S->ep_s[0].p, st);
        ep_base = cur_ep = S->ep_s[0].p;
    }
    for (int s = 0; s < tab.stages; ++s) {
        const bool last = !prime && s == tab.stages - 1;
        StageCoefs c{};
        c.stage = s;
        c.last = last ? 1 : 0;
        float cp[3] = {0.f, 0.f, 0.f};
        if (!last) {
            for (int j = 0; j < s && j < 3; ++j) cp[j] = (float)(tab.a[s + 1][j] * (double)S->dt_sub);
            c.c_self = (float)(tab.a[s + 1][s] * (double)S->dt_sub);
        }
        c.c_prev0 = cp[0];
        c.c_prev1 = cp[1];
        c.c_prev2 = cp[2];
        c.c_acc = prime ? 0.0f : (float)(tab.b[s] * (double)S->dt_sub);
        c.acc_first = acc_started ? 0 : 1;
        c.kick = verlet ? 1 : 0;
        if (c.c_acc != 0.0f) acc_started = true;
        bool store_k = false;
        for (int t = s + 2; t < tab.stages; ++t)
            if (tab.a[t][s] != 0.0) store_k = true;
        B.store_pd = verlet ? S->vforce.pd.p : store_k ? S->kst[s].pd.p : nullptr;
        B.store_vm = verlet ? S->vforce.vm.p : store_k ? S->kst[s].vm.p : nullptr;
        B.prev0_pd = cp[0] != 0.f ? S->kst[0].pd.p : nullptr;
        B.prev0_vm = cp[0] != 0.f ? S->kst[0].vm.p : nullptr;
        B.prev1_pd = cp[1] != 0.f ? S->kst[1].pd.p : nullptr;
        B.prev1_vm = cp[1] != 0.f ? S->kst[1].vm.p : nullptr;
        B.prev2_pd = cp[2] != 0.f ? S->kst[2].pd.p : nullptr;
        B.prev2_vm = cp[2] != 0.f ? S->kst[2].vm.p : nullptr;

        if (s > 0) {
            if (S->profiling && s > 0) mark(S, mk, 0);
            l0 = S->launches;
            S->launches += build_grid(cur_pd, cur_vm, nullptr, n, S->tables, S->gb, S->d_stats.p, bstart, st, zero);
            SolidScatter sol;  // this stage's solid copies
            if (sb && ns) {
                sol.sid_of_slot = S->sid.p;
                sol.coord_of_slot = S->gb.coord;
                sol.sx = S->sx.p;
                sol.sv = S->sv.p;
                sol.sc = S->sc.p;
            }
            S->launches += gather_state(S->gb.perm, n, cur_pd, S->X.pd.p, cur_vm, S->X.vm.p, sb ? S->sid.p : nullptr,
                                        sb ? S->sid_sorted.p : nullptr, nullptr, nullptr, nullptr, nullptr, S->ps.p,
                                        S->d_mats.p, st, sol);
            nl += S->launches - l0;
        }
        const float4* xs = s == 0 ? S->Y.pd.p : S->X.pd.p;
        const float4* vs = s == 0 ? S->Y.vm.p : S->X.vm.p;
        const uint32_t* perm = s == 0 ? nullptr : S->gb.perm;
        const uint32_t* sid_sorted = s == 0 ? S->sid.p : S->sid_sorted.p;
        float4* next_pd = last ? S->T.pd.p : S->S[s % 2].pd.p;
        float4* next_vm = last ? S->T.vm.p : S->S[s % 2].vm.p;
        mark(S, mk, 1);
        if (R) {
            CUDA_TRY(keep(R->pd[s], cur_pd, n, st));
            CUDA_TRY(keep(R->vm[s], cur_vm, n, st));
            CUDA_TRY(keep(R->start[s], (const uint32_t*)S->gb.start, size_t(S->ncells) + 2, st));
            R->has_perm[s] = s > 0;
            if (s > 0) CUDA_TRY(keep(R->perm[s], (const uint32_t*)S->gb.perm, n, st));
        }

        uint64_t sl = 0;
        if (sb) {
            SolidArgs a{};
            a.ref = S->ref.p;
            a.L = S->L.p;
            a.rl = SolidRefList{S->rl_off.p, S->rl_nbr.p, S->rl_gw.p, S->rl_nnz};
            a.ep = cur_ep;
            a.ep0 = ep_base;
            a.ep_next = last ? S->ep_t.p : S->ep_s[s % 2].p;
            a.ep_acc = S->ep_acc.p;
            a.ep_store = verlet ? S->ep_force.p : store_k ? S->ep_kst[s].p : nullptr;
            a.ep_prev0 = cp[0] != 0.f ? S->ep_kst[0].p : nullptr;
            a.ep_prev1 = cp[1] != 0.f ? S->ep_kst[1].p : nullptr;
            a.ep_prev2 = cp[2] != 0.f ? S->ep_kst[2].p : nullptr;
            a.F = S->F.p;
            a.A = S->A.p;
            a.ksol = S->ksol.p;
            a.contact_bound = S->contact_bound.p;
            a.counters_cleared = n > 0 ? 1 : 0;
            a.xs = xs;
            a.vs = vs;
            a.start = S->gb.start;
            a.sid_sorted = sid_sorted;
            a.ns = ns;
            a.all_order2 = S->all_order2 ? 1 : 0;
            a.any_plastic = S->any_plastic ? 1 : 0;
            a.sx = S->sx.p;
            a.sv = S->sv.p;
            a.sc = S->sc.p;
            a.stiff = S->have_stiff ? S->stiff.p : nullptr;
            sl = launch_solid(a, S->tables, c, st);
            S->launches += sl;
            cur_ep = a.ep_next;
            if (R) {
                CUDA_TRY(keep(R->F[s], (const float4*)S->F.p, 3 * size_t(ns), st));
                CUDA_TRY(keep(R->A[s], (const float4*)S->A.p, 3 * size_t(ns), st));
                CUDA_TRY(keep(R->sx[s], (const float4*)S->sx.p, ns, st));
                CUDA_TRY(keep(R->sv[s], (const float4*)S->sv.p, ns, st));
                CUDA_TRY(keep(R->sc[s], (const uint2*)S->sc.p, ns, st));
                CUDA_TRY(keep(R->cb[s], (const uint32_t*)S->contact_bound.p, 2, st));
                if (S->any_plastic) CUDA_TRY(keep(R->ep[s], a.ep, 4 * size_t(ns), st));
            }
        }
        mark(S, mk, 2);

        FluidArgs f{};
        f.xs = xs;
        f.vs = vs;
        f.start = S->gb.start;
        f.bxs = S->b_pd.p;
        f.bvs = S->b_vm.p;
        f.bstart = bstart;
        f.perm = perm;
        f.sid = S->sid.p;
        f.sid_of_boundary_index = S->sid_of_bidx.p;
        f.borig = S->b_orig.p;
        f.ps = S->ps.p;
        f.bps = S->bps.p;
        f.ksol = sb ? S->ksol.p : nullptr;
        f.n = n;
        f.solid_branch = sb ? 1 : 0;
        f.overflow = S->overflow.p;
        f.overflow_count = S->overflow_count.p;
        f.counters_cleared = 1;  // by this stage's grid build
        f.any_stiff_immobile = S->any_stiff_immobile ? 1 : 0;
        B.next_pd = next_pd;
        B.next_vm = next_vm;
        const int fl = launch_fluid(f, S->tables, S->kdim, c, B, S->fluid_variant, S->tile_counter.p, st);
        S->launches += fl;
        mark(S, mk, 3);
        if (S->profiling) {
            S->marks.push_back(mk);
            S->prof_l[0] += nl;
            S->prof_l[1] += sl;
            S->prof_l[2] += (uint64_t)fl;
            S->prof_stages++;
            nl = 0;
            mk = arp_sim::Mark{};
            if (S->marks.size() > 256) harvest_marks(S);
        }
        cur_pd = next_pd;
        cur_vm = next_vm;
    }
    if (!prime) {
        std::swap(S->Y, S->T);
        if (sb && S->any_plastic) std::swap(S->ep, S->ep_t);  // without plastic materials ep stays zero
    }
    if (verlet) S->vforce_valid = true;
    if (S->profiling) S->prof_steps++;
    return check_launch("step");
}

// Validate one scene and append it to the batch: particles, boundary and
// materials are concatenated in scene order, material ids remapped into the
// batch's table, the interaction matrix resolved into the scene's block.
arp_status append_scene(const arp_scene* sc, arp_sim* S) {
    if (!sc) return fail(ARP_ERR_INVALID_ARG, "scene is null");
    if (sc->n_materials == 0 || !sc->materials) return fail(ARP_ERR_INVALID_ARG, "scene has no materials");
    if (sc->n_materials > (uint32_t)kMaxMaterials)
        return fail(ARP_ERR_UNSUPPORTED, "more than 32 materials in one scene");
    if (sc->n_particles && !sc->particles) return fail(ARP_ERR_INVALID_ARG, "particles is null");
    if (sc->n_boundary && !sc->boundary) return fail(ARP_ERR_INVALID_ARG, "boundary is null");
    if (!(sc->kernel_radius > 0.0f) || !std::isfinite(sc->kernel_radius))
        return fail(ARP_ERR_INVALID_ARG, "kernel_radius must be positive");
    if (!std::isfinite(sc->timestep)) return fail(ARP_ERR_INVALID_ARG, "timestep must be finite");
    Tableau tab;
    if (!make_tableau(sc->integrator, tab)) return fail(ARP_ERR_INVALID_ARG, "unknown integrator id");
    if (sc->bounds.dim[3] > 0.0f) return fail(ARP_ERR_UNSUPPORTED, "4-dimensional boxes are not supported");
    for (int a = 0; a < 4; ++a)
        if (!std::isfinite(sc->bounds.min[a]) || !std::isfinite(sc->bounds.dim[a]) || sc->bounds.dim[a] < 0.0f)
            return fail(ARP_ERR_INVALID_ARG, "bounds must be finite with non-negative extent");
    const uint32_t subticks = sc->subticks ? sc->subticks : 1;
    const bool first = S->scenes.empty();
    if (first) {
        S->tab = tab;
        S->integrator = sc->integrator;
        S->timestep = sc->timestep;
        S->subticks = subticks;
        S->dt_sub = sc->timestep / (float)subticks;
        S->h = sc->kernel_radius;
    } else if (sc->integrator != S->integrator || sc->timestep != S->timestep || subticks != S->subticks) {
        return fail(ARP_ERR_UNSUPPORTED, "all scenes of a batch must share integrator, time step and subticks");
    }
    uint32_t dim = 0;
    for (int a = 0; a < 4; ++a)
        if (sc->bounds.dim[a] > 0.0f) dim++;
    if (dim == 0) return fail(ARP_ERR_INVALID_ARG, "bounds have no extent");
    if (first) S->dim = dim;

    arp_sim::SceneHost H{};
    H.p_base = S->n;
    H.n = sc->n_particles;
    H.b_base = S->nb;
    H.nb = sc->n_boundary;
    H.mat_base = S->M;
    H.nmat = sc->n_materials;
    H.inter_base = (uint32_t)S->inter.size();
    H.bounds = sc->bounds;
    H.h = sc->kernel_radius;
    H.gravity = sc->gravity;
    H.alpha = sc->artificial_viscocity;
    const uint32_t scene_idx = (uint32_t)S->scenes.size();
    const uint32_t M = sc->n_materials;
    const arp_material* mats = sc->materials;

    bool flat_z = sc->bounds.dim[2] == 0.0f;
    float z0 = 0.0f;
    bool have_z = false;
    auto check_p = [&](const arp_particle& p, bool boundary) -> arp_status {
        if (p.mat >= M) return fail(ARP_ERR_INVALID_ARG, "particle material index out of range");
        const bool imm = mats[p.mat].immobile != 0;
        if (imm != boundary)
            return fail(ARP_ERR_INVALID_ARG, boundary ? "boundary particle uses a mobile material"
                                                      : "mobile particle uses an immobile material");
        if (!std::isfinite(p.pos[3])) return fail(ARP_ERR_INVALID_ARG, "non-finite w coordinate");
        if (!S->have_w) {
            S->pos_w = p.pos[3];
            S->have_w = true;
        } else if (p.pos[3] != S->pos_w) {
            return fail(ARP_ERR_UNSUPPORTED, "positions must share one w coordinate (4D motion is not supported)");
        }
        if (p.vel[3] != 0.0f) return fail(ARP_ERR_UNSUPPORTED, "velocities must have zero w component");
        if (!have_z) {
            z0 = p.pos[2];
            have_z = true;
        } else if (p.pos[2] != z0) {
            flat_z = false;
        }
        if (p.vel[2] != 0.0f) flat_z = false;
        return ARP_OK;
    };
    for (uint32_t i = 0; i < sc->n_particles; ++i) ARP_TRY(check_p(sc->particles[i], false));
    for (uint32_t i = 0; i < sc->n_boundary; ++i) ARP_TRY(check_p(sc->boundary[i], true));
    H.flat_z = flat_z;
    for (uint32_t i = 0; i < sc->n_particles; ++i) {
        arp_particle p = sc->particles[i];
        p.mat += H.mat_base;
        S->host_particles.push_back(p);
    }
    for (uint32_t i = 0; i < sc->n_boundary; ++i) {
        arp_particle p = sc->boundary[i];
        p.mat += H.mat_base;
        S->host_boundary.push_back(p);
    }
    for (uint32_t i = 0; i < M; ++i) {
        S->mats.push_back(mats[i]);
        S->scene_of_material.push_back(scene_idx);
        if (mats[i].immobile && is_stiff(mats[i])) S->any_stiff_immobile = true;
        if (is_stiff(mats[i]) && mats[i].strain_order != 2) S->all_order2 = false;
        if (is_stiff(mats[i]) && mats[i].plastic) S->any_plastic = true;
    }
    // mod.rs:93-111 interaction matrix of the scene
    std::vector<arp_interaction> block(size_t(M) * M, arp_interaction{0, 0, 0, 0, 0});
    auto given = [&](uint32_t i, uint32_t j) -> bool {
        if (!sc->interactions) return false;
        if (!sc->interaction_given) return true;
        return sc->interaction_given[size_t(i) * M + j] != 0;
    };
    for (uint32_t i = 0; i < M; ++i)
        for (uint32_t j = i; j < M; ++j) {
            arp_interaction x{0, 0, 0, 0, 0};
            if (given(i, j)) x = sc->interactions[size_t(i) * M + j];
            else if (given(j, i)) x = sc->interactions[size_t(j) * M + i];
            else if (i != j) {
                const arp_material& a = mats[i];
                const arp_material& b = mats[j];
                if (a.state_eq != ARP_EOS_ZERO && b.state_eq != ARP_EOS_ZERO) x = arp_interaction{0, 0, 0, 0, 0};
                else x = arp_interaction{ARP_CONTACT_LINEAR, 10000.0f, sc->kernel_radius * 2.0f, 0.0f, a.visc + b.visc};
            }
            block[size_t(i) * M + j] = x;
            block[size_t(j) * M + i] = x;
        }
    S->inter.insert(S->inter.end(), block.begin(), block.end());
    // particles within h of a particle, ~ (h / s)^dim with s = (m / rho0)^(1/dim) the mean spacing
    if (sc->n_particles > 0 && dim > 0) {
        double vol = 0.0;
        for (uint32_t i = 0; i < sc->n_particles; ++i) {
            const arp_material& m = mats[sc->particles[i].mat];
            vol += m.start_den > 0.0f ? (double)m.mass / (double)m.start_den : 0.0;
        }
        const double s = std::pow(vol / sc->n_particles, 1.0 / dim);
        H.dense = s > 0.0 && std::pow((double)H.h / s, (double)dim) >= kDenseNeighbors;
    }
    ARP_TRY(scene_params(H, dim));
    if ((uint64_t)S->ncells + H.sp.sgrid.ncells + 2 > (1ull << 31))
        return fail(ARP_ERR_UNSUPPORTED, "the batch's grids have more than 2^31 cells");
    H.sp.cell_base = S->ncells;
    S->ncells += H.sp.sgrid.ncells;
    H.sp.ccell_base = S->nccells;
    S->nccells += H.sp.grid.ncells;
    S->n += H.n;
    S->nb += H.nb;
    S->M += M;
    S->max_nmat = std::max(S->max_nmat, M);
    S->scenes.push_back(H);
    return ARP_OK;
}

// Solid ids in particle order for stiff materials (particles.rs:488-506), in
// the concatenated caller order of the batch.  `creating` marks the first call
// for a handle, which decides each scene's placeholder solid entry.
void finalize_scenes(arp_sim* S, bool creating) {
    bool all_flat = true;
    for (const auto& H : S->scenes) all_flat = all_flat && H.flat_z;
    S->kdim = all_flat ? 2 : 3;
    S->sid_of_caller.assign(S->n, kInvalid);
    S->part_of_solid.clear();
    for (uint32_t i = 0; i < S->n; ++i)
        if (is_stiff(S->mats[S->host_particles[i].mat])) {
            S->sid_of_caller[i] = (uint32_t)S->part_of_solid.size();
            S->part_of_solid.push_back(i);
        }
    S->ns = (uint32_t)S->part_of_solid.size();
    uint32_t base = 0;
    S->any_solid_branch = false;
    for (auto& H : S->scenes) {
        uint32_t cnt = 0;
        for (uint32_t i = H.p_base; i < H.p_base + H.n; ++i) cnt += S->sid_of_caller[i] != kInvalid;
        if (creating) H.dummy_solid = cnt == 0 ? 1u : 0u;
        H.sp.solid_branch = cnt + H.dummy_solid > 1 ? 1u : 0u;
        S->any_solid_branch = S->any_solid_branch || H.sp.solid_branch;
        H.s_base = base;
        base += cnt;
    }
}

arp_status allocate(arp_sim* S) {
    const size_t n = std::max(S->n, 1u), nb = std::max(S->nb, 1u), ns = std::max(S->ns, 1u);
    const size_t nc = S->ncells;
    ARP_TRY(alloc_state(S->Y, n));
    ARP_TRY(alloc_state(S->T, n));
    ARP_TRY(alloc_state(S->S[0], n));
    if (S->tab.stages > 2) ARP_TRY(alloc_state(S->S[1], n));
    ARP_TRY(alloc_state(S->X, n));
    ARP_TRY(alloc_state(S->acc, n));
    if (S->verlet()) {
        ARP_TRY(alloc_state(S->vforce, n));
        CUDA_TRY(S->ep_force.alloc(4 * ns));
    }
    for (int j = 0; j < S->tab.stages; ++j) {
        bool needed = false;
        for (int t = j + 2; t < S->tab.stages; ++t)
            if (S->tab.a[t][j] != 0.0) needed = true;
        if (needed) ARP_TRY(alloc_state(S->kst[j], n));
    }
    CUDA_TRY(S->orig.alloc(n));
    CUDA_TRY(S->orig_r.alloc(n));
    CUDA_TRY(S->sid.alloc(n));
    CUDA_TRY(S->sid_r.alloc(n));
    CUDA_TRY(S->sid_sorted.alloc(n));
    CUDA_TRY(S->slot_of.alloc(ns));
    CUDA_TRY(S->ps.alloc(n));
    CUDA_TRY(S->sid_of_caller_d.alloc(n));
    CUDA_TRY(S->mat_of_caller_d.alloc(n));
    CUDA_TRY(S->check_flag.alloc(1));
    {
        std::vector<uint32_t> mo(S->n);
        for (uint32_t i = 0; i < S->n; ++i) mo[i] = S->host_particles[i].mat;
        if (S->n)
            CUDA_TRY(cudaMemcpy(S->mat_of_caller_d.p, mo.data(), S->n * sizeof(uint32_t), cudaMemcpyHostToDevice));
    }
    if (S->n)
        CUDA_TRY(cudaMemcpy(S->sid_of_caller_d.p, S->sid_of_caller.data(), S->n * sizeof(uint32_t),
                            cudaMemcpyHostToDevice));
    CUDA_TRY(S->bps.alloc(nb));
    CUDA_TRY(S->b_pd.alloc(nb));
    CUDA_TRY(S->b_vm.alloc(nb));
    CUDA_TRY(S->b_orig.alloc(nb));
    CUDA_TRY(S->b_start.alloc(nc + 2));
    CUDA_TRY(S->sid_of_bidx.alloc(nb));
    CUDA_TRY(S->ref.alloc(ns));
    CUDA_TRY(S->mat_of_solid.alloc(ns));
    CUDA_TRY(S->L.alloc(3 * ns));
    CUDA_TRY(S->F.alloc(3 * ns));
    CUDA_TRY(S->A.alloc(3 * ns));
    CUDA_TRY(S->ksol.alloc(ns));
    CUDA_TRY(S->contact_bound.alloc(2));
    CUDA_TRY(S->tile_counter.alloc(1));
    CUDA_TRY(S->overflow.alloc(2 * n));  // two queues of n entries
    CUDA_TRY(S->overflow_count.alloc(2));
    CUDA_TRY(S->ep.alloc(4 * ns));
    CUDA_TRY(S->ep_t.alloc(4 * ns));
    CUDA_TRY(S->sx.alloc(ns));
    CUDA_TRY(S->sv.alloc(ns));
    CUDA_TRY(S->sc.alloc(ns));
    CUDA_TRY(S->ep_s[0].alloc(4 * ns));
    CUDA_TRY(S->ep_s[1].alloc(4 * ns));
    CUDA_TRY(S->ep_acc.alloc(4 * ns));
    for (int j = 0; j < 4; ++j)
        if (S->kst[j].pd.p) CUDA_TRY(S->ep_kst[j].alloc(4 * ns));
    CUDA_TRY(S->d_stats.alloc(1));
    CUDA_TRY(cudaMemset(S->d_stats.p, 0, sizeof(DevStats)));
    // materials
    std::vector<DevMat> dm(S->M);
    for (uint32_t i = 0; i < S->M; ++i) {
        const arp_material& m = S->mats[i];
        DevMat d{};
        d.mass = m.mass; d.start_den = m.start_den; d.sound_speed = m.sound_speed; d.target_den = m.target_den;
        d.visc = m.visc; d.bulk_visc = m.bulk_visc; d.lam = m.normal_stiffness; d.mu = m.shear_stiffness;
        d.lam_d = m.normal_damp; d.mu_d = m.shear_damp; d.yield_strength = m.yield_strength;
        d.work_hardening = m.work_hardening; d.work_hardening_exp = m.work_hardening_exp;
        d.kinematic_hardening = m.kinematic_hardening; d.relaxation_time = m.relaxation_time;
        d.vol0 = m.mass / m.start_den;
        d.state_eq = m.state_eq; d.stiff = is_stiff(m) ? 1u : 0u; d.plastic = m.plastic ? 1u : 0u;
        d.strain_order = m.strain_order;
        d.scene = S->scene_of_material[i];
        d.local = i - S->scenes[d.scene].mat_base;
        d.solid_base = S->scenes[d.scene].s_base - S->scenes[d.scene].dummy_solid;  // reported id = global - base
        dm[i] = d;
    }
    CUDA_TRY(S->d_mats.alloc(S->M));
    CUDA_TRY(cudaMemcpy(S->d_mats.p, dm.data(), S->M * sizeof(DevMat), cudaMemcpyHostToDevice));
    std::vector<FluidMat> fm(S->M);
    for (uint32_t i = 0; i < S->M; ++i)
        fm[i] = FluidMat{dm[i].mass, dm[i].sound_speed, dm[i].target_den, dm[i].visc, dm[i].bulk_visc, dm[i].state_eq,
                         dm[i].stiff, 0u};
    CUDA_TRY(S->d_fmats.alloc(S->M));
    CUDA_TRY(cudaMemcpy(S->d_fmats.p, fm.data(), S->M * sizeof(FluidMat), cudaMemcpyHostToDevice));
    std::vector<SceneP> sp;
    for (const auto& H : S->scenes) sp.push_back(H.sp);
    CUDA_TRY(S->d_scenes.alloc(sp.size()));
    CUDA_TRY(cudaMemcpy(S->d_scenes.p, sp.data(), sp.size() * sizeof(SceneP), cudaMemcpyHostToDevice));
    std::vector<DevInter> di(S->inter.size());
    for (size_t i = 0; i < di.size(); ++i) {
        const arp_interaction& x = S->inter[i];
        di[i] = DevInter{x.potential, x.strength, x.radius, x.dampening, x.friction};
    }
    CUDA_TRY(S->d_inter.alloc(di.size()));
    CUDA_TRY(cudaMemcpy(S->d_inter.p, di.data(), di.size() * sizeof(DevInter), cudaMemcpyHostToDevice));
    S->tables.scenes = S->d_scenes.p;
    S->tables.mats = S->d_mats.p;
    S->tables.fmats = S->d_fmats.p;
    S->tables.inter = S->d_inter.p;
    S->tables.ncells = S->ncells;
    S->tables.max_nmat = S->max_nmat;
    S->tables.nscenes = (uint32_t)S->scenes.size();
    return ARP_OK;
}

// ---- autotuner -----------------------------------------------------------------
// Chooses the fluid kernel's launch shape (hit-list capacity, one tile per
// block or persistent tile queue) by timing every variant on the live stage-0
// state.  All variants evaluate the same pairs in the same order, so the
// choice changes speed, never results.  Choices are cached per (kernel
// dimension, log2 particle count, quarter-octave of h / particle spacing).
std::mutex g_tune_mu;
std::map<std::tuple<int, int, int>, int> g_tune_cache;

std::tuple<int, int, int> tune_key(const arp_sim* S) {
    double acc = 0.0;
    for (uint32_t i = 0; i < S->n; ++i) {
        const uint32_t m = S->host_particles[i].mat;
        const auto& H = S->scenes[S->scene_of_material[m]];
        const double vol = (double)S->mats[m].mass / (double)S->mats[m].start_den;
        const double spacing = vol > 0 ? std::pow(vol, 1.0 / std::max(1u, H.sp.dim)) : H.h;
        acc += std::log2((double)H.h / spacing);
    }
    const double ratio = S->n ? acc / S->n : 0.0;
    const int nbits = S->n ? (int)std::ceil(std::log2((double)S->n)) : 0;
    return std::make_tuple(S->kdim, nbits, (int)std::lround(4.0 * ratio));
}

arp_status run_autotune(arp_sim* S, bool force) {
    const auto key = tune_key(S);
    if (!force) {
        std::lock_guard<std::mutex> lock(g_tune_mu);
        auto it = g_tune_cache.find(key);
        if (it != g_tune_cache.end()) {
            S->fluid_variant = it->second;
            return ARP_OK;
        }
    }
    const uint32_t n = S->n;
    if (n == 0) return ARP_OK;
    cudaStream_t st = S->stream;
    // stage-0 inputs: y0 sorted into cell order (the state itself is unchanged)
    S->launches += build_grid(S->Y.pd.p, S->Y.vm.p, nullptr, n, S->tables, S->gb, nullptr, S->b_start.p, st);
    S->launches += gather_state(S->gb.perm, n, S->Y.pd.p, S->T.pd.p, S->Y.vm.p, S->T.vm.p, S->orig.p, S->orig_r.p,
                                S->sid.p, S->sid_r.p, nullptr, nullptr, S->ps.p, S->d_mats.p, st);
    std::swap(S->Y, S->T);
    std::swap(S->orig, S->orig_r);
    std::swap(S->sid, S->sid_r);
    if (S->verlet() && S->vforce_valid) {  // the carried force record follows the reorder
        S->launches += gather_sorted(S->gb.perm, n, S->vforce.pd.p, S->X.pd.p, S->vforce.vm.p, S->X.vm.p, nullptr,
                                     nullptr, nullptr, nullptr, st);
        std::swap(S->vforce, S->X);
    }
    const Tableau& tab = S->tab;
    const bool last = tab.stages == 1;
    StageCoefs c{};
    c.last = last ? 1 : 0;
    if (!last) c.c_self = (float)(tab.a[1][0] * (double)S->dt_sub);
    c.c_acc = (float)(tab.b[0] * (double)S->dt_sub);
    c.acc_first = 1;
    StageBuffers B{};
    B.y0_pd = S->Y.pd.p;
    B.y0_vm = S->Y.vm.p;
    B.acc_pd = S->acc.pd.p;
    B.acc_vm = S->acc.vm.p;
    B.next_pd = last ? S->T.pd.p : S->S[0].pd.p;  // scratch at this point
    B.next_vm = last ? S->T.vm.p : S->S[0].vm.p;
    FluidArgs f{};
    f.xs = S->Y.pd.p;
    f.vs = S->Y.vm.p;
    f.start = S->gb.start;
    f.bxs = S->b_pd.p;
    f.bvs = S->b_vm.p;
    f.bstart = S->b_start.p;
    f.sid = S->sid.p;
    f.sid_of_boundary_index = S->sid_of_bidx.p;
    f.borig = S->b_orig.p;
    f.ps = S->ps.p;
    f.bps = S->bps.p;
    f.n = n;
    f.any_stiff_immobile = S->any_stiff_immobile ? 1 : 0;
    f.overflow = S->overflow.p;
    f.overflow_count = S->overflow_count.p;
    cudaEvent_t e0 = take_event(S), e1 = take_event(S);
    float best = 1e30f;
    int best_v = 0;
    for (int v = 0; v < kNumFluidVariants; ++v) {
        S->launches += launch_fluid(f, S->tables, S->kdim, c, B, v, S->tile_counter.p, st);  // warm-up
        CUDA_TRY(cudaEventRecord(e0, st));
        for (int r = 0; r < 3; ++r) S->launches += launch_fluid(f, S->tables, S->kdim, c, B, v, S->tile_counter.p, st);
        CUDA_TRY(cudaEventRecord(e1, st));
        CUDA_TRY(cudaEventSynchronize(e1));
        float ms = 0;
        CUDA_TRY(cudaEventElapsedTime(&ms, e0, e1));
        if (ms < best) {
            best = ms;
            best_v = v;
        }
    }
    S->ev_free.push_back(e0);
    S->ev_free.push_back(e1);
    ARP_TRY(check_launch("autotune"));
    S->fluid_variant = best_v;
    std::lock_guard<std::mutex> lock(g_tune_mu);
    g_tune_cache[key] = best_v;
    return ARP_OK;
}

arp_status need_init(const arp_sim* S) {
    if (!S) return fail(ARP_ERR_INVALID_ARG, "sim is null");
    if (!S->initialized) return fail(ARP_ERR_INVALID_ARG, "arp_sim_init must be called first");
    return ARP_OK;
}

}  // namespace

extern "C" {

const char* arp_last_error(void) { return g_last_error.c_str(); }
uint32_t arp_abi_version(void) { return ARP_ABI_VERSION; }

arp_status arp_sim_create_batch(const arp_scene* scenes, uint32_t count, arp_sim** out) {
    g_last_error.clear();
    if (!out) return fail(ARP_ERR_INVALID_ARG, "out is null");
    *out = nullptr;
    if (!scenes || count == 0) return fail(ARP_ERR_INVALID_ARG, scenes ? "no scenes" : "scene is null");
    arp_sim* S = new (std::nothrow) arp_sim();
    if (!S) return fail(ARP_ERR_OUT_OF_MEMORY, "host allocation failed");
    arp_status s = ARP_OK;
    for (uint32_t k = 0; k < count && s == ARP_OK; ++k) s = append_scene(&scenes[k], S);
    if (s == ARP_OK) {
        finalize_scenes(S, true);
        cudaError_t e = cudaStreamCreateWithFlags(&S->own_stream, cudaStreamNonBlocking);
        if (e != cudaSuccess) s = fail(ARP_ERR_CUDA, std::string("cudaStreamCreate: ") + cudaGetErrorString(e));
        S->stream = S->own_stream;
    }
    if (s == ARP_OK) s = allocate(S);
    if (s != ARP_OK) {
        delete S;
        return s;
    }
    *out = S;
    return ARP_OK;
}

arp_status arp_sim_create(const arp_scene* scene, arp_sim** out) {
    if (!scene) {
        if (out) *out = nullptr;
        return fail(ARP_ERR_INVALID_ARG, "scene is null");
    }
    return arp_sim_create_batch(scene, 1, out);
}

arp_status arp_sim_num_scenes(const arp_sim* sim, uint32_t* out) {
    if (!sim || !out) return fail(ARP_ERR_INVALID_ARG, "null argument");
    *out = (uint32_t)sim->scenes.size();
    return ARP_OK;
}

arp_status arp_sim_scene_range(const arp_sim* sim, uint32_t scene, uint32_t* first_particle, uint32_t* n_particles,
                               uint32_t* first_boundary, uint32_t* n_boundary, uint32_t* first_cell,
                               uint32_t* n_cells) {
    if (!sim) return fail(ARP_ERR_INVALID_ARG, "sim is null");
    if (scene >= sim->scenes.size()) return fail(ARP_ERR_INVALID_ARG, "scene index out of range");
    const auto& H = sim->scenes[scene];
    if (first_particle) *first_particle = H.p_base;
    if (n_particles) *n_particles = H.n;
    if (first_boundary) *first_boundary = H.b_base;
    if (n_boundary) *n_boundary = H.nb;
    if (first_cell) *first_cell = H.sp.ccell_base;
    if (n_cells) *n_cells = H.sp.grid.ncells;
    return ARP_OK;
}

arp_status arp_sim_create_from_toml(const char* path, arp_sim** out) {
    g_last_error.clear();
    if (!path || !out) return fail(ARP_ERR_INVALID_ARG, "null argument");
    *out = nullptr;
    arp::LoadedScene ls;
    std::string err;
    arp_status s = arp::load_scene_toml(path, ls, err);
    if (s != ARP_OK) return fail(s, err);
    arp_scene sc = ls.as_scene();
    return arp_sim_create(&sc, out);
}

struct arp_scene_file {
    arp::LoadedScene scene;
    mutable std::vector<float> densities;  // ramp centres handed out by arp_scene_file_render_settings
};

arp_status arp_scene_file_load(const char* path, arp_scene_file** out) {
    g_last_error.clear();
    if (!path || !out) return fail(ARP_ERR_INVALID_ARG, "null argument");
    *out = nullptr;
    auto f = std::make_unique<arp_scene_file>();
    std::string err;
    arp_status s = arp::load_scene_toml(path, f->scene, err);
    if (s != ARP_OK) return fail(s, err);
    *out = f.release();
    return ARP_OK;
}

arp_status arp_scene_file_scene(const arp_scene_file* file, arp_scene* out) {
    if (!file || !out) return fail(ARP_ERR_INVALID_ARG, "null argument");
    *out = file->scene.as_scene();
    return ARP_OK;
}

arp_status arp_scene_file_name(const arp_scene_file* file, const char** name) {
    if (!file || !name) return fail(ARP_ERR_INVALID_ARG, "null argument");
    *name = file->scene.name.c_str();
    return ARP_OK;
}

arp_status arp_scene_file_on_click_count(const arp_scene_file* file, uint32_t* count) {
    if (!file || !count) return fail(ARP_ERR_INVALID_ARG, "null argument");
    *count = (uint32_t)file->scene.on_click.size();
    return ARP_OK;
}

arp_status arp_scene_file_on_click(const arp_scene_file* file, uint32_t index, const arp_particle** particles,
                                   uint32_t* n, arp_material* material, int* relative) {
    if (!file) return fail(ARP_ERR_INVALID_ARG, "null argument");
    if (index >= file->scene.on_click.size()) return fail(ARP_ERR_INVALID_ARG, "on_click index out of range");
    const auto& a = file->scene.on_click[index];
    if (particles) *particles = a.particles.data();
    if (n) *n = (uint32_t)a.particles.size();
    if (material) *material = a.material;
    if (relative) *relative = a.relative ? 1 : 0;
    return ARP_OK;
}

arp_status arp_scene_file_render_settings(const arp_scene_file* file, arp_view* view, arp_render_style* style) {
    if (!file || !view || !style) return fail(ARP_ERR_INVALID_ARG, "null argument");
    const auto& S = file->scene;
    view->angle = (float)S.view_angle;
    view->pos[0] = (float)S.view_pos[0];
    view->pos[1] = (float)S.view_pos[1];
    view->scale = (float)S.view_scale;
    style->render_h = S.render_h;
    style->lighting = S.lighting ? 1 : 0;
    for (int k = 0; k < 3; ++k) {
        style->light_pos[k] = S.light_pos[k];
        style->light_color[k] = S.light_color[k];
    }
    style->ambient = S.ambient;
    style->diffuse = S.diffuse;
    style->specular = S.specular;
    style->n_materials = (uint32_t)S.materials.size();
    style->colors = S.colors.data();
    file->densities.resize(S.materials.size());
    for (size_t m = 0; m < S.materials.size(); ++m) file->densities[m] = S.materials[m].start_den;
    style->densities = file->densities.data();
    return ARP_OK;
}

arp_status arp_scene_file_free(arp_scene_file* file) {
    delete file;
    return ARP_OK;
}

arp_status arp_sim_destroy(arp_sim* sim) {
    if (!sim) return ARP_OK;
    if (sim->stream) cudaStreamSynchronize(sim->stream);
    delete sim;
    return ARP_OK;
}

arp_status arp_sim_init(arp_sim* sim) {
    if (!sim) return fail(ARP_ERR_INVALID_ARG, "sim is null");
    ARP_TRY(do_init(sim));
    return run_autotune(sim, false);
}

arp_status arp_sim_autotune(arp_sim* sim, int* variant) {
    ARP_TRY(need_init(sim));
    sim->drop_graph();
    ARP_TRY(run_autotune(sim, true));
    if (variant) *variant = sim->fluid_variant;
    return ARP_OK;
}

arp_status arp_sim_set_fluid_variant(arp_sim* sim, int variant) {
    if (!sim) return fail(ARP_ERR_INVALID_ARG, "sim is null");
    if (variant < 0 || variant >= kNumFluidVariants) return fail(ARP_ERR_INVALID_ARG, "variant out of range");
    sim->drop_graph();
    sim->fluid_variant = variant;
    return ARP_OK;
}

int arp_fluid_variant_count(void) { return kNumFluidVariants; }

arp_status arp_sim_fluid_variant(const arp_sim* sim, int* variant, int* block, int* persistent) {
    // (the hit-list capacity of the shape is kFluidVariants[variant].cap)
    if (!sim) return fail(ARP_ERR_INVALID_ARG, "sim is null");
    if (variant) *variant = sim->fluid_variant;
    if (block) *block = kFluidVariants[sim->fluid_variant].block;
    if (persistent) *persistent = kFluidVariants[sim->fluid_variant].persistent;
    return ARP_OK;
}

// The buffer pointers a step's launches depend on and swaps.
static void step_signature(const arp_sim* S, const void* sig[4]) {
    sig[0] = S->Y.pd.p;
    sig[1] = S->orig.p;
    sig[2] = S->sid.p;
    sig[3] = S->ep.p;
}

// Capture one step on the handle's stream into the graph slot `k`; the host
// side of the step (buffer swaps, time, launch count) happens here, so the
// caller launches the graph once to run the step it stands for.
arp_status capture_step_graph(arp_sim* S, int k) {
    arp_sim::StepGraph& G = S->graphs[k];
    if (G.exec) cudaGraphExecDestroy(G.exec);
    if (G.g) cudaGraphDestroy(G.g);
    G = arp_sim::StepGraph{};
    step_signature(S, G.sig);
    const uint64_t l0 = S->launches;
    const bool prof = S->prof_on;
    S->prof_on = false;
    CUDA_TRY(cudaStreamBeginCapture(S->stream, cudaStreamCaptureModeThreadLocal));
    arp_status st = do_step(S);
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(S->stream, &g);
    S->prof_on = prof;
    G.launches = S->launches - l0;
    if (st != ARP_OK) {
        if (g) cudaGraphDestroy(g);
        S->drop_graph();
        return st;
    }
    if (e != cudaSuccess) {
        S->drop_graph();
        return fail(ARP_ERR_CUDA, std::string("cudaStreamEndCapture: ") + cudaGetErrorString(e));
    }
    G.g = g;
    e = cudaGraphInstantiate(&G.exec, g, 0);
    if (e != cudaSuccess) {
        S->drop_graph();
        return fail(ARP_ERR_CUDA, std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e));
    }
    S->graph_stream = S->stream;
    return ARP_OK;
}

// One step from a graph: replay the graph captured for the current buffer
// pointers (capturing it first if there is none) and apply the step's host
// side: the buffer swaps of do_step, time and launch count.
arp_status graph_step(arp_sim* S) {
    if (S->graph_stream != S->stream) S->drop_graph();
    const void* sig[4];
    step_signature(S, sig);
    int k = -1, free_slot = -1;
    for (int q = 0; q < 2; ++q) {
        const auto& G = S->graphs[q];
        if (G.exec && std::equal(sig, sig + 4, G.sig)) k = q;
        if (!G.exec && free_slot < 0) free_slot = q;
    }
    if (k < 0) {  // capture; do_step's host side happens during the capture
        k = free_slot >= 0 ? free_slot : 0;
        const float t = S->time;
        ARP_TRY(capture_step_graph(S, k));
        S->time = t;
    } else {
        std::swap(S->orig, S->orig_r);
        std::swap(S->sid, S->sid_r);
        if (S->solid_branch() && S->any_plastic) std::swap(S->ep, S->ep_t);
        S->launches += S->graphs[k].launches;
    }
    CUDA_TRY(cudaGraphLaunch(S->graphs[k].exec, S->stream));
    S->time += S->dt_sub;
    if (S->prof_on) S->prof_phase++;  // a step not sampled by the profiler
    return ARP_OK;
}

arp_status arp_sim_step(arp_sim* sim, uint32_t nsteps) {
    ARP_TRY(need_init(sim));
    for (uint32_t i = 0; i < nsteps; ++i) {
        const bool sampled = sim->prof_on && sim->prof_phase % sim->prof_every == 0;
        const bool graphed = sim->use_graph && !sim->tape && !sampled;
        // velocity Verlet starts from a force evaluation at the current state:
        // plain launches before a graphed step (the graph replays only steps
        // that carry the record); a plain step makes it itself
        if (graphed && sim->verlet() && !sim->vforce_valid) ARP_TRY(do_step(sim, true));
        if (graphed) ARP_TRY(graph_step(sim));
        else ARP_TRY(do_step(sim));
    }
    return ARP_OK;
}

arp_status arp_sim_set_graph(arp_sim* sim, int enable) {
    if (!sim) return fail(ARP_ERR_INVALID_ARG, "sim is null");
    if (!enable) sim->drop_graph();
    sim->use_graph = enable != 0;
    return ARP_OK;
}

arp_status arp_sim_update(arp_sim* sim) {
    ARP_TRY(need_init(sim));
    return arp_sim_step(sim, sim->subticks);
}

arp_status arp_sim_time(const arp_sim* sim, float* out) {
    if (!sim || !out) return fail(ARP_ERR_INVALID_ARG, "null argument");
    *out = sim->time;
    return ARP_OK;
}
arp_status arp_sim_kernel_radius(const arp_sim* sim, float* out) {
    if (!sim || !out) return fail(ARP_ERR_INVALID_ARG, "null argument");
    *out = sim->h;
    return ARP_OK;
}
arp_status arp_sim_num_materials(const arp_sim* sim, uint32_t* out) {
    if (!sim || !out) return fail(ARP_ERR_INVALID_ARG, "null argument");
    *out = sim->M;
    return ARP_OK;
}
arp_status arp_sim_counts(const arp_sim* sim, uint32_t* n, uint32_t* nb, uint32_t* ns) {
    if (!sim) return fail(ARP_ERR_INVALID_ARG, "sim is null");
    if (n) *n = sim->n;
    if (nb) *nb = sim->nb;
    if (ns) *ns = sim->ns;
    return ARP_OK;
}
arp_status arp_sim_dim(const arp_sim* sim, uint32_t* out) {
    if (!sim || !out) return fail(ARP_ERR_INVALID_ARG, "null argument");
    *out = sim->dim;
    return ARP_OK;
}

arp_status arp_sim_get_particles(arp_sim* sim, arp_particle* out, uint32_t cap) {
    if (!sim || (!out && sim->n)) return fail(ARP_ERR_INVALID_ARG, "null argument");
    if (cap < sim->n) return fail(ARP_ERR_CAPACITY, "output holds fewer records than n_particles");
    if (!sim->initialized) {
        std::memcpy(out, sim->host_particles.data(), sim->n * sizeof(arp_particle));
        for (uint32_t i = 0; i < sim->n; ++i) {
            const auto& H = sim->scenes[sim->scene_of_material[out[i].mat]];
            const uint32_t sg = sim->sid_of_caller[i];
            out[i].solid_id = sg == kInvalid ? sg : sg - (H.s_base - H.dummy_solid);
            out[i].mat -= H.mat_base;
        }
        return ARP_OK;
    }
    const uint32_t n = sim->n;
    if (!sim->records.p) CUDA_TRY(sim->records.alloc(n));
    sim->launches += soa_to_records(sim->Y.pd.p, sim->Y.vm.p, sim->orig.p, sim->sid.p, n, sim->pos_w, sim->d_mats.p,
                                    sim->records.p, sim->stream);
    if (n) CUDA_TRY(cudaMemcpyAsync(out, sim->records.p, n * sizeof(arp_particle), cudaMemcpyDeviceToHost, sim->stream));
    CUDA_TRY(cudaStreamSynchronize(sim->stream));
    return check_launch("get_particles");
}

arp_status arp_sim_get_solids(arp_sim* sim, arp_solid_particle* out, uint32_t cap) {
    if (!sim || (!out && sim->ns)) return fail(ARP_ERR_INVALID_ARG, "null argument");
    if (cap < sim->ns) return fail(ARP_ERR_CAPACITY, "output holds fewer records than n_solids");
    const uint32_t ns = sim->ns;
    std::vector<float4> ep(4 * size_t(ns));
    if (sim->initialized && ns) {
        CUDA_TRY(cudaMemcpyAsync(ep.data(), sim->ep.p, 4 * ns * sizeof(float4), cudaMemcpyDeviceToHost, sim->stream));
        CUDA_TRY(cudaStreamSynchronize(sim->stream));
    }
    for (uint32_t s = 0; s < ns; ++s) {
        arp_solid_particle& r = out[s];
        std::memset(&r, 0, sizeof(r));
        const uint32_t caller = sim->part_of_solid[s];
        const arp_particle& p = sim->host_particles[caller];
        r.part_id = caller - sim->scenes[sim->scene_of_material[p.mat]].p_base;  // index inside its scene
        if (s < sim->host_ref.size()) {
            r.ref_pos[0] = sim->host_ref[s].x;
            r.ref_pos[1] = sim->host_ref[s].y;
            r.ref_pos[2] = sim->host_ref[s].z;
        } else {
            for (int a = 0; a < 3; ++a) r.ref_pos[a] = p.pos[a];
        }
        r.ref_pos[3] = sim->pos_w;
        for (int c = 0; c < 4; ++c) {
            r.stress[4 * c + 0] = ep[4 * s + c].x;
            r.stress[4 * c + 1] = ep[4 * s + c].y;
            r.stress[4 * c + 2] = ep[4 * s + c].z;
            r.stress[4 * c + 3] = ep[4 * s + c].w;
        }
    }
    return ARP_OK;
}

arp_status arp_sim_get_boundary(arp_sim* sim, arp_particle* out, uint32_t cap) {
    if (!sim || (!out && sim->nb)) return fail(ARP_ERR_INVALID_ARG, "null argument");
    if (cap < sim->nb) return fail(ARP_ERR_CAPACITY, "output holds fewer records than n_boundary");
    std::memcpy(out, sim->host_boundary.data(), sim->nb * sizeof(arp_particle));
    for (uint32_t i = 0; i < sim->nb; ++i) {
        out[i].solid_id = kInvalid;
        out[i].mat -= sim->scenes[sim->scene_of_material[out[i].mat]].mat_base;
    }
    return ARP_OK;
}

arp_status arp_sim_get_materials(const arp_sim* sim, arp_material* out, uint32_t cap) {
    if (!sim || !out) return fail(ARP_ERR_INVALID_ARG, "null argument");
    if (cap < sim->M) return fail(ARP_ERR_CAPACITY, "output holds fewer records than n_materials");
    std::memcpy(out, sim->mats.data(), sim->M * sizeof(arp_material));
    return ARP_OK;
}

arp_status arp_sim_get_interactions(const arp_sim* sim, arp_interaction* out, uint32_t cap) {
    if (!sim || !out) return fail(ARP_ERR_INVALID_ARG, "null argument");
    if (cap < sim->inter.size())
        return fail(ARP_ERR_CAPACITY, "output holds fewer records than the interaction blocks of all scenes");
    std::memcpy(out, sim->inter.data(), sim->inter.size() * sizeof(arp_interaction));
    return ARP_OK;
}

arp_status arp_sim_set_particles(arp_sim* sim, const arp_particle* in, uint32_t n) {
    ARP_TRY(need_init(sim));
    if (sim->tape && sim->tape->steps) return fail(ARP_ERR_INVALID_ARG, "a tape is recording steps");
    if (!in && n) return fail(ARP_ERR_INVALID_ARG, "null argument");
    if (n != sim->n) return fail(ARP_ERR_INVALID_ARG, "particle count differs from the handle's");
    cudaStream_t st = sim->stream;
    if (n) {
        if (!sim->records.p) CUDA_TRY(sim->records.alloc(n));
        CUDA_TRY(cudaMemcpyAsync(sim->records.p, in, n * sizeof(arp_particle), cudaMemcpyHostToDevice, st));
        uint32_t flag = 0;
        CUDA_TRY(cudaMemsetAsync(sim->check_flag.p, 0, sizeof(uint32_t), st));
        sim->launches += check_records(sim->records.p, n, sim->mat_of_caller_d.p, sim->d_mats.p, sim->pos_w,
                                       sim->check_flag.p, st);
        CUDA_TRY(cudaMemcpyAsync(&flag, sim->check_flag.p, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
        CUDA_TRY(cudaStreamSynchronize(st));
        if (flag & 1u) return fail(ARP_ERR_INVALID_ARG, "material of a particle changed");
        if (flag & 2u) return fail(ARP_ERR_UNSUPPORTED, "w components must keep their values");
        sim->launches += records_to_soa(sim->records.p, n, sim->sid_of_caller_d.p, sim->mat_of_caller_d.p,
                                        sim->Y.pd.p, sim->Y.vm.p, sim->orig.p, sim->sid.p, st);
        sim->vforce_valid = false;  // a new state: velocity Verlet evaluates its forces again
        CUDA_TRY(cudaStreamSynchronize(st));
        ARP_TRY(check_launch("set_particles"));
    }
    return ARP_OK;
}

namespace {
// Streams, events, staging slots and the sticky flag of the asynchronous
// exchange, made on first use.
arp_status ensure_io(arp_sim* S) {
    auto& io = S->io;
    if (io.ready && io.cap >= S->n) return ARP_OK;
    if (!io.ready) {
        CUDA_TRY(cudaStreamCreateWithFlags(&io.copy_in, cudaStreamNonBlocking));
        CUDA_TRY(cudaStreamCreateWithFlags(&io.copy_out, cudaStreamNonBlocking));
        for (int q = 0; q < 2; ++q)
            for (cudaEvent_t* e : {&io.in_copied[q], &io.in_used[q], &io.out_ready[q], &io.out_copied[q]})
                CUDA_TRY(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
        CUDA_TRY(io.flag.alloc(1));
        CUDA_TRY(cudaMemsetAsync(io.flag.p, 0, sizeof(uint32_t), S->stream));
        io.ready = true;
    }
    // (re)size the slots: particles were added since they were made
    CUDA_TRY(cudaStreamSynchronize(io.copy_in));
    CUDA_TRY(cudaStreamSynchronize(io.copy_out));
    CUDA_TRY(cudaStreamSynchronize(S->stream));
    for (int q = 0; q < 2; ++q) {
        CUDA_TRY(io.in_rec[q].alloc(S->n));
        CUDA_TRY(io.out_rec[q].alloc(S->n));
    }
    io.cap = S->n;
    return ARP_OK;
}
}  // namespace

arp_status arp_sim_set_particles_async(arp_sim* sim, const arp_particle* in, uint32_t n) {
    ARP_TRY(need_init(sim));
    if (sim->tape && sim->tape->steps) return fail(ARP_ERR_INVALID_ARG, "a tape is recording steps");
    if (!in && n) return fail(ARP_ERR_INVALID_ARG, "null argument");
    if (n != sim->n) return fail(ARP_ERR_INVALID_ARG, "particle count differs from the handle's");
    if (!n) return ARP_OK;
    ARP_TRY(ensure_io(sim));
    auto& io = sim->io;
    const int q = io.in_slot;
    io.in_slot ^= 1;
    cudaStream_t st = sim->stream;
    // the slot's previous records have been converted before they are overwritten
    CUDA_TRY(cudaStreamWaitEvent(io.copy_in, io.in_used[q], 0));
    CUDA_TRY(cudaMemcpyAsync(io.in_rec[q].p, in, n * sizeof(arp_particle), cudaMemcpyHostToDevice, io.copy_in));
    CUDA_TRY(cudaEventRecord(io.in_copied[q], io.copy_in));
    CUDA_TRY(cudaStreamWaitEvent(st, io.in_copied[q], 0));
    // the conversion takes materials and solid ids from the handle's own
    // tables, so a record that fails the check cannot reach outside them
    sim->launches += check_records(io.in_rec[q].p, n, sim->mat_of_caller_d.p, sim->d_mats.p, sim->pos_w,
                                   io.flag.p, st);
    sim->launches += records_to_soa(io.in_rec[q].p, n, sim->sid_of_caller_d.p, sim->mat_of_caller_d.p,
                                    sim->Y.pd.p, sim->Y.vm.p, sim->orig.p, sim->sid.p, st);
    CUDA_TRY(cudaEventRecord(io.in_used[q], st));
    sim->vforce_valid = false;  // a new state: velocity Verlet evaluates its forces again
    return check_launch("set_particles_async");
}

arp_status arp_sim_get_particles_async(arp_sim* sim, arp_particle* out, uint32_t cap) {
    ARP_TRY(need_init(sim));
    if (!out && sim->n) return fail(ARP_ERR_INVALID_ARG, "null argument");
    if (cap < sim->n) return fail(ARP_ERR_CAPACITY, "output holds fewer records than n_particles");
    const uint32_t n = sim->n;
    if (!n) return ARP_OK;
    ARP_TRY(ensure_io(sim));
    auto& io = sim->io;
    const int q = io.out_slot;
    io.out_slot ^= 1;
    cudaStream_t st = sim->stream;
    // the slot's previous records have left for the host before they are overwritten
    CUDA_TRY(cudaStreamWaitEvent(st, io.out_copied[q], 0));
    sim->launches += soa_to_records(sim->Y.pd.p, sim->Y.vm.p, sim->orig.p, sim->sid.p, n, sim->pos_w, sim->d_mats.p,
                                    io.out_rec[q].p, st);
    CUDA_TRY(cudaEventRecord(io.out_ready[q], st));
    CUDA_TRY(cudaStreamWaitEvent(io.copy_out, io.out_ready[q], 0));
    CUDA_TRY(cudaMemcpyAsync(out, io.out_rec[q].p, n * sizeof(arp_particle), cudaMemcpyDeviceToHost, io.copy_out));
    CUDA_TRY(cudaEventRecord(io.out_copied[q], io.copy_out));
    return check_launch("get_particles_async");
}

arp_status arp_sim_synchronize(arp_sim* sim) {
    if (!sim) return fail(ARP_ERR_INVALID_ARG, "sim is null");
    if (sim->io.ready) CUDA_TRY(cudaStreamSynchronize(sim->io.copy_in));
    if (sim->stream) CUDA_TRY(cudaStreamSynchronize(sim->stream));
    if (!sim->io.ready) return check_launch("synchronize");
    CUDA_TRY(cudaStreamSynchronize(sim->io.copy_out));
    uint32_t flag = 0;
    CUDA_TRY(cudaMemcpy(&flag, sim->io.flag.p, sizeof(uint32_t), cudaMemcpyDeviceToHost));
    if (flag) CUDA_TRY(cudaMemset(sim->io.flag.p, 0, sizeof(uint32_t)));
    if (flag & 1u) return fail(ARP_ERR_INVALID_ARG, "material of a particle changed (asynchronous set)");
    if (flag & 2u) return fail(ARP_ERR_UNSUPPORTED, "w components must keep their values (asynchronous set)");
    return check_launch("synchronize");
}

arp_status arp_sim_device_state(arp_sim* sim, arp_device_view* out) {
    ARP_TRY(need_init(sim));
    if (!out) return fail(ARP_ERR_INVALID_ARG, "null argument");
    out->pos_den = sim->Y.pd.p;
    out->vel_mat = sim->Y.vm.p;
    out->orig_id = sim->orig.p;
    out->n = sim->n;
    return ARP_OK;
}

// The derived PartialEq of Material (material.rs:9-27): every field equal.
static bool same_material(const arp_material& a, const arp_material& b) {
    return a.immobile == b.immobile && a.mass == b.mass && a.start_den == b.start_den && a.state_eq == b.state_eq &&
           a.sound_speed == b.sound_speed && a.target_den == b.target_den && a.visc == b.visc &&
           a.bulk_visc == b.bulk_visc && a.strain_order == b.strain_order &&
           a.normal_stiffness == b.normal_stiffness && a.shear_stiffness == b.shear_stiffness &&
           a.normal_damp == b.normal_damp && a.shear_damp == b.shear_damp && a.plastic == b.plastic &&
           a.yield_strength == b.yield_strength && a.work_hardening == b.work_hardening &&
           a.work_hardening_exp == b.work_hardening_exp && a.kinematic_hardening == b.kinematic_hardening &&
           a.thermal_softening == b.thermal_softening && a.relaxation_time == b.relaxation_time;
}

// interaction.rs:42-50
static arp_interaction default_between(const arp_material& a, const arp_material& b, float h) {
    if (a.state_eq != ARP_EOS_ZERO && b.state_eq != ARP_EOS_ZERO) return arp_interaction{0, 0, 0, 0, 0};
    return arp_interaction{ARP_CONTACT_LINEAR, 10000.0f, h * 2.0f, 0.0f, a.visc + b.visc};
}

arp_status arp_sim_add_particles(arp_sim* sim, const arp_particle* p, uint32_t n, const arp_material* material,
                                 const float* offset, int* material_added) {
    ARP_TRY(need_init(sim));
    if (material_added) *material_added = 0;
    if (!material || (n && !p)) return fail(ARP_ERR_INVALID_ARG, "null argument");
    if (n == 0) return ARP_OK;  // particles.rs:548: nothing added, no material
    if (sim->scenes.size() != 1) return fail(ARP_ERR_UNSUPPORTED, "add_particles on a batch of scenes");
    // asynchronous copies in flight finish before the state is rebuilt
    if (sim->io.ready) {
        CUDA_TRY(cudaStreamSynchronize(sim->io.copy_in));
        CUDA_TRY(cudaStreamSynchronize(sim->io.copy_out));
    }
    if (material->immobile)
        return fail(ARP_ERR_UNSUPPORTED, "added particles join the mobile set; an immobile material is not supported");
    if (sim->tape) return fail(ARP_ERR_UNSUPPORTED, "add_particles while a tape records");
    if (sim->have_stiff) return fail(ARP_ERR_UNSUPPORTED, "add_particles with per-solid stiffness set");
    if ((uint64_t)sim->n + n > (1ull << 31)) return fail(ARP_ERR_UNSUPPORTED, "more than 2^31 particles");
    arp_sim::SceneHost& H = sim->scenes[0];
    // particles.rs:550-566: a solid material is always new, any other reuses
    // the first equal material
    const bool stiff = is_stiff(*material);
    uint32_t id = sim->M;
    if (!stiff)
        for (uint32_t i = 0; i < sim->M; ++i)
            if (same_material(sim->mats[i], *material)) {
                id = i;
                break;
            }
    const bool add_mat = id == sim->M;
    if (add_mat && sim->M + 1 > (uint32_t)kMaxMaterials)
        return fail(ARP_ERR_UNSUPPORTED, "more than 32 materials in one scene");
    // mod.rs:184-191: the offset is added in f32 to every component
    std::vector<arp_particle> added(p, p + n);
    for (auto& x : added) {
        if (offset)
            for (int a = 0; a < 4; ++a) x.pos[a] += offset[a];
        x.mat = id;
        x.solid_id = kInvalid;
        for (int a = 0; a < 4; ++a)
            if (!std::isfinite(x.pos[a]) || !std::isfinite(x.vel[a]))
                return fail(ARP_ERR_INVALID_ARG, "non-finite position or velocity");
        if (sim->have_w && x.pos[3] != sim->pos_w)
            return fail(ARP_ERR_UNSUPPORTED, "positions must share one w coordinate (4D motion is not supported)");
        if (x.vel[3] != 0.0f) return fail(ARP_ERR_UNSUPPORTED, "velocities must have zero w component");
    }
    // the current state in caller order, with each solid's reference position
    // and plastic strain
    std::vector<arp_particle> cur(sim->n);
    if (sim->n) ARP_TRY(arp_sim_get_particles(sim, cur.data(), sim->n));
    const uint32_t ns_old = sim->ns;
    std::vector<float4> ep_old(4 * size_t(ns_old));
    if (ns_old) {
        CUDA_TRY(cudaMemcpyAsync(ep_old.data(), sim->ep.p, ep_old.size() * sizeof(float4), cudaMemcpyDeviceToHost,
                                 sim->stream));
        CUDA_TRY(cudaStreamSynchronize(sim->stream));
    }
    sim->drop_graph();

    // new material and its interaction row and column (particles.rs:571-604)
    if (add_mat) {
        const uint32_t old = sim->M;
        sim->mats.push_back(*material);
        sim->scene_of_material.push_back(0);
        if (stiff && material->strain_order != 2) sim->all_order2 = false;
        if (stiff && material->plastic) sim->any_plastic = true;
        std::vector<arp_interaction> ni;
        ni.reserve(size_t(old + 1) * (old + 1));
        for (uint32_t i = 0; i < old; ++i) {
            for (uint32_t j = 0; j < old; ++j) ni.push_back(sim->inter[size_t(i) * old + j]);
            ni.push_back(default_between(sim->mats[i], sim->mats[old], sim->h));
        }
        for (uint32_t i = 0; i < old; ++i) ni.push_back(default_between(sim->mats[old], sim->mats[i], sim->h));
        ni.push_back(stiff ? arp_interaction{0, 0, 0, 0, 0} : default_between(sim->mats[old], sim->mats[old], sim->h));
        sim->inter = ni;
        sim->M = old + 1;
        H.nmat = sim->M;
        sim->max_nmat = std::max(sim->max_nmat, sim->M);
    }
    // the state becomes the initial state of a handle with the particles appended
    sim->host_particles = cur;
    for (auto& x : sim->host_particles) x.solid_id = kInvalid;
    sim->host_particles.insert(sim->host_particles.end(), added.begin(), added.end());
    if (!sim->have_w) {
        sim->pos_w = added[0].pos[3];
        sim->have_w = true;
    }
    bool flat = H.bounds.dim[2] == 0.0f;
    const float z0 = sim->host_particles[0].pos[2];
    for (const auto& x : sim->host_particles) flat = flat && x.pos[2] == z0 && x.vel[2] == 0.0f;
    for (const auto& x : sim->host_boundary) flat = flat && x.pos[2] == z0;
    H.flat_z = flat;
    H.n += n;
    sim->n += n;
    ARP_TRY(scene_params(H, H.sp.dim));  // material count and flatness enter the scene parameters
    finalize_scenes(sim, false);
    // solid ids of existing particles are unchanged (they precede the new ones)
    sim->host_ep = std::move(ep_old);
    sim->host_ep.resize(4 * size_t(sim->ns), make_float4(0.f, 0.f, 0.f, 0.f));
    sim->records.release();
    sim->initialized = false;
    ARP_TRY(allocate(sim));
    ARP_TRY(do_init(sim));
    ARP_TRY(run_autotune(sim, false));
    if (material_added) *material_added = add_mat ? 1 : 0;
    return ARP_OK;
}

arp_status arp_sim_grid(const arp_sim* sim, uint32_t subdivisions[4], uint32_t* n_cells) {
    if (!sim) return fail(ARP_ERR_INVALID_ARG, "sim is null");
    if (subdivisions) {
        for (int a = 0; a < 3; ++a) subdivisions[a] = sim->scenes[0].sp.grid.sub[a];
        subdivisions[3] = 1;
    }
    if (n_cells) *n_cells = sim->nccells;
    return ARP_OK;
}

// Reference cell (neighbor_list.rs:95) of a position in scene `scene`, in the
// C ABI's numbering; nccells for a non-finite position.
static uint32_t ref_cell_key(const arp_sim* S, float4 p, uint32_t scene) {
    if (!finite3(p)) return S->nccells;
    const SceneP& P = S->scenes[scene].sp;
    return P.ccell_base + cell_id(cell_coord(p, P.grid), P.grid);
}

// CSR of keys (caller order) over nc cells plus the non-finite bucket:
// start[0..nc+1], members in ascending caller id inside each cell.
static void cells_csr(const std::vector<uint32_t>& key, uint32_t nc, uint32_t* start_out, uint32_t* members) {
    std::vector<uint32_t> start(size_t(nc) + 2, 0u);
    for (uint32_t k : key) ++start[size_t(k) + 1];
    for (size_t c = 0; c + 1 < start.size(); ++c) start[c + 1] += start[c];
    if (start_out) std::memcpy(start_out, start.data(), (size_t(nc) + 1) * 4);
    if (members) {
        std::vector<uint32_t> fill(start.begin(), start.end() - 1);
        for (uint32_t i = 0; i < (uint32_t)key.size(); ++i) members[fill[key[i]]++] = i;
    }
}

arp_status arp_sim_neighbors(arp_sim* sim, uint32_t* cell_of, uint32_t* cell_start, uint32_t* members,
                             uint32_t* nbr_count) {
    ARP_TRY(need_init(sim));
    const uint32_t n = sim->n;
    cudaStream_t st = sim->stream;
    sim->launches += build_grid(sim->Y.pd.p, sim->Y.vm.p, nullptr, n, sim->tables, sim->gb, nullptr, nullptr, st);
    sim->launches += gather_sorted(sim->gb.perm, n, sim->Y.pd.p, sim->X.pd.p, sim->Y.vm.p, sim->X.vm.p, nullptr,
                                   nullptr, nullptr, nullptr, st);
    DevBuf<uint32_t> cnt;
    CUDA_TRY(cnt.alloc(n));
    sim->launches += count_neighbors(sim->X.pd.p, sim->X.vm.p, sim->gb.start, n, sim->b_pd.p, sim->b_start.p, sim->tables,
                                     cnt.p, st);
    std::vector<uint32_t> perm(n), orig(n), c(n);
    std::vector<float4> pd(n), vm(n);
    if (n) {
        CUDA_TRY(cudaMemcpyAsync(pd.data(), sim->Y.pd.p, n * sizeof(float4), cudaMemcpyDeviceToHost, st));
        CUDA_TRY(cudaMemcpyAsync(vm.data(), sim->Y.vm.p, n * sizeof(float4), cudaMemcpyDeviceToHost, st));
        CUDA_TRY(cudaMemcpyAsync(perm.data(), sim->gb.perm, n * 4, cudaMemcpyDeviceToHost, st));
        CUDA_TRY(cudaMemcpyAsync(orig.data(), sim->orig.p, n * 4, cudaMemcpyDeviceToHost, st));
        CUDA_TRY(cudaMemcpyAsync(c.data(), cnt.p, n * 4, cudaMemcpyDeviceToHost, st));
    }
    CUDA_TRY(cudaStreamSynchronize(st));
    ARP_TRY(check_launch("neighbors"));
    // reference cells of the current positions, in caller order
    const uint32_t nc = sim->nccells;
    std::vector<uint32_t> key(n);
    for (uint32_t k = 0; k < n; ++k) {
        uint32_t m;
        std::memcpy(&m, &vm[k].w, 4);
        key[orig[k]] = ref_cell_key(sim, pd[k], sim->scene_of_material[m]);
    }
    if (cell_of)
        for (uint32_t i = 0; i < n; ++i) cell_of[i] = key[i] >= nc ? kInvalid : key[i];
    cells_csr(key, nc, cell_start, members);
    if (nbr_count)
        for (uint32_t k = 0; k < n; ++k) nbr_count[orig[perm[k]]] = c[k];
    return ARP_OK;
}

arp_status arp_sim_boundary_cells(arp_sim* sim, uint32_t* cell_start, uint32_t* members) {
    ARP_TRY(need_init(sim));
    const uint32_t nb = sim->nb;
    std::vector<uint32_t> key(nb);
    for (uint32_t i = 0; i < nb; ++i) {
        const arp_particle& p = sim->host_boundary[i];
        key[i] = ref_cell_key(sim, make_float4(p.pos[0], p.pos[1], p.pos[2], p.den), sim->scene_of_material[p.mat]);
    }
    cells_csr(key, sim->nccells, cell_start, members);
    return ARP_OK;
}

arp_status arp_sim_set_stream(arp_sim* sim, void* stream) {
    if (!sim) return fail(ARP_ERR_INVALID_ARG, "sim is null");
    CUDA_TRY(cudaStreamSynchronize(sim->stream));
    sim->stream = stream ? (cudaStream_t)stream : sim->own_stream;
    if (sim->graph_stream != sim->stream) sim->drop_graph();
    return ARP_OK;
}

arp_status arp_sim_profile_enable(arp_sim* sim, int enable) {
    if (!sim) return fail(ARP_ERR_INVALID_ARG, "sim is null");
    if (enable < 0) return fail(ARP_ERR_INVALID_ARG, "enable must be 0 or a sampling period >= 1");
    if (!enable) harvest_marks(sim);
    sim->prof_on = enable != 0;
    sim->prof_every = enable > 0 ? (uint32_t)enable : 1u;
    sim->prof_phase = 0;
    sim->profiling = false;
    return ARP_OK;
}

arp_status arp_sim_profile_read(arp_sim* sim, arp_profile* out) {
    if (!sim || !out) return fail(ARP_ERR_INVALID_ARG, "null argument");
    harvest_marks(sim);
    out->steps = sim->prof_steps;
    out->stages = sim->prof_stages;
    out->launches = sim->prof_l[0] + sim->prof_l[1] + sim->prof_l[2];
    out->neighbor_ms = sim->acc_ms[0];
    out->solid_ms = sim->acc_ms[1];
    out->fluid_ms = sim->acc_ms[2];
    out->integrate_ms = 0.0;
    out->neighbor_launches = sim->prof_l[0];
    out->solid_launches = sim->prof_l[1];
    out->fluid_launches = sim->prof_l[2];
    for (double& x : sim->acc_ms) x = 0;
    for (auto& x : sim->prof_l) x = 0;
    sim->prof_steps = 0;
    sim->prof_stages = 0;
    return ARP_OK;
}

arp_status arp_sim_stats(arp_sim* sim, arp_stats* out) {
    if (!sim || !out) return fail(ARP_ERR_INVALID_ARG, "null argument");
    DevStats d{};
    CUDA_TRY(cudaMemcpyAsync(&d, sim->d_stats.p, sizeof(d), cudaMemcpyDeviceToHost, sim->stream));
    CUDA_TRY(cudaStreamSynchronize(sim->stream));
    out->max_cell_occupancy = d.max_cell_occupancy;
    out->overflow_cells = d.overflow_cells;
    out->nonfinite_positions = d.nonfinite_positions;
    out->clamped_coordinates = d.clamped_coordinates;
    return ARP_OK;
}

arp_status arp_sim_launch_count(const arp_sim* sim, uint64_t* out) {
    if (!sim || !out) return fail(ARP_ERR_INVALID_ARG, "null argument");
    *out = sim->launches;
    return ARP_OK;
}

arp_status arp_sim_render_rgb24(arp_sim* sim, const arp_view* view, const arp_render_style* style, uint32_t width,
                                uint32_t height, uint8_t* out_rgb) {
    ARP_TRY(need_init(sim));
    if (!view || !style || !out_rgb || !style->colors || !style->densities)
        return fail(ARP_ERR_INVALID_ARG, "null argument");
    if (width == 0 || height == 0 || (uint64_t)width * height > (1ull << 28))
        return fail(ARP_ERR_INVALID_ARG, "frame size must be positive and at most 2^28 pixels");
    if (style->n_materials < sim->M)
        return fail(ARP_ERR_INVALID_ARG, "the style has fewer materials than the handle");
    if (!(style->render_h > 0.0f) || !std::isfinite(style->render_h))
        return fail(ARP_ERR_INVALID_ARG, "render_h must be positive");
    cudaStream_t st = sim->stream;
    auto& R = sim->rbuf;
    auto fit = [](auto& b, size_t count) -> cudaError_t { return b.n >= count ? cudaSuccess : b.alloc(count); };
    RenderCfg c{};
    c.W = width;
    c.H = height;
    const uint32_t s2 = std::min(width, height);
    c.s2 = (float)s2;
    c.vx0 = (float)((width - s2) / 2);
    c.vy0 = (float)((height - s2) / 2);
    c.S = (float)s2 * style->render_h;  // gl::PointSize(s2 * render_h)
    c.ca = std::cos(view->angle);
    c.sa = std::sin(view->angle);
    c.tx = -view->pos[0];
    c.ty = view->pos[1];  // the matrix holds -trans_y with trans_y = -view_pos[1] (renderer.rs:347)
    c.tz = -view->scale + 1.0f;
    c.render_h = style->render_h;
    c.kconst = norm_const_f32(3, 3.0f);  // normalization_constant(3, 3) in the fragment shader
    c.lighting = style->lighting ? 1 : 0;
    for (int k = 0; k < 3; ++k) {
        c.light[k] = style->light_pos[k];
        c.lcol[k] = style->light_color[k];
    }
    c.amb = style->ambient;
    c.dif = style->diffuse;
    c.spec = style->specular;
    c.nmat = sim->M;
    c.nprims = sim->nb + sim->n;
    const uint32_t ts = render_tile_size();
    c.tiles_x = (width + ts - 1) / ts;
    c.tiles_y = (height + ts - 1) / ts;
    {
        std::vector<float4> h1(sim->M), h2(sim->M), h3(sim->M);
        for (uint32_t m = 0; m < sim->M; ++m) {
            const float* q = style->colors + 12 * size_t(m);
            h2[m] = make_float4(q[0], q[1], q[2], q[3]);
            h1[m] = make_float4(q[4], q[5], q[6], q[7]);
            h3[m] = make_float4(q[8], q[9], q[10], q[11]);
        }
        CUDA_TRY(fit(R.c1, sim->M));
        CUDA_TRY(fit(R.c2, sim->M));
        CUDA_TRY(fit(R.c3, sim->M));
        CUDA_TRY(fit(R.d0, sim->M));
        CUDA_TRY(cudaMemcpyAsync(R.c1.p, h1.data(), sim->M * sizeof(float4), cudaMemcpyHostToDevice, st));
        CUDA_TRY(cudaMemcpyAsync(R.c2.p, h2.data(), sim->M * sizeof(float4), cudaMemcpyHostToDevice, st));
        CUDA_TRY(cudaMemcpyAsync(R.c3.p, h3.data(), sim->M * sizeof(float4), cudaMemcpyHostToDevice, st));
        CUDA_TRY(cudaMemcpyAsync(R.d0.p, style->densities, sim->M * sizeof(float), cudaMemcpyHostToDevice, st));
        CUDA_TRY(cudaStreamSynchronize(st));
    }
    c.c1 = R.c1.p;
    c.c2 = R.c2.p;
    c.c3 = R.c3.p;
    c.d0 = R.d0.p;
    const size_t np = std::max(c.nprims, 1u);
    CUDA_TRY(fit(R.PR, np));
    CUDA_TRY(fit(R.PC, np));
    CUDA_TRY(fit(R.PP, np));
    CUDA_TRY(fit(R.rgb, (size_t)width * height * 3));
    sim->launches += render_project(sim->b_pd.p, sim->b_vm.p, sim->b_orig.p, sim->nb, 0, c, R.PR.p, R.PC.p, R.PP.p, st);
    sim->launches += render_project(sim->Y.pd.p, sim->Y.vm.p, sim->orig.p, sim->n, sim->nb, c, R.PR.p, R.PC.p, R.PP.p,
                                    st);
    if (!c.lighting) {
        const uint64_t nchunks = (c.nprims + render_chunk_size() - 1) / render_chunk_size();
        const uint64_t K = std::max<uint64_t>(nchunks, 1) * c.tiles_x * c.tiles_y;
        if (K + 1 > (1ull << 31)) return fail(ARP_ERR_UNSUPPORTED, "too many sprite bins for this frame size");
        CUDA_TRY(fit(R.counts, K + 1));
        CUDA_TRY(fit(R.start, K + 1));
        CUDA_TRY(fit(R.fill, K + 1));
        CUDA_TRY(fit(R.bsums, scan_block_sums_needed((uint32_t)(K + 1))));
        CUDA_TRY(cudaMemsetAsync(R.counts.p, 0, (K + 1) * sizeof(uint32_t), st));
        CUDA_TRY(cudaMemsetAsync(R.fill.p, 0, (K + 1) * sizeof(uint32_t), st));
        sim->launches += render_bin_count(R.PR.p, R.PC.p, c, R.counts.p, st);
        sim->launches += exclusive_scan(R.counts.p, (uint32_t)(K + 1), R.start.p, R.bsums.p, st);
        uint32_t total = 0;
        CUDA_TRY(cudaMemcpyAsync(&total, R.start.p + K, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
        CUDA_TRY(cudaStreamSynchronize(st));
        CUDA_TRY(fit(R.list, std::max(total, 1u)));
        sim->launches += render_bin_scatter(R.PR.p, R.PC.p, c, R.start.p, R.fill.p, R.list.p, st);
        sim->launches += render_composite(R.PR.p, R.PC.p, c, R.start.p, R.list.p, R.rgb.p, st);
    } else {
        CUDA_TRY(fit(R.zkey, (size_t)width * height));
        CUDA_TRY(cudaMemsetAsync(R.zkey.p, 0xFF, (size_t)width * height * sizeof(unsigned long long), st));
        sim->launches += render_lit(R.PR.p, R.PC.p, R.PP.p, c, R.zkey.p, R.rgb.p, st);
    }
    CUDA_TRY(cudaMemcpyAsync(out_rgb, R.rgb.p, (size_t)width * height * 3, cudaMemcpyDeviceToHost, st));
    CUDA_TRY(cudaStreamSynchronize(st));
    return check_launch("render");
}

arp_status arp_sim_set_solid_stiffness(arp_sim* sim, const float* normal_shear, uint32_t ns) {
    if (!sim) return fail(ARP_ERR_INVALID_ARG, "sim is null");
    if (!normal_shear) {
        sim->have_stiff = false;
        return ARP_OK;
    }
    if (ns != sim->ns) return fail(ARP_ERR_INVALID_ARG, "stiffness count differs from the number of solids");
    sim->drop_graph();
    if (ns) {
        CUDA_TRY(sim->stiff.alloc(ns));
        CUDA_TRY(cudaMemcpyAsync(sim->stiff.p, normal_shear, ns * sizeof(float2), cudaMemcpyHostToDevice,
                                 sim->stream));
        CUDA_TRY(cudaStreamSynchronize(sim->stream));
    }
    sim->have_stiff = true;
    return ARP_OK;
}

// Checkpoints of an ended tape go back to the handle's pool.
static void retire_tape(arp_sim* sim) {
    if (!sim->tape) return;
    for (auto& c : sim->tape->ckpts) sim->adj.spare.push_back(std::move(c));
    sim->tape.reset();
}

arp_status arp_tape_begin(arp_sim* sim, uint32_t checkpoint_every) {
    ARP_TRY(need_init(sim));
    if (checkpoint_every == 0) return fail(ARP_ERR_INVALID_ARG, "checkpoint interval must be positive");
    if (sim->tab.stages > kMaxStages) return fail(ARP_ERR_UNSUPPORTED, "more than 4 stages");
    sim->drop_graph();
    retire_tape(sim);
    // velocity Verlet: the tape starts with a force evaluation at the current
    // state (recorded, so the gradient reaches y_0 through it), as after init
    if (sim->verlet()) sim->vforce_valid = false;
    sim->tape.reset(new Tape());
    sim->tape->every = checkpoint_every;
    return ARP_OK;
}

arp_status arp_tape_end(arp_sim* sim) {
    if (!sim) return fail(ARP_ERR_INVALID_ARG, "sim is null");
    retire_tape(sim);
    return ARP_OK;
}

arp_status arp_tape_steps(const arp_sim* sim, uint64_t* steps) {
    if (!sim || !steps) return fail(ARP_ERR_INVALID_ARG, "null argument");
    *steps = sim->tape ? sim->tape->steps : 0;
    return ARP_OK;
}

arp_status arp_tape_backward(arp_sim* sim, const float* dl_dstate, float* grad_state0, float* grad_stiffness) {
    ARP_TRY(need_init(sim));
    if (!sim->tape) return fail(ARP_ERR_INVALID_ARG, "no tape is recording");
    if (!dl_dstate || !grad_state0) return fail(ARP_ERR_INVALID_ARG, "null argument");
    Tape& tp = *sim->tape;
    const uint32_t n = sim->n, ns = sim->ns;
    const uint64_t total = tp.steps;
    cudaStream_t st = sim->stream;
    const int S = sim->tab.stages;
    AdjointPool& P = sim->adj;
    // the forward state is put back when the pass ends
    Checkpoint& now = P.now;
    CUDA_TRY(keep(now.pd, (const float4*)sim->Y.pd.p, n, st));
    CUDA_TRY(keep(now.vm, (const float4*)sim->Y.vm.p, n, st));
    CUDA_TRY(keep(now.orig, (const uint32_t*)sim->orig.p, n, st));
    CUDA_TRY(keep(now.sid, (const uint32_t*)sim->sid.p, n, st));
    if (sim->any_plastic) CUDA_TRY(keep(now.ep, (const float4*)sim->ep.p, 4 * size_t(ns), st));
    now.fvalid = sim->verlet() && sim->vforce_valid;
    if (now.fvalid) {
        CUDA_TRY(keep(now.fpd, (const float4*)sim->vforce.pd.p, n, st));
        CUDA_TRY(keep(now.fvm, (const float4*)sim->vforce.vm.p, n, st));
        if (sim->any_plastic) CUDA_TRY(keep(now.fep, (const float4*)sim->ep_force.p, 4 * size_t(ns), st));
    }
    now.time = sim->time;
    // adjoint buffers: caller order (lc), storage order (ls, out), per stage (lY), stage weights (mu)
    const size_t nn = std::max(n, 1u);
    auto fit = [](auto& b, size_t count) -> cudaError_t { return b.n >= count ? cudaSuccess : b.alloc(count); };
    for (DevBuf<float4>* b :
         {&P.lc_p, &P.lc_v, &P.ls_p, &P.ls_v, &P.out_p, &P.out_v, &P.mu_p, &P.mu_v, &P.w, &P.e, &P.xs})
        CUDA_TRY(fit(*b, nn));
    for (int q = 0; q < S; ++q) {
        CUDA_TRY(fit(P.lY_p[q], nn));
        CUDA_TRY(fit(P.lY_v[q], nn));
    }
    CUDA_TRY(fit(P.lamF, 3 * size_t(std::max(ns, 1u))));
    CUDA_TRY(fit(P.lamFd, 3 * size_t(std::max(ns, 1u))));
    CUDA_TRY(fit(P.gst, std::max(ns, 1u)));
    const bool plastic = sim->any_plastic && sim->solid_branch() && ns > 0;
    const size_t ne = 4 * size_t(std::max(ns, 1u));
    if (plastic) {
        for (DevBuf<float4>* b : {&P.lam_ep, &P.out_ep, &P.mu_ep}) CUDA_TRY(fit(*b, ne));
        for (int q = 0; q < S; ++q) CUDA_TRY(fit(P.lY_ep[q], ne));
        CUDA_TRY(cudaMemsetAsync(P.lam_ep.p, 0, ne * sizeof(float4), st));  // the loss reads no plastic strain
    }
    CUDA_TRY(fit(P.flags, 1));
    CUDA_TRY(fit(P.io, 2 * nn));
    DevBuf<float4>&lc_p = P.lc_p, &lc_v = P.lc_v, &ls_p = P.ls_p, &ls_v = P.ls_v, &out_p = P.out_p,
                  &out_v = P.out_v, &mu_p = P.mu_p, &mu_v = P.mu_v, &lamF = P.lamF, &lamFd = P.lamFd;
    DevBuf<float4>* lY_p = P.lY_p;
    DevBuf<float4>* lY_v = P.lY_v;
    DevBuf<double2>& gst = P.gst;
    DevBuf<uint32_t>& flags = P.flags;
    CUDA_TRY(cudaMemsetAsync(gst.p, 0, std::max(ns, 1u) * sizeof(double2), st));
    CUDA_TRY(cudaMemsetAsync(flags.p, 0, sizeof(uint32_t), st));
    if (n) {  // one copy of the caller's array, split on the device
        CUDA_TRY(cudaMemcpyAsync(P.io.p, dl_dstate, n * 2 * sizeof(float4), cudaMemcpyHostToDevice, st));
        sim->launches += adjoint_unpack(n, P.io.p, lc_p.p, lc_v.p, st);
    }
    // lam_Y += J_f(Y)^T mu for stage q of a recorded step
    auto stage_vjp = [&](const StepRecord& R, int q, const float4* mup, const float4* muv, float4* lyp, float4* lyv,
                         const float4* muep, float4* lyep) {
        AdjArgs a{};
        a.st.pd = R.pd[q].p;
        a.st.vm = R.vm[q].p;
        a.st.perm = R.has_perm[q] ? R.perm[q].p : nullptr;
        a.st.start = R.start[q].p;
        const bool sb = sim->solid_branch();
        a.st.F = sb ? R.F[q].p : nullptr;
        a.st.A = sb ? R.A[q].p : nullptr;
        a.st.sx = sb ? R.sx[q].p : nullptr;
        a.st.sv = sb ? R.sv[q].p : nullptr;
        a.st.sc = sb ? R.sc[q].p : nullptr;
        a.st.contact_bound = sb ? R.cb[q].p : nullptr;
        a.sid = R.sid.p;
        a.slot_of = R.slot_of.p;
        a.mu_pd = mup;
        a.mu_vm = muv;
        a.lam_pd = lyp;
        a.lam_vm = lyv;
        a.bxs = sim->b_pd.p;
        a.bvs = sim->b_vm.p;
        a.bstart = sim->b_start.p;
        a.bps = sim->bps.p;
        a.ref = sim->ref.p;
        a.L = sim->L.p;
        a.rl = SolidRefList{sim->rl_off.p, sim->rl_nbr.p, sim->rl_gw.p, sim->rl_nnz};
        a.stiff = sim->have_stiff ? sim->stiff.p : nullptr;
        a.lamF = lamF.p;
        a.lamFd = lamFd.p;
        a.g_stiff = gst.p;
        a.flags = flags.p;
        a.w = P.w.p;
        a.eq = P.e.p;
        a.xs = P.xs.p;
        a.n = n;
        a.ns = ns;
        a.solid_branch = sb ? 1 : 0;
        a.all_order2 = sim->all_order2 ? 1 : 0;
        a.st.ep = plastic ? R.ep[q].p : nullptr;
        a.mu_ep = plastic ? muep : nullptr;
        a.lam_ep = plastic ? lyep : nullptr;
        sim->launches += launch_adjoint_stage(a, sim->tables, sim->kdim, st);
    };
    // Velocity Verlet, one step (reverse): y* = kick-drift(y_n, f_n),
    // f_{n+1} = f(y*), y_{n+1} = y* + (dt/2) P f_{n+1}.  With lam the state's
    // adjoint and lf the carried record's (both caller order):
    //   mu = lf + (dt/2) P lam;  lam* = lam + J_f(y*)^T mu;  then the
    //   kick-drift's adjoint gives lam_n and lf_n from lam*;  a step that began
    //   with the force evaluation f_n = f(y_n) adds J_f(y_n)^T lf_n to lam_n.
    const bool verlet = sim->verlet();
    const float vh = (float)(sim->tab.b[0] * (double)sim->dt_sub);
    if (verlet) {
        for (DevBuf<float4>* b : {&P.lf_p, &P.lf_v}) {
            CUDA_TRY(fit(*b, nn));
            CUDA_TRY(cudaMemsetAsync(b->p, 0, nn * sizeof(float4), st));  // the loss reads no force record
        }
        if (plastic) {
            CUDA_TRY(fit(P.lf_ep, ne));
            CUDA_TRY(cudaMemsetAsync(P.lf_ep.p, 0, ne * sizeof(float4), st));
        }
        P.prime_recorded = false;
    }
    auto verlet_step_vjp = [&](const StepRecord& R, bool with_prime) -> arp_status {
        const float one = 1.0f;
        sim->launches += adjoint_gather(n, R.orig.p, lc_p.p, lc_v.p, ls_p.p, ls_v.p, st);
        sim->launches += adjoint_gather(n, R.orig.p, P.lf_p.p, P.lf_v.p, out_p.p, out_v.p, st);
        sim->launches += verlet_adjoint_weights(n, ls_p.p, ls_v.p, out_p.p, out_v.p, vh, mu_p.p, mu_v.p, st);
        if (plastic) {
            const float4* lfe[1] = {P.lf_ep.p};
            sim->launches += adjoint_stage_weights_all(4 * ns, vh, P.lam_ep.p, 1, &one, lfe, P.mu_ep.p, st);
            CUDA_TRY(cudaMemsetAsync(P.lY_ep[0].p, 0, 4 * size_t(ns) * sizeof(float4), st));
        }
        if (n) {
            CUDA_TRY(cudaMemsetAsync(lY_p[0].p, 0, n * sizeof(float4), st));
            CUDA_TRY(cudaMemsetAsync(lY_v[0].p, 0, n * sizeof(float4), st));
        }
        stage_vjp(R, 0, mu_p.p, mu_v.p, lY_p[0].p, lY_v[0].p, P.mu_ep.p, P.lY_ep[0].p);
        const float4* yp[1] = {lY_p[0].p};
        const float4* yv[1] = {lY_v[0].p};
        sim->launches += adjoint_step_sum(n, ls_p.p, ls_v.p, 1, yp, yv, out_p.p, out_v.p, st);
        sim->launches += adjoint_scatter(n, R.orig.p, out_p.p, out_v.p, lc_p.p, lc_v.p, st);
        sim->launches += verlet_kick_drift_adjoint(n, lc_p.p, lc_v.p, vh, sim->dt_sub, P.lf_p.p, P.lf_v.p, st);
        if (plastic) {
            const float4* ye[1] = {P.lY_ep[0].p};
            sim->launches += adjoint_step_sum_all(4 * ns, P.lam_ep.p, 1, ye, P.out_ep.p, st);
            std::swap(P.lam_ep, P.out_ep);
            sim->launches += adjoint_stage_weights_all(4 * ns, vh, P.lam_ep.p, 0, nullptr, nullptr, P.lf_ep.p, st);
        }
        if (!with_prime) return ARP_OK;
        // the force evaluation at y_0: lam_0 += J_f(y_0)^T lf_0 (the record's
        // position part is zero), in the storage order of that evaluation
        const StepRecord& R0 = P.prime;
        sim->launches += adjoint_gather(n, R0.orig.p, P.lf_p.p, P.lf_v.p, mu_p.p, mu_v.p, st);
        if (n) {
            CUDA_TRY(cudaMemsetAsync(lY_p[0].p, 0, n * sizeof(float4), st));
            CUDA_TRY(cudaMemsetAsync(lY_v[0].p, 0, n * sizeof(float4), st));
        }
        if (plastic) CUDA_TRY(cudaMemsetAsync(P.lY_ep[0].p, 0, 4 * size_t(ns) * sizeof(float4), st));
        stage_vjp(R0, 0, mu_p.p, mu_v.p, lY_p[0].p, lY_v[0].p, P.lf_ep.p, P.lY_ep[0].p);
        sim->launches += adjoint_scatter(n, R0.orig.p, lY_p[0].p, lY_v[0].p, out_p.p, out_v.p, st);
        const float4* op[1] = {out_p.p};
        const float4* ov[1] = {out_v.p};
        sim->launches += adjoint_step_sum(n, lc_p.p, lc_v.p, 1, op, ov, ls_p.p, ls_v.p, st);
        std::swap(P.lc_p, P.ls_p);
        std::swap(P.lc_v, P.ls_v);
        if (plastic) {
            const float4* ye[1] = {P.lY_ep[0].p};
            sim->launches += adjoint_step_sum_all(4 * ns, P.lam_ep.p, 1, ye, P.out_ep.p, st);
            std::swap(P.lam_ep, P.out_ep);
        }
        return ARP_OK;
    };
    const uint32_t every = tp.every;
    if (P.recs.size() < every) P.recs.resize(every);
    const uint64_t nseg = (total + every - 1) / every;
    sim->replaying = true;
    arp_status status = ARP_OK;
    for (uint64_t seg = nseg; seg-- > 0 && status == ARP_OK;) {
        const uint64_t t0 = seg * every, t1 = std::min<uint64_t>(t0 + every, total);
        status = restore_checkpoint(sim, tp.ckpts[seg]);
        for (uint64_t t = t0; t < t1 && status == ARP_OK; ++t) {
            sim->rec = &P.recs[t - t0];
            status = do_step(sim);
            sim->rec = nullptr;
        }
        for (uint64_t t = t1; t-- > t0 && status == ARP_OK;) {
            const StepRecord& R = P.recs[t - t0];
            if (verlet) {
                status = verlet_step_vjp(R, t == 0 && P.prime_recorded);
                continue;
            }
            sim->launches += adjoint_gather(n, R.orig.p, lc_p.p, lc_v.p, ls_p.p, ls_v.p, st);
            for (int q = S - 1; q >= 0; --q) {
                float ca[kMaxStages];
                const float4* lp[kMaxStages];
                const float4* lv[kMaxStages];
                int nl = 0;
                for (int u = q + 1; u < S; ++u)
                    if (sim->tab.a[u][q] != 0.0) {
                        ca[nl] = (float)(sim->tab.a[u][q] * (double)sim->dt_sub);
                        lp[nl] = lY_p[u].p;
                        lv[nl] = lY_v[u].p;
                        ++nl;
                    }
                const float cb = (float)(sim->tab.b[q] * (double)sim->dt_sub);
                sim->launches += adjoint_stage_weights(n, cb, ls_p.p, ls_v.p, nl, ca, lp, lv, mu_p.p, mu_v.p, st);
                if (plastic) {  // the same weights for the plastic strain's record
                    const float4* le[kMaxStages];
                    int ne_later = 0;
                    for (int u = q + 1; u < S; ++u)
                        if (sim->tab.a[u][q] != 0.0) le[ne_later++] = P.lY_ep[u].p;
                    sim->launches += adjoint_stage_weights_all(4 * ns, cb, P.lam_ep.p, ne_later, ca, le, P.mu_ep.p, st);
                    CUDA_TRY(cudaMemsetAsync(P.lY_ep[q].p, 0, 4 * size_t(ns) * sizeof(float4), st));
                }
                if (n) {
                    cudaMemsetAsync(lY_p[q].p, 0, n * sizeof(float4), st);
                    cudaMemsetAsync(lY_v[q].p, 0, n * sizeof(float4), st);
                }
                stage_vjp(R, q, mu_p.p, mu_v.p, lY_p[q].p, lY_v[q].p, P.mu_ep.p, P.lY_ep[q].p);
            }
            const float4* yp[kMaxStages];
            const float4* yv[kMaxStages];
            for (int q = 0; q < S; ++q) {
                yp[q] = lY_p[q].p;
                yv[q] = lY_v[q].p;
            }
            sim->launches += adjoint_step_sum(n, ls_p.p, ls_v.p, S, yp, yv, out_p.p, out_v.p, st);
            if (plastic) {
                const float4* ye[kMaxStages];
                for (int q = 0; q < S; ++q) ye[q] = P.lY_ep[q].p;
                sim->launches += adjoint_step_sum_all(4 * ns, P.lam_ep.p, S, ye, P.out_ep.p, st);
                std::swap(P.lam_ep, P.out_ep);
            }
            sim->launches += adjoint_scatter(n, R.orig.p, out_p.p, out_v.p, lc_p.p, lc_v.p, st);
        }
        if (status == ARP_OK) {
            cudaError_t e = cudaStreamSynchronize(st);
            if (e != cudaSuccess) status = fail(ARP_ERR_CUDA, std::string("adjoint: ") + cudaGetErrorString(e));
        }
    }
    sim->replaying = false;
    sim->rec = nullptr;
    ARP_TRY(status);
    ARP_TRY(restore_checkpoint(sim, now));
    ARP_TRY(check_launch("adjoint"));
    uint32_t hflags = 0;
    if (n) {  // interleaved on the device, one copy into the caller's array
        sim->launches += adjoint_pack(n, lc_p.p, lc_v.p, P.io.p, st);
        CUDA_TRY(cudaMemcpyAsync(grad_state0, P.io.p, n * 2 * sizeof(float4), cudaMemcpyDeviceToHost, st));
    }
    // accumulated in double; float2 (normal, shear) per solid is the caller's layout
    std::vector<double2> gst_host(grad_stiffness ? ns : 0);
    if (ns && grad_stiffness)
        CUDA_TRY(cudaMemcpyAsync(gst_host.data(), gst.p, ns * sizeof(double2), cudaMemcpyDeviceToHost, st));
    CUDA_TRY(cudaMemcpyAsync(&hflags, flags.p, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    CUDA_TRY(cudaStreamSynchronize(st));
    for (uint32_t q = 0; q < gst_host.size(); ++q) {
        grad_stiffness[2 * q] = (float)gst_host[q].x;
        grad_stiffness[2 * q + 1] = (float)gst_host[q].y;
    }
    if (hflags & 1u) return fail(ARP_ERR_UNSUPPORTED, "a self-contact pair was active; it is not differentiated");
    return ARP_OK;
}

}  // extern "C"
