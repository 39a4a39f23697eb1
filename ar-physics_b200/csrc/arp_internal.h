// arp_internal.h -- device-side data layout and kernel entry points of libarphys.
//
// State layout in HBM (structure of arrays, cell-sorted):
//   pos_den  float4[N]  x, y, z, density          (the reference's pos.xyz + den)
//   vel_mat  float4[N]  vx, vy, vz, material bits  (vel.xyz + mat)
//   orig     uint32[N]  caller-order particle id of each slot
//   sid      uint32[N]  solid id of each slot or ARP_INVALID_INDEX
// Solid data stays in solid-id order (solid ids never change):
//   ref      float4[Ns] reference position
//   ep       float4[4*Ns] plastic strain mat4, column-major (SolidParticle.stress)
//   L        float4[3*Ns] correction matrix columns (constant, built at init)
// Particles are re-sorted by cell at the start of every integrator step; the
// grid of each later RK stage is a permutation over those slots.
#pragma once

#include <cstdint>
#include <string>

#include <cuda_runtime.h>

#include "../../include/arphys.h"

namespace arp {

constexpr uint32_t kInvalid = 0xFFFFFFFFu;
constexpr uint32_t kBucketSlots = 128;  // neighbor_list.rs:45
constexpr int kMaxMaterials = 32;  // per scene
// Axes (bit a = axis a) along which the search grid halves the reference
// cells.  Halving x alone keeps a warp's 32 consecutive particles inside a
// compact 4h x h x h block (the rows stay x-fastest) while its rows of 5
// half-width cells hold 5/6 of the candidates of 3 reference cells.
#ifndef ARP_SEARCH_HALVE
#define ARP_SEARCH_HALVE 1
#endif
constexpr uint32_t kSearchHalve = ARP_SEARCH_HALVE;
// A scene whose particles have at least this many neighbors within h,
// estimated as (h / spacing)^dim, also halves y: its rows of 5 x 5 half
// cells hold ~40 % fewer candidates than 5 x 3, which outweighs the grid's
// four times as many cells (the batched workload: 23.0 k -> 25.8 k scene
// steps/s with every scene halved so; the 1M workload, (h/s)^3 = 8, loses 4 %
// that way and keeps x alone).
constexpr double kDenseNeighbors = 10.0;

// Uniform grid of NeighborList::new (neighbor_list.rs:199-217), one scene.
struct Grid {
    float min[3];
    float dim[3];
    uint32_t sub[3];
    uint32_t ncells;
};

// Per-material constants the kernels read (a subset of `Material`), in one
// table over all scenes of a batch.
struct DevMat {
    float mass, start_den, sound_speed, target_den;
    float visc, bulk_visc, lam, mu;
    float lam_d, mu_d, yield_strength, work_hardening;
    float work_hardening_exp, kinematic_hardening, relaxation_time, vol0;  // vol0 = mass / start_den
    uint32_t state_eq, stiff, plastic;
    int32_t strain_order;
    uint32_t scene;       // scene the material belongs to
    uint32_t local;       // index inside that scene's material list
    uint32_t solid_base;  // first batch-wide solid id of that scene
};

struct DevInter {
    uint32_t potential;
    float strength, radius, dampening, friction;
};

// Scalars of one scene.  Products are rounded exactly as the shaders group
// them (e.g. EPSILON*h*h = (0.1*h)*h).  A single simulation is a batch of one
// scene.
//
// Two grids cover the scene's box.  `grid` is the reference's (cells of at
// least h); the hourglass and self-contact stencils, the cell statistics and
// the cell queries of the C ABI use it.  `sgrid`, the search grid, halves the
// cells along the axes of kSearchHalve that have non-zero extent, and along y
// too in a dense scene (kDenseNeighbors) (sub doubled), so along such an axis a sphere of radius h spans at most 5 cells
// of width h/2 instead of 3 of width h; particles are sorted by search cell,
// and the search cells of one reference cell c are 2c and 2c+1 along each
// halved axis.  Because 2 * (t * sub) is rounded exactly like t * (2 sub),
// floor(search) >> 1 is the reference cell bit for bit.  Search cells of
// scene k are global cells cell_base .. cell_base + sgrid.ncells; its
// reference cells, numbered for the C ABI only, start at ccell_base.
struct SceneP {
    Grid grid;
    Grid sgrid;
    uint32_t halved[3];               // 1 where sgrid halves grid's cells
    uint32_t cell_base;
    uint32_t ccell_base;
    uint32_t dim;                     // the reference's count of non-zero box axes
    uint32_t mat_base, nmat;          // global material range of the scene
    uint32_t inter_base;              // first entry of its nmat x nmat interaction block
    float h, h2, kconst, g;
    float eps_hh;                     // (0.1f * h) * h
    float eps_h;                      // 0.1f * h
    float hg_h;                       // (10 * 0.1f) * h
    float rcut, rcut2, r_geom;        // 8h, (8h)^2, h*h/(8h)
    float contact_slack;              // r_cut - largest in-stencil |dx|, 0 when unbounded
    uint32_t solid_branch;            // the scene has more than one solid (shaders/mod.rs:51)
};

// The fields of a material the fluid pair loop reads (32 B).
struct FluidMat {
    float mass, c, d0, visc, bulk;
    uint32_t eos, stiff, pad;
};

// Kernel-wide view of the batch tables.
struct Tables {
    const SceneP* scenes;
    const DevMat* mats;
    const FluidMat* fmats;
    const DevInter* inter;
    uint32_t ncells;                  // total search cells of all scenes (the non-finite bucket follows)
    uint32_t max_nmat;                // largest per-scene material count
    uint32_t nscenes;
};

// Health counters written by device code.
struct DevStats {
    uint32_t max_cell_occupancy;
    uint32_t overflow_cells;
    uint32_t nonfinite_positions;
    uint32_t clamped_coordinates;
};

// One stage of the Runge-Kutta epilogue (fused into the fluid kernel).
// y_next = y0 + (c_prev0 k_0 + c_prev1 k_1 + c_prev2 k_2 + c_self k_stage)
// (terms with a zero coefficient skipped, in stage order), acc += c_acc *
// k_stage, and on the last stage y_new = y0 + acc.  Stage derivatives that a
// later stage reads are stored (non-diagonal tableaus only).
struct StageCoefs {
    int stage;          // 0-based
    int last;           // 1 when this stage ends the step
    float c_prev0, c_prev1, c_prev2;  // a[stage+1][j] * dt for j < stage
    float c_self;       // a[stage+1][stage] * dt (unused when last)
    float c_acc;        // b[stage] * dt
    int acc_first;      // 1 when no earlier stage contributed to acc
    int kick;           // 1: a velocity-Verlet kick, which leaves positions as they are
};

struct StageBuffers {
    const float4* y0_pd;   // y0 (storage order)
    const float4* y0_vm;
    float4* next_pd;       // y_{s+1} or y_new (storage order)
    float4* next_vm;
    float4* acc_pd;        // b-weighted derivative accumulator
    float4* acc_vm;
    float4* store_pd;      // where k of this stage is kept, or null
    float4* store_vm;
    const float4* prev0_pd;  // stored k_0, k_1, k_2 (null when not read)
    const float4* prev0_vm;
    const float4* prev1_pd;
    const float4* prev1_vm;
    const float4* prev2_pd;
    const float4* prev2_vm;
};

// Record `msg` as the calling thread's last error and return `code`.
arp_status set_error(arp_status code, const std::string& msg);

// ---- neighbor grid (neighbor.cu) -------------------------------------------
struct GridBuffers {
    uint32_t* key;         // [cap] cell id of each slot (ncells for non-finite)
    uint32_t* rank;        // [cap] arrival rank inside the cell
    uint32_t* count;       // [ncells + 1] occupancy (zeroed by the scan)
    uint32_t* start;       // [ncells + 2] exclusive prefix of count
    uint32_t* perm;        // [cap] sorted index -> slot
    uint2* coord;          // [cap] packed cell coordinates of each slot: x | y << 16, z
    uint32_t* block_sums;  // scan partials
    uint32_t block_sums_cap;
};

// Build cell_start / perm for `n` positions.  Counting sort: keys and
// histogram, exclusive scan, scatter, then ascending slot order within each
// cell.  Returns the number of kernel launches issued.
// The scene of item i is mats[material].scene, the material read from
// vm[i].w (bits) when vm is given, else from mat_u32[i].
// Counters a stage's later kernels start from zero (the fluid kernel's
// overflow counts and tile counter, the self-contact gate): the grid build's
// first kernel clears them, which saves a memset per counter per stage.
struct StageCounters {
    uint32_t* p[3] = {nullptr, nullptr, nullptr};
    uint32_t n[3] = {0, 0, 0};  // words at each pointer (at most 2)
};
int build_grid(const float4* pos, const float4* vm, const uint32_t* mat_u32, uint32_t n, const Tables& T,
               GridBuffers& gb, DevStats* stats, const uint32_t* boundary_start, cudaStream_t st,
               const StageCounters& zero = StageCounters{});

// Exclusive scan of `len` counts into out (len entries); clears `count`.
int exclusive_scan(uint32_t* count, uint32_t len, uint32_t* out, uint32_t* block_sums, cudaStream_t st);
// Scratch entries exclusive_scan needs for `len` items.
uint32_t scan_block_sums_needed(uint32_t len);

// out[k] = in[perm[k]] for float4 / uint32 arrays (nullptr entries skipped).
int gather_sorted(const uint32_t* perm, uint32_t n, const float4* a_in, float4* a_out, const float4* b_in,
                  float4* b_out, const uint32_t* c_in, uint32_t* c_out, const uint32_t* d_in, uint32_t* d_out,
                  cudaStream_t st);
// Gather a state into sorted order (out[k] = in[perm[k]]) and evaluate the
// pressure term p / rho^2 of every gathered particle (fluid.rs:45-52,
// :128,165).  Any pointer pair may be null.
// Solid-order copies a gather writes on the side: for a gathered particle
// whose solid id (sid_of_slot at its source slot) is valid, sx/sv/sc[sid] =
// its state and cell coordinates, and slot_of[sid] = its new index (when
// slot_of is given).
struct SolidScatter {
    const uint32_t* sid_of_slot = nullptr;
    const uint2* coord_of_slot = nullptr;
    float4* sx = nullptr;
    float4* sv = nullptr;
    uint2* sc = nullptr;
    uint32_t* slot_of = nullptr;
};
int gather_state(const uint32_t* perm, uint32_t n, const float4* pd_in, float4* pd_out, const float4* vm_in,
                 float4* vm_out, const uint32_t* a_in, uint32_t* a_out, const uint32_t* b_in, uint32_t* b_out,
                 const uint2* c_in, uint2* c_out, float* ps_out, const DevMat* mats, cudaStream_t st,
                 const SolidScatter& sol = SolidScatter{});

// Particle records (caller order) to structure of arrays in caller order, and
// back from cell order into caller order (the state exchange of the C ABI).
// Records carry each scene's own material index; the device state carries the
// batch-wide one (mat_of[i] for caller id i; mats[].local maps back).
int records_to_soa(const arp_particle* in, uint32_t n, const uint32_t* sid_of, const uint32_t* mat_of, float4* pd,
                   float4* vm, uint32_t* orig, uint32_t* sid, cudaStream_t st);
int soa_to_records(const float4* pd, const float4* vm, const uint32_t* orig, const uint32_t* sid, uint32_t n,
                   float pos_w, const DevMat* mats, arp_particle* out, cudaStream_t st);
// Sets flag bit 0 when a record's material differs from the handle's, bit 1
// when a w component differs from pos_w / zero.
int check_records(const arp_particle* in, uint32_t n, const uint32_t* mat_of, const DevMat* mats, float pos_w,
                  uint32_t* flag, cudaStream_t st);

// Neighbor counts within h of each sorted particle (mobile + boundary),
// computed with separately rounded float products for bit-exact output.
int count_neighbors(const float4* xs, const float4* vs, const uint32_t* start, uint32_t n, const float4* bxs,
                    const uint32_t* bstart, const Tables& T, uint32_t* out_sorted, cudaStream_t st);

// ---- fluid forces + stage update (fluid.cu) ---------------------------------
struct FluidArgs {
    const float4* xs;        // sorted stage positions/density
    const float4* vs;        // sorted stage velocity/material
    const uint32_t* start;   // mobile cell start (ncells + 1)
    const float4* bxs;       // boundary sorted
    const float4* bvs;
    const uint32_t* bstart;  // boundary cell start
    const uint32_t* perm;    // sorted -> storage slot (nullptr = identity)
    const uint32_t* sid;     // storage-order solid id
    const uint32_t* sid_of_boundary_index;  // per boundary caller id: solid id of the scene's mobile particle
                                            // with the same in-scene index, or invalid
    const uint32_t* borig;   // boundary caller ids, sorted
    const float* ps;         // p / rho^2 of each sorted particle
    const float* bps;        // p / rho^2 of each sorted boundary particle
    const float4* ksol;      // per-solid solid-term acceleration (nullptr when the solid branch is off)
    uint32_t* overflow;        // [2n] two queues: particles whose hit list filled up ([0, n)), and those
                               // whose list filled up inside one row ([n, 2n))
    uint32_t* overflow_count;  // [2] their numbers (cleared before each launch)
    uint32_t n;
    int solid_branch;
    int any_stiff_immobile;
    int counters_cleared;  // the stage's grid build cleared overflow_count and the tile counter
};
// Launch shapes of the fluid kernel the autotuner chooses between: threads
// per block, hit-list capacity, one tile per block or persistent blocks
// taking tiles from an atomic work counter, and whether a warp empties its
// lists by a vote before each search row (suited to dense scenes, where
// lists overflow).  Every shape evaluates the same pairs in the same order
// (a particle whose list fills up is finished by an overflow kernel in
// candidate order), so results do not depend on the choice.
struct FluidVariant {
    int block;       // threads per block
    int cap;         // hit-list entries per thread
    int persistent;  // tile-queue form
    int flush;       // warp-voted list flushes (kFlush) instead of pass 1 then pass 2
    int staged;      // candidates staged in shared memory per tile before the scan
                     // (1: cooperative loads, 2: bulk copies on an mbarrier)
};
constexpr int kNumFluidVariants = 15;
extern const FluidVariant kFluidVariants[kNumFluidVariants];
// `tile_counter` (one uint32 on the device) is used by persistent variants.
int launch_fluid(const FluidArgs& a, const Tables& T, int kdim, const StageCoefs& c, const StageBuffers& b,
                 int variant, uint32_t* tile_counter, cudaStream_t st);

// Velocity Verlet's kick and drift, in storage order: v' = v + (dt/2) a,
// rho' = rho + (dt/2) drho/dt, x' = x + dt v' from the derivative record
// (fpd, fvm) of the previous force evaluation; and the kick of a 4-float4
// per-solid field (the plastic strain).  Return the launches issued.
int verlet_kick_drift(const float4* pd, const float4* vm, const float4* fpd, const float4* fvm, uint32_t n, float half,
                      float full, float4* out_pd, float4* out_vm, cudaStream_t st);
int verlet_kick4(const float4* e, const float4* k4, uint32_t count, float half, float4* out, cudaStream_t st);

// ---- solids (solid.cu) ------------------------------------------------------
struct SolidRefList {
    uint32_t* off;   // [ns + 1]
    uint32_t* nbr;   // [nnz] solid id | 0x80000000 when same material
    float4* gw;      // [nnz] grad_w(X_j - X_i).xyz, w = vol0 of j
    uint32_t nnz;
};
// Reference-neighbor lists: counts per solid (pass 1), then after an
// exclusive scan of the counts into rl.off, the entries and L (pass 2).
// `gb` holds a grid built over the reference positions.
int ref_lists_count(const float4* ref, const uint32_t* mat_of_solid, uint32_t ns, const GridBuffers& gb,
                    const Tables& T, uint32_t* count, cudaStream_t st);
int ref_lists_fill(const float4* ref, const uint32_t* mat_of_solid, uint32_t ns, const GridBuffers& gb,
                   const Tables& T, SolidRefList& rl, float4* L, cudaStream_t st);

struct SolidArgs {
    const float4* ref;        // reference positions, w = rest volume m / rho0
    const float4* L;
    SolidRefList rl;
    const float4* ep;         // stage plastic strain (4 per solid)
    const float4* ep0;        // step-start plastic strain
    float4* ep_next;          // stage / step output
    float4* ep_acc;
    float4* ep_store;         // k of this stage, or null
    const float4* ep_prev0;   // stored k_0, k_1, k_2
    const float4* ep_prev1;
    const float4* ep_prev2;
    float4* F;                // [3*ns] deformation gradient columns (stage scratch)
    float4* A;                // [3*ns] sigma * L columns (stage scratch)
    float4* ksol;             // [ns] solid-term acceleration
    uint32_t* contact_bound;  // [2] max |u_i - u_0| bits, outside-box flag (cleared per stage)
    const float4* xs;         // sorted stage positions (current-neighbor loop)
    const float4* vs;
    const uint32_t* start;
    const uint32_t* sid_sorted;
    float4* sx;               // [ns] stage position + density in solid-id order (gathered per stage)
    float4* sv;               // [ns] stage velocity + material bits in solid-id order
    uint2* sc;                // [ns] packed cell coordinates in solid-id order
    const float2* stiff;      // [ns] per-solid (normal, shear) stiffness overriding the material's, or null
    uint32_t ns;
    int all_order2;           // every solid material has strain_order 2
    int any_plastic;          // some solid material is plastic; otherwise the plastic strain stays zero
    int counters_cleared;     // the stage's grid build cleared contact_bound
};
int launch_solid(const SolidArgs& a, const Tables& T, const StageCoefs& c, cudaStream_t st);

// ---- headless renderer ------------------------------------------------------------
struct RenderCfg {
    uint32_t W, H;                 // frame, pixels
    float s2, vx0, vy0;            // square viewport: size and lower-left corner
    float S;                       // sprite size, pixels
    float ca, sa, tx, ty, tz;      // view matrix terms
    float render_h;
    float kconst;                  // poly6 constant the fragment shader weighs alpha with
    int lighting;
    float light[3], lcol[3], amb, dif, spec;
    const float4* c1;              // per material: low-density colour
    const float4* c2;              // colour
    const float4* c3;              // high-density colour
    const float* d0;               // ramp centre density
    uint32_t nmat, nprims, tiles_x, tiles_y;
};
// sprites of boundary (prim_base 0) or mobile (prim_base = n_boundary)
// particles in caller order: PR = (window x, window y, clip w, window z),
// PC = colour, PP = view-space position
int render_project(const float4* pd, const float4* vm, const uint32_t* orig, uint32_t n, uint32_t prim_base,
                   const RenderCfg& c, float4* PR, float4* PC, float4* PP, cudaStream_t st);
uint32_t render_chunk_size();
uint32_t render_tile_size();
int render_bin_count(const float4* PR, const float4* PC, const RenderCfg& c, uint32_t* counts, cudaStream_t st);
int render_bin_scatter(const float4* PR, const float4* PC, const RenderCfg& c, const uint32_t* start,
                       uint32_t* fill, uint32_t* list, cudaStream_t st);
int render_composite(const float4* PR, const float4* PC, const RenderCfg& c, const uint32_t* start,
                     const uint32_t* list, uint8_t* rgb, cudaStream_t st);
int render_lit(const float4* PR, const float4* PC, const float4* PP, const RenderCfg& c, unsigned long long* zkey,
               uint8_t* rgb, cudaStream_t st);

// ---- adjoint (reverse mode of one integrator step) ------------------------------
// Quantities of one RK stage saved by a recording forward step.
struct AdjStage {
    const float4* pd;          // stage state, storage order (x, y, z, rho)
    const float4* vm;          // (vx, vy, vz, material bits)
    const uint32_t* perm;      // sorted index -> slot of the stage grid (null: identity)
    const uint32_t* start;     // cell starts of the stage grid
    const float4* F;           // [3*ns] deformation gradient columns
    const float4* A;           // [3*ns] sigma * L columns
    const float4* sx;          // [ns] solid-order state
    const float4* sv;
    const uint2* sc;           // [ns] packed cell coordinates
    const uint32_t* contact_bound;  // [2] self-contact gate of the stage
    const float4* ep;          // [4*ns] plastic strain of the stage (columns), null without plastic materials
};
struct AdjArgs {
    AdjStage st;
    const uint32_t* sid;       // slot -> solid id
    const uint32_t* slot_of;   // solid id -> slot
    const float4* mu_pd;       // adjoint of the stage derivative k_s, storage order: (x, y, z, rho)
    const float4* mu_vm;       // (vx, vy, vz, 0)
    float4* lam_pd;            // adjoint of the stage state Y_s (accumulated)
    float4* lam_vm;
    const float4* bxs;         // boundary, cell order
    const float4* bvs;
    const uint32_t* bstart;
    const float* bps;
    const float4* ref;         // reference positions, w = rest volume m / rho0
    const float4* L;
    SolidRefList rl;
    const float2* stiff;       // per-solid stiffness override or null
    float4* lamF;              // [3*ns] adjoint of F (columns), scratch
    float4* lamFd;             // [3*ns] adjoint of dF/dt
    double2* g_stiff;          // [ns] accumulated dL/d(normal, shear) stiffness
    uint32_t* flags;           // bit 0: an active self-contact pair (not differentiated)
    float4* w;                 // [n] scratch: per-particle weights of the stage
    float4* eq;                // [n] scratch: per-particle state-equation terms
    float4* xs;                // [n] scratch: the stage positions in cell order
    uint32_t n, ns;
    int solid_branch;
    int all_order2;            // every solid material has strain order 2
    const float4* mu_ep;       // [4*ns] adjoint of the stage's plastic-strain rate (columns), or null
    float4* lam_ep;            // [4*ns] adjoint of the stage's plastic strain (accumulated)
};
// One stage VJP: lam_{Y_s} += J_f(Y_s)^T mu_s (+ stiffness gradients).  Returns launches.
int launch_adjoint_stage(const AdjArgs& a, const Tables& T, int kdim, cudaStream_t st);
// The same weights for a plain array of `n` float4 (the plastic strain:
// every component kept).
int adjoint_stage_weights_all(uint32_t n, float cb, const float4* lam, int nlater, const float* ca,
                              const float4* const* lamY, float4* mu, cudaStream_t st);
// out = lam + sum_s lamY[s] for a plain array of `n` float4.
int adjoint_step_sum_all(uint32_t n, const float4* lam, int stages, const float4* const* lamY, float4* out,
                         cudaStream_t st);
// Velocity Verlet: the weights of a step's force evaluation,
// mu = lam_f + (dt/2) P lam (P keeps the density and velocity parts), and the
// kick-drift's adjoint in place (caller order), writing the adjoint of the
// carried record it read.  h = dt/2.
int verlet_adjoint_weights(uint32_t n, const float4* lsp, const float4* lsv, const float4* lfp, const float4* lfv,
                           float h, float4* mp, float4* mv, cudaStream_t st);
int verlet_kick_drift_adjoint(uint32_t n, float4* lp, float4* lv, float h, float dt, float4* lfp, float4* lfv,
                              cudaStream_t st);
// mu = cb * lam_next + sum_t ca[t] * lamY[t] over the given later stages.
int adjoint_stage_weights(uint32_t n, float cb, const float4* lam_pd, const float4* lam_vm, int nlater,
                          const float* ca, const float4* const* lamY_pd, const float4* const* lamY_vm,
                          float4* mu_pd, float4* mu_vm, cudaStream_t st);
// lam_out = lam_next + sum_s lamY[s]
int adjoint_step_sum(uint32_t n, const float4* lam_pd, const float4* lam_vm, int stages,
                     const float4* const* lamY_pd, const float4* const* lamY_vm, float4* out_pd, float4* out_vm,
                     cudaStream_t st);
// Caller order <-> storage order by orig (slot -> caller id).
int adjoint_gather(uint32_t n, const uint32_t* orig, const float4* in_pd, const float4* in_vm, float4* out_pd,
                   float4* out_vm, cudaStream_t st);
int adjoint_scatter(uint32_t n, const uint32_t* orig, const float4* in_pd, const float4* in_vm, float4* out_pd,
                    float4* out_vm, cudaStream_t st);
// 8 floats per particle (x, y, z, rho, vx, vy, vz, unused) <-> two float4
// arrays, the unused one written and read as 0.
int adjoint_unpack(uint32_t n, const float4* in2, float4* p, float4* v, cudaStream_t st);
int adjoint_pack(uint32_t n, const float4* p, const float4* v, float4* out2, cudaStream_t st);

}  // namespace arp
