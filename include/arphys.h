/*
 * arphys.h -- C ABI of the B200-native SPH time step.
 *
 * This is the drop-in boundary for the simulation-step interface of
 * jsmith628/ar-physics, `FluidSim` (src/soft_body/mod.rs:23-275).  Each entry
 * point names the reference method it replaces.  The reference binds its GPU
 * work through OpenGL buffers; here the state lives in CUDA device memory
 * owned by an opaque `arp_sim` handle, and the host exchanges particles in the
 * reference's own std430 record layouts (`Particle`, `SolidParticle`,
 * `Material`, `MatInteraction`), so a caller that already builds those records
 * passes them unchanged.
 *
 * Rules shared by every call:
 *   - every call returns an `arp_status`; ARP_OK is 0.  No call aborts the
 *     process.  `arp_last_error()` gives a message for the calling thread's
 *     last failure.
 *   - a handle is used by one host thread at a time; different handles are
 *     independent and may be driven from different threads.
 *   - each handle owns a CUDA stream (or uses the one given by
 *     `arp_sim_set_stream`); device work of a call is ordered on that stream.
 *   - host buffers passed in are only read during the call; host buffers
 *     passed out are written before the call returns -- except for the two
 *     `_async` exchange calls, whose buffers belong to the library until the
 *     next `arp_sim_synchronize`.
 */
#ifndef ARPHYS_H
#define ARPHYS_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ARP_ABI_VERSION 1u
#define ARP_INVALID_INDEX 0xFFFFFFFFu

typedef enum arp_status {
    ARP_OK = 0,
    ARP_ERR_INVALID_ARG = 1,  /* null pointer, bad count, bad enum, init order */
    ARP_ERR_CUDA = 2,         /* a CUDA runtime call failed (message has the name) */
    ARP_ERR_NAN_STATE = 3,    /* a non-finite position reached the neighbor build */
    ARP_ERR_CELL_OVERFLOW = 4,/* strict mode only: a cell held more than 128 entries */
    ARP_ERR_TIMEOUT = 5,      /* a bounded device-side wait gave up */
    ARP_ERR_UNSUPPORTED = 6,  /* a scene feature this build does not implement */
    ARP_ERR_OUT_OF_MEMORY = 7,
    ARP_ERR_PARSE = 8,        /* scene file syntax or schema error */
    ARP_ERR_IO = 9,           /* scene file could not be read */
    ARP_ERR_CAPACITY = 10     /* a caller-provided output buffer is too small */
} arp_status;

/* Equation of state ids, src/soft_body/material_region/material.rs:54-59 and
 * the shader switch in src/soft_body/shaders/fluid.rs:45-52. */
enum { ARP_EOS_ZERO = 0, ARP_EOS_CONSTANT = 1, ARP_EOS_IDEAL_GAS = 2, ARP_EOS_TAIT = 3 };

/* Contact potential ids, src/soft_body/material_region/interaction.rs:21-28. */
enum {
    ARP_CONTACT_ZERO = 0, ARP_CONTACT_CONSTANT = 1, ARP_CONTACT_LINEAR = 2,
    ARP_CONTACT_TAIT = 3, ARP_CONTACT_LENNARD_JONES = 4, ARP_CONTACT_HERTZ = 5
};

/* Explicit integrators named by the reference's scene loader
 * (examples/test.rs:165-180).  The tableaus are the textbook ones; the
 * reference takes them from the un-vendored crate numerical-integration
 * 0.0.1, so the exact stage arithmetic there is not observable. */
typedef enum arp_integrator {
    ARP_INT_EULER = 0,     /* "euler", "rk1" */
    ARP_INT_MIDPOINT = 1,  /* "midpoint", "rk2" */
    ARP_INT_HEUN2 = 2,     /* "heun2", "heun" */
    ARP_INT_RALSTON = 3,   /* "ralston" */
    ARP_INT_RK3 = 4,       /* "rk3" (Kutta's third-order method) */
    ARP_INT_HEUN3 = 5,     /* "heun3" */
    ARP_INT_RK4 = 6,       /* "rk4" */
    ARP_INT_RK_3_8 = 7,    /* "rk_3_8" */
    ARP_INT_VERLET = 8     /* "verlet": velocity Verlet, kick-drift-kick (see arp_sim_step) */
} arp_integrator;

/* `Material`, std430, 80 bytes (src/soft_body/material_region/material.rs:11-28).
 * GLSL `bool` fields are 4-byte integers. */
typedef struct arp_material {
    uint32_t immobile;
    float mass, start_den;
    uint32_t state_eq;
    float sound_speed, target_den, visc, bulk_visc;
    int32_t strain_order;
    float normal_stiffness, shear_stiffness, normal_damp, shear_damp;
    uint32_t plastic;
    float yield_strength, work_hardening, work_hardening_exp, kinematic_hardening, thermal_softening;
    float relaxation_time;
} arp_material;

/* `MatInteraction`, std430, 20 bytes (src/soft_body/material_region/interaction.rs:10-14). */
typedef struct arp_interaction {
    uint32_t potential;
    float strength, radius;
    float dampening, friction;
} arp_interaction;

/* `Particle`, std430, 48 bytes (src/soft_body/particle_state/mod.rs:24-29):
 * den@0 mat@4 solid_id@8 pos@16 vel@32.  The same record carries time
 * derivatives where the reference uses it as a derivative container. */
typedef struct arp_particle {
    float den;
    uint32_t mat;
    uint32_t solid_id;
    uint32_t _pad0;
    float pos[4];
    float vel[4];
} arp_particle;

/* `SolidParticle`, std430, 96 bytes (src/soft_body/particle_state/mod.rs:31-35).
 * `stress` is the accumulated plastic strain, column-major mat4. */
typedef struct arp_solid_particle {
    uint32_t part_id;
    uint32_t _pad0[3];
    float ref_pos[4];
    float stress[16];
} arp_solid_particle;

/* `AABB` (src/soft_body/material_region/region.rs:11-14). */
typedef struct arp_aabb {
    float min[4];
    float dim[4];
} arp_aabb;

/* Everything `FluidSim::new` receives (src/soft_body/mod.rs:58-66), after the
 * regions have been turned into particles (the reference does that inside
 * `new` with `MaterialRegion::gen_particles`; `arp_sim_create_from_toml`
 * does it here).  Particle `mat` fields index `materials`.  Mobile particles
 * must use materials with immobile == 0, boundary particles materials with
 * immobile != 0.  `solid_id` fields of the input are ignored: solid ids are
 * assigned in particle order to particles whose material has non-zero
 * stiffness, as `Particles::init_solid_particles` does
 * (src/soft_body/particle_state/particles.rs:488-506). */
typedef struct arp_scene {
    const arp_particle* particles;     /* mobile particles, n_particles */
    uint32_t n_particles;
    const arp_particle* boundary;      /* immobile particles, n_boundary (may be 0) */
    uint32_t n_boundary;
    const arp_material* materials;     /* n_materials */
    uint32_t n_materials;
    /* Optional n_materials x n_materials interaction table (row-major) and
     * matching "given" flags.  Pairs not given are resolved exactly as
     * src/soft_body/mod.rs:93-111 does (symmetric copy, else
     * MatInteraction::default_between for i != j, else zero).  With
     * interactions == NULL every pair is resolved by default; with
     * interaction_given == NULL every entry of `interactions` is used. */
    const arp_interaction* interactions;
    const uint8_t* interaction_given;
    arp_aabb bounds;
    float kernel_radius;
    int32_t integrator;                /* arp_integrator */
    float timestep;
    uint32_t subticks;
    float gravity;
    float artificial_viscocity;        /* kept for the record: the step reads bulk_visc */
} arp_scene;

typedef struct arp_sim arp_sim;

/* Per-segment device time, the reference's profiler segments
 * (src/profiler.rs:10-81; "Bucketting", "Forces", "Arith").  Filled from CUDA
 * events when profiling is enabled; reading resets the accumulators. */
typedef struct arp_profile {
    uint64_t steps;              /* integrator steps since the last read */
    uint64_t launches;           /* kernels launched by the handle since the last read */
    double neighbor_ms;          /* grid build: keys, histogram, scan, scatter, reorder */
    double solid_ms;             /* deformation gradient, stress, solid forces */
    double fluid_ms;             /* fluid forces + fused stage update */
    double integrate_ms;         /* stand-alone stage arithmetic (non-fused paths) */
    uint64_t fluid_launches;
    uint64_t neighbor_launches;
    uint64_t solid_launches;
    uint64_t stages;             /* Runge-Kutta stages evaluated */
} arp_profile;

/* Health counters collected on the device during steps. */
typedef struct arp_stats {
    uint32_t max_cell_occupancy;   /* largest mobile+boundary count of one cell seen */
    uint32_t overflow_cells;       /* cells seen above the reference's 128-slot bucket */
    uint32_t nonfinite_positions;  /* positions the grid build found NaN/Inf */
    uint32_t clamped_coordinates;  /* coordinates exactly on the upper box face */
} arp_stats;

/* Device view of the current state (the headless stand-in for the GL buffers
 * that `FluidSim::particles()` hands to the renderer,
 * src/soft_body/mod.rs:172-174).  Pointers are owned by the handle and valid
 * until the next call that steps or changes the particle set.  Particles are
 * stored in cell order; `orig_id[k]` gives the caller-order index of slot k. */
typedef struct arp_device_view {
    const void* pos_den;   /* float4[n]: x, y, z, density */
    const void* vel_mat;   /* float4[n]: vx, vy, vz, material id as uint32 bits */
    const void* orig_id;   /* uint32[n] */
    uint32_t n;
} arp_device_view;

/* ---- lifecycle (FluidSim::new / init / drop) ------------------------------ */

/* FluidSim::new, src/soft_body/mod.rs:58-166. */
arp_status arp_sim_create(const arp_scene* scene, arp_sim** out);
/* Several independent scenes stepped together (the batched form; the
 * reference has no batching).  Scenes keep their own box, kernel radius,
 * gravity, materials and interactions; they must share the integrator, time
 * step and subticks.  Particles of scene k occupy the caller-order range
 * reported by arp_sim_scene_range, and records carry each scene's own
 * material indices.  arp_sim_create(s) is arp_sim_create_batch(s, 1). */
arp_status arp_sim_create_batch(const arp_scene* scenes, uint32_t count, arp_sim** out);
arp_status arp_sim_num_scenes(const arp_sim* sim, uint32_t* out);
/* Caller-order particle range, boundary range and global cell range of one
 * scene (any output may be NULL). */
arp_status arp_sim_scene_range(const arp_sim* sim, uint32_t scene, uint32_t* first_particle,
                               uint32_t* n_particles, uint32_t* first_boundary, uint32_t* n_boundary,
                               uint32_t* first_cell, uint32_t* n_cells);
/* FluidSim::new after examples/test_mods/config.rs:298-474 parses a scene
 * file and src/soft_body/material_region/mod.rs:56-155 seeds its regions. */
arp_status arp_sim_create_from_toml(const char* path, arp_sim** out);

/* ---- scene files (host only; no CUDA call) ----------------------------------- */

/* A scene file in the schema of examples/test_mods/config.rs, parsed and
 * seeded on the host.  Replaces `Config::parse` (config.rs:298-474) followed by
 * the seeding loop of `FluidSim::new` (src/soft_body/mod.rs:70-86, which calls
 * `MaterialRegion::gen_particles`, material_region/mod.rs:56-156): materials in
 * object order (boundaries, then objects, each by name), boundary and mobile
 * particles in that order, the n_materials^2 interaction table with a `given`
 * flag per entry.  STL regions ("model", examples/test_mods/mesh.rs) are read
 * from paths relative to the working directory; objects with "on_click" are
 * interactive additions and are skipped; an integrator name outside the
 * reference's list gives ARP_ERR_PARSE, as does an unreadable STL file or any
 * schema error the reference would panic on. */
typedef struct arp_scene_file arp_scene_file;
arp_status arp_scene_file_load(const char* path, arp_scene_file** out);
/* Points `out` at the file's records; valid until arp_scene_file_free. */
arp_status arp_scene_file_scene(const arp_scene_file* file, arp_scene* out);
/* The scene's "name" (default "Fluid Test"), NUL-terminated, owned by `file`. */
arp_status arp_scene_file_name(const arp_scene_file* file, const char** name);
arp_status arp_scene_file_free(arp_scene_file* file);
/* The file's objects marked "on_click" (config.rs:426-446), by name: seeded
 * with the file's kernel radius and material id 0, as FluidSim::add_particles
 * seeds them (src/soft_body/mod.rs:180-182).  A host passes one to
 * arp_sim_add_particles, with the pointer position as `offset` when
 * `*relative` is 1 (examples/test_mods/renderer.rs:388-409). */
arp_status arp_scene_file_on_click_count(const arp_scene_file* file, uint32_t* count);
arp_status arp_scene_file_on_click(const arp_scene_file* file, uint32_t index, const arp_particle** particles,
                                   uint32_t* n, arp_material* material, int* relative);
/* FluidSim::init, src/soft_body/mod.rs:213-233. */
arp_status arp_sim_init(arp_sim* sim);
/* Drop of FluidSim. */
arp_status arp_sim_destroy(arp_sim* sim);

/* ---- stepping -------------------------------------------------------------- */

/* FluidSim::update, src/soft_body/mod.rs:235-274: `subticks` integrator steps
 * of timestep/subticks. */
arp_status arp_sim_update(arp_sim* sim);
/* `nsteps` integrator steps of timestep/subticks (update() without the
 * subtick grouping).
 * Velocity Verlet (ARP_INT_VERLET; the reference's default integrator,
 * examples/test_mods/config.rs:451) is taken as the textbook kick-drift-kick
 * over the derivative record f = (drho/dt, a) of the force evaluation
 * (src/soft_body/shaders/mod.rs:11-86), with dt' = timestep/subticks:
 *   v' = v + (dt'/2) a_n, rho' = rho + (dt'/2) drho_n/dt, x_{n+1} = x + dt' v',
 *   f_{n+1} = f(x_{n+1}, v', rho'),
 *   v_{n+1} = v' + (dt'/2) a_{n+1}, rho_{n+1} = rho' + (dt'/2) drho_{n+1}/dt
 * (the plastic strain is kicked like the density).  Positions move only in
 * the drift, with the velocity closure of FluidSim::update (state.velocity(),
 * src/soft_body/mod.rs:256), so the position part of f is not used.  f_n is
 * carried from the previous step; the first step after init, set_particles
 * or add_particles first evaluates f at the current state, as init_with_vel
 * does in FluidSim::init (src/soft_body/mod.rs:213-233).  The scheme inside
 * the un-vendored crate numerical-integration is not observable, so this is
 * a stated assumption, like the Runge-Kutta tableaus. */
arp_status arp_sim_step(arp_sim* sim, uint32_t nsteps);
/* Time every launch shape of the fluid kernel (128 or 256 threads per block,
 * 48 or 96 listed neighbors per thread, one tile per block or persistent
 * blocks on a tile queue, lists evaluated after the scan or emptied whenever
 * a warp's next row could overfill one, or the tile's candidates staged in
 * shared memory before the scan, 64 or 128 threads per block) on the current
 * state and keep the fastest; arp_sim_init does this once per (dimension,
 * particle count, h/spacing) bucket and reuses the choice afterwards.  The
 * shapes evaluate identical arithmetic, so results do not depend on it. */
arp_status arp_sim_autotune(arp_sim* sim, int* variant);
arp_status arp_sim_fluid_variant(const arp_sim* sim, int* variant, int* block, int* persistent);
/* Pin the fluid kernel's launch shape (0 .. arp_fluid_variant_count() - 1). */
arp_status arp_sim_set_fluid_variant(arp_sim* sim, int variant);
/* The number of launch shapes of the fluid kernel. */
int arp_fluid_variant_count(void);
/* Replay each step from a CUDA graph captured on the handle's stream (two
 * graphs, one for each of the two buffer sets consecutive steps alternate
 * between; captured on first use and again after the stream or the buffers
 * change).  Steps sampled by arp_sim_profile_enable and steps on a tape run
 * as plain launches.  Off by default. */
arp_status arp_sim_set_graph(arp_sim* sim, int enable);

/* ---- queries (FluidSim accessors, src/soft_body/mod.rs:168-178) ------------ */

arp_status arp_sim_time(const arp_sim* sim, float* out);
arp_status arp_sim_kernel_radius(const arp_sim* sim, float* out);
arp_status arp_sim_num_materials(const arp_sim* sim, uint32_t* out);
arp_status arp_sim_counts(const arp_sim* sim, uint32_t* n_particles, uint32_t* n_boundary,
                          uint32_t* n_solids);
arp_status arp_sim_dim(const arp_sim* sim, uint32_t* out);

/* FluidSim::particles() read back, src/soft_body/particle_state/particles.rs:534-541:
 * mobile particles in caller order (`cap` >= n_particles). */
arp_status arp_sim_get_particles(arp_sim* sim, arp_particle* out, uint32_t cap);
/* Solid records in solid-id order (`cap` >= n_solids). */
arp_status arp_sim_get_solids(arp_sim* sim, arp_solid_particle* out, uint32_t cap);
arp_status arp_sim_get_boundary(arp_sim* sim, arp_particle* out, uint32_t cap);
arp_status arp_sim_get_materials(const arp_sim* sim, arp_material* out, uint32_t cap);
/* The resolved interaction tables (src/soft_body/mod.rs:93-111): one
 * n_materials^2 block per scene, in scene order. */
arp_status arp_sim_get_interactions(const arp_sim* sim, arp_interaction* out, uint32_t cap);
/* Replace the mobile state (den, pos, vel) of all particles, caller order;
 * mat and solid_id of the input must match the handle's. */
arp_status arp_sim_set_particles(arp_sim* sim, const arp_particle* in, uint32_t n);
/* Asynchronous forms of arp_sim_set_particles / arp_sim_get_particles (no
 * counterpart in the reference, whose particles() hands out GL buffers): the
 * records cross PCIe on copy streams of the handle's own through two device
 * staging slots each way, ordered with the steps on the handle's stream by
 * events, so that the copy of the next state in, a step and the copy of the
 * last result out overlap.  Both return before their copies finish: `in`
 * must stay unchanged and `out` is valid only after arp_sim_synchronize.
 * Page-locked host memory lets the copies run truly asynchronously.  The
 * record checks of arp_sim_set_particles run on the device and are
 * reported by the next arp_sim_synchronize (ARP_ERR_INVALID_ARG for a
 * changed material, ARP_ERR_UNSUPPORTED for a changed w component); the
 * state they replaced takes materials and solid ids from the handle's own
 * tables either way. */
arp_status arp_sim_set_particles_async(arp_sim* sim, const arp_particle* in, uint32_t n);
arp_status arp_sim_get_particles_async(arp_sim* sim, arp_particle* out, uint32_t cap);
/* Wait for the handle's device work and asynchronous copies; reports the
 * checks of asynchronous sets since the last call. */
arp_status arp_sim_synchronize(arp_sim* sim);
arp_status arp_sim_device_state(arp_sim* sim, arp_device_view* out);

/* FluidSim::add_particles, src/soft_body/mod.rs:180-206 with
 * Particles::add_particles, src/soft_body/particle_state/particles.rs:547-631.
 * `p` holds particles already seeded for `material` (their `mat` and
 * `solid_id` fields are ignored); `offset` (4 floats, may be NULL) is added to
 * their positions in f32.  They take the first material equal to `material`
 * in every field, or a new one (always new for a material with stiffness),
 * and are appended after the existing particles; the simulated time and the
 * reference positions and plastic strain of existing solids are kept, new
 * solids take their current positions as reference.  A new material gets
 * MatInteraction::default_between with every other material (and itself,
 * unless it is a solid).  `*material_added` receives 1 when a material entry
 * was appended.  n == 0 adds nothing.  Requires arp_sim_init; a batch of
 * scenes or an immobile material gives ARP_ERR_UNSUPPORTED.  Any captured
 * CUDA graph is dropped. */
arp_status arp_sim_add_particles(arp_sim* sim, const arp_particle* p, uint32_t n,
                                 const arp_material* material, const float* offset,
                                 int* material_added);

/* ---- neighbor grid (src/soft_body/neighbor_list.rs) ------------------------ */

/* Grid shape: subdivisions as NeighborList::new computes them (:199-217) for
 * scene 0, and the cell count of all scenes. */
arp_status arp_sim_grid(const arp_sim* sim, uint32_t subdivisions[4], uint32_t* n_cells);
/* Build the grid for the current positions and copy it out in the reference's
 * terms: `cell_of[i]` = bucket of mobile particle i (caller order), or
 * ARP_INVALID_INDEX for a non-finite position; `cell_start` (n_cells+1) and
 * `members` (n_particles) = mobile particles of each cell in ascending caller
 * id; `nbr_count[i]` = mobile + boundary particles within the kernel radius
 * among the 27 cells around i (i itself included).  Any output may be NULL. */
arp_status arp_sim_neighbors(arp_sim* sim, uint32_t* cell_of, uint32_t* cell_start,
                             uint32_t* members, uint32_t* nbr_count);
/* Boundary section of the grid: `cell_start` (n_cells+1), `members`
 * (n_boundary) in ascending boundary id. */
arp_status arp_sim_boundary_cells(arp_sim* sim, uint32_t* cell_start, uint32_t* members);

/* ---- allocation-free grid build -------------------------------------------- */

/* No counterpart in the reference (whose buckets live in a GL buffer the
 * simulation allocates).  Builds the cell grid of NeighborList::new's shape
 * for `n` caller-owned device positions without allocating any memory, for
 * callers that cannot call cudaMalloc on this path: code running inside a
 * host framework that owns the device allocator (a caching allocator or an
 * engine's pre-reserved heap), or a real-time loop that forbids allocation
 * after start-up.
 *   pos_den     device float4[n] (x, y, z used; 16-byte aligned), n <= 1048576
 *   cell_start  device uint32[n_cells + 2], n_cells = prod_a max(1, floor(dim_a / h))
 *               <= 4194302: entries c..c+1 bound the slots of cell c, the last
 *               two bound the non-finite positions
 *   perm        device uint32[n]: slot -> input index, ascending inside a cell
 *   stream      cudaStream_t (NULL = the legacy default stream); the call is
 *               asynchronous on it.
 * Scratch (ranks and scan partials) is a file-scope device array of 4 MiB +
 * 4 KiB that every GPU which loads the library holds until the process
 * exits.  The first call on a device looks up that array's device address
 * (cudaGetSymbolAddress) with the device current; make that first call
 * before any stream capture.  All calls share the one array, so calls whose
 * work overlaps on the GPU (different streams or threads without ordering)
 * race and corrupt each other's output.  Sizes beyond the maxima (a kernel
 * radius so small against the box that a cell count would not fit in 32 bits
 * included) return ARP_ERR_CAPACITY without launching anything. */
arp_status arp_grid_build_noalloc(const void* pos_den, uint32_t n, const arp_aabb* bounds, float kernel_radius,
                                  uint32_t* cell_start, uint32_t cell_start_capacity, uint32_t* perm,
                                  void* stream);

/* ---- streams, profiling, health ------------------------------------------- */

/* Use a caller-owned CUDA stream (cudaStream_t passed as void*); NULL returns
 * to the handle's own stream. */
arp_status arp_sim_set_stream(arp_sim* sim, void* stream);
/* (arp_sim_synchronize is declared with the asynchronous exchange above.) */
/* Per-segment timing (grid build, solid, fluid) with CUDA events between the
 * launches of a step.  enable = 0 stops it; enable = N >= 1 records the events
 * on one step in every N (1: every step; each event costs the step a few
 * microseconds, so a long timed run samples); arp_sim_profile_read reports
 * the sampled steps only. */
arp_status arp_sim_profile_enable(arp_sim* sim, int enable);
arp_status arp_sim_profile_read(arp_sim* sim, arp_profile* out);
arp_status arp_sim_stats(arp_sim* sim, arp_stats* out);
/* Kernels launched by this handle since creation. */
arp_status arp_sim_launch_count(const arp_sim* sim, uint64_t* out);

/* Thread-local message of the last failing call ("" when none). */
const char* arp_last_error(void);
uint32_t arp_abi_version(void);

/* ---- headless rendering (examples/test_mods/renderer.rs) --------------------- */

/* The camera of renderer.rs:338-349: the view matrix rotates by `angle`
 * (radians) about y, translates by -view_pos and moves by 1 - scale along z;
 * clip w = z + 1. */
typedef struct arp_view {
    float angle;      /* view_angle, in radians */
    float pos[2];     /* view_pos */
    float scale;      /* view_scale */
} arp_view;

/* The shader settings of renderer.rs:189-210.  `colors` holds 12 floats per
 * material (RGBA of "color", "color_low_density", "color_high_density") and
 * `densities` the density the colour ramp is centred on (the material's
 * start density), both indexed by material id. */
typedef struct arp_render_style {
    float render_h;            /* kernel_radius * particle_render_factor */
    int32_t lighting;          /* sphere shading with depth test, else density-ramp splats */
    float light_pos[3], light_color[3];
    float ambient, diffuse, specular;
    uint32_t n_materials;
    const float* colors;
    const float* densities;
} arp_render_style;

/* One frame of the recording path (renderer.rs:305-478) without a graphics API:
 * boundary particles then mobile particles, each in caller order, drawn as
 * point sprites of render_h * min(width, height) pixels into a square viewport
 * centred in the frame, over a white background; without lighting each sprite
 * is a poly6-weighted disc in the density-ramp colour, composited in draw order
 * with the blend the reference configures (src*(1-dst.a) + dst*(1-src.a), the
 * destination alpha staying 0) into 8-bit channels; with lighting the nearest
 * sprite of each pixel is shaded as a sphere.  `out_rgb` (host) receives
 * width * height * 3 bytes, rows from bottom to top as glReadnPixels returns
 * them.  A scene's particles are drawn with global material ids. */
arp_status arp_sim_render_rgb24(arp_sim* sim, const arp_view* view, const arp_render_style* style, uint32_t width,
                                uint32_t height, uint8_t* out_rgb);
/* The view and style a scene file sets (config.rs:302-323,466-470); `colors`
 * and `densities` point into `file`. */
arp_status arp_scene_file_render_settings(const arp_scene_file* file, arp_view* view, arp_render_style* style);

/* ---- per-particle stiffness and reverse mode (no counterpart in the reference) -- */

/* Per-solid (normal, shear) stiffness — the Lame pair the reference keeps per
 * material in `normal_stiffness`/`shear_stiffness` (same sign convention) —
 * overriding the materials' values in the stress (solid.rs:139-141,339), 2
 * floats per solid in solid-id order; NULL restores the material values.
 * `ns` must equal the handle's solid count. */
arp_status arp_sim_set_solid_stiffness(arp_sim* sim, const float* normal_shear, uint32_t ns);

/* Reverse-mode differentiation of the steps taken after arp_tape_begin.  The
 * state before every `checkpoint_every`-th step is kept; arp_tape_backward
 * re-runs each segment from its checkpoint recording the stage states, then
 * applies the hand-written adjoint of every stage (neighbor sets reused, not
 * differentiated) in reverse.  CUDA-graph replay is off while a tape records.
 * Refused (ARP_ERR_UNSUPPORTED) for plastic materials, strain orders other
 * than 2 and contact friction; a self-contact pair found active during the
 * backward pass makes it return ARP_ERR_UNSUPPORTED after filling the outputs
 * (that term is not differentiated). */
arp_status arp_tape_begin(arp_sim* sim, uint32_t checkpoint_every);
arp_status arp_tape_end(arp_sim* sim);
arp_status arp_tape_steps(const arp_sim* sim, uint64_t* steps);
/* `dl_dstate`: dL/d(state after the last recorded step), 8 floats per mobile
 * particle in caller order (dx, dy, dz, drho, dvx, dvy, dvz, unused).
 * `grad_state0` receives dL/d(state when the tape began) in the same layout;
 * `grad_stiffness` (may be NULL) dL/d(normal, shear) per solid in solid-id
 * order, with the materials' values where no per-solid stiffness is set.  The
 * handle's current state is unchanged. */
arp_status arp_tape_backward(arp_sim* sim, const float* dl_dstate, float* grad_state0, float* grad_stiffness);

#ifdef __cplusplus
}
#endif

#endif /* ARPHYS_H */
