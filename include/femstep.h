/*
 * femstep.h -- C ABI of the B200 explicit structural FEM step.
 *
 * One shared library, libfemstep.so, built for sm_100a.  Plain C types only: host
 * pointers and sizes in, status codes out.  Every entry point below names the
 * reference interface it replaces (paths relative to the solarbaron/sinking-simulator
 * source tree).
 *
 * Status codes: 0 is success.  FEMSTEP_SKIP means "no usable CUDA device": callers
 * degrade exactly as the reference's Vulkan back-ends do when there is no device
 * (engine/gpu/fem_gpu.hpp:21-22, engine/gpu/zone_gpu.hpp:186-202).  Every other
 * non-zero code is an error whose text is available from the *_error function of the
 * handle, or femstep_last_error() when no handle was made.
 *
 * Threading: a handle is used from one host thread at a time, like the reference's
 * solvers.  Handles are independent; each owns its device memory and stream.
 */
#ifndef FEMSTEP_H
#define FEMSTEP_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FEMSTEP_OK 0
#define FEMSTEP_SKIP 1      /* no CUDA device */
#define FEMSTEP_EINVAL 2    /* a size, index or adjacency that does not describe a mesh */
#define FEMSTEP_ENOMEM 3    /* device or host allocation failed / over the memory budget */
#define FEMSTEP_ECUDA 4     /* a CUDA call failed */
#define FEMSTEP_ESTATE 5    /* call out of order (e.g. run before upload) */
#define FEMSTEP_ETIMEOUT 6  /* a bounded device-side wait gave up; the outputs of that launch are undefined */

/* Text of the last error raised on this thread by a call that has no handle yet. */
const char *femstep_last_error(void);
/* Name of the current CUDA device, or FEMSTEP_SKIP.  Mirrors gpu::FemGpuSolver::deviceName
   (engine/gpu/fem_gpu.hpp:37). */
int femstep_device_name(char *buffer, size_t length);
/* Select the CUDA device the calling thread's subsequent handles are made on (one
   process per GPU: device = local rank).  No reference counterpart: the reference
   picks the first discrete Vulkan device (engine/gpu/fem_gpu.cpp:207-213). */
int femstep_set_device(int device);

/* =====================================================================================
 * Linear-tet step.  Replaces gpu::FemGpuSolver (engine/gpu/fem_gpu.hpp:17-45) and
 * extends it to the J2 tet.
 * ===================================================================================== */

typedef enum {
    /* Co-rotational linear-elastic tet in float, arithmetic of fem::tetForces /
       fem::stepCpu (engine/sim/fem.cpp:73-117, 187-215): bit-identical to the
       reference CPU step.  Uses the caller's mass / restInv / restVolume. */
    FEMSTEP_TET_REF32 = 0,
    /* J2 tet (linear isotropic hardening), FP32, displacement state, no compensation. */
    FEMSTEP_TET_J2_F32 = 1,
    /* J2 tet, FP32 with Kahan-compensated displacement and plastic strain. */
    FEMSTEP_TET_J2_F32K = 2,
    /* J2 tet in FP64: fem.cpp's kinematics with plasticity::update
       (engine/sim/plasticity.cpp:319-505) at the single point; bit-identical to the
       FP64 CPU composition of those two. */
    FEMSTEP_TET_J2_F64 = 3
} femstep_tet_mode;

/* The reference's sim::fem::TetMesh (engine/sim/fem.hpp:38-68), as raw arrays. */
typedef struct {
    size_t nodes, tets;
    const float *position;          /* 3N, fem.hpp:40 */
    const float *velocity;          /* 3N, fem.hpp:41; NULL = at rest */
    const float *mass;              /* N,  fem.hpp:42 (REF32; J2 modes lump it from density) */
    const uint32_t *fixed;          /* N,  fem.hpp:43; non-zero pins the node; NULL = none */
    const uint32_t *index;          /* 4T, fem.hpp:46 */
    const float *rest_inv;          /* 9T, fem.hpp:47 (REF32) */
    const float *rest_volume;       /* T,  fem.hpp:48 (REF32) */
    const uint32_t *adjacency_offset; /* N+1, fem.hpp:56 */
    const uint32_t *adjacency_entry;  /* 4T,  fem.hpp:57, entry = tet*4 + corner */
    const double *external_force;   /* 3N full-amplitude nodal load, NULL = none (J2 modes) */
    double density;                 /* kg/m^3, J2 modes: rest state is formed from it */
} femstep_tet_mesh;

typedef struct {
    double youngs_modulus, poisson_ratio;   /* fem.hpp:24-27 Material */
    double yield_strength, hardening_modulus; /* J2 modes: plasticity.hpp:115-118 linear curve */
    double dt, gravity, damping;            /* FemGpuSolver::run arguments (fem_gpu.hpp:31) */
    int ramp_steps;                         /* external load factor min((step+1)/ramp, 1); 0 = full */
} femstep_tet_params;

typedef struct femstep_tet femstep_tet;

/* gpu::FemGpuSolver::initialise (fem_gpu.hpp:23, fem_gpu.cpp:183): validate and upload. */
int femstep_tet_create(const femstep_tet_mesh *mesh, int mode, femstep_tet **out);
/* gpu::FemGpuSolver::run (fem_gpu.hpp:31, fem_gpu.cpp:374): `substeps` steps on the
   device, returns the device-measured milliseconds in *gpu_ms (may be NULL). */
int femstep_tet_run(femstep_tet *solver, int substeps, const femstep_tet_params *params, double *gpu_ms);
/* gpu::FemGpuSolver::readback (fem_gpu.hpp:35, fem_gpu.cpp:424): positions and
   velocities back into the caller's 3N float arrays (either may be NULL). */
int femstep_tet_readback(femstep_tet *solver, float *position, float *velocity);
/* The same in double (exact for J2_F64; the FP32 modes add rest + displacement in double). */
int femstep_tet_readback_f64(femstep_tet *solver, double *position, double *velocity);
/* Per-tet plastic state, 7 doubles each: plastic strain [xx,yy,zz,xy,yz,zx]
   (engineering shears, plasticity.hpp:74-88) and equivalent plastic strain. */
int femstep_tet_plastic(femstep_tet *solver, double *plastic);
/* Energy account reduced on the device in FP64 and fixed order:
   [0] external work  [1] plastic dissipation  [2] strain energy (last force pass)
   [3] kinetic  [4] gravity work.  Zeros for REF32, which keeps no account. */
int femstep_tet_energy(femstep_tet *solver, double out[5]);
/* Critical time step by the FP64 element eigenvalue bound, on the device:
   safety * 2 / sqrt(max_e omega_e^2), omega_e^2 = (4/rho) lambda_max(B^T C B).
   Replaces the edge heuristic fem::criticalTimestep (fem.cpp:183-185) with a bound. */
int femstep_tet_critical_dt(femstep_tet *solver, double youngs, double poisson, double density,
                            double safety, double *dt);
/* Per-kernel device time: runs `steps` steps with CUDA events around each launch and
   writes the mean milliseconds of [0] the element kernel and [1] the node kernel.
   The same arithmetic as femstep_tet_run; used by the benchmark's roofline. */
int femstep_tet_profile(femstep_tet *solver, int steps, const femstep_tet_params *params, double out[2]);
/* Number of kernel launches the last femstep_tet_run issued. */
long long femstep_tet_launches(const femstep_tet *solver);
const char *femstep_tet_error(const femstep_tet *solver);
void femstep_tet_destroy(femstep_tet *solver);

/* A tet mesh already in the caller's device memory, in the reference's TetMesh layout
   (engine/sim/fem.hpp:38-68).  All pointers are device pointers. */
typedef struct {
    size_t nodes, tets;
    float *position;                  /* 3N, advanced in place */
    float *velocity;                  /* 3N, advanced in place */
    const float *mass;                /* N */
    const uint32_t *fixed;            /* N, may be NULL */
    const uint32_t *index;            /* 4T */
    const float *rest_inv;            /* 9T, column-major per tet */
    const float *rest_volume;         /* T */
    const uint32_t *adjacency_offset; /* N+1 */
    const uint32_t *adjacency_entry;  /* 4T */
} femstep_tet_device_mesh;

/* No counterpart in the reference.  The REF32 step (bit-identical to
   femstep_tet_create + femstep_tet_run in FEMSTEP_TET_REF32 mode) for callers that
   cannot allocate device memory -- an engine or plugin that owns all device memory
   through its own allocator or a fixed budget.  It allocates nothing: the caller passes
   its device arrays, and the only scratch, the per-tet corner forces, is a fixed
   library-resident array of 65,536 tets (3 MiB per GPU that loads the library, held
   until the process exits).  Larger meshes are rejected with FEMSTEP_EINVAL.  The
   step is elastic: yield_strength, hardening_modulus and ramp_steps must be 0
   (FEMSTEP_EINVAL otherwise).  The first call in each CUDA context on a device looks
   up that array's device address in that context (a new context after
   cudaDeviceReset gets a new lookup), so make that call before any stream capture.
   Every call on a device shares the array: calls whose kernels overlap on the GPU
   race; calls ordered on one stream do not.  A CUDA error pending from before the
   call is returned as FEMSTEP_ECUDA without launching.  Launches on `stream` (a
   cudaStream_t, NULL for the legacy default stream) and returns without
   synchronising. */
int femstep_tet_step_noalloc(const femstep_tet_device_mesh *mesh, int substeps, const femstep_tet_params *params,
                             void *stream);

/* =====================================================================================
 * Pool of many tet meshes: the batched and the served step.  No reference
 * counterpart: the reference solves one mesh at a time (fem::stepCpu,
 * engine/sim/fem.cpp:187; gpu::FemGpuSolver::run, engine/gpu/fem_gpu.cpp:374).  Every
 * mesh keeps its own material, load, time step and step count; the arithmetic per
 * mesh is the J2_F32K tet step's (its displacement, velocity and plastic state are
 * bit-identical to a femstep_tet handle in FEMSTEP_TET_J2_F32K mode given the same
 * dt), and a mesh's result does not depend on what else is in the pool.
 *
 * Every pool call is ordered on the pool's one stream, so admit / release may be
 * called while a chunk from femstep_pool_run_async is still running: their device
 * work lands behind it.  Admission does its host work while the GPU runs.
 * ===================================================================================== */

typedef struct {
    size_t nodes, tets;
    const float *position;            /* 3N (TetMesh::position) */
    const uint32_t *index;            /* 4T, mesh-local node ids */
    const uint32_t *fixed;            /* N, may be NULL */
    const double *external_force;     /* 3N full-amplitude load, may be NULL */
    double density, youngs_modulus, poisson_ratio, yield_strength, hardening_modulus;
    double dt;                        /* 0: 0.9 x the FP64 element eigenvalue bound, on the GPU */
    double gravity, damping;          /* damping 0 means 1 (none) */
    int ramp_steps;                   /* load factor min((step+1)/ramp, 1); 0 = full */
} femstep_pool_mesh;

typedef struct femstep_pool femstep_pool;

#define FEMSTEP_POOL_AUTO 0        /* the pool's schedule (set by autotune or set_schedule) */
#define FEMSTEP_POOL_GRAPH 1       /* two launches per step, replayed from a CUDA graph */
#define FEMSTEP_POOL_PERSISTENT 2  /* one cooperative launch per chunk, grid barriers */
#define FEMSTEP_POOL_GRAPH_STAGED 3 /* GRAPH, each tile's per-tet rows staged in shared memory by
                                       bulk async copies (tiles of 128 and 256) */
#define FEMSTEP_POOL_GRAPH_TILED 4  /* GRAPH, tiles of 128: a tile gathers its distinct nodes once and
                                       writes one force partial per (tile, node); the node pass sums a
                                       node's partials in tile order.  Same bits alone or in the mix;
                                       the per-tile association differs from the other schedules' in
                                       rounding.  Its tables are allocated at first use (about 21 B
                                       per tet and 4 B per node of capacity, beyond the pool's own)
                                       and rebuilt whenever the set of meshes changes */

/* A pool holding up to `tet_capacity` tets and `node_capacity` nodes (each mesh also
   takes one spare node slot) of at most `max_meshes` meshes; tile = threads per block
   (128, 256 or 512; 0 = 256).  Device memory: femstep_pool_bytes_per_tet() per tet and
   femstep_pool_bytes_per_node() per node of capacity, all allocated here.
   tet_capacity <= 1e9 (slot ids are 32-bit). */
int femstep_pool_create(size_t tet_capacity, size_t node_capacity, int max_meshes, int tile, femstep_pool **out);
size_t femstep_pool_bytes_per_tet(void);
size_t femstep_pool_bytes_per_node(void);
/* Admit a mesh that will take `steps` steps (at rest, zero plastic strain).
   FEMSTEP_ENOMEM when it does not fit in the free space now: the caller keeps it
   queued and retries after a release. */
int femstep_pool_admit(femstep_pool *pool, const femstep_pool_mesh *mesh, long long steps, int *id);
/* Admit meshes[0..count) in order while they fit (a prefix is admitted; *admitted says
   how many, their ids in ids[]).  The host work of all of them (rest state, CSR, slot
   map) runs on all host cores at once.  FEMSTEP_ENOMEM when the rest did not fit now;
   FEMSTEP_EINVAL, with nothing admitted, when a mesh is not valid. */
int femstep_pool_admit_many(femstep_pool *pool, const femstep_pool_mesh *meshes, const long long *steps, int count,
                            int *ids, int *admitted);
/* Free a mesh's space.  Its device state is frozen behind any queued work. */
int femstep_pool_release(femstep_pool *pool, int id);
/* Eviction.  checkpoint copies one mesh's whole mutable state (displacement and
   velocity, plastic strain, both with their compensation, its energy partials and step
   counter) into a host buffer of femstep_pool_checkpoint_size bytes; release it, and
   admit_resume the same mesh later -- anywhere in this or another pool -- with that
   buffer and a target >= the steps already taken.  It then steps on bit-identically
   to a mesh that never left (and its energy sums are bit-identical too when the pool's
   tile is the same).  Not while a chunk is in flight. */
int femstep_pool_checkpoint_size(femstep_pool *pool, int id, size_t *bytes);
int femstep_pool_checkpoint(femstep_pool *pool, int id, void *buffer, size_t bytes);
int femstep_pool_admit_resume(femstep_pool *pool, const femstep_pool_mesh *mesh, long long steps,
                              const void *checkpoint, size_t bytes, int *id);
/* Queue one chunk: every admitted mesh that has steps left advances by up to `steps`
   steps (meshes that reach their count stop there).  Returns without waiting. */
int femstep_pool_run_async(femstep_pool *pool, int steps, int mode);
/* Build what the next chunk launches -- the work list and, in the graph schedules,
   the captured graph of 16 steps -- without running a step, so that a timed chunk
   that follows does no set-up.  Waits for the pool's stream. */
int femstep_pool_prepare(femstep_pool *pool);
/* Wait for the queued chunk; its device milliseconds (CUDA events). */
int femstep_pool_wait(femstep_pool *pool, double *gpu_ms);
/* run_async + wait. */
int femstep_pool_run(femstep_pool *pool, int steps, int mode, double *gpu_ms);
/* Ids of the meshes whose step count was reached by the last chunk that was waited
   for (up to `capacity` of them; *count = how many there are). */
int femstep_pool_finished(femstep_pool *pool, int *ids, int capacity, int *count);
/* Steps taken and requested of one mesh (waits for queued work). */
int femstep_pool_status(femstep_pool *pool, int id, long long *steps_done, long long *steps_target);
/* Positions (rest + displacement) and velocities of one mesh, 3N doubles each. */
int femstep_pool_readback(femstep_pool *pool, int id, double *position, double *velocity);
/* The same for ids[0..count): positions[k] / velocities[k] receive mesh ids[k]'s (3N
   doubles each; velocities may be NULL).  The copies of all meshes are queued at once
   through pinned buffers and converted on all host cores as they land: for reading a
   whole batch back, one call instead of one per mesh. */
int femstep_pool_readback_many(femstep_pool *pool, int count, const int *ids, double *const *positions,
                               double *const *velocities);
/* Plastic strain of one mesh, 7 per tet (6 engineering components, equivalent). */
int femstep_pool_plastic(femstep_pool *pool, int id, double *plastic);
/* [0] external work (load and gravity) [1] dissipation [2] strain energy [3] kinetic
   of one mesh, reduced on the GPU in FP64 in a fixed order. */
int femstep_pool_energy(femstep_pool *pool, int id, double out[4]);
/* The time step a mesh runs with (its own, or the bound computed at admission). */
int femstep_pool_dt(femstep_pool *pool, int id, double *dt);
/* The autotuner: times every tile size in {128, 256, 512} with every schedule for
   `steps` steps on the pool as it is, restores the pool's state after each trial (so
   tuning does not change any result), keeps the fastest, and reports it. */
int femstep_pool_autotune(femstep_pool *pool, int steps, int *tile, int *mode, double *ms_per_step);
/* Set the schedule by hand (tile 128 / 256 / 512; GRAPH, PERSISTENT, GRAPH_STAGED, or
   GRAPH_TILED at tile 128). */
int femstep_pool_set_schedule(femstep_pool *pool, int tile, int mode);
/* Mean device milliseconds per launch of [0] the element pass and [1] the node pass,
   over `steps` steps taken one launch at a time (the steps count as taken). */
int femstep_pool_profile(femstep_pool *pool, int steps, double out[2]);
/* [0] tets in use [1] nodes in use [2] meshes admitted [3] tile [4] mode [5] kernel
   launches of the last chunk [6] device bytes held [7] pinned staging buffers */
int femstep_pool_info(femstep_pool *pool, long long out[8]);
const char *femstep_pool_error(const femstep_pool *pool);
void femstep_pool_destroy(femstep_pool *pool);

/* =====================================================================================
 * Solid-shell zone step.  Replaces gpu::ZoneGpuSolver (engine/gpu/zone_gpu.hpp:179-234):
 * the 8-node ANS + 7-parameter EAS solid-shell with J2 plasticity (linear isotropic
 * hardening, failure off), the CSR gather and the lumped-mass node update of
 * zone::Solver::step (engine/sim/zone.cpp:928-989, 1094-1121, 1200-1202), in FP32 with
 * optional Kahan-compensated displacement and plastic strain.
 * ===================================================================================== */

/* A solid-shell mesh: the reference's solidshell::HexMesh (solid_shell.hpp:464-477)
   plus what zone::Solver hands its accelerator (zone.hpp:903-961). */
typedef struct {
    size_t nodes, elements;
    const double *rest;             /* 3N rest positions (HexMesh::position) */
    const double *position;         /* 3N current positions (Solver::position), NULL = rest */
    const double *velocity;         /* 3N (Solver::velocity), NULL = at rest */
    const uint32_t *index;          /* 8E, node order of solid_shell.hpp:115-126 */
    const uint8_t *pinned;          /* 3N (Solver::pinnedDof / HexMesh::fixed), NULL = none */
    const double *load;             /* 3N full-amplitude external nodal load, NULL = none */
    const double *forms;            /* NULL, or the caller's RestForms, 1505 doubles per
                                       element in the order of engine/gpu/zone_gpu.cpp:28-34
                                       (b, g, weight, J0^-1).  The step forms B and G in FP32
                                       from the rest positions itself; given forms must be the
                                       solid-shell forms of those positions (every weight, and
                                       all of the first 64 elements, to 1e-9), else EINVAL */
    const double *mass;             /* N lumped mass (Solver::nodalMass), NULL = lumped on device */
    const double *state;            /* 129 doubles per element (zone_gpu.cpp:36-40 layout), NULL = virgin */
    const uint32_t *adjacency_offset; /* N+1 (Solver::adjacencyOffset), NULL = built */
    const uint32_t *adjacency_entry;  /* 8E, entry = element*8 + corner */
    double density;                 /* kg/m^3, for the lumped mass when mass is NULL */
} femstep_shell_mesh;

/* The general point law (plasticity::update, engine/sim/plasticity.cpp:319-505): the
   flow curve (plasticity.hpp:112-128), kinematic hardening and the ductile damage law
   (plasticity.hpp:193-199).  Each element's failure strain comes from the state handed
   to femstep_shell_create (ElementPlasticState::failureStrain; +inf without one). */
#define FEMSTEP_SHELL_LINEAR 0
#define FEMSTEP_SHELL_SWIFT 1
typedef struct {
    int hardening;                 /* FEMSTEP_SHELL_LINEAR (yield_strength, hardening_modulus of
                                      femstep_shell_params) or FEMSTEP_SHELL_SWIFT: K (eps0 + p)^n */
    double strength_coefficient, reference_strain, hardening_exponent;  /* Swift K, eps0, n */
    double kinematic_modulus;      /* back-stress modulus, Pa */
    double triaxiality_sensitivity, reference_triaxiality, cutoff_triaxiality;  /* Failure */
} femstep_shell_material;

typedef struct {
    double youngs_modulus, poisson_ratio;      /* plasticity::Material (plasticity.hpp:220-228) */
    double yield_strength, hardening_modulus;  /* linear curve (plasticity.hpp:115-118) */
    double dt, damping;                        /* SolveParams::timestep / damping (zone.hpp:698-699) */
    double rise_time;                          /* load factor min((step+1) dt / rise, 1); 0 = full */
    int max_iterations;                        /* EAS Newton cap (CPU: 40) */
    double tol_residual, tol_work;             /* Newton stops on ||r|| or |delta.r| below tol * sigma_y V
                                                  (0: the reference's 1e-12 and 1e-16), or once ||r|| is at
                                                  FP32 rounding (16 ulps of the magnitude of its terms) */
    int compensated;                           /* 1: Kahan-compensated displacement and plastic strain */
    const femstep_shell_material *material;    /* NULL: the linear law, no back stress, no damage;
                                                  else the general law and the element failure rules
                                                  (no enhanced modes after a point fails, one retry
                                                  without them, torn when all eight points have) */
    int eas_fp64;                              /* how much of the enhanced-strain block runs in FP64
                                                  (gpu::EasPrecision, zone_gpu.hpp:153-162): 0 none;
                                                  1 the 7x7 factor and substitutions; 2 also K_aa and
                                                  the residual summed in double; 3 also alpha, its
                                                  correction and its stored state.  1-3 need the
                                                  compensated step and a material */
} femstep_shell_params;

typedef struct femstep_shell femstep_shell;

/* gpu::ZoneGpuSolver::initialise (zone_gpu.hpp:203-207, zone_gpu.cpp:495). */
int femstep_shell_create(const femstep_shell_mesh *mesh, femstep_shell **out);
/* gpu::ZoneGpuSolver::run (zone_gpu.hpp:214, zone_gpu.cpp:877): device milliseconds. */
int femstep_shell_run(femstep_shell *solver, int substeps, const femstep_shell_params *params, double *gpu_ms);
/* gpu::ZoneGpuSolver::readback (zone_gpu.hpp:218, zone_gpu.cpp:932): positions (rest +
   displacement, in double) and velocities; either may be NULL. */
int femstep_shell_readback(femstep_shell *solver, double *position, double *velocity);
/* Per-element plastic state in the 129-double layout of zone_gpu.cpp:36-40 (eight points
   of plastic strain, back stress, eq. plastic strain, damage, failed; seven enhanced
   parameters; failure strain; torn), the ElementPlasticState zone::Solver::adopt takes. */
int femstep_shell_state(femstep_shell *solver, double *state);
/* [0] external work [1] plastic dissipation [2] strain energy [3] kinetic, FP64 reduced
   on the device in fixed order (zone::Solver::accumulateEnergy, zone.cpp:1014-1044). */
int femstep_shell_energy(femstep_shell *solver, double out[4]);
/* The punch of zone::Solver::step (engine/sim/zone.cpp:1147-1198).
   mass == 0: the prescribed punch, as the reference's GPU zone step drives it
   (engine/gpu/shaders/solidshell_integrate.comp, zone_gpu.cpp:889-919): every step each
   node in `driven` has its velocity along `axis` set to -speed, after the force update,
   the damping and the driven edge; the speed rises linearly over ramp_time seconds from
   the time the punch is set.
   mass > 0: the inertial punch (Drive::Inertial, zone.cpp:1154-1185), which the
   reference runs on the CPU only: a striking body of that mass arrives at `speed` and
   the grip is a perfectly inelastic collision with the gripped nodes; ramp_time is
   ignored, as the reference ignores it.  Once the body has stopped, every later step is
   skipped on the device (the run has ended, zone.cpp:1225-1230).  speed must be > 0.
   Either way the impulse it takes is the punch's work, summed in FP64 in a fixed order
   (the shader used a fixed-point atomic).  count 0 removes the punch. */
int femstep_shell_set_punch(femstep_shell *solver, const uint32_t *driven, size_t count, const double axis[3],
                            double speed, double ramp_time, double mass);
/* [0] punch work (J) [1] penetration (m) [2] time (s) [3] steps since the punch was set:
   ZoneGpuState::work / penetration / time / steps (zone_gpu.hpp:116-126). */
int femstep_shell_punch_state(femstep_shell *solver, double out[4]);
/* The driven edge (zone.cpp:833-842, 1123-1145): each pinned DOF d with prescribed[d]
   != 0 follows meshed[d] + prescribed[d] * smoothstep(t / edge_ramp) (t at the step's
   end; edge_ramp 0: the whole drive at once) instead of staying clamped; the others stay
   clamps.  meshed (3N) is the position the drive is measured from; NULL takes the rest
   position.  The boundary's work is kept in FP64 (femstep_shell_account).  prescribed
   NULL, or all zero, removes the drive. */
int femstep_shell_set_edge(femstep_shell *solver, const double *prescribed, const double *meshed,
                           double edge_ramp);
/* Constraint fibres (engine/sim/constraint.hpp; zone.cpp:990-1002): the axial bars an
   eccentric stiffener is made of, each end tied to a through-thickness node pair as
   (1 - w) x[bottom] + w x[top].  Every step each fibre's co-rotational strain
   (l - L) / L goes through the uniaxial return (isotropic hardening on the solver's
   flow curve, damage with the bar's triaxiality +-1/3, tearing at the fibre's failure
   strain), in FP64, and N = sigma A is added to the four tie nodes after the plating's
   gather, in fibre order.  Their dissipation and strain energy join
   femstep_shell_energy's.  count 0 removes them. */
typedef struct {
    size_t count;
    const uint32_t *tie;           /* 4 per fibre: end 0 bottom, top; end 1 bottom, top */
    const double *weight;          /* 2 per fibre: the ties' weights (constraint::tieWeight) */
    const double *area;            /* m^2 per fibre */
    const double *rest_length;     /* m per fibre; NULL: from the rest positions (restFibers) */
    const double *failure_strain;  /* per fibre (constraint::fiberFailureStrain); NULL: never fails */
    double density;                /* > 0: add the fibres' lumped mass (lumpFiberMass); 0: the
                                      solver's mass already holds it, as zone::Solver's does */
} femstep_shell_fibers;
int femstep_shell_set_fibers(femstep_shell *solver, const femstep_shell_fibers *fibers);
/* 4 doubles per fibre: plastic strain, eq. plastic strain, damage, failed (FiberState). */
int femstep_shell_fiber_state(femstep_shell *solver, double *out);
/* The rest of zone::Solver's account (SolveResult, zone.hpp:750-815): [0] damping loss
   (J) [1] boundary work of the driven edge (J) [2] the punch's speed now (m/s) [3] the
   striking body's kinetic energy (J; 0 for a prescribed punch) [4] 1 once an inertial
   punch has stopped [5] driven edge DOFs. */
int femstep_shell_account(femstep_shell *solver, double out[6]);
/* [0] element-steps whose EAS Newton hit its cap, [1] yielded Gauss points last step. */
int femstep_shell_stats(femstep_shell *solver, long long out[2]);
/* Smallest element critical step, FP64 power iteration per element on the device
   (solidshell::criticalTimestep, solid_shell.cpp:1088-1133, 1187-1198). */
int femstep_shell_critical_dt(femstep_shell *solver, double youngs, double poisson, double density,
                              double safety, double *dt);
/* Mean device ms of [0] the element kernel and [1] the node kernel over `steps` steps. */
int femstep_shell_profile(femstep_shell *solver, int steps, const femstep_shell_params *params, double out[2]);
long long femstep_shell_launches(const femstep_shell *solver);
/* Bytes of device memory the solver holds. */
size_t femstep_shell_device_bytes(const femstep_shell *solver);
/* Checkpoint and resume (ZoneGpuState's role in zone_gpu.hpp:116-126, kept whole):
   the solver's entire mutable device state -- displacement with its compensation,
   velocity, element state with its compensation, enhanced parameters, step counter,
   the FP64 energy and punch partials -- and the punch clock, as one host buffer of
   femstep_shell_checkpoint_size bytes.  Restore into a solver created from the same
   mesh with the same punch and driven edge set; running on from it is bit-identical to
   never having stopped (also across destroy / create, e.g. to evict a zone from the
   GPU and bring it back later). */
int femstep_shell_checkpoint_size(femstep_shell *solver, size_t *bytes);
int femstep_shell_checkpoint(femstep_shell *solver, void *buffer, size_t bytes);
int femstep_shell_restore(femstep_shell *solver, const void *buffer, size_t bytes);
const char *femstep_shell_error(const femstep_shell *solver);
void femstep_shell_destroy(femstep_shell *solver);

/* RestForms of `elements` elements formed on the device in FP64
   (solidshell::computeRestForms, solid_shell.cpp:237-375), with elementMass (:655) and
   criticalTimestep (:1088).  nodes: 24 doubles per element.  forms_out: 1507 doubles per
   element (1505 in zone_gpu.cpp order, then easCount, ok); mass_out: 8 per element;
   dt_out: 1 per element; each may be NULL. */
int femstep_shell_forms(const double *nodes, size_t elements, int formulation, double youngs, double poisson,
                        double density, double safety, double *forms_out, double *mass_out, double *dt_out);

#ifdef __cplusplus
}
#endif
#endif
