/*
 * femoracle.h -- CPU oracle for the explicit structural FEM step.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product (the CUDA library, the compat
 * classes, the Python binding) links, loads or calls anything declared here.  Only
 * tests/, __graft_entry__.smoke() and the cpu_baseline / --impl reference legs of
 * bench.py use it, and only as the checker.
 *
 * Two implementations share this interface:
 *
 *   liboracle.so            a plain-C restatement of the reference algorithm
 *                           (femoracle.c), each function citing the reference
 *                           file:line it follows;
 *   _ref/libshipsim_ref.so  the reference's own C++ sources compiled unchanged
 *                           (engine/sim/{fem,plasticity,solid_shell,zone,...}.cpp)
 *                           plus ref_shim.cpp, which exposes them with the same
 *                           C signatures under a `ref_` prefix.
 *
 * The restatement is pinned against the compiled reference (bit-for-bit where the
 * arithmetic order is the same) and against golden vectors in tests/golden/.
 *
 * Conventions, all inherited from the reference:
 *   - Voigt order [xx, yy, zz, xy, yz, zx]; strain shears are engineering (2 eps),
 *     stress shears are tensor components (engine/sim/plasticity.hpp:74-88).
 *   - 3x3 matrices in the tet path are column-major m[col*3+row]
 *     (engine/sim/fem.cpp:10-16); in the solid-shell path row-major
 *     (engine/sim/solid_shell.cpp:35).
 */
#ifndef FEMORACLE_H
#define FEMORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- J2 point law ---------------------------------------------------------
 * Material as a flat array (engine/sim/plasticity.hpp:112-128, 193-228):
 *   [0] E  [1] nu  [2] sigma_y0  [3] H (linear)  [4] H_kin  [5] kind (0 linear, 1 Swift)
 *   [6] Swift K  [7] Swift eps0  [8] Swift n
 *   [9] failure uniformStrain  [10] fractureStrain  [11] triaxialitySensitivity
 *   [12] referenceTriaxiality  [13] cutoffTriaxiality
 * Point state, 15 doubles (engine/sim/plasticity.hpp:313-319):
 *   [0..5] plastic strain  [6..11] back stress  [12] eq. plastic strain
 *   [13] damage  [14] failed (0/1)
 * Increment, 9 doubles (engine/sim/plasticity.hpp:323-340):
 *   [0] yielded [1] failedNow [2] dgamma [3] d eps_p [4] dissipation
 *   [5] plasticWork [6] vonMises [7] triaxiality [8] iterations
 */
#define OR_MAT_LEN 14
#define OR_POINT_LEN 15
#define OR_INCR_LEN 9

int or_plastic_update(const double *mat, double failure_strain, const double strain[6],
                      double state[OR_POINT_LEN], double stress[6], double *tangent /*36 or NULL*/,
                      double incr[OR_INCR_LEN]);

/* ---- Linear tet, float, elastic: engine/sim/fem.cpp --------------------- */
typedef struct {
    size_t nodes, tets;
    float *position;          /* 3N */
    float *velocity;          /* 3N */
    float *mass;              /* N  */
    uint32_t *fixed;          /* N  */
    uint32_t *index;          /* 4T */
    float *rest_inv;          /* 9T, column-major */
    float *rest_volume;       /* T  */
    float *tet_force;         /* 12T scratch */
    uint32_t *adj_offset;     /* N+1 */
    uint32_t *adj_entry;      /* 4T  */
} or_tet32;

/* makeBoxTetMesh (fem.cpp:217-263): sizes first, then fill. */
void or_box_tet_sizes(int nx, int ny, int nz, size_t *nodes, size_t *tets);
void or_box_tet_mesh(float lx, float ly, float lz, int nx, int ny, int nz, float *position,
                     uint32_t *index);
/* computeRestState (fem.cpp:119-158). position/index in, the rest out. */
void or_tet32_rest_state(or_tet32 *m, float E, float nu, float rho);
void or_tet32_forces(const or_tet32 *m, size_t t, float lambda, float mu, float out[12]);
/* stepCpu (fem.cpp:187-215), `steps` times. */
void or_tet32_step(or_tet32 *m, float E, float nu, float rho, float dt, float gravity,
                   float damping, int steps);
float or_tet32_critical_dt(const or_tet32 *m, float E, float nu, float rho, float safety);

/* ---- Linear tet, double, J2 (O-tet64) -----------------------------------
 * fem.cpp's tet kinematics (fem.cpp:73-117) restated in double, with the J2 point
 * law (plasticity.cpp:319) at the tet's single integration point, lumped mass as
 * fem.cpp:143-145, an explicit nodal external force ramped over `ramp_steps`, and
 * the node update of fem.cpp:196-214.  Plastic state is 7 doubles per tet
 * (plastic strain[6], eq. plastic strain); back stress and damage are not carried
 * (linear isotropic hardening, failure off). */
typedef struct {
    size_t nodes, tets;
    double *position;         /* 3N */
    double *velocity;         /* 3N */
    double *mass;             /* N  */
    uint32_t *fixed;          /* N  */
    uint32_t *index;          /* 4T */
    double *rest_inv;         /* 9T column-major */
    double *rest_volume;      /* T  */
    double *tet_force;        /* 12T scratch */
    uint32_t *adj_offset;     /* N+1 */
    uint32_t *adj_entry;      /* 4T  */
    double *plastic;          /* 7T  */
    double *stress;           /* 6T  last stress, Voigt */
    double *fext;             /* 3N full-load external force, or NULL */
    /* energy[0] external work, [1] plastic dissipation, [2] strain energy (last
       force pass), [3] kinetic (last velocities), [4] gravity work */
    double energy[5];
    long step;                /* steps taken; drives the load ramp */
} or_tet64;

typedef struct {
    double E, nu, rho, yield, hardening;
    double dt, gravity, damping;
    int ramp_steps;           /* load factor min((step+1)/ramp_steps, 1); 0 = full */
    int polar_fixed;          /* 0: converge (solid_shell.cpp:473), >0: that many iterations */
} or_tet64_params;

/* Rest state in double from float positions promoted: Dm^-1, |det|/6, rho V/4. */
void or_tet64_rest_state(or_tet64 *m, double rho);
void or_tet64_step(or_tet64 *m, const or_tet64_params *p, int steps);
void or_tet64_step_threads(or_tet64 *m, const or_tet64_params *p, int steps, int threads);
/* Element eigenvalue bound (lumped mass): largest omega^2 of the element, FP64.
   dt = safety * 2 / sqrt(max). */
double or_tet64_critical_dt(const or_tet64 *m, double E, double nu, double rho, double safety);

/* ---- Solid-shell (engine/sim/solid_shell.cpp) ----------------------------
 * RestForms as 1505 doubles: b[8][6][24] | g[8][6][7] | weight[8] | J0inv[9]
 * (row-major), then [1505] = easCount, [1506] = ok.  Same order as
 * engine/gpu/zone_gpu.cpp:28-34. */
#define OR_FORMS_LEN 1507
#define OR_SHELL_STATE_LEN 129  /* 8 x 15 point state, 7 enhanced, failure strain, torn */
/* formulation: 0 displacement, 1 ANS, 2 solid-shell */
int or_shell_forms(const double rest[24], int formulation, double out[OR_FORMS_LEN]);
void or_shell_mass(const double nodes[24], double density, double out[8]);
void or_shell_gauss_volumes(const double nodes[24], double out[8]);
void or_shell_init_state(const double nodes[24], const double *mat, double state[OR_SHELL_STATE_LEN]);
/* info: [0] converged [1] iterations [2] yielded [3] failed [4] dissipation
         [5] enhancedResidual [6] enhancedWork */
int or_shell_plastic_update(const double forms[OR_FORMS_LEN], const double rest[24],
                            const double current[24], const double *mat,
                            double state[OR_SHELL_STATE_LEN], double force[24],
                            double stress[48], double info[7]);
void or_shell_rotation(const double forms[OR_FORMS_LEN], const double current[24], double out[9]);
void or_shell_stiffness(const double nodes[24], double E, double nu, int formulation, double out[576]);
double or_shell_critical_dt(const double nodes[24], double E, double nu, double rho,
                            int formulation, double safety);
/* makePlateMesh (solid_shell.cpp:1152) */
void or_plate_sizes(int nx, int ny, int nz, size_t *nodes, size_t *elements);
void or_plate_mesh(double lx, double ly, double thickness, int nx, int ny, int nz,
                   double *position, uint32_t *index);
/* uniformPressureLoad (solid_shell.cpp:1505) for a structured plate (nz = 1 top
   faces are exactly the +zeta faces of every element). */
void or_plate_pressure_load(const double *position, const uint32_t *index, size_t nodes,
                            size_t elements, double pressure, double *load);

/* The composed explicit shell step: element loop (zone.cpp:928-975), CSR gather
   (zone.cpp:976-989), external force, pinned DOF, velocity/position update
   (zone.cpp:1094-1111, 1200). */
typedef struct {
    size_t nodes, elements;
    double *rest;             /* 3N */
    double *position;         /* 3N */
    double *velocity;         /* 3N */
    double *mass;             /* N  */
    uint8_t *pinned;          /* 3N */
    uint32_t *index;          /* 8E */
    double *forms;            /* OR_FORMS_LEN * E */
    double *state;            /* OR_SHELL_STATE_LEN * E */
    double *element_force;    /* 24E scratch */
    double *stress;           /* 48E last stress */
    double *gauss_volume;     /* 8E  */
    uint32_t *adj_offset;     /* N+1 */
    uint32_t *adj_entry;      /* 8E  */
    double *fext;             /* 3N load at full amplitude, or NULL */
    double energy[5];         /* work, dissipation, strain, kinetic, punch work */
    long step;
    uint8_t *driven;          /* N: 1 for a node the punch grips, or NULL (no punch) */
    double axis[3];           /* the punch travels along -axis */
    /* The driven edge (zone.cpp:833-842, 1123-1145): a pinned DOF whose prescribed value
       is non-zero follows meshed + prescribed * smoothstep(t / edge_ramp), t the time at
       the step's end; NULL = every pinned DOF is a clamp. */
    double *prescribed;       /* 3N or NULL */
    double *meshed;           /* 3N: the position the drive is measured from; NULL = rest */
    double edge_ramp;         /* s; 0 = the whole drive at once */
    /* The inertial punch (zone.cpp:1154-1185): mass > 0 makes the grip a perfectly
       inelastic collision with a striking body of that mass; 0 = the prescribed punch. */
    double punch_mass;
    double punch_velocity;    /* m/s along -axis (state of the striking body) */
    int arrested;             /* the striking body has stopped: no further steps run */
    double account[4];        /* damping loss, boundary work, penetration, time */
    /* Constraint fibres (engine/sim/constraint.hpp, zone.cpp:990-1002): the axial bars of
       eccentric stiffeners, each end tied to a through-thickness node pair as
       (1 - w) x[bottom] + w x[top].  Their forces are added after the plating's gather,
       in fibre order. */
    size_t fibers;
    uint32_t *fiber_tie;      /* 4 per fibre: end 0 bottom, top; end 1 bottom, top */
    double *fiber_weight;     /* 2 per fibre: the ties' weights */
    double *fiber_area;       /* m^2 */
    double *fiber_length;     /* rest length, m (restFibers) */
    double *fiber_fail;       /* failure strain (fiberFailureStrain); inf never fails */
    double *fiber_state;      /* 4 per fibre: plastic strain, eq. plastic strain, damage, failed */
    double fiber_energy;      /* the fibres' recoverable strain energy after the last step */
} or_shell;

typedef struct {
    double dt, damping;
    double rise_time;         /* load factor min(t / rise_time, 1), t = (step+1) dt */
    double punch_speed;       /* the prescribed punch (zone.cpp:1150-1198) */
    double punch_ramp;        /* s over which its speed rises linearly from rest */
} or_shell_params;

/* A flat plate stepped by the reference's zone::Solver itself (ref_shim.cpp only; the
   port has no twin: tests run or_shell_step on the arrays it returns and compare).  The
   plate is built as the reference's own zone tests build theirs: makePlateMesh, the
   perimeter pinned, the punch footprint round the centre of the outer face. */
typedef struct {
    double lx, ly, thickness;
    int nx, ny, nz;
    double half_length, half_width;   /* the punch footprint; 0 = no punch */
    double speed, ramp_time;          /* prescribed punch; the arrival speed if mass > 0 */
    double mass;                      /* > 0: the inertial punch (Drive::Inertial) */
    double damping, edge_ramp;
    double edge_drive[3];             /* a perimeter DOF's prescribed value: edge_drive * x / lx */
    int steps;
    /* flat-bar stiffeners along x, as constraint fibres (constraint::addStiffener) */
    int stiffeners;                   /* lines at y = ly (s + 1) / (stiffeners + 1), on grid lines */
    double web_height, web_thickness;
    int fiber_failure;                /* SolveParams::fiberFailure */
} or_zone_case;
typedef struct {
    double *rest;                     /* 3N meshed position (= rest) */
    uint32_t *index;                  /* 8E */
    uint8_t *pinned;                  /* 3N */
    double *prescribed;               /* 3N */
    uint8_t *driven;                  /* N: the solver's driven nodes */
    double *mass;                     /* N lumped */
    double *state0;                   /* OR_SHELL_STATE_LEN * E, at construction */
    double *position, *velocity;      /* 3N after the steps */
    double *state;                    /* OR_SHELL_STATE_LEN * E after the steps */
    double mat[OR_MAT_LEN];           /* plasticity::shipSteel() */
    double density, dt;
    double account[10];               /* work, dissipation, penetration, time, damping loss,
                                         boundary work, indenter speed, steps, arrested,
                                         driven edge DOFs */
    /* the fibres as or_shell takes them, and their state after the steps */
    uint32_t *fiber_tie;              /* 4F */
    double *fiber_weight;             /* 2F */
    double *fiber_area, *fiber_length, *fiber_fail;  /* F */
    double *fiber_state;              /* 4F */
} or_zone_out;

void or_shell_setup(or_shell *m, const double *mat, double density);
void or_shell_step(or_shell *m, const double *mat, const or_shell_params *p, int steps);
void or_shell_step_threads(or_shell *m, const double *mat, const or_shell_params *p, int steps, int threads);
void or_shell_energy(or_shell *m, const double *mat);

#ifdef __cplusplus
}
#endif
#endif
