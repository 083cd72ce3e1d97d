// shell.hpp -- device layout of a solid-shell zone and its kernel launchers.
//
// The element is the reference's 8-node ANS + 7-parameter EAS solid-shell
// (engine/sim/solid_shell.{hpp,cpp}); the step is zone::Solver::step's element loop,
// CSR gather and node update (engine/sim/zone.cpp:928-989, 1094-1121, 1200-1202).
//
// Work mapping: one element = 8 lanes of a warp, lane g owning Gauss point g, so a
// warp holds 4 elements.  Each lane forms its point's strain-displacement and
// enhanced-strain operators in FP32 from the element's rest corners every step
// (shell_geom.cuh), so per element only a 64-byte row of rest data is stored:
//
//   elem    float4 [E][4]                  J0^-1 at the centre (row-major, 9) and the
//                                          enhanced modes' scales det J0 n_j (7); all
//                                          zero for an element without valid forms
//   state   float  [groups][14][32]        per lane: plastic strain (6), eq. plastic
//                                          strain, and their Kahan compensations (7)
//   alpha   float  [E][8]                  the seven enhanced parameters (+ pad)
//   index   uint32 [E][8]; slot uint32 [E][8] (node-major CSR position of each corner)
//
//   nodes:  rest double[3N] (rest positions), disp/disp_c float[3N] (displacement and
//           its compensation), velocity float[3N], mass/inv_mass float[N],
//           pinned uint8[N] (bit k pins DOF k; bit 3+k: DOF k is a driven edge DOF),
//           load float[3N] (full-amplitude load),
//           offset uint32[N+1] (CSR)
//   slots:  float[3 * 8E] in CSR order
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace fs {

constexpr int kShellElemQ = 4;       // float4 per element row: J0^-1 (9), enhanced-mode scales (7)
constexpr int kShellStateQ = 14;     // floats of state per lane
constexpr int kShellState2Q = 8;     // back stress (6), damage, failed: the general point law
constexpr int kShellLanesPerElement = 8;
constexpr int kShellElementsPerWarp = 4;

struct ShellDevice {
    long long nodes = 0, elements = 0, groups = 0;
    int sms = 148;                  // the device's SM count (the element pass's launch form)
    const float4* elem = nullptr;  // [E][kShellElemQ]
    float* state = nullptr;
    float* alpha = nullptr;
    double* alpha64 = nullptr;         // [E][8]: alpha in double (the EAS64 = 3 variant only)
    const uint32_t* index = nullptr;
    const uint32_t* slot = nullptr;
    const double* rest = nullptr;
    float* disp = nullptr;
    float* disp_c = nullptr;
    float* velocity = nullptr;
    const float* mass = nullptr;
    const float* inv_mass = nullptr;
    const uint8_t* pinned = nullptr;
    const float* load = nullptr;
    const uint32_t* offset = nullptr;
    float* slots = nullptr;
    const float* kaa_factor = nullptr; // [E][32]: Cholesky factor of the elastic K_aa (may be null)
    // the general point law (ShellParams::general): per lane back stress (6), damage,
    // failed flag, in the state's lane-interleaved layout; per element failure strain
    float* state2 = nullptr;          // [groups][kShellState2Q][32]
    // the punch (zone.cpp:1150-1198): 1 for a node the indenter grips; null without one
    const uint8_t* driven = nullptr;
    double* n_punch = nullptr;        // FP64 punch work per node block (+=)
    // The inertial punch (zone.cpp:1154-1185, ShellParams::inertial): the gripped nodes
    // as a list for the one-block punch kernel, the striking body's account, and a halt
    // flag that every kernel of the step reads first (set once the body has stopped).
    const uint32_t* driven_list = nullptr;
    int n_driven = 0;
    double* punch_state = nullptr;    // [0] speed, [1] work, [2] penetration, [3] time, [4] steps
    double* punch_kin = nullptr;      // kinetic energy of the gripped nodes (= per step)
    int* halt = nullptr;
    // The driven edge (zone.cpp:833-842, 1123-1145): pinned bit 3+k marks DOF k as
    // driven rather than clamped.  Rows of the edge arrays are read only for marked nodes.
    const int* edge_map = nullptr;    // [N]: the node's row
    const double* edge_base = nullptr;   // [rows][3]: meshed - rest
    const double* edge_drive = nullptr;  // [rows][3]: the prescribed value
    double* n_edge = nullptr;         // FP64 boundary work per node block (+=)
    double* n_damp = nullptr;         // FP64 damping loss per node block (+=)
    // Constraint fibres (constraint.hpp; zone.cpp:990-1002): axial bars of eccentric
    // stiffeners, each end tied to a through-thickness node pair.  One FP64 thread per
    // fibre writes the force on its four tie nodes into fiber_slots; the node pass adds
    // them after the element gather through a second CSR, in fibre order.
    long long fibers = 0;
    const uint4* fiber_tie = nullptr;       // [F]: end 0 bottom, top; end 1 bottom, top
    const double2* fiber_weight = nullptr;  // [F]: the two ties' weights
    const double* fiber_area = nullptr;     // [F]
    const double* fiber_length = nullptr;   // [F] rest length
    const double* fiber_fail = nullptr;     // [F] failure strain (inf: never)
    double* fiber_state = nullptr;          // [F][4]: plastic strain, eq. plastic strain, damage, failed
    float* fiber_slots = nullptr;           // [F][4][3]
    const uint32_t* fiber_offset = nullptr; // [N+1]
    const uint32_t* fiber_entry = nullptr;  // [4F]: fibre * 4 + tie node (0..3), ascending per node
    double* f_diss = nullptr;               // FP64 fibre dissipation per fibre block (+=)
    double* f_energy = nullptr;             // FP64 fibre strain energy per fibre block (=)
    const float* fail_strain = nullptr;  // [E]; +inf never fails
    long long* counter = nullptr;     // [0] steps taken, [1] step of the current node pass
    // FP64 partials with a fixed mapping: one entry per warp of the element kernel
    // (a warp = a group of 4 elements), one per block of the node kernel
    double* e_diss = nullptr;         // += per element warp
    double* e_strain = nullptr;       // =
    double* n_work = nullptr;         // += per node block
    double* n_kin = nullptr;          // =
    int* e_stats = nullptr;           // per element warp: [0] += non-converged, [1] = yielded points
};

struct ShellParams {
    float mu, kappa, yield, hardening;   // J2 point law, linear isotropic hardening
    // The general point law of plasticity::update (plasticity.cpp:319-505): a Swift
    // curve K (eps0 + p)^n instead of the linear one, linear kinematic hardening (back
    // stress), ductile damage D += d(eps_p) / (eps_f f(eta)) with eps_f the element's
    // failure strain and f(eta) = exp(-c (eta - eta_ref)) above the cutoff, a point
    // failing at D = 1; and the element rules that go with it (solid_shell.cpp:870-1000):
    // no enhanced modes once a point has failed, one retry without them in the step a
    // point fails, torn when all eight have.
    int general;
    int swift;                            // 1: Swift curve; 0: linear
    float swift_k, swift_eps0, swift_n;
    float kinematic;
    float tri_sens, tri_ref, tri_cut;
    // the punch: speed along -axis, ramped linearly over punch_ramp seconds from rest;
    // or, with inertial set, a striking body of punch_mass whose speed the grip sets
    float punch_speed;
    double punch_ramp;
    int inertial;
    double punch_mass;
    double edge_ramp;                     // smoothstep ramp of the driven edge, s (0: at once)
    float axis_x, axis_y, axis_z;
    double inv_2mu, inv_3kappa;           // 1 / (2 mu), 1 / (3 kappa) in double (energy account)
    // the fibres' uniaxial law, in double (constraint.cpp:39-95): E, the flow curve,
    // and the Rice-Tracey factor's constants
    struct FiberLaw {
        double youngs, yield, hardening, swift_k, swift_eps0, swift_n, tri_sens, tri_ref, tri_cut;
        int swift;
    } fiber;
    float dt, damping;
    double damping64;                     // the damping as given: velocities are scaled in double
    double dt64, rise_time;               // load factor min((step+1) dt / rise, 1)
    int max_iterations;                   // EAS Newton cap
    float tol_residual, tol_work;         // relative to sigma_y V
    int compensated;                      // Kahan on displacement and plastic strain
    int eas64;                            // FP64 in the enhanced-strain block: 0-3 (shell_forces)
};

constexpr int kShellBlock = 128;          // 16 elements per block
// The step's per-element corner record in shared memory (floats): the corners' rest
// differences to corner 0 (8 x 3), the bottom corners' directors (4 x 3), the
// displacement differences to corner 0 (8 x 3), the co-rotated displacements (8 x 3)
// and the centre's Voigt transform T0 (4 columns x 6).
constexpr int kGeoX = 0, kGeoD = 24, kGeoDd = 36, kGeoU = 60, kGeoT = 84, kShellGeo = 108;
constexpr int kShellNodeBlock = 256;
constexpr int kShellPunchBlock = 256;   // the inertial punch: one block
constexpr int kShellFiberBlock = 128;

void launch_shell_step(const ShellDevice& d, const ShellParams& p, cudaStream_t stream, int parts);
// Factor of the elastic K_aa per element for this material (into `out`, [E][32]).
void launch_shell_elastic_factor(const ShellDevice& d, double youngs, double poisson, float* out,
                                 cudaStream_t stream);

// Rest forms in FP64 on the device (solid_shell.cpp:237-375).  The solver's set-up
// (eight lanes per element) writes the element rows and, in double, the lumped corner
// masses (into CSR slots) and the Gauss volumes; the per-element form (one thread per
// element) writes the double forms (forms64, 1507 doubles per element), the masses
// and, if dt_out is non-null, the element's critical step (solid_shell.cpp:1088-1133).
struct ShellSetupArgs {
    long long elements, groups;
    const double* rest;        // 3N
    const uint32_t* index;     // 8E
    const uint32_t* slot;      // 8E
    int formulation;           // 0 displacement, 1 ANS, 2 solid-shell
    double density, youngs, poisson, safety;
    float4* elem;              // [E][kShellElemQ] element rows (may be null)
    double* corner_mass;       // CSR slots (may be null)
    double* gauss_volume;      // [E][8] (may be null)
    double* dt_out;            // [E] (may be null)
    double* forms64;           // [E][1507] (may be null)
    int* ok;                   // [E] (may be null)
};
void launch_shell_setup(const ShellSetupArgs& a, cudaStream_t stream);
// The node -> corner adjacency in element order and the corner -> CSR slot map, on the
// device (csr.cu): offset [nodes + 1], slot [total]; index values must be < nodes.
// `entry_out` [total], if given, receives the adjacency entries themselves; `base` is
// added to every offset and slot (a CSR placed at that position of a larger one).
cudaError_t build_csr_device(const uint32_t* index, long long total, long long nodes, uint32_t* offset, uint32_t* slot,
                             cudaStream_t stream, uint32_t* entry_out = nullptr, uint32_t base = 0);
// Sum the CSR corner masses per node in CSR order (the element order zone.cpp:709-712
// accumulates them in), then the FP32 mass and 1/mass.
void launch_shell_mass(long long nodes, const uint32_t* offset, const double* corner_mass, double* mass64,
                       float* mass, float* inv_mass, cudaStream_t stream);

}  // namespace fs
