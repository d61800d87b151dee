// kyn_types.h -- data structures shared by the host setup and the CUDA kernels.
//
// Layout in HBM: every beam system (an element, or elements sharing nodes, or
// the nodes of a model without beam elements) owns one contiguous "slab" of
// doubles holding its constant geometry (shape tables, quadrature data,
// sectional 6x6 matrices) followed by its resident node state in local node
// order, its constraints' inputs and multipliers, and the hub-chain records
// of a jointed model.  Beam systems share no nodes, so one slab is everything
// its CTA reads and writes during a step; what couples the systems of a model
// (its hub chain) is kept as identical copies in every slab of the model.
#pragma once

#include <cstdint>

#if defined(__CUDACC__)
#define KYN_HD __host__ __device__
#else
#define KYN_HD
#endif

namespace kyn {

constexpr int kMaxBeamConstraints = 16;  // constraint records of one system (dense models)
constexpr int kMaxBeamSystemConstraints = 8;  // FixedBC / PrescribedBC / joints per beam system
constexpr int kMaxFP64SystemNodes = 21;  // nodes of one beam system in the FP64 form (shared memory)
constexpr int kMaxClusterBeams = 8;      // beams per model (portable cluster size)
constexpr int kMaxNewtonIters = 64;      // convergence-history capacity
constexpr int kRefineSweeps = 8;         // FP32 form: most refinement sweeps per linear solve
constexpr double kRefineTol = 1e-10;     // FP32 form: backward error the sweeps aim for
constexpr int kDenseModelMaxDofs = 120;  // unknowns of a model solved as a dense bordered system
// A dense model with beam elements keeps each beam component's constant data
// (a slab in SlabLayout(Nc, Qc)) after its own records; a header of
// kCompHead doubles per component precedes them: [offset of the component's
// slab from the header start, Nc, Qc, model node of each local node (32),
// offset of the component's condensation workspace from the header start].
constexpr int kCompHead = 36;
constexpr int kCompWork = 35;
constexpr int kMaxDenseComps = 8;
// A condensed dense model (KBeam::cond_nd > 0) eliminates the interior nodes
// of each beam component -- nodes of one component only, without masses,
// springs or constraints -- inside the component's own system, and solves
// the bordered system of the remaining nodes and the constraints (at most
// kCondMaxDofs unknowns).  The workspace of a component holds its system
// [6Nc][6Nc + 1] during the condensation and its factored interior rows for
// the back substitution.
constexpr int kCondMaxDofs = 160;
constexpr int kThreads = 256;            // threads per CTA of the step kernel

// Offsets (in doubles) of the arrays inside one beam slab.
struct SlabLayout {
    int32_t phi, dphi;          // [Q][N] shape values / derivatives (qp-major)
    int32_t dphiJ;              // [Q][N] derivatives divided by the Jacobian
    int32_t qpw;                // [Q][4]  w, J, w*J, w/J
    int32_t x0p;                // [Q][3]  unit tangent of the reference line
    int32_t r0;                 // [Q][4]  reference rotation
    int32_t mstar, cstar;       // [Q][36] sectional mass / stiffness (material frame)
    int32_t x0;                 // [N][7]
    int32_t q, q_prev, x;       // [N][7]
    int32_t v, vd, a, q_delta;  // [N][6]
    int32_t fx, f;              // [N][6]  node_FX and state.f
    int32_t tangent;            // [N][9]  rotational block of the stored tangent
    int32_t con_input;          // [kMaxBeamConstraints][7]
    int32_t lambda;             // [kMaxBeamConstraints][6]
    int32_t hub;                // [kHubChain][kHubDoubles] hub chain of a jointed model (hubrec)
    int32_t total;
};

// Hub node of a model whose beam roots are rigidly jointed to it: a node in
// no beam element, held by one FixedBC / PrescribedBC.  Every beam of the
// model keeps an identical copy of the hub's state in its slab; every CTA of
// the model's cluster updates its copy with the same arithmetic.
//
// A drive train extends the hub to a chain of up to kHubChain massless nodes:
// record 0 is the node held by the BC (shaft base), record 1 the target of a
// revolute joint from it (azimuth), record 2 an optional node rigidly jointed
// to record 1 (hub).  The beam roots join the last record.  Each record holds
// its node's state and the constraint that leads into the node: the BC
// (record 0), the revolute joint with its frame in `axes` and its torque in
// input[0] (record 1), the rigid joint (record 2).
namespace hubrec {
constexpr int x0 = 0;       // [7]
constexpr int q = 7;        // [7]
constexpr int q_prev = 14;  // [7]
constexpr int x = 21;       // [7]
constexpr int v = 28;       // [6]
constexpr int vd = 34;      // [6]
constexpr int a = 40;       // [6]
constexpr int q_delta = 46; // [6]
constexpr int tangent = 52; // [9] rotational block of the stored tangent
constexpr int input = 61;   // [7] hub BC input (PrescribedBC displacement); revolute torque
constexpr int lambda = 68;  // [6] multipliers of the constraint leading into the node
constexpr int X0 = 74;      // [3] hub BC X0 (FixedBC); joints: node x0 - previous node x0
constexpr int axes = 77;    // [9] revolute joint frame, row 0 = joint axis
}  // namespace hubrec
constexpr int kHubDoubles = 86;  // one record
constexpr int kHubChain = 3;

KYN_HD inline SlabLayout make_slab_layout(int N, int Q) {
    SlabLayout L{};
    int o = 0;
    auto take = [&](int n) {
        const int r = o;
        o += (n + 1) & ~1;  // keep 16-byte alignment of every array
        return r;
    };
    L.phi = take(Q * N);
    L.dphi = take(Q * N);
    L.dphiJ = take(Q * N);
    L.qpw = take(Q * 4);
    L.x0p = take(Q * 3);
    L.r0 = take(Q * 4);
    L.mstar = take(Q * 36);
    L.cstar = take(Q * 36);
    L.x0 = take(N * 7);
    L.q = take(N * 7);
    L.q_prev = take(N * 7);
    L.x = take(N * 7);
    L.v = take(N * 6);
    L.vd = take(N * 6);
    L.a = take(N * 6);
    L.q_delta = take(N * 6);
    L.fx = take(N * 6);
    L.f = take(N * 6);
    L.tangent = take(N * 9);
    L.con_input = take(kMaxBeamConstraints * 7);
    L.lambda = take(kMaxBeamConstraints * 6);
    L.hub = take(kHubChain * kHubDoubles);
    L.total = o;
    return L;
}

// One beam as seen by the step kernel (built per launch plan).
// Point-mass and spring records behind KBeam::lumped (doubles):
//   mass   [kMassRec]   = node, M_star[36] (material frame), r0[4] (node x0 rotation)
//   spring [kSpringRec] = node 1, node 2, x0[3] (x0 of node 2 - x0 of node 1), l_ref, k
constexpr int kMassRec = 41;
constexpr int kSpringRec = 7;

// Joints between the hub node and a target node (six rows, base blocks on the
// hub): KYN_CONSTRAINT_RIGID_JOINT (3) and KYN_CONSTRAINT_ROTATION_CONTROL (5).
KYN_HD inline bool is_hub_joint(int type) { return type == 3 || type == 5; }
// Node freedom signatures (src/dof_management/freedom_signature.hpp): all six
// components, or the three positions of a position-only node.
constexpr int kSigAll = 0b111111;
constexpr int kSigPosition = 0b111000;
// Rows of a constraint (src/constraints/constraint_type.hpp NumRowsForConstraint).
KYN_HD inline int constraint_rows(int type) { return type == 4 ? 5 : type >= 6 ? 3 : 6; }

struct KBeam {
    double* slab;             // device slab of this beam
    int32_t N, Q, nc;         // nodes, quadrature points, constraints on this beam
    int32_t plan_model;       // model index inside the launch plan
    int32_t rank;             // beam index inside its model (cluster rank)
    int32_t model_beams;      // beams of the model (= cluster size of the launch)
    int32_t model_dofs;       // Solver::num_dofs of the model
    int32_t con_node[kMaxBeamConstraints];   // beam-local target node
    int32_t con_type[kMaxBeamConstraints];   // KYN_CONSTRAINT_*
    int32_t con_row[kMaxBeamConstraints];    // constraint index within the model
    double con_X0[kMaxBeamConstraints][3];   // joints: target x0 - hub x0
    double con_axis[kMaxBeamConstraints][3]; // RotationControl: unit rotation axis
    const double* lumped;     // point masses then springs at this beam's nodes, or null
    int32_t n_mass, n_spring; // (records of kMassRec / kSpringRec doubles, node-local indices)
    int32_t hub;              // hub chain length: 0 none, 1 hub, 2-3 drive train
    int32_t dense;            // 1: a model without beams solved as its dense bordered system
    int32_t con_base[kMaxBeamConstraints];   // dense models: joint base node (local), or -1
    int32_t hub_con_type;     // KYN_CONSTRAINT_FIXED_BC / PRESCRIBED_BC on the hub
    double gravity[3];
    const double* comps;      // dense models with beams: component records (kCompHead), or null
    int32_t n_comps;          // beam components (connected element groups) of a dense model
    int32_t comp_maxN, comp_maxQ;  // their largest node and quadrature-point counts
    int32_t cond_nd;          // condensed dense models: unknowns of the bordered system, else 0
    double* cond_md;          // condensed dense models: that system in device memory, or null (shared)
    const double* con_frames; // dense models: [nc][9] frame (x0, y0, z0) of each revolute joint, or null
    double* conv;             // [kMaxNewtonIters] model convergence history (rank 0)
    double* dump;             // optional: last assembled system (see kyn_capi.cu)
    unsigned long long* prof; // optional: per-phase SM cycles, summed over beams
};

// Phases of the step kernel timed when KYN_OPT_PHASE_TIMING is set.
enum Phase {
    kPhaseLoadPredict = 0,
    kPhaseQuadrature = 1,   // tangent operator + quadrature-point physics
    kPhaseIntegrate = 2,    // residual + stiffness/inertia integration into A
    kPhaseConstraints = 3,  // constraint residual/gradient + right-hand side
    kPhaseEliminate = 4,    // boundary-condition elimination
    kPhaseFactor = 5,       // LU of the free block
    kPhaseSubstitute = 6,   // back substitution + multipliers
    kPhaseUpdate = 7,       // convergence error + Newton update
    kPhaseStore = 8,        // post-step and write-back
    kPhaseLUDiag = 9,       // LU: diagonal-block factorisation (part of the factor phase)
    kPhaseLUPanel = 10,     // LU: panel solves (part of the factor phase)
    kPhaseIntEpilogue = 11, // LU: L21 rows solved by all threads (part of the factor phase)
    kPhaseRefine = 12,      // FP32 form: FP64-residual refinement sweeps of the correction
    kNumPhases = 13
};

// Step coefficients (src/step/step_parameters.hpp:37-52).
struct StepCoeffs {
    double h, alpha_m, alpha_f, gamma, beta, gamma_prime, beta_prime, conditioner;
    double atol, rtol;
    int32_t max_iter;
    int32_t dynamic;
    int32_t refine_iters;  // extra corrections after convergence (FP32 form)
    int32_t solver;        // KYN_SOLVER_*: free-block solve (register Gauss-Jordan or panel LU)
    int32_t refine_sweeps; // FP32 form: most refinement sweeps of one linear solve
    double refine_tol;     // FP32 form: target relative FP64 residual of the linear solve
    unsigned long long* diag;  // solve counters (kDiag*), or null
    int32_t bulk_sections;     // 1: stage each iteration's sections with one bulk copy
};

// Solve counters of a context (StepCoeffs::diag), summed over the beams of
// every step: Gauss-Jordan solves whose backward error was checked, those
// above kGJBackwardErrorMax, the largest backward error seen (bits of a
// non-negative double, so integer max orders them), FP32 refinement sweeps
// taken, and FP32 solves still above the refinement tolerance after the last
// sweep.
enum : int {
    kDiagChecked = 0,
    kDiagGuardTrips = 1,
    kDiagMaxBackwardError = 2,
    kDiagRefineSweeps = 3,
    kDiagRefineShort = 4,
    kNumDiag = 8
};

}  // namespace kyn
