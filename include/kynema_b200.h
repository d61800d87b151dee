/*
 * kynema_b200.h -- C ABI of the B200-native per-step beam path.
 *
 * This library replaces the device side of Kynema's (formerly OpenTurbine's)
 * per-time-step beam path: the GEBT beam quadrature-point kernels, node-pair
 * integration, assembly of the bordered constraint system, the linear solve and
 * the Lie-group generalized-alpha Newton predictor/update.  The host keeps the
 * reference's Model / Elements / State / Constraints / Solver / Step() surface
 * and calls the path through the entry points below.
 *
 * Conventions
 *   - Plain C types only; every array is row-major and caller-owned.  The
 *     library copies inputs in and results out and never retains caller
 *     pointers.
 *   - Quaternions are (w, x, y, z), as in src/math/quaternion_operations.hpp.
 *   - Node state rows: position/rotation fields have 7 components
 *     (x, y, z, w, i, j, k); velocity-like fields have 6.
 *   - Every entry point returns an int status: KYN_OK (0) on success, a
 *     negative KYN_ERR_* code on failure (kyn_last_error() gives the text).
 *     kyn_step() additionally reports per-model step status, where
 *     KYN_NOT_CONVERGED (1) is the reference's `Step() == false`.
 *   - One context per host thread; all work of a context is serialised on its
 *     own CUDA stream.  kyn_step() returns after results are resident on the
 *     device and the per-model status has been copied back.
 */
#ifndef KYNEMA_B200_H
#define KYNEMA_B200_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define KYN_API __attribute__((visibility("default")))
#else
#define KYN_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
enum {
    KYN_OK = 0,
    KYN_NOT_CONVERGED = 1,   /* Newton loop hit max_iter: Step() returned false
                                (src/step/step.hpp:55-57) */
    KYN_ERR_INVALID = -1,    /* bad argument or malformed model description */
    KYN_ERR_UNSUPPORTED = -2,/* topology or constraint type outside this path */
    KYN_ERR_CUDA = -3,       /* a CUDA runtime call failed */
    KYN_ERR_BUDGET = -4,     /* model admission refused: HBM budget exceeded */
    KYN_ERR_NONFINITE = -5,  /* a non-finite value appeared in the Newton loop */
    KYN_ERR_SINGULAR = -6,   /* zero pivot in the linear solve */
    KYN_ERR_NOT_FOUND = -7,  /* unknown model id */
    KYN_ERR_NO_DEVICE = -8   /* no CUDA device / library built without it */
};

/* Constraint types: same numbering as constraints::ConstraintType
 * (src/constraints/constraint_type.hpp:9-24).  This path implements the two
 * single-node boundary conditions used by beams and rotors, the two six-row
 * joints that tie blade roots to a hub node, the five-row revolute joint that
 * lets a drive train (hub, or azimuth node rigidly holding the hub) turn about
 * a shaft held by a boundary condition, and the three-row constraints on
 * position-only nodes of models without beam elements. */
enum {
    KYN_CONSTRAINT_FIXED_BC = 1,
    KYN_CONSTRAINT_PRESCRIBED_BC = 2,
    KYN_CONSTRAINT_RIGID_JOINT = 3,  /* base node (hub) to target node, six DOFs
                                        (src/constraints/calculate_rigid_joint_constraint.hpp) */
    KYN_CONSTRAINT_REVOLUTE_JOINT = 4, /* five rows: the target turns freely about the
                                        joint axis (constraint_axis, or the base-to-target
                                        direction when it is zero; src/constraints/
                                        constraints.hpp:294-319); a torque about that axis,
                                        u[0] of kyn_model_set_prescribed, acts on the target
                                        (src/constraints/calculate_revolute_joint_constraint.hpp,
                                        calculate_revolute_joint_force.hpp) */
    KYN_CONSTRAINT_ROTATION_CONTROL = 5  /* a rigid joint whose target is turned by a
                                        commanded angle about constraint_axis (normalised
                                        here as in src/constraints/constraints.hpp:321-328);
                                        the angle is u[0] of kyn_model_set_prescribed, the
                                        slot Constraints::UpdateViews fills from the control
                                        pointer (src/constraints/constraints.hpp:345-352;
                                        src/constraints/calculate_rotation_control_constraint.hpp:17-144,
                                        src/model/model.hpp:550-562) */,
    KYN_CONSTRAINT_FIXED_BC_3DOF = 6,      /* three rows on a position-only node (model.hpp:570-583) */
    KYN_CONSTRAINT_PRESCRIBED_BC_3DOF = 7, /* three rows, input = the node's displacement */
    KYN_CONSTRAINT_RIGID_JOINT_6DOF_TO_3DOF = 8 /* three rows: a position-only target rigidly
                                        carried by a six-DOF base (model.hpp:599-611;
                                        src/constraints/calculate_rigid_joint_3DOF_constraint.hpp) */
};

/* Node-state fields readable with kyn_get_state (src/state/state.hpp:18-68,
 * src/constraints/constraints.hpp lambda). */
enum {
    KYN_FIELD_X0 = 0,      /* [nodes][7] initial position/orientation      */
    KYN_FIELD_X = 1,       /* [nodes][7] current global position           */
    KYN_FIELD_Q = 2,       /* [nodes][7] displacement                      */
    KYN_FIELD_Q_PREV = 3,  /* [nodes][7] displacement at the previous step */
    KYN_FIELD_Q_DELTA = 4, /* [nodes][6] displacement increment            */
    KYN_FIELD_V = 5,       /* [nodes][6] velocity                          */
    KYN_FIELD_VD = 6,      /* [nodes][6] acceleration                      */
    KYN_FIELD_A = 7,       /* [nodes][6] algorithmic acceleration          */
    KYN_FIELD_F = 8,       /* [nodes][6] external nodal forces (state.f)   */
    KYN_FIELD_LAMBDA = 9,  /* [constraints][6] Lagrange multipliers        */
    KYN_FIELD_TANGENT = 10, /* [nodes][6][6] tangent operator, stored
                              transposed as in CalculateTangentOperator     */
    KYN_FIELD_CONSTRAINT_OUTPUT = 11 /* [constraints][3] Constraints::output: for a
                              revolute joint the rotation, angular velocity and
                              angular acceleration about its axis
                              (src/constraints/calculate_revolute_joint_output.hpp);
                              zero for the other types                          */
};

/* Load channels for kyn_model_set_loads. */
enum {
    KYN_LOAD_NODE_FX = 0,  /* Beams::node_FX: [element nodes][6] in the order
                              of desc.beam_node_ids (element, node-in-element) */
    KYN_LOAD_STATE_F = 1   /* State::f: [nodes][6] */
};

/* Arithmetic of the tangent blocks and the linear solve. */
enum {
    KYN_PRECISION_FP64 = 0,          /* plain form: everything FP64            */
    KYN_PRECISION_FP32_REFINED = 1   /* FP32 tangent + FP32 LU, FP64 residual,
                                        rotation update and refinement        */
};

/* Model description: the data Model::AddNode / AddBeamElement /
 * AddMassElement / AddSpringElement / AddFixedBC / AddPrescribedBC /
 * SetGravity collect on the host
 * (src/model/model.hpp:74-693, src/model/node.hpp:35-60,
 * src/elements/beams/beam_section.hpp, src/constraints/constraint.hpp). */
typedef struct kyn_model_desc {
    int32_t num_nodes;
    const double* node_x0;  /* [num_nodes][7] Node::x0                    */
    const double* node_u;   /* [num_nodes][7] Node::u   (NULL: identity)  */
    const double* node_v;   /* [num_nodes][6] Node::v   (NULL: zero)      */
    const double* node_vd;  /* [num_nodes][6] Node::vd  (NULL: zero)      */
    const double* node_s;   /* [num_nodes]    Node::s, element location   */

    int32_t num_beams;
    const int32_t* beam_node_offsets;    /* [num_beams+1] into beam_node_ids */
    const int32_t* beam_node_ids;        /* node ids of each beam element    */
    const int32_t* beam_section_offsets; /* [num_beams+1]                    */
    const double* section_position;      /* BeamSection::position in [0,1]   */
    const double* section_mass;          /* [sections][6][6] M_star          */
    const double* section_stiffness;     /* [sections][6][6] C_star          */
    const int32_t* beam_qp_offsets;      /* [num_beams+1]                    */
    const double* qp_xi;                 /* quadrature locations in [-1,1]   */
    const double* qp_weight;             /* quadrature weights               */

    int32_t num_constraints;
    const int32_t* constraint_type;        /* KYN_CONSTRAINT_*               */
    const int32_t* constraint_base_node;   /* Constraint::node_ids[0]        */
    const int32_t* constraint_target_node; /* Constraint::node_ids[1]        */
    const double* constraint_axis;         /* [constraints][3] or NULL       */
    const double* constraint_initial_displacement; /* [constraints][7] or NULL */

    double gravity[3];

    /* Point masses and springs (src/model/model.hpp:294-415 AddMassElement,
     * AddSpringElement).  A model of masses and springs only (num_beams = 0) runs
     * on the lumped-element kernel; see KYN_LUMPED_* for its limits. */
    int32_t num_masses;
    const int32_t* mass_node;          /* [num_masses] MassElement::node_id        */
    const double* mass_matrix;         /* [num_masses][6][6] M_star, material frame */
    int32_t num_springs;
    const int32_t* spring_nodes;       /* [num_springs][2] SpringElement::node_ids */
    const double* spring_stiffness;    /* [num_springs] k                          */
    const double* spring_length;       /* [num_springs] undeformed length l_ref    */
} kyn_model_desc;

/* Limits of a lumped model (masses, springs and single-node boundary
 * conditions, no beam element): one CTA holds its dense system. */
enum {
    KYN_LUMPED_MAX_NODES = 24,
    KYN_LUMPED_MAX_MASSES = 32,
    KYN_LUMPED_MAX_SPRINGS = 64
};

/* Step controls: the arguments of the StepParameters constructor
 * (src/step/step_parameters.hpp:37-52) plus the arithmetic choice. */
typedef struct kyn_step_params {
    int32_t is_dynamic_solve;
    int32_t max_iter;
    double h;
    double rho_inf;
    double absolute_convergence_tol; /* reference default 1e-5 */
    double relative_convergence_tol; /* reference default 1e-3 */
    int32_t precision;               /* KYN_PRECISION_*         */
    int32_t refine_iters;            /* FP32 form: extra Newton corrections after
                                        the convergence test passes (each with
                                        the FP64 residual); ignored in FP64 */
} kyn_step_params;

/* Sizes of one model's system (Solver::num_system_dofs / num_dofs / nnz). */
typedef struct kyn_model_info {
    int32_t num_nodes;
    int32_t num_beams;
    int32_t num_constraints;
    int32_t num_system_dofs;
    int32_t num_dofs;
    int32_t nnz;
    int32_t max_beam_nodes;
    int32_t max_beam_qps;
    int64_t device_bytes;   /* HBM held by this model's resident state */
    /* Condensed models (a multi-element beam longer than one FP64 beam system,
     * or beams coupled by joints beyond 120 unknowns): unknowns of the
     * bordered system left after each element's interior nodes are eliminated
     * inside the element; 0 for every other model.  No reference counterpart
     * (the reference factors the whole sparse system). */
    int32_t condensed_dofs;
} kyn_model_info;

typedef struct kyn_ctx kyn_ctx;

/* Context: owns every device buffer.  hbm_budget_bytes caps the resident
 * model state admitted by kyn_model_create (0 = no cap).
 * Replaces the Kokkos::initialize + per-model View allocation done by
 * Model::CreateSystemWithSolver (src/model/model.hpp:647-656). */
KYN_API kyn_ctx* kyn_ctx_create(int device, size_t hbm_budget_bytes);
KYN_API void kyn_ctx_destroy(kyn_ctx* ctx);
KYN_API const char* kyn_last_error(const kyn_ctx* ctx);
/* The context's CUDA stream (a cudaStream_t), for callers that order their own
 * work or timing events against the library's work. */
KYN_API void* kyn_ctx_stream(kyn_ctx* ctx);
/* Device bytes currently held by admitted models. */
KYN_API size_t kyn_ctx_used_bytes(const kyn_ctx* ctx);

/* Replaces Model::CreateSystemWithSolver (src/model/model.hpp:647-656):
 * copies the nodes to resident state (src/model/copy_nodes_to_state.hpp),
 * builds beam geometry (src/elements/beams/create_beams.hpp:27-165), the
 * constraints (src/constraints/constraints.hpp:76-266), the DOF map and the
 * CRS graph (src/model/model.hpp:42-63, src/solver/create_full_matrix.hpp).
 * Returns the model id (>= 0) or a negative KYN_ERR_* code. */
KYN_API int kyn_model_create(kyn_ctx* ctx, const kyn_model_desc* desc);
KYN_API int kyn_model_destroy(kyn_ctx* ctx, int model_id);
KYN_API int kyn_model_info_get(kyn_ctx* ctx, int model_id, kyn_model_info* info);

/* Host only (no device, no context): validates a description as
 * kyn_model_create does and reports its sizes and, when row_ptrs / col_inds are
 * not NULL, its CRS graph (row_ptrs [num_dofs + 1], col_inds [nnz]; the graph of
 * Model::CreateSystemWithSolver, src/solver/create_full_matrix.hpp:27-73).
 * info->device_bytes is the slab footprint a model would take.  err (errlen
 * bytes, may be NULL) receives the reason of a negative return code.  No
 * counterpart in the reference: lets a caller check a model, and tests check the
 * DOF map and CRS graph of every model type, without a GPU. */
KYN_API int kyn_model_describe(const kyn_model_desc* desc, kyn_model_info* info, int32_t* row_ptrs,
                               int32_t* col_inds, char* err, int errlen);

/* A new model that is a copy of an existing one in its current state (same
 * description, node state, multipliers and loads; its own device memory,
 * counted against the HBM budget).  No counterpart in the reference: a server
 * that admits many copies of the same description keeps one resident template
 * and clones it, which costs a device-to-device copy instead of a rebuild of
 * the shape tables, sections and CRS graph.  Returns the new id or a negative
 * KYN_ERR_* code. */
KYN_API int kyn_model_clone(kyn_ctx* ctx, int model_id);

/* Replaces writes of Beams::node_FX (tests/regression_tests/regression/
 * test_cantilever_beam.cpp:105-107) or State::f. */
KYN_API int kyn_model_set_loads(kyn_ctx* ctx, int model_id, int which, const double* values);

/* Replaces Constraints::UpdateDisplacement (src/constraints/constraints.hpp:338-343).
 * For a KYN_CONSTRAINT_ROTATION_CONTROL constraint u[0] is the commanded angle
 * (rad), for a KYN_CONSTRAINT_REVOLUTE_JOINT the torque about the joint axis;
 * u[1..6] are ignored for both. */
KYN_API int kyn_model_set_prescribed(kyn_ctx* ctx, int model_id, int constraint_id, const double u[7]);

/* Replaces kynema::Step (src/step/step.hpp:42-124) for a batch of models:
 * every listed model advances one time step.  status_out[i] is KYN_OK,
 * KYN_NOT_CONVERGED or a negative code; iters_out[i] is the Newton iteration
 * count (= solver.convergence_err.size()).  Either output may be NULL. */
KYN_API int kyn_step(kyn_ctx* ctx, const int* model_ids, int n, const kyn_step_params* params,
             int* status_out, int* iters_out);

/* Asynchronous form used by the serving loop: enqueue the step on the
 * context stream and return; kyn_step_wait() blocks until it is complete and
 * fills status/iterations for the models of the last kyn_step_async call. */
KYN_API int kyn_step_async(kyn_ctx* ctx, const int* model_ids, int n, const kyn_step_params* params);
KYN_API int kyn_step_wait(kyn_ctx* ctx, int* status_out, int* iters_out);

/* Batched forms of kyn_model_set_loads / kyn_get_state for many models in one
 * transfer: `values` / `out` hold the models' arrays back to back in the order
 * of model_ids (NODE_FX: [element nodes][6]; STATE_F and node fields:
 * [nodes][width]).  With on_device != 0 the pointer is device memory and no
 * host copy is made; otherwise it is host memory (pinned memory is fastest).
 * These replace the per-model Kokkos::deep_copy of node_FX / state.f before
 * Step() and of state.q after it (src/interfaces/cfd/interface.cpp:283-309). */
KYN_API int kyn_set_loads_batch(kyn_ctx* ctx, const int* model_ids, int n, int which,
                                const double* values, int on_device);
KYN_API int kyn_get_state_batch(kyn_ctx* ctx, const int* model_ids, int n, int field,
                                double* out, int on_device);

/* kyn_set_loads_batch without any allocation (no counterpart in the reference).
 * For callers that cannot let a library allocate while they run, e.g. a CFD
 * solver that owns the device memory through its own pool and shares the GPU:
 * device staging comes from one fixed 9.19 MiB array inside the library instead
 * of cudaMalloc'd buffers.  Limits per call: 8192 beam elements, 262144 node
 * rows, and (host values) 1048576 load doubles; larger batches return
 * KYN_ERR_INVALID with a message and change nothing.  The first call on each
 * device does a one-time set-up (looks up the array's device address, which
 * may load the library's device code): make it before any stream capture.
 * The array is shared by every call and context on the device and keeps the
 * last call's contents: calls that overlap on the device race on it.  A call
 * returns before its copy kernel runs, so calls from two contexts (two streams)
 * race even when the host makes them one after the other: order them on the
 * device (synchronise the first stream, or make the second wait on an event
 * recorded after the first call).  The device address found at set-up is kept
 * for the life of the process; do not call this again on a device after
 * cudaDeviceReset.  Results equal those of kyn_set_loads_batch. */
KYN_API int kyn_set_loads_batch_static(kyn_ctx* ctx, const int* model_ids, int n, int which,
                                       const double* values, int on_device);

/* Autotuner (no counterpart in the reference): for every size class of the
 * listed models (beams per model, nodes, quadrature points, constraints,
 * precision), times the step kernel with 128, 256 and 512 threads per CTA --
 * in the FP64 form, for beam systems, each with the panel LU and with the
 * register Gauss-Jordan solve of the free block (the same FP64 accuracy
 * class; Gauss-Jordan is the faster for small beams) -- on temporary copies
 * of all the class's models (repeated up to 4 x SMs copies, at most 16384;
 * four steps after one warm-up step)
 * and keeps the fastest for later kyn_step calls on this context.  The
 * listed models' states are not changed. */
KYN_API int kyn_autotune(kyn_ctx* ctx, const int* model_ids, int n, const kyn_step_params* params);

/* Threads per CTA kyn_step uses for a model at a precision (tuned or default). */
KYN_API int kyn_tuned_threads(kyn_ctx* ctx, int model_id, int precision);

/* Free-block solver (KYN_SOLVER_*) kyn_step uses for a model at a precision:
 * the tuned one, else the context's KYN_OPT_LINEAR_SOLVER.  No counterpart in
 * the reference. */
KYN_API int kyn_tuned_solver(kyn_ctx* ctx, int model_id, int precision);

/* Batched Constraints::UpdateDisplacement for many models: values holds
 * [sum of the listed models' constraints][7] (model order, then constraint
 * order).  Replaces the per-blade prescribed hub motion updates of
 * src/interfaces/turbine/turbine_interface.cpp:117-150. */
KYN_API int kyn_set_prescribed_batch(kyn_ctx* ctx, const int* model_ids, int n, const double* values,
                                     int on_device);

/* Writes one node field ([nodes][7] or [nodes][6], model node order) into the
 * resident state: the inverse of kyn_get_state for x0, x, q, q_prev, q_delta,
 * v, vd, a and f. */
KYN_API int kyn_set_state(kyn_ctx* ctx, int model_id, int field, const double* values);

/* Restart record of WriteStateToFile / ReadStateFromFile
 * (src/state/write_state_to_file.hpp:20-58, read_state_from_file.hpp:23-65):
 * size_t num_system_nodes, then x0, x, q_delta, q_prev, q, v, vd, a, f as
 * doubles, node-major.  kyn_state_write with buf NULL only reports the size;
 * kyn_state_read rejects a record whose node count differs from the model's
 * (the reference's std::length_error) with KYN_ERR_INVALID. */
KYN_API int kyn_state_write(kyn_ctx* ctx, int model_id, void* buf, size_t capacity, size_t* bytes);
KYN_API int kyn_state_read(kyn_ctx* ctx, int model_id, const void* buf, size_t size);

/* CopyStateData (src/state/copy_state_data.hpp:21-34) between two models of the
 * same structure: x, q_delta, q_prev, q, v, vd, a, f and the tangent blocks
 * (the save / restore of the CFD predictor-corrector loop,
 * src/interfaces/cfd/interface.cpp:312-327). */
KYN_API int kyn_state_copy(kyn_ctx* ctx, int dst_model_id, int src_model_id);

/* Replaces host reads of State / Constraints views after Step(). */
KYN_API int kyn_get_state(kyn_ctx* ctx, int model_id, int field, double* out);

/* Replaces reads of solver.convergence_err (src/solver/solver.hpp:83):
 * errs must hold max_iter values; *n receives the count. */
KYN_API int kyn_get_convergence(kyn_ctx* ctx, int model_id, double* errs, int* n);

/* Replaces solver.A / solver.b / solver.x reads (src/solver/solver.hpp:79-81).
 * row_ptrs [num_dofs+1] and col_inds [nnz] are the reference's CRS graph
 * (src/solver/create_full_matrix.hpp:47-72), bit-exact.  values [nnz], rhs
 * [num_dofs] and solution [num_dofs] are the system of the last Newton
 * iteration of the last step; they are only recorded while the context
 * option KYN_OPT_RECORD_SYSTEM is set (any pointer may be NULL). */
KYN_API int kyn_get_crs(kyn_ctx* ctx, int model_id, int* row_ptrs, int* col_inds, double* values);
KYN_API int kyn_get_system_vectors(kyn_ctx* ctx, int model_id, double* rhs, double* solution);

enum {
    KYN_OPT_RECORD_SYSTEM = 1, /* keep the last assembled system for kyn_get_crs */
    KYN_OPT_PHASE_TIMING = 2,  /* count SM cycles per step-kernel phase (tracing) */
    KYN_OPT_CUDA_GRAPH = 3,    /* capture each model set's step launches in a CUDA
                                  graph and replay it (re-captured when the model
                                  set or the step coefficients change) */
    KYN_OPT_LINEAR_SOLVER = 4, /* KYN_SOLVER_*: how the step kernel solves a beam's
                                  free block (default KYN_SOLVER_PANEL_LU) */
    KYN_OPT_RESET_SOLVE_STATS = 5, /* any value: zero the KYN_STAT_SOLVES_CHECKED ..
                                      KYN_STAT_REFINE_SHORT counters */
    KYN_OPT_BULK_SECTIONS = 6  /* 1 (default): each Newton iteration's sectional
                                  data (x0', r0, M*, C*) reach shared memory in one
                                  bulk copy issued during the previous iteration;
                                  0: every quadrature point loads its own */
};

/* Free-block solves of the step kernel (the reference's sparse direct solve,
 * src/step/solve_system.hpp:27-31, after the boundary conditions are
 * eliminated).  Neither pivots.
 * PANEL_LU (default): right-looking LU in shared memory, 8-column look-ahead
 *   panels, trailing updates on the FP64 tensor cores, block back substitution.
 * GAUSS_JORDAN: the block held in registers across the CTA, one barrier per
 *   2x2 pivot block.  FP64 form: the backward error
 *   max|b - A x| / (|A| |x| + |b|) of every solve is measured and counted
 *   (KYN_STAT_SOLVES_CHECKED, _GUARD_TRIPS above 1e-10, _MAX_BACKWARD_ERROR).
 *   FP32 form: the block is inverted in FP32 and every Newton correction is
 *   refined with FP64 residuals of the assembled system until that backward
 *   error is at most 1e-10 (at most 8 sweeps; KYN_STAT_REFINE_*).  Blocks
 *   larger than the register grid of their thread count take PANEL_LU. */
enum { KYN_SOLVER_GAUSS_JORDAN = 0, KYN_SOLVER_PANEL_LU = 1 };
KYN_API int kyn_ctx_set_option(kyn_ctx* ctx, int option, int64_t value);

/* Context counters (diagnostics; no counterpart in the reference). */
enum {
    KYN_STAT_KERNEL_LAUNCHES = 1,  /* kernels launched by this context so far */
    KYN_STAT_STEP_BUCKETS = 2,     /* step-kernel launches of the last step call */
    KYN_STAT_ALLOCATIONS = 3,      /* device (cudaMalloc, cudaMallocAsync) and pinned host
                                      (cudaMallocHost) allocations made by this context */
    /* Gauss-Jordan solves (KYN_SOLVER_GAUSS_JORDAN), summed since the context
       was created or KYN_OPT_RESET_SOLVE_STATS: */
    KYN_STAT_SOLVES_CHECKED = 4,   /* solves whose backward error was measured */
    KYN_STAT_GUARD_TRIPS = 5,      /* FP64 solves with a backward error above 1e-10 */
    KYN_STAT_MAX_BACKWARD_ERROR = 6, /* largest backward error seen: the bits of a double */
    KYN_STAT_REFINE_SWEEPS = 7,    /* FP32 form: refinement sweeps taken */
    KYN_STAT_REFINE_SHORT = 8,     /* FP32 form: solves above 1e-10 after the last sweep */
    KYN_STAT_PHASE_CYCLES = 100    /* + phase (0..12): SM cycles summed over beams since
                                      KYN_OPT_PHASE_TIMING was set: load/predict,
                                      quadrature, integrate, constraints, eliminate,
                                      factor, substitute, update, store, then the
                                      panel LU's sub-phases (9..11) and the FP32
                                      form's refinement sweeps (12) */
};
KYN_API int kyn_ctx_stat(kyn_ctx* ctx, int stat, int64_t* value);

#ifdef __cplusplus
}
#endif

#endif /* KYNEMA_B200_H */
