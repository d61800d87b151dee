/*
 * kyn_oracle.h -- CPU FP64 oracle for the per-step beam path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a restatement of the reference's
 * algorithm (Kynema, formerly Exawind/openturbine) used as the checker for the
 * CUDA path and as the timed CPU baseline.  Only tests/, __graft_entry__.smoke()
 * and bench.py's CPU-baseline leg may load it; the product library never links
 * or calls it.
 *
 * Parity pinning: the oracle is checked against the reference's own golden
 * vectors (regression tests test_cantilever_beam.cpp, test_solver.cpp,
 * test_rotor.cpp, test_rotating_beam.cpp; unit tests test_curved_beam.cpp,
 * test_compute_row_ptrs.cpp, test_compute_col_inds.cpp, math and state
 * tests).  The fixtures are extracted by tests/golden/make_golden.py.
 */
#ifndef KYN_ORACLE_H
#define KYN_ORACLE_H

#include "../include/kynema_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_model orc_model;

/* Model::CreateSystemWithSolver restated (host FP64). NULL on error. */
orc_model* orc_model_create(const kyn_model_desc* desc, char* err, int errlen);
void orc_model_destroy(orc_model* m);
/* Bit flags: 0 = dense partial-pivot LU of the bordered system (default);
 * 1 = boundary-condition elimination + LU without pivoting; 2 = quadrature
 * sums in reverse order.  Flagged runs are cross-checks of rounding noise. */
void orc_set_solver_mode(orc_model* m, int mode);
int orc_model_info(const orc_model* m, kyn_model_info* info);
int orc_set_loads(orc_model* m, int which, const double* values);
int orc_set_prescribed(orc_model* m, int constraint_id, const double u[7]);

/* kynema::Step restated: returns KYN_OK or KYN_NOT_CONVERGED. */
int orc_step(orc_model* m, const kyn_step_params* p, int* iters);

/* The assembly sequence of test_solver.cpp SetUpSolverAndAssemble:
 * PredictNextState, ResetConstraints, ResetSolver, UpdateSystemVariables,
 * AssembleSystemMatrix, AssembleSystemResidual, UpdateConstraintVariables,
 * AssembleConstraintsMatrix, AssembleConstraintsResidual (no solve). */
int orc_predict_and_assemble(orc_model* m, const kyn_step_params* p);

int orc_get_state(const orc_model* m, int field, double* out);
int orc_get_crs(const orc_model* m, int* row_ptrs, int* col_inds, double* values);
/* b and x of the solver, as left by the last iteration */
int orc_get_system_vectors(const orc_model* m, double* rhs, double* solution);
int orc_get_convergence(const orc_model* m, double* errs, int* n);
/* residual_vector_terms [N][6] and system_matrix_terms [N][N][6][6] of beam e */
int orc_get_element_terms(const orc_model* m, int beam, double* residual, double* sysmat);

/* Batch runner for the CPU baseline: advance each model `steps` steps with
 * OpenMP threads over models; loads[i] (may be NULL) gives per-step tip loads
 * through a callback-free schedule: node_fx_amp/freq arrays drive
 * node_FX[last node of beam 0][2] = amp*sin(2*pi*freq*t_{k+1}).
 * Returns the number of converged model-steps; *seconds gets wall time. */
long orc_run_batch(orc_model** models, int n, const kyn_step_params* p, int steps,
                   const double* amp, const double* freq, int nthreads,
                   double* seconds, int* iters_total);

/* The same schedule starting at time step `first_step` (the tip load of step k
 * uses t = h (first_step + k + 1)), recording every model's status and Newton
 * iterations per step: status[i*steps + k], iters[i*steps + k] (either may be
 * NULL).  A step the reference's loop ends because its error norm is NaN
 * (Step() returns true) is recorded as KYN_ERR_NONFINITE and not counted.
 * Returns the number of converged model-steps. */
long orc_run_batch_record(orc_model** models, int n, const kyn_step_params* p, int first_step,
                          int steps, const double* amp, const double* freq, int nthreads,
                          double* seconds, int* status, int* iters);

/* FLOP tally of the counting build (-DORC_COUNT_FLOPS, libkyn_oracle_flops.so;
 * always 0 in the normal build): reset, then read all counted operations or
 * (qp_only) those of the quadrature-point physics of every beam update. */
void orc_flops_reset(void);
long long orc_flops_read(int qp_only);

/* ---- kernel-level restatements (curved-beam and unit known-answer tests) -- */
void orc_lagrange_interp_weights(double x, const double* xs, int n, double* w);
void orc_lagrange_deriv_weights(double x, const double* xs, int n, double* w);
void orc_gll_points(int order, double* pts);
void orc_rotate_section(const double xr[4], const double cstar[36], double out[36]);
void orc_revolute_joint(const double X0[3], const double axes[9], const double base_u[7],
                        const double target_u[7], double torque, double res[6], double base_grad[36],
                        double target_grad[36], double sys_res[6]);
void orc_constraint_kernel(int type, const double X0[3], const double axis[3], const double input[7],
                           const double base_u[7], const double target_u[7], double res[6],
                           double base_grad[36], double target_grad[36]);
void orc_revolute_output(const double axes[9], const double u[7], const double udot[6],
                         const double uddot[6], double out[3]);
void orc_calc_strain(const double x0p[3], const double up[3], const double r[4],
                     const double rp[4], double strain[6]);
void orc_calc_fc(const double cuu[36], const double strain[6], double fc[6]);
void orc_calc_fd(const double ss[9], const double fc[6], double fd[6]);
void orc_calc_ouu(const double cuu[36], const double ss[9], const double mt[9],
                  const double nt[9], double out[36]);
void orc_calc_puu(const double cuu[36], const double ss[9], const double nt[9], double out[36]);
void orc_calc_quu(const double cuu[36], const double ss[9], const double nt[9], double out[36]);
void orc_calc_jacobian(int nn, int nq, const double* shape_deriv /*[nn][nq]*/,
                       const double* node_x0 /*[nn][7]*/, double* x0p /*[nq][3]*/,
                       double* jac /*[nq]*/);
void orc_integrate_residual(int nn, int nq, const double* w, const double* jac,
                            const double* phi, const double* dphi, const double* fx,
                            const double* fc, const double* fd, const double* fi,
                            const double* fe, const double* fg, double* out);
void orc_integrate_stiffness(int nn, int nq, const double* w, const double* jac,
                             const double* phi, const double* dphi, const double* kuu,
                             const double* puu, const double* cuu, const double* ouu,
                             const double* quu, double* out /*[nn][nn][36]*/);
void orc_integrate_inertia(int nn, int nq, const double* w, const double* jac,
                           const double* phi, const double* muu, const double* guu,
                           double beta_prime, double gamma_prime, double* out);
void orc_inertial_qp(double mass_scale_unused, const double mstar[36], const double r0[4],
                     const double r[4], const double uddot[3], const double omega[3],
                     const double omegadot[3], const double gravity[3], double fi[6],
                     double fg[6], double muu[36], double guu[36], double kuu[36]);
void orc_tangent_operator(double h, const double qdelta[6], double t_stored[36]);

/* ComputeRowPtrs / ComputeColInds / sort_crs_graph restated for arbitrary
 * connectivity (tests/unit_tests/solver/test_compute_{row_ptrs,col_inds}.cpp).
 * elem_nodes: [num_elems][max_nodes] state indices; nodes_per_elem [num_elems].
 * Constraint tables: base/target active dofs, [c][6] freedom tables, row
 * ranges as [c][2].  col_inds may be NULL to only size the graph.
 * Returns nnz. */
long orc_crs_build(int num_system_dofs, int num_dofs, int num_nodes, const long* active_dofs,
                   const long* node_freedom_map_table, int num_elems, int max_nodes,
                   const long* nodes_per_elem, const long* elem_nodes, int num_constraints,
                   const long* base_active, const long* target_active,
                   const long* base_table, const long* target_table, const long* row_range,
                   long* row_ptrs, long* col_inds, int sort_rows);

#ifdef __cplusplus
}
#endif

#endif
