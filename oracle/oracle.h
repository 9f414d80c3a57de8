/*
 * oracle.h -- TEST INFRASTRUCTURE ONLY (never linked by the product).
 *
 * A plain-C restatement of micm's Rosenbrock path (NCAR/micm 3.13.0) for
 * checking the B200 kernels, plus the FP64 discrete adjoint micm does not
 * have.  Everything is restated from the reference's algorithm, with the
 * scatter loops in micm's own order:
 *   reaction sort           include/micm/solver/solver_builder.inl:274-329
 *   Markowitz reordering    include/micm/solver/linear_solver.inl:30-124
 *   Jacobian sparsity       include/micm/process/process_set.hpp:425-457, util/jacobian.hpp:15-32
 *   LU fill / Decompose     include/micm/solver/lu_decomposition_mozart_in_place.inl:121-210
 *   forcing / -J            include/micm/process/process_set.hpp:256-422, 524-670
 *   linear solve            include/micm/solver/linear_solver_in_place.inl:113-167
 *   rate constants          include/micm/process/rate_constant/rate_constant_functions.hpp:52-136
 *   Rosenbrock + control    include/micm/solver/rosenbrock.inl:12-402
 * Arrays are row-major [cell][column] in state columns.
 */
#ifndef MICMB_ORACLE_H
#define MICMB_ORACLE_H

#include "../include/micmb.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct om_mech om_mech;

om_mech* om_create(const micmb_mechanism_desc* desc);
void om_destroy(om_mech* m);
const char* om_last_error(void);
int om_n_params(const om_mech* m);
int om_nnz(const om_mech* m);
void om_species_columns(const om_mech* m, int32_t* out);
void om_reaction_columns(const om_mech* m, int32_t* out);
void om_jacobian_pattern(const om_mech* m, int32_t* rows, int32_t* cols);

/* rate constants of n cells: params [cell][P], k_out [cell][R] */
void om_rate_constants(const om_mech* m, int n, const double* T, const double* P, const double* rho,
                       const double* params, double* k_out);

/* Per-cell Rosenbrock over n cells (one independent solve per cell, n_threads
 * host threads).  y [cell][S] in/out (clamped at zero on exit); stats_out
 * [cell][10] = function_calls, jacobian_updates, number_of_steps, accepted,
 * rejected, decompositions, solves, state, (final time bits), 0. */
int om_solve_per_cell(const om_mech* m, const micmb_rosenbrock_params* p, int n, double dt, const double* k,
                      const double* atol, double rtol, double* y, int64_t* stats_out, int n_threads);

/* Discrete adjoint of the accepted steps (step sizes frozen) of a per-cell
 * solve.  Runs the forward solve from y0, then sweeps back.
 *   ybar_final [cell][S]: dL/d(final clamped y)
 *   y_final    [cell][S]: out, final clamped y
 *   ybar0      [cell][S]: out, dL/dy0
 *   kbar       [cell][R]: out, dL/d log k_r (rate columns) */
int om_adjoint_per_cell(const om_mech* m, const micmb_rosenbrock_params* p, int n, double dt, const double* k,
                        const double* atol, double rtol, const double* y0, const double* ybar_final,
                        double* y_final, double* ybar0, double* kbar, int max_steps_stored, int n_threads);

/* Fixed-step replay of given step sizes (no error control), final clamp as the
 * solve: the map whose derivative om_adjoint_per_cell computes.  For finite-
 * difference checks.  h [cell][max_steps], n_steps [cell], y [cell][S] in/out. */
int om_replay_per_cell(const om_mech* m, const micmb_rosenbrock_params* p, int n, const double* k, const double* h,
                       const int32_t* n_steps, int max_steps, double* y);
/* Accepted step sizes of a per-cell solve from y0 [cell][S]. */
/* Backward Euler (micm's backward_euler.inl, default parameters), a 1-cell
 * State per cell, one Solve(dt) each; y [cell][column] in/out, stats [cell][10]. */
/* Global step control (one step size for all n cells) with the error sum in
 * the fixed order a GPU reproduces (per cell, per 256-cell block tree, per
 * shard, shards in order).  exchange != NULL: the cells are this rank's
 * shard; exchange(shard sum, OM_EXCHANGE_SUM, user) returns the job's sum over
 * total_cells, and exchange(v, OM_EXCHANGE_MAX, user) the job's combination of
 * every rank's encoded maximum (om_max_combine in rank order: NaN when any is
 * NaN, +Inf when any is infinite, else the largest), which the constraint
 * initialisation uses.  keq [cell][n_eq] may be NULL without equilibrium
 * constraints. */
#define OM_EXCHANGE_SUM 0
#define OM_EXCHANGE_MAX 1
typedef double (*om_exchange_fn)(double value, int op, void* user);
double om_max_combine(double a, double b);
int om_solve_global(const om_mech* m, const micmb_rosenbrock_params* p, int n, double dt, const double* k,
                    const double* keq, const double* atol, double rtol, double* y, int64_t* stats_out,
                    int n_shards, const int* shard_start, om_exchange_fn exchange, void* user,
                    int64_t total_cells);
/* Algebraic constraints: K_eq(T) of every equilibrium constraint per cell
 * ([cell][n_eq], Van't Hoff with the handle's exp), and the per-cell solve
 * with those values (keq may be NULL without equilibrium constraints). */
void om_constraint_params(const om_mech* m, int n, const double* T, double* keq);
int om_n_eq(const om_mech* m);
int om_solve_per_cell_keq(const om_mech* m, const micmb_rosenbrock_params* p, int n, double dt, const double* k,
                          const double* keq, const double* atol, double rtol, double* y, int64_t* stats_out,
                          int n_threads);
/* 0 (default): exp, pow and log10 of the rate constants and the step-size
 * factor from the C library, as micm calls them; 1: correctly rounded (quad
 * precision).  om_math_eval evaluates exp (0), log10 (1) or pow (2)
 * element-wise in the handle's mode. */
void om_set_correctly_rounded(om_mech* m, int on);
void om_math_eval(const om_mech* m, int fn, const double* x, const double* y, double* out, int64_t n);
int om_backward_euler_per_cell(const om_mech* m, int n, double dt, const double* k, const double* atol, double rtol,
                               double* y, int64_t* stats_out);
/* Backward Euler on one n-cell State (one step size, one convergence test over
 * all cells), micm's multi-cell semantics; stats_out [10]. */
int om_backward_euler_global(const om_mech* m, int n, double dt, const double* k, const double* atol, double rtol,
                             double* y, int64_t* stats_out);
int om_step_sizes_per_cell(const om_mech* m, const micmb_rosenbrock_params* p, int n, double dt, const double* k,
                           const double* atol, double rtol, const double* y0, int max_steps, double* h,
                           int32_t* n_steps);

#ifdef __cplusplus
}
#endif

#endif
