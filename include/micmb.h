/*
 * micmb.h -- C ABI of the B200-native Rosenbrock chemistry solver.
 *
 * Plain C types only (pointers, sizes, doubles, 32/64-bit integers): this is
 * the boundary a Fortran/C/Python host or micm's own C++ layer binds to.  No
 * exceptions cross it; every call returns MICMB_OK (0) or a negative status
 * and micmb_last_error() gives the message of the last failure on the calling
 * thread.
 *
 * Each entry point names the micm (NCAR/micm 3.13.0) interface it replaces.
 * Paths are relative to the micm source tree.
 *
 * Data layout at the boundary is micm's own vector ordering with L cells per
 * group (include/micm/util/vector_matrix.hpp:254-345): element (cell c,
 * column j) of an n-column dense matrix lives at
 *     (c / L) * L * n + j * L + c % L
 * and element e of the LU-filled sparse Jacobian at
 *     (c / L) * L * nnz + e * L + c % L
 * (sparse_matrix_vector_ordering_compressed_sparse_row.hpp:79-88), with the
 * nonzeros in row-major order.  Columns of `variables` follow micm's species
 * map after Markowitz reordering, columns of `rate_constants` follow micm's
 * reaction order after the stable sort by rate-constant type, exactly as the
 * reference solver numbers them.
 */
#ifndef MICMB_H
#define MICMB_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------ */
/* status codes                                                        */
/* ------------------------------------------------------------------ */
#define MICMB_OK 0
#define MICMB_ERR_INVALID_ARGUMENT (-1)
#define MICMB_ERR_CUDA (-2)
#define MICMB_ERR_UNSUPPORTED (-3)
#define MICMB_ERR_OUT_OF_MEMORY (-4)
#define MICMB_ERR_INTERNAL (-5)
#define MICMB_ERR_NO_DEVICE (-6)
#define MICMB_ERR_TIMEOUT (-7)

/* micm::SolverState values (include/micm/solver/solver_result.hpp:13-35) */
#define MICMB_SOLVER_NOT_YET_CALLED 0
#define MICMB_SOLVER_RUNNING 1
#define MICMB_SOLVER_CONVERGED 2
#define MICMB_SOLVER_CONVERGENCE_EXCEEDED_MAX_STEPS 3
#define MICMB_SOLVER_STEP_SIZE_TOO_SMALL 4
#define MICMB_SOLVER_REPEATEDLY_SINGULAR_MATRIX 5
#define MICMB_SOLVER_NAN_DETECTED 6
#define MICMB_SOLVER_INF_DETECTED 7
#define MICMB_SOLVER_ACCEPTING_UNCONVERGED 8 /* Backward Euler: AcceptingUnconvergedIntegration */
#define MICMB_SOLVER_CONSTRAINT_INITIALIZATION_FAILED 9 /* DAE: ConstraintInitializationFailed */

/* ------------------------------------------------------------------ */
/* mechanism description                                               */
/* ------------------------------------------------------------------ */

/* Rate-constant kinds; the numeric value is micm's sort key
 * (include/micm/solver/solver_builder.inl:274-329). */
#define MICMB_RATE_ARRHENIUS 0
#define MICMB_RATE_TROE 1
#define MICMB_RATE_TERNARY_CHEMICAL_ACTIVATION 2
#define MICMB_RATE_BRANCHED 3
#define MICMB_RATE_TUNNELING 4
#define MICMB_RATE_TAYLOR_SERIES 5
#define MICMB_RATE_REVERSIBLE 6
#define MICMB_RATE_USER_DEFINED 7
#define MICMB_RATE_SURFACE 8

/* doubles per reaction in micmb_mechanism_desc::rate_params */
#define MICMB_RATE_PARAM_STRIDE 24
/* maximum parameterized reactants per reaction
 * (include/micm/process/reaction_rate_store.hpp:57-76, kMaxFuncs) */
#define MICMB_MAX_PARAMETERIZED 4

/*
 * A chemical mechanism in flat form.  Species are numbered 0..n_species-1 in
 * the order of micm's gas phase (System::UniqueNames,
 * include/micm/system/system.hpp:38-63).  Reactions are numbered
 * 0..n_reactions-1 in the order given to SolverBuilder::SetReactions.
 *
 * rate_params[r * MICMB_RATE_PARAM_STRIDE + i] by rate_type[r]:
 *   ARRHENIUS   A, B, C, D, E             (arrhenius_rate_constant.hpp:9-22)
 *   TROE        k0_A k0_B k0_C kinf_A kinf_B kinf_C Fc N (troe_rate_constant.hpp)
 *   TERNARY_CHEMICAL_ACTIVATION  same eight as TROE
 *   BRANCHED    branch(0 alkoxy, 1 nitrate), X, Y, a0, n
 *   TUNNELING   A, B, C
 *   TAYLOR_SERIES A, B, C, D, E, n_coefficients, c0 .. c15
 *   REVERSIBLE  A, C, k_r
 *   USER_DEFINED scaling_factor            (one custom rate parameter)
 *   SURFACE     diffusion_coefficient [m2 s-1], molecular_weight [kg mol-1],
 *               reaction_probability       (two custom rate parameters)
 *
 * reactant_species[i] >= 0 is a species index; a value -(p+1) names
 * parameterized reactant p whose concentration is
 *   c0 + cT*T + cP*P + crho*air_density   (parameterized_function.hpp)
 * with coefficients parameterized_coef[4p .. 4p+3].
 */
typedef struct micmb_mechanism_desc {
  int32_t n_species;
  int32_t n_reactions;
  const int32_t* rate_type;        /* [n_reactions] */
  const double* rate_params;       /* [n_reactions * MICMB_RATE_PARAM_STRIDE] */
  const int32_t* reactant_start;   /* [n_reactions + 1] */
  const int32_t* reactant_species; /* [reactant_start[n_reactions]] */
  const int32_t* product_start;    /* [n_reactions + 1] */
  const int32_t* product_species;  /* [product_start[n_reactions]] */
  const double* product_yield;     /* [product_start[n_reactions]] */
  int32_t n_parameterized;
  const double* parameterized_coef; /* [4 * n_parameterized] */
  int32_t reorder_state;            /* SolverBuilder::SetReorderState, default 1 */
  /* Algebraic constraints (DAE form; include/micm/constraint/types/
   * linear_constraint.hpp, equilibrium_constraint.hpp), as
   * SolverBuilder::SetConstraints passes them.  Each constraint replaces the
   * ODE row of its algebraic species (mass-matrix diagonal 0 there):
   *   LINEAR       G = sum_t coef_t * y[species_t] - params[0]
   *   EQUILIBRIUM  G = K_eq(T) * prod_reactants y^coef - prod_products y^coef,
   *                the first n_reactants terms are reactants,
   *                K_eq(T) = params[0] * exp((params[1] / params[2]) * (1/T - 1/params[3]))
   *                (K_HLC_ref, delta_H [J mol-1], R [J mol-1 K-1], T_ref [K]).
   * n_constraints = 0 (and null arrays) for a plain ODE mechanism. */
  int32_t n_constraints;
  const int32_t* constraint_type;         /* [n_constraints] MICMB_CONSTRAINT_* */
  const int32_t* constraint_species;      /* [n_constraints] algebraic species */
  const int32_t* constraint_term_start;   /* [n_constraints + 1] */
  const int32_t* constraint_term_species; /* [constraint_term_start[n_constraints]] */
  const double* constraint_term_coef;     /* coefficient (linear) or stoichiometry (equilibrium) */
  const int32_t* constraint_n_reactants;  /* [n_constraints] equilibrium: leading reactant terms */
  const double* constraint_params;        /* [n_constraints * 4], see above */
} micmb_mechanism_desc;

#define MICMB_CONSTRAINT_LINEAR 0
#define MICMB_CONSTRAINT_EQUILIBRIUM 1

/* Rosenbrock tableau and step control
 * (include/micm/solver/rosenbrock_solver_parameters.hpp:22-67). */
typedef struct micmb_rosenbrock_params {
  int32_t stages;
  int32_t max_number_of_steps;
  double round_off;
  double factor_min;
  double factor_max;
  double rejection_factor_decrease;
  double safety_factor;
  double h_min;
  double h_max;
  double h_start;
  int32_t new_function_evaluation[6];
  double estimator_of_local_order;
  double a[15];
  double c[15];
  double m[6];
  double e[6];
  double alpha[6];
  double gamma[6];
  /* DAE constraint initialisation (Newton on the algebraic variables at the
   * start of each Solve; rosenbrock.inl:407-576): iterations and tolerance on
   * the largest |G| */
  int32_t constraint_init_max_iterations; /* 10 */
  double constraint_init_tolerance;       /* 1e-10 */
} micmb_rosenbrock_params;

/* micm::SolverStats (include/micm/solver/solver_result.hpp:37-57), summed
 * over cells in per-cell step control. */
typedef struct micmb_solver_stats {
  int64_t function_calls;
  int64_t jacobian_updates;
  int64_t number_of_steps;
  int64_t accepted;
  int64_t rejected;
  int64_t decompositions;
  int64_t solves;
  double final_time;
  int32_t state; /* MICMB_SOLVER_*: worst over cells in per-cell mode */
  int32_t cells_not_converged;
  int64_t constraint_init_iterations; /* DAE: Newton iterations of the constraint initialisation */
} micmb_solver_stats;

typedef struct micmb_mechanism_info {
  int32_t n_species;
  int32_t n_reactions;
  int32_t n_custom_params;
  int32_t jacobian_nnz;       /* LU-filled nonzeros per cell */
  int32_t jacobian_nnz_unfilled;
  int32_t lu_updates;         /* a_jk -= a_ji * a_ik terms per factorisation */
  int32_t lu_lower;           /* multipliers a_ji per factorisation */
  int32_t n_jacobian_terms;   /* product/reactant contributions to -J */
  int32_t n_forcing_terms;
  int32_t n_jacobian_infos;   /* (independent species, process) pairs */
  int32_t lu_levels;
  int32_t forward_levels;
  int32_t backward_levels;
  int32_t blocked_schedules;  /* 1: the register-blocked LU and solves are in use (they
                                 reproduced the serial schedules bit for bit when built) */
  int32_t lu_blocked_ops;     /* shared-operand steps of the blocked LU */
} micmb_mechanism_info;

typedef struct micmb_mechanism micmb_mechanism;
typedef struct micmb_solver micmb_solver;
typedef struct micmb_state micmb_state;

/* Message of the last failed call on this thread ("" if none). */
const char* micmb_last_error(void);

/* Symbolic compile of a mechanism: reaction sort by rate type, Markowitz
 * species order, Jacobian sparsity with diagonal, LU fill and the level
 * schedules of every kernel.  Host only, needs no GPU.
 * Replaces SolverBuilder::Build (include/micm/solver/solver_builder.inl:227-548),
 * DiagonalMarkowitzReorder (include/micm/solver/linear_solver.inl:30-124),
 * ProcessSet ctor (include/micm/process/process_set.hpp:256-422),
 * LuDecompositionMozartInPlace::Initialize/GetLUMatrix
 * (include/micm/solver/lu_decomposition_mozart_in_place.inl:60-169). */
int micmb_mechanism_create(const micmb_mechanism_desc* desc, micmb_mechanism** out);
void micmb_mechanism_destroy(micmb_mechanism* mech);
int micmb_mechanism_get_info(const micmb_mechanism* mech, micmb_mechanism_info* out);
/* column of each system species in `variables` (micm State::variable_map_) */
int micmb_mechanism_species_columns(const micmb_mechanism* mech, int32_t* out /*[n_species]*/);
/* column of each input reaction in `rate_constants` */
int micmb_mechanism_reaction_columns(const micmb_mechanism* mech, int32_t* out /*[n_reactions]*/);
/* first custom-parameter column of each input reaction, -1 if it has none
 * (SolverBuilder::GetCustomParameterMap, solver_builder.inl:129-188) */
int micmb_mechanism_custom_param_columns(const micmb_mechanism* mech, int32_t* out /*[n_reactions]*/);
/* LU-filled sparsity in storage order (row-major), in state columns */
int micmb_mechanism_jacobian_pattern(const micmb_mechanism* mech, int32_t* rows, int32_t* cols);
/* the unfilled Jacobian sparsity (ProcessSet::NonZeroJacobianElements + diagonal) */
int micmb_mechanism_jacobian_pattern_unfilled(const micmb_mechanism* mech, int32_t* rows, int32_t* cols);
/* Shape of the fused kernel's streamed schedule, per phase (forcing, -J,
 * LU, forward, backward, forward-transposed, backward-transposed):
 * out[p*4 + 0] blocks, [1] segments, [2] lane steps (sum of segment lengths),
 * [3] terms (nonzero work).  Returns MICMB_ERR_UNSUPPORTED when the
 * mechanism has no streamed schedule. */
int micmb_mechanism_stream_stats(const micmb_mechanism* mech, int64_t* out /*[28]*/);
/* 64-bit FNV-1a hash of the compiled tables (autotuner cache key) */
uint64_t micmb_mechanism_hash(const micmb_mechanism* mech);

/* Rosenbrock tableaus, identical to RosenbrockSolverParameters::*Parameters()
 * (rosenbrock_solver_parameters.hpp:152-434): stages 2, 3, 4 (L-stable
 * order 4), 40 (4-stage DAE variant), 60 (6-stage DAE variant). */
int micmb_rosenbrock_params_default(int32_t kind, micmb_rosenbrock_params* out);

/* Device: the solver uploads the mechanism tables to the current CUDA device.
 * Replaces CudaProcessSet::InitDevStruct / CopyConstData
 * (include/micm/cuda/process/cuda_process_set.hpp:141-157, src/process/process_set.cu:154-227),
 * CudaLuDecompositionMozartInPlace and CudaLinearSolverInPlace ctors
 * (include/micm/cuda/solver/cuda_lu_decomposition_mozart_in_place.hpp:12-96,
 *  include/micm/cuda/solver/cuda_linear_solver_in_place.hpp:51-84). */
int micmb_solver_create(const micmb_mechanism* mech, const micmb_rosenbrock_params* params,
                        micmb_solver** out);
void micmb_solver_destroy(micmb_solver* solver);
int micmb_solver_set_params(micmb_solver* solver, const micmb_rosenbrock_params* params);
/* per-reaction multiplicative scale of the rate constant, in input reaction
 * order (1.0 = as given).  d(log k)/d(log scale) = 1, so gradients reported
 * by micmb_solve_adjoint are also d loss / d log(scale). */
int micmb_solver_set_rate_scale(micmb_solver* solver, const double* scale /*[n_reactions]*/);

/* Device state for n_cells grid cells with vector length L.
 * Replaces Solver::GetState / CudaState ctor
 * (include/micm/solver/solver.hpp:174-195, include/micm/cuda/solver/cuda_state.hpp:40-78). */
int micmb_state_create(micmb_solver* solver, int64_t n_cells, int32_t vector_length,
                       micmb_state** out);
void micmb_state_destroy(micmb_state* state);
/* run this state's work on `stream` (a cudaStream_t); NULL restores the
 * state's own stream. */
int micmb_state_set_stream(micmb_state* state, void* stream);
int micmb_state_synchronize(micmb_state* state);

/* Host <-> device copies, all in micm's vector layout of the state's L.
 * variables: CudaState::SyncInputsToDevice / SyncOutputsToHost
 * (include/micm/cuda/solver/cuda_state.hpp:132-148). */
#define MICMB_BUF_VARIABLES 0
#define MICMB_BUF_CUSTOM_PARAMS 1
#define MICMB_BUF_RATE_CONSTANTS 2
#define MICMB_BUF_JACOBIAN 3
#define MICMB_BUF_CONDITIONS 4 /* 3 columns: temperature, pressure, air density */
#define MICMB_BUF_ABSOLUTE_TOLERANCE 5 /* [n_species], one per column */
#define MICMB_BUF_FORCING 6    /* initial forcing scratch, n_species columns */
#define MICMB_BUF_SCRATCH_Y 7  /* Ynew scratch, n_species columns */
int micmb_state_upload(micmb_state* state, int32_t buffer, const double* host);
int micmb_state_download(micmb_state* state, int32_t buffer, double* host);
/* device pointer and element count of a state buffer (zero-copy interop) */
int micmb_state_device_buffer(micmb_state* state, int32_t buffer, double** ptr, int64_t* count);
int micmb_state_set_relative_tolerance(micmb_state* state, double rtol);

/* Rate constants on the GPU from conditions and custom parameters.
 * Replaces Solver::UpdateStateParameters -> CudaProcessSet::GpuCalculateRateConstants
 * (include/micm/solver/solver.hpp:217-247, include/micm/cuda/process/cuda_process_set.hpp:88-114,
 *  src/process/cuda_rate_constant_kernel.cu:97-170). */
int micmb_update_state_parameters(micmb_solver* solver, micmb_state* state);

/* Step control: one step size for all cells (micm's own semantics,
 * rosenbrock.inl:353-402) or an independent adaptive solve per cell. */
#define MICMB_STEP_GLOBAL 0
#define MICMB_STEP_PER_CELL 1
/* Methods: one kernel per stage over all cells, or one persistent kernel. */
#define MICMB_METHOD_PLAIN 0
#define MICMB_METHOD_FUSED 1

/* Solve(time_step, state): advance every cell by dt and clamp at zero.
 * Replaces Solver::Solve -> AbstractRosenbrockSolver::Solve and
 * Solver::PostSolveClamp (include/micm/solver/solver.hpp:133-142, 275-297,
 * include/micm/solver/rosenbrock.inl:12-304).  per_cell_status (device
 * results copied to host, may be NULL) receives MICMB_SOLVER_* per cell and
 * per_cell_steps the accepted-step count per cell.  With algebraic
 * constraints every solve starts with micm's constraint initialisation
 * (rosenbrock.inl:407-576; over all cells of the state together under
 * MICMB_STEP_GLOBAL, per cell under MICMB_STEP_PER_CELL), and the clamp
 * leaves the algebraic variables as solved; the fused method takes them with
 * per-cell step control. */
int micmb_solve(micmb_solver* solver, micmb_state* state, double dt, int32_t method,
                int32_t step_control, micmb_solver_stats* stats, int32_t* per_cell_status,
                int32_t* per_cell_accepted);

/* Fused-kernel launch configuration (autotuner knobs). */
typedef struct micmb_fused_config {
  int32_t cells_per_cta;   /* consumer warps (one cell each) per CTA, 0..12, 0 = as many as fit */
  int32_t lu_in_shared;    /* 1 LU factor in shared memory, 0 in a per-warp global (L2) slot */
  int32_t ctas_per_sm;     /* persistent grid = ctas_per_sm * SM count (0 = occupancy); variant 2
                              also picks its kernel build by it: 1..5 the 96-register kernel,
                              6..8 the 64-register one, 9..12 the 40-register one, 0 or above 12
                              the 32-register one (every warp slot of the SM) */
  int32_t ring_slots;      /* streamed variant: shared-memory slots for table blocks (0 = 4) */
  int32_t variant;         /* 0 streamed (TMA-fed, warp-specialised), 1 direct (warp per cell),
                              2 one cell per thread (working sets in global memory) */
} micmb_fused_config;
int micmb_solver_set_fused_config(micmb_solver* solver, const micmb_fused_config* config);
int micmb_solver_get_fused_config(micmb_solver* solver, micmb_fused_config* config);
/* Time candidate fused configurations on this state (its current inputs are
 * preserved) and keep the fastest; the choice is cached in `cache_path`
 * (may be NULL) under the mechanism hash. */
int micmb_autotune(micmb_solver* solver, micmb_state* state, double dt, const char* cache_path,
                   micmb_fused_config* chosen);

/* CUDA-graph replay of repeated Solve calls with the fused method: captures
 * UpdateStateParameters + Solve once per (state, dt) and replays it. */
int micmb_solve_graph(micmb_solver* solver, micmb_state* state, double dt, int32_t n_repeats);

/* Discrete adjoint of the accepted Rosenbrock steps of one per-cell solve
 * (no counterpart in micm).  Runs the forward solve from the current
 * variables, checkpoints every accepted step, then sweeps back.
 *   dloss_dy_final: [vector layout, n_species columns] dL/d(final clamped y)
 *   dloss_dy0:      [vector layout] dL/d(initial y), may be NULL
 *   dloss_dlogk:    [n_reactions, input order] sum over cells of dL/d log k_r,
 *                   may be NULL
 * Buffers are host pointers.  The state's variables hold the final values
 * afterwards, as after micmb_solve.  max_checkpoints bounds accepted steps
 * per cell (cells beyond it report MICMB_SOLVER_CONVERGENCE_EXCEEDED_MAX_STEPS).
 * Checkpoints take max_checkpoints * (n_species + 1) doubles per cell, plus
 * max_checkpoints * stages * n_species when the accepted steps' stage vectors
 * are kept.  Cells are solved and swept in chunks (multiples of the vector
 * length) that fit the solver's adjoint memory limit; stage vectors are kept
 * unless that would make a chunk smaller than the cells the forward kernel
 * keeps resident, in which case the sweep recomputes them.  Results do not
 * depend on the chunking. */
int micmb_solve_adjoint(micmb_solver* solver, micmb_state* state, double dt,
                        const double* dloss_dy_final, double* dloss_dy0, double* dloss_dlogk,
                        int32_t max_checkpoints, micmb_solver_stats* stats);
/* Device bytes micmb_solve_adjoint may hold in checkpoints (0, the default:
 * 80 % of the device memory free at the call, counting checkpoints it already
 * holds).  A limit below one vector-length group of cells makes
 * micmb_solve_adjoint return MICMB_ERR_OUT_OF_MEMORY. */
int micmb_set_adjoint_memory_limit(micmb_solver* solver, int64_t bytes);

/* ---- single-stage entry points (per-kernel parity with micm's drivers) ---- */
/* ProcessSet::AddForcingTerms (process_set.hpp:524-590; src/process/process_set.cu:10-74):
 * forcing += f(y) with y = state variables; forcing is MICMB_BUF_FORCING */
int micmb_add_forcing_terms(micmb_solver* solver, micmb_state* state);
/* ProcessSet::SubtractJacobianTerms (process_set.hpp:594-670; process_set.cu:77-149):
 * jacobian -= J(y) into MICMB_BUF_JACOBIAN (add to existing values) */
int micmb_subtract_jacobian_terms(micmb_solver* solver, micmb_state* state);
/* AlphaMinusJacobian (rosenbrock.inl:308-326; src/solver/rosenbrock.cu:37-68) */
int micmb_alpha_minus_jacobian(micmb_solver* solver, micmb_state* state, double alpha);
/* LuDecompositionMozartInPlace::Decompose (lu_decomposition_mozart_in_place.inl:171-210) */
int micmb_lu_decompose(micmb_solver* solver, micmb_state* state);
/* LinearSolverInPlace::Solve (linear_solver_in_place.inl:113-167): x = (LU)^-1 b,
 * b and x in MICMB_BUF_FORCING */
int micmb_linear_solve(micmb_solver* solver, micmb_state* state);
/* NormalizedError (rosenbrock.inl:353-402): y = variables, ynew = MICMB_BUF_SCRATCH_Y,
 * errors = MICMB_BUF_FORCING; global (all cells) or per cell into per_cell_out */
int micmb_normalized_error(micmb_solver* solver, micmb_state* state, double* global_out,
                           double* per_cell_out);

/* The global value of micmb_normalized_error, computed without allocating
 * (no counterpart in micm).  For callers that cannot call cudaMalloc while they
 * run: a host model that has handed the device's memory to its own pool
 * allocator up front, or one whose error-control loop runs where a device
 * allocation would stall or fail (an allocation synchronises the device and
 * can fail once the device is full).  Scratch is a fixed file-scope device
 * array for at most 65536 cells (512 KB, held on every device that loads the
 * library until the process exits); larger states return
 * MICMB_ERR_INVALID_ARGUMENT.  The buffers read (variables,
 * MICMB_BUF_SCRATCH_Y, MICMB_BUF_FORCING, absolute tolerances) must already
 * exist: upload them first.  Nothing in the scratch needs to start at zero:
 * every slot a call reads, the same call wrote first.  The first call on a
 * device looks up the scratch address (cudaGetSymbolAddress) and keeps it;
 * make that first call before any stream capture, and make no call after a
 * cudaDeviceReset in the same process (the kept address is then stale).
 * There is one scratch area per device: calls that overlap on the same device
 * (different streams or host threads) race on it, so serialise them. */
int micmb_normalized_error_noalloc(micmb_solver* solver, micmb_state* state, double* global_out);

/* ---- global step control over several GPUs (one process per GPU) ---- */
/* All-gather of one double per rank: recv[r] = rank r's send[0], in rank
 * order (device pointers), queued on `stream` (a cudaStream_t) after the work
 * already queued there.  Called on the host once per step attempt while a
 * solve queues its kernels; it must not wait for the stream.  Returns 0 on
 * success. */
typedef int (*micmb_allgather_fn)(const double* send, double* recv, int32_t world, void* stream, void* user);
/* Makes MICMB_STEP_GLOBAL plain solves of this state one shard of a job over
 * `world` ranks: per step attempt the shard's sum of scaled squared errors
 * goes through `fn`, every rank adds the gathered sums in rank order and
 * divides by total_cells * n_species, so every rank takes the same step-size
 * decisions -- micm's global NormalizedError (include/micm/solver/
 * rosenbrock.inl:353-402) over the whole job, one 8-byte exchange per
 * attempt.  Every rank must call micmb_solve the same number of times with
 * the same dt.  fn = NULL restores the single-GPU solve. */
int micmb_state_set_global_exchange(micmb_state* state, micmb_allgather_fn fn, void* user, int32_t world,
                                    int64_t total_cells);

/* ---- Backward Euler (micm's second integrator) ---- */
/* micm::BackwardEulerSolverParameters
 * (include/micm/solver/backward_euler_solver_parameters.hpp:17-29). */
typedef struct micmb_backward_euler_params {
  double small;                    /* residuals below this count as converged (1e-40) */
  double h_start;                  /* first step size; 0 = the whole time step */
  int32_t max_number_of_steps;     /* Newton iterations per attempt (11) */
  int32_t n_time_step_reductions;  /* entries of time_step_reductions in use (5, at most 8) */
  double time_step_reductions[8];  /* H factor after the k-th failed attempt ({0.5, 0.5, 0.5, 0.5, 0.1}) */
} micmb_backward_euler_params;
/* micm's defaults (the CAM-Chem set). */
int micmb_backward_euler_params_default(micmb_backward_euler_params* out);
/* Backward Euler Solve(time_step, state) over every cell, then the clamp at
 * zero; replaces AbstractBackwardEuler::Solve
 * (include/micm/solver/backward_euler.inl:10-186, IsConverged :188-246) and
 * Solver::PostSolveClamp.  params may be NULL (micm's defaults).
 * step_control MICMB_STEP_GLOBAL follows micm's multi-cell State exactly: one
 * step size and one convergence test over all cells (device-side control, one
 * launch group per Newton iteration).  MICMB_STEP_PER_CELL solves each cell as
 * micm solves a 1-cell State (one persistent kernel, one cell per thread,
 * cells taken from an atomic queue).  stats are summed over cells (global:
 * the single control's); per_cell_status / per_cell_accepted as micmb_solve. */
int micmb_solve_backward_euler(micmb_solver* solver, micmb_state* state, double dt,
                               const micmb_backward_euler_params* params, int32_t step_control,
                               micmb_solver_stats* stats, int32_t* per_cell_status,
                               int32_t* per_cell_accepted);

/* ---- math check ---- */
#define MICMB_MATH_EXP 0
#define MICMB_MATH_LOG10 1
#define MICMB_MATH_POW 2
/* The correctly rounded exp, log10 and pow every kernel uses in place of the C
 * library calls micm makes (std::exp / std::pow / std::log10 in
 * include/micm/process/rate_constant/rate_constant_functions.hpp:52-136, and
 * the step-size factor std::pow(error, 1 / order) in
 * include/micm/solver/rosenbrock.inl:232-235), evaluated element-wise:
 * out[i] = f(x[i]) or pow(x[i], y[i]).  on_device = 0 runs the host build of
 * the same code on host arrays; 1 runs it in a kernel on device arrays (the
 * current device, default stream, synchronised).  A diagnostic: it lets a
 * caller check the device results against the host's bit for bit. */
int micmb_math_eval(int32_t function, const double* x, const double* y, double* out, int64_t n,
                    int32_t on_device);

#ifdef __cplusplus
}
#endif

#endif /* MICMB_H */
