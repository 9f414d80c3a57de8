// runtime.hpp -- host-side objects behind the C ABI handles.
#pragma once

#include "device.cuh"
#include "mechanism.hpp"

#include <cuda_runtime.h>

#include <memory>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

struct micmb_mechanism
{
  micmb::CompiledMechanism m;
};

namespace micmb
{
  // exception carrying a C-ABI status code
  struct Error : std::runtime_error
  {
    int code;
    Error(int c, const std::string& what)
        : std::runtime_error(what),
          code(c)
    {
    }
  };

  void CudaCheck(cudaError_t e, const char* what);
#define MICMB_CUDA(call) ::micmb::CudaCheck((call), #call)

  // owning device allocation
  struct DeviceMemory
  {
    void* p = nullptr;
    size_t bytes = 0;
    DeviceMemory() = default;
    explicit DeviceMemory(size_t b);
    ~DeviceMemory();
    DeviceMemory(const DeviceMemory&) = delete;
    DeviceMemory& operator=(const DeviceMemory&) = delete;
    DeviceMemory(DeviceMemory&& o) noexcept
        : p(o.p),
          bytes(o.bytes)
    {
      o.p = nullptr;
      o.bytes = 0;
    }
    DeviceMemory& operator=(DeviceMemory&& o) noexcept;
    template<class T>
    T* as() const
    {
      return static_cast<T*>(p);
    }
  };

  DevParams ToDevParams(const micmb_rosenbrock_params& p);

  // per-launch arguments of the fused kernel
  struct FusedArgs
  {
    int64_t n_cells;
    int32_t L;
    const double* variables_in;
    double* variables_out;
    const double* rate_constants;
    const double* atol;
    double rtol;
    const double* keq;           // [vector layout, n_eq columns] K_eq of the equilibrium constraints
    int32_t* next_cell;          // work-stealing counter
    int32_t* cell_status;        // [n_cells] or null
    int32_t* cell_accepted;      // [n_cells] or null
    unsigned long long* stats;   // [9] accumulators (the seven counters, cells not converged,
                                 // constraint-initialisation iterations)
    double* lu_global;           // per-warp LU slots when not staged in shared memory
    int64_t lu_slot_stride;      // doubles per slot
    // adjoint checkpoints (null for a plain forward solve)
    double* ckpt_y;              // [n_cells][max_ckpt][S]
    double* ckpt_h;              // [n_cells][max_ckpt]
    double* ckpt_k;              // [n_cells][max_ckpt][stages][S] stage vectors of each accepted step,
                                 // or null (one-cell-per-thread variant only)
    int32_t max_ckpt;
  };
}  // namespace micmb

struct micmb_solver
{
  std::shared_ptr<const micmb::CompiledMechanism> mech;
  int device = 0;
  int sm_count = 0;
  size_t smem_optin = 0;
  micmb::DeviceMemory tables;
  micmb::DeviceMemory scale_dev;  // [R] by rate column
  micmb::DevMech dev{};
  const int32_t* diag_row_of = nullptr;  // [nnz]: row if diagonal, else -1
  micmb_rosenbrock_params host_params{};
  micmb::DevParams params{};
  micmb_fused_config fused{ 0, 1, 0, 0, 0 };
  micmb::DeviceMemory stream_blocks;       // StreamProgram bytes
  micmb::DeviceMemory stream_block_bytes;  // [n_blocks]
  micmb::DeviceMemory stream_coef;         // StreamProgram coef_table
  int32_t n_stream_coef = 0;
  int64_t adjoint_memory_limit = 0;  // bytes of adjoint checkpoints (0 = from free device memory)
};

struct micmb_state
{
  micmb_solver* solver = nullptr;
  int64_t n_cells = 0;
  int32_t L = 1;
  int64_t n_groups = 0;
  int64_t n_pad = 0;
  cudaStream_t own_stream = nullptr;
  cudaStream_t stream = nullptr;
  double rtol = 1e-6;

  micmb::DeviceMemory variables, custom_params, rate_constants, conditions, atol;
  micmb::DeviceMemory keq;   // K_eq of the equilibrium constraints, vector layout (UpdateStateParameters)
  micmb::DeviceMemory cjac;  // plain path: constraint Jacobian terms per cell
  // plain-path working set (allocated on first use)
  micmb::DeviceMemory jacobian, forcing0, fcur, ynew, stages, scratch, inv_diag, err_cell;
  micmb::DeviceMemory ctl, status, accepted;
  micmb::DeviceMemory counters;  // device counters / stats accumulators
  int32_t* host_counters = nullptr;  // pinned
  // fused path
  micmb::DeviceMemory lu_slots;
  int64_t lu_slot_count = 0;  // doubles allocated in lu_slots
  micmb::DeviceMemory thread_ws;  // one-cell-per-thread variant: per-thread working sets
  micmb::DeviceMemory attempt_order;  // streamed kernel: block order of one attempt
  std::vector<int32_t> attempt_order_host;  // what attempt_order holds
  int64_t solve_limit = 0;                  // fused solves: only the first solve_limit cells (0 = all)
  // CUDA graph of UpdateStateParameters + fused Solve (micmb_solve_graph)
  cudaGraphExec_t graph_exec = nullptr;
  double graph_dt = 0.0;
  micmb_fused_config graph_config{};
  // adjoint working set (allocated on first use)
  micmb::DeviceMemory adj_y0, adj_ybar, adj_ckpt_y, adj_ckpt_h, adj_ckpt_k, adj_kbar_cells, adj_kbar;
  micmb::DeviceMemory be_ctl;     // Backward Euler global control block
  // global step control over several ranks (micmb_state_set_global_exchange)
  micmb_allgather_fn gx_fn = nullptr;
  void* gx_user = nullptr;
  int32_t gx_world = 1;
  int64_t gx_total_cells = 0;
  micmb::DeviceMemory gx_buf;     // [0]: this shard's sum; [1, 1 + world): the gathered sums
  micmb::DeviceMemory cinit_slots;  // global constraint initialisation: 3 words per iteration
  micmb::DeviceMemory adj_order;  // backward sweep: cells by decreasing step count, then bins
  int64_t adj_ckpt_capacity = 0;  // doubles in adj_ckpt_y
  double dt_for_launch = 0.0;

  size_t dense_bytes(int32_t ncols) const
  {
    return (size_t)n_pad * (size_t)ncols * sizeof(double);
  }
};

namespace micmb
{
  extern thread_local std::string g_last_error;  // micmb_last_error()

  // Runs an entry point's body and turns every C++ exception into a status
  // code and a micmb_last_error() message, so none crosses the C ABI
  // (kStdCode: the status of a standard-library exception).
  template<int kStdCode = MICMB_ERR_INTERNAL, class F>
  int GuardCall(F&& f) noexcept
  {
    try
    {
      f();
      g_last_error.clear();
      return MICMB_OK;
    }
    catch (const Error& e)
    {
      g_last_error = e.what();
      return e.code;
    }
    catch (const std::bad_alloc&)
    {
      g_last_error = "host allocation failed";
      return MICMB_ERR_OUT_OF_MEMORY;
    }
    catch (const std::exception& e)
    {
      g_last_error = e.what();
      return kStdCode;
    }
    catch (...)
    {
      g_last_error = "unknown error";
      return MICMB_ERR_INTERNAL;
    }
  }
  void EnsurePlainBuffers(micmb_state& st);
  // plain path: one kernel per stage; returns after the whole solve
  void SolvePlain(micmb_solver& s, micmb_state& st, double dt, int32_t step_control, micmb_solver_stats* stats,
                  int32_t* per_cell_status, int32_t* per_cell_accepted);
  void SolveFused(micmb_solver& s, micmb_state& st, double dt, micmb_solver_stats* stats, int32_t* per_cell_status,
                  int32_t* per_cell_accepted, const FusedArgs* adjoint_ckpt);
  void LaunchRateConstants(micmb_solver& s, micmb_state& st);
  // single-stage launchers (per-kernel parity entry points)
  void LaunchAddForcing(micmb_solver& s, micmb_state& st);
  void LaunchSubtractJacobian(micmb_solver& s, micmb_state& st);
  void LaunchAlphaMinusJacobian(micmb_solver& s, micmb_state& st, double alpha);
  void LaunchDecompose(micmb_solver& s, micmb_state& st);
  void LaunchLinearSolve(micmb_solver& s, micmb_state& st);
  void NormalizedError(micmb_solver& s, micmb_state& st, double* global_out, double* per_cell_out);
  size_t FusedSharedBytes(const micmb_solver& s, bool lu_in_shared);
  // streamed warp-specialised variant; returns false when it does not apply
  bool SolveFusedStream(micmb_solver& s, micmb_state& st, double dt, const FusedArgs& A);
  // whether the streamed variant runs for the solver's mechanism and configuration
  bool StreamVariantApplies(const micmb_solver& s);
  // one cell per thread, working sets in global memory
  bool SolveFusedThread(micmb_solver& s, micmb_state& st, const FusedArgs& A, double dt);
  int StreamWarpsPerCta(const micmb_solver& s, int slots, int cap, bool lu_shared);
  // discrete adjoint sweep over the checkpoints of a fused solve of cells
  // [begin, begin + count) (begin a multiple of L; checkpoints hold those cells only)
  void LaunchAdjoint(micmb_solver& s, micmb_state& st, int32_t max_ckpt, int64_t begin, int64_t count);
  // dloss/dlog k summed over all cells in a fixed order, after every chunk's sweep
  void ReduceAdjointParameters(micmb_solver& s, micmb_state& st);
  // doubles of per-thread working set the backward sweep needs for n_cells cells
  int64_t AdjointThreadWorkspaceDoubles(const micmb_solver& s, int64_t n_cells);
  // doubles of per-thread working set the one-cell-per-thread forward needs
  int64_t FusedThreadWorkspaceDoubles(const micmb_solver& s, int64_t n_cells);
  // cells the one-cell-per-thread forward keeps resident at once
  int64_t FusedThreadResidentCells(const micmb_solver& s);
  int FusedWarpsPerCta(const micmb_solver& s, const micmb_fused_config& cfg);
  // Backward Euler (global: micm's multi-cell State; per cell: one persistent kernel)
  void DefaultBackwardEulerParams(micmb_backward_euler_params* p);
  void SolveBackwardEuler(micmb_solver& s, micmb_state& st, double dt, const micmb_backward_euler_params& params,
                          int32_t step_control, micmb_solver_stats* stats, int32_t* per_cell_status,
                          int32_t* per_cell_accepted);
}  // namespace micmb
