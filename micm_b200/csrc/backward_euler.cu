// backward_euler.cu -- micm's second integrator on the GPU: Backward Euler
// with Newton iterations (include/micm/solver/backward_euler.inl:10-186,
// IsConverged :188-246), built on the same forcing, -J, LU and triangular
// solve routines as the Rosenbrock kernels.
//
// Each Newton iteration at y_{n+1}: f = f(y), J = -J(y) + (1/H) I, LU in
// place, r = f - (y - y_n) / H, solve (LU) d = r, y = max(0, y + d); from the
// second iteration on, the attempt converges when every |d_i| is below small,
// atol_i or rtol |y_i|.  An attempt that fails max_number_of_steps iterations
// is retried from y_n with H scaled by the next time-step reduction; when the
// reductions are used up micm accepts the unconverged step and stops.  Two
// accepted attempts in a row double H.
//
// Two forms:
//   * per cell (k_backward_euler_thread): one persistent kernel, one cell per
//     thread, each cell solved as micm solves a 1-cell State; a warp runs its
//     cells' Newton iterations in lockstep and a thread whose cell finishes
//     takes the next cell from an atomic counter.  Working sets live in global
//     memory, warp-interleaved (entry e of lane l at e * 32 + l).
//   * global (k_be_iterate / k_be_control / k_be_apply): micm's multi-cell
//     State, one step size and one convergence test for all cells.  One
//     thread per cell does the Newton iteration; a one-thread control kernel
//     takes micm's decisions on the device, so the host only checks for the
//     end of the solve between batches of iterations.  The convergence test is
//     a logical AND over all cells and species, so the result is independent
//     of the cell count's grouping: bit for bit micm's.
#include "runtime.hpp"

#include <algorithm>
#include <cmath>

namespace micmb
{
  namespace
  {
    constexpr int kBlock = 256;
    constexpr int kThreadsPerBlock = 128;

    __device__ __forceinline__ size_t cell_base(int64_t c, int32_t L, int32_t ncol)
    {
      return (size_t)(c / L) * (size_t)L * (size_t)ncol + (size_t)(c % L);
    }

    inline unsigned Blocks(int64_t n, int block = kBlock)
    {
      return (unsigned)std::max<int64_t>(1, (n + block - 1) / block);
    }

    struct BeParams
    {
      double small, h_start;
      int32_t max_iter, n_red;
      double red[8];
    };

    BeParams ToDevice(const micmb_backward_euler_params& p)
    {
      BeParams b{};
      b.small = p.small;
      b.h_start = p.h_start;
      b.max_iter = p.max_number_of_steps;
      b.n_red = p.n_time_step_reductions;
      for (int i = 0; i < 8; ++i)
        b.red[i] = p.time_step_reductions[i];
      return b;
    }

    // One Newton iteration of one cell: y <- max(0, y + (LU)^-1 (f(y) - (y - yn)/H)).
    // Leaves the correction d in F.  Same routines as the Rosenbrock kernels.
    template<class YV, class NV, class FV, class LV, class IV, class KV, class SV>
    __device__ __forceinline__ void newton_iteration(const DevMech& M, double H, YV Y, NV Yn, FV F, LV LU, IV inv,
                                                     KV kk, SV scr)
    {
      const int32_t S = M.S;
      reaction_rates<1>(M, kk, Y, scr, 0);
      forcing_gather<1>(M, scr, F, 0);
      jacobian_rates<1>(M, kk, Y, scr, 0);
      // J = -J(y) in micm's term order, then + 1/H on the diagonal (AddToDiagonal), then the LU
      thread_lu_gathered(M, scr, 1.0 / H, LU, inv);
      for (int32_t i = 0; i < S; ++i)
        F[i] = F[i] - (Y[i] - Yn[i]) / H;
      thread_solve(M, LU, F);
      for (int32_t i = 0; i < S; ++i)
      {
        const double v = Y[i] + F[i];
        Y[i] = (0.0 > v) ? 0.0 : v;
      }
    }

    // IsConverged for one cell (backward_euler.inl:188-246)
    template<class FV, class YV>
    __device__ __forceinline__ bool cell_converged(const DevMech& M, const BeParams& P, const double* atol,
                                                   double rtol, FV F, YV Y)
    {
      bool ok = true;
      for (int32_t i = 0; i < M.S; ++i)
      {
        const double r = F[i];
        if (!isfinite(r))
          ok = false;
        else if (fabs(r) > P.small && fabs(r) > atol[i] && fabs(r) > rtol * fabs(Y[i]))
          ok = false;
      }
      return ok;
    }

    // ------------------------------------------------------------------
    // per cell: persistent kernel, one cell per thread
    // ------------------------------------------------------------------
    struct BeLayout
    {
      int32_t oY, oYn, oF, oLU, oInv, oKk, oScr, per_slot;
    };

    BeLayout MakeBeLayout(int32_t S, int32_t R, int32_t n_info, int32_t nnz)
    {
      BeLayout t;
      int32_t o = 0;
      t.oY = o;
      o += S;
      t.oYn = o;
      o += S;
      t.oF = o;
      o += S;
      t.oLU = o;
      o += nnz;
      t.oInv = o;
      o += S;
      t.oKk = o;
      o += R;
      t.oScr = o;
      o += (R > n_info ? R : n_info);
      t.per_slot = o;
      return t;
    }

    struct BeCell
    {
      double H, t;
      int32_t n_ok, n_fail, iterations, state;
      int32_t st[7];  // function_calls, jacobian_updates, number_of_steps, accepted, rejected, decompositions, solves
    };

    __global__ void __launch_bounds__(kThreadsPerBlock, 8)
        k_backward_euler_thread(DevMech M, BeParams P, double dt, FusedArgs A, double* ws, BeLayout T)
    {
      const int lane = threadIdx.x & 31;
      const int64_t wslot = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
      double* w = ws + (size_t)wslot * (size_t)T.per_slot * 32 + lane;
      const int32_t S = M.S, R = M.R, L = A.L;
      Strided Y{ w + (size_t)T.oY * 32, 32 };
      Strided Yn{ w + (size_t)T.oYn * 32, 32 };
      Strided F{ w + (size_t)T.oF * 32, 32 };
      Strided LU{ w + (size_t)T.oLU * 32, 32 };
      Strided inv{ w + (size_t)T.oInv * 32, 32 };
      Strided kk{ w + (size_t)T.oKk * 32, 32 };
      Strided scr{ w + (size_t)T.oScr * 32, 32 };

      __shared__ unsigned long long block_stats[8];
      if (threadIdx.x < 8)
        block_stats[threadIdx.x] = 0;
      __syncthreads();
      BeCell c{};
      int64_t cell = 0;
      bool have = false;

      auto write_out = [&]() {
        const size_t by = cell_base(cell, L, S);
        for (int32_t i = 0; i < S; ++i)
        {
          const double v = Y[i];
          A.variables_out[by + (size_t)i * L] = (v < 0.0) ? 0.0 : v;
        }
        if (A.cell_status)
          A.cell_status[cell] = c.state;
        if (A.cell_accepted)
          A.cell_accepted[cell] = c.st[3];
        for (int q = 0; q < 7; ++q)
          atomicAdd(block_stats + q, (unsigned long long)c.st[q]);
        if (c.state != MICMB_SOLVER_CONVERGED)
          atomicAdd(block_stats + 7, 1ull);
      };
      // take the next cell; returns with `have` false when none are left
      auto claim = [&]() {
        cell = atomicAdd(A.next_cell, 1);
        if (cell >= A.n_cells)
        {
          have = false;
          return;
        }
        const size_t by = cell_base(cell, L, S);
        const size_t bk = cell_base(cell, L, R);
        for (int32_t i = 0; i < S; ++i)
        {
          const double v = A.variables_in[by + (size_t)i * L];
          Y[i] = v;
          Yn[i] = v;
        }
        for (int32_t r = 0; r < R; ++r)
          kk[r] = A.rate_constants[bk + (size_t)r * L];
        c = BeCell{};
        c.H = P.h_start == 0.0 ? dt : P.h_start;
        c.state = MICMB_SOLVER_RUNNING;
        have = true;
      };

      claim();
      while (__any_sync(0xffffffffu, have))
      {
        if (!have)
          continue;
        c.st[2] += 1;  // number_of_steps
        newton_iteration(M, c.H, Y, Yn, F, LU, inv, kk, scr);
        c.st[0] += 1;  // function_calls
        c.st[1] += 1;  // jacobian_updates
        c.st[5] += 1;  // decompositions
        c.st[6] += 1;  // solves
        const bool converged = (c.iterations++ != 0) && cell_converged(M, P, A.atol, A.rtol, F, Y);
        if (!converged && c.iterations < P.max_iter)
          continue;
        bool done = false;
        if (!converged)
        {
          c.st[4] += 1;
          c.n_ok = 0;
          if (c.n_fail >= P.n_red)
          {
            c.t = c.t + c.H;
            bool any_nan = false, any_inf = false;
            for (int32_t i = 0; i < S; ++i)
            {
              any_nan = any_nan || isnan(Y[i]);
              any_inf = any_inf || isinf(Y[i]);
            }
            c.state = any_nan ? MICMB_SOLVER_NAN_DETECTED
                              : (any_inf ? MICMB_SOLVER_INF_DETECTED : MICMB_SOLVER_ACCEPTING_UNCONVERGED);
            done = true;
          }
          else
          {
            for (int32_t i = 0; i < S; ++i)
              Y[i] = Yn[i];
            c.H = c.H * P.red[c.n_fail++];
          }
        }
        else
        {
          c.st[3] += 1;
          c.state = MICMB_SOLVER_CONVERGED;
          c.t = c.t + c.H;
          for (int32_t i = 0; i < S; ++i)
            Yn[i] = Y[i];
          if (++c.n_ok >= 2)
          {
            c.n_ok = 0;
            c.H = c.H * 2.0;
          }
        }
        if (!done)
        {
          const double rem = dt - c.t;
          c.H = (rem < c.H) ? rem : c.H;  // std::min(H, time_step - present_time)
          c.iterations = 0;
          if (c.t < dt)
            c.state = MICMB_SOLVER_RUNNING;
          else
            done = true;
        }
        if (done)
        {
          write_out();
          claim();
        }
      }
      __syncthreads();
      if (threadIdx.x < 8 && block_stats[threadIdx.x])
        atomicAdd(A.stats + threadIdx.x, block_stats[threadIdx.x]);
    }

    // ------------------------------------------------------------------
    // global: one step size and one convergence test for all cells
    // ------------------------------------------------------------------
    struct BeCtl
    {
      double H, t;
      int32_t n_ok, n_fail, iterations, state;
      int32_t phase;          // 0 iterating, 1 done
      int32_t action;         // for k_be_apply: 0 none, 1 yn <- y (accepted), 2 y <- yn (rejected)
      int32_t not_converged;  // set by any cell in this iteration's test
      int32_t any_nan, any_inf;
      int32_t pad;
      long long st[7];
    };

    struct BeArgs
    {
      int64_t n;
      int32_t L, scratch_cols;
      double* y;
      double* yn;
      double* f;
      double* jac;
      double* inv;
      double* scratch;
      const double* k;
      const double* atol;
      double rtol;
      BeCtl* ctl;
    };

    __global__ void k_be_init(BeCtl* ctl, BeParams P, double dt)
    {
      BeCtl c{};
      c.H = P.h_start == 0.0 ? dt : P.h_start;
      c.state = MICMB_SOLVER_RUNNING;
      c.phase = (0.0 < dt) ? 0 : 1;
      c.action = 1;  // yn <- y before the first iteration
      *ctl = c;
    }

    __global__ void k_be_iterate(DevMech M, BeParams P, BeArgs a)
    {
      const int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
      const BeCtl* ctl = a.ctl;
      if (c >= a.n || ctl->phase != 0)
        return;
      const int32_t L = a.L, S = M.S;
      const double H = ctl->H;
      const bool check = ctl->iterations != 0;
      Strided Y{ a.y + cell_base(c, L, S), L };
      Strided Yn{ a.yn + cell_base(c, L, S), L };
      Strided F{ a.f + cell_base(c, L, S), L };
      Strided J{ a.jac + cell_base(c, L, M.nnz), L };
      Strided inv{ a.inv + cell_base(c, L, S), L };
      Strided k{ const_cast<double*>(a.k) + cell_base(c, L, M.R), L };
      Strided scr{ a.scratch + cell_base(c, L, a.scratch_cols), L };
      newton_iteration(M, H, Y, Yn, F, J, inv, k, scr);
      bool any_nan = false, any_inf = false;
      for (int32_t i = 0; i < S; ++i)
      {
        any_nan = any_nan || isnan(Y[i]);
        any_inf = any_inf || isinf(Y[i]);
      }
      BeCtl* w = a.ctl;
      if (check && !cell_converged(M, P, a.atol, a.rtol, F, Y))
        atomicOr(&w->not_converged, 1);
      if (any_nan)
        atomicOr(&w->any_nan, 1);
      if (any_inf)
        atomicOr(&w->any_inf, 1);
    }

    // micm's decisions after one Newton iteration (backward_euler.inl:55-179)
    __global__ void k_be_control(BeParams P, double dt, BeCtl* ctl)
    {
      BeCtl c = *ctl;
      if (c.phase != 0)
      {
        ctl->action = 0;
        return;
      }
      c.st[2] += 1;
      c.st[0] += 1;
      c.st[1] += 1;
      c.st[5] += 1;
      c.st[6] += 1;
      const bool converged = (c.iterations++ != 0) && !c.not_converged;
      c.action = 0;
      if (converged || c.iterations >= P.max_iter)
      {
        bool done = false;
        if (!converged)
        {
          c.st[4] += 1;
          c.n_ok = 0;
          if (c.n_fail >= P.n_red)
          {
            c.t = c.t + c.H;
            c.state = c.any_nan ? MICMB_SOLVER_NAN_DETECTED
                                : (c.any_inf ? MICMB_SOLVER_INF_DETECTED : MICMB_SOLVER_ACCEPTING_UNCONVERGED);
            done = true;
          }
          else
          {
            c.action = 2;
            c.H = c.H * P.red[c.n_fail++];
          }
        }
        else
        {
          c.st[3] += 1;
          c.state = MICMB_SOLVER_CONVERGED;
          c.t = c.t + c.H;
          c.action = 1;
          if (++c.n_ok >= 2)
          {
            c.n_ok = 0;
            c.H = c.H * 2.0;
          }
        }
        if (!done)
        {
          const double rem = dt - c.t;
          c.H = (rem < c.H) ? rem : c.H;
          c.iterations = 0;
          if (c.t < dt)
            c.state = MICMB_SOLVER_RUNNING;
          else
            done = true;
        }
        if (done)
          c.phase = 1;
      }
      c.not_converged = 0;
      c.any_nan = 0;
      c.any_inf = 0;
      *ctl = c;
    }

    __global__ void k_be_apply(BeArgs a, int32_t S)
    {
      const int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
      const int32_t action = a.ctl->action;
      if (action == 0 || idx >= a.n * (int64_t)S)
        return;
      const int64_t c = idx / S;
      const int32_t i = (int32_t)(idx - c * S);
      const size_t p = cell_base(c, a.L, S) + (size_t)i * a.L;
      if (action == 1)
        a.yn[p] = a.y[p];
      else
        a.y[p] = a.yn[p];
    }

    __global__ void k_be_clamp(double* y, int64_t n, int32_t L, int32_t S)
    {
      const int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
      if (idx >= n * (int64_t)S)
        return;
      const int64_t c = idx / S;
      const int32_t i = (int32_t)(idx - c * S);
      const size_t p = cell_base(c, L, S) + (size_t)i * L;
      const double v = y[p];
      y[p] = (v < 0.0) ? 0.0 : v;
    }

    __global__ void k_be_fill_per_cell(const BeCtl* ctl, int64_t n, int32_t* status, int32_t* accepted)
    {
      const int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
      if (c >= n)
        return;
      status[c] = ctl->state;
      accepted[c] = (int32_t)ctl->st[3];
    }

    void FillStats(micmb_solver_stats* stats, const unsigned long long* hs, int32_t worst, int32_t not_conv,
                   double final_time)
    {
      stats->function_calls = (int64_t)hs[0];
      stats->jacobian_updates = (int64_t)hs[1];
      stats->number_of_steps = (int64_t)hs[2];
      stats->accepted = (int64_t)hs[3];
      stats->rejected = (int64_t)hs[4];
      stats->decompositions = (int64_t)hs[5];
      stats->solves = (int64_t)hs[6];
      stats->cells_not_converged = not_conv;
      stats->final_time = final_time;
      stats->state = worst;
    }

    void SolveBackwardEulerGlobal(micmb_solver& s, micmb_state& st, double dt, const BeParams& P,
                                  micmb_solver_stats* stats, int32_t* per_cell_status, int32_t* per_cell_accepted)
    {
      EnsurePlainBuffers(st);
      const auto& m = *s.mech;
      const int64_t n = st.n_cells;
      if (!st.be_ctl.p)
        st.be_ctl = DeviceMemory(sizeof(BeCtl));
      BeArgs a{};
      a.n = n;
      a.L = st.L;
      a.scratch_cols = std::max<int32_t>(m.R, (int32_t)m.info_rxn.size());
      a.y = st.variables.as<double>();
      a.yn = st.ynew.as<double>();
      a.f = st.forcing0.as<double>();
      a.jac = st.jacobian.as<double>();
      a.inv = st.inv_diag.as<double>();
      a.scratch = st.scratch.as<double>();
      a.k = st.rate_constants.as<double>();
      a.atol = st.atol.as<double>();
      a.rtol = st.rtol;
      a.ctl = st.be_ctl.as<BeCtl>();
      cudaStream_t stream = st.stream;
      const int32_t S = m.S;
      const unsigned grid_c = Blocks(n);
      const unsigned grid_e = Blocks(n * (int64_t)S);
      k_be_init<<<1, 1, 0, stream>>>(a.ctl, P, dt);
      if (n > 0)
        k_be_apply<<<grid_e, kBlock, 0, stream>>>(a, S);
      MICMB_CUDA(cudaGetLastError());
      // bound on Newton iterations: every attempt either ends the solve, halves
      // H at most n_red times in a row, or advances t; far more than any solve takes
      const int64_t max_iterations = (int64_t)(P.max_iter + 1) * 4000000;
      int64_t iterations = 0, batch = 8;
      BeCtl hc{};
      if (n > 0)
        for (;;)
        {
          for (int64_t it = 0; it < batch; ++it)
          {
            k_be_iterate<<<grid_c, kBlock, 0, stream>>>(s.dev, P, a);
            k_be_control<<<1, 1, 0, stream>>>(P, dt, a.ctl);
            k_be_apply<<<grid_e, kBlock, 0, stream>>>(a, S);
          }
          MICMB_CUDA(cudaGetLastError());
          iterations += batch;
          MICMB_CUDA(cudaMemcpyAsync(&hc, a.ctl, sizeof(BeCtl), cudaMemcpyDeviceToHost, stream));
          MICMB_CUDA(cudaStreamSynchronize(stream));
          if (hc.phase != 0)
            break;
          if (iterations > max_iterations)
            throw Error(MICMB_ERR_INTERNAL, "Backward Euler solve did not terminate");
          batch = std::min<int64_t>(batch * 2, 64);
        }
      else
      {
        MICMB_CUDA(cudaMemcpyAsync(&hc, a.ctl, sizeof(BeCtl), cudaMemcpyDeviceToHost, stream));
        MICMB_CUDA(cudaStreamSynchronize(stream));
      }
      if (n > 0)
      {
        k_be_clamp<<<grid_e, kBlock, 0, stream>>>(a.y, n, st.L, S);
        MICMB_CUDA(cudaGetLastError());
      }
      if (per_cell_status || per_cell_accepted)
      {
        if (!st.status.p)
          st.status = DeviceMemory(sizeof(int32_t) * std::max<int64_t>(n, 1));
        if (!st.accepted.p)
          st.accepted = DeviceMemory(sizeof(int32_t) * std::max<int64_t>(n, 1));
        if (n > 0)
          k_be_fill_per_cell<<<grid_c, kBlock, 0, stream>>>(a.ctl, n, st.status.as<int32_t>(),
                                                            st.accepted.as<int32_t>());
        MICMB_CUDA(cudaGetLastError());
        if (per_cell_status && n > 0)
          MICMB_CUDA(cudaMemcpyAsync(per_cell_status, st.status.p, sizeof(int32_t) * n, cudaMemcpyDeviceToHost,
                                     stream));
        if (per_cell_accepted && n > 0)
          MICMB_CUDA(cudaMemcpyAsync(per_cell_accepted, st.accepted.p, sizeof(int32_t) * n,
                                     cudaMemcpyDeviceToHost, stream));
      }
      MICMB_CUDA(cudaStreamSynchronize(stream));
      if (stats)
      {
        unsigned long long hs[8];
        for (int q = 0; q < 7; ++q)
          hs[q] = (unsigned long long)hc.st[q];
        const int32_t nc = hc.state == MICMB_SOLVER_CONVERGED ? 0 : (int32_t)n;
        FillStats(stats, hs, hc.state, nc, hc.t);
      }
    }

    void SolveBackwardEulerPerCell(micmb_solver& s, micmb_state& st, double dt, const BeParams& P,
                                   micmb_solver_stats* stats, int32_t* per_cell_status, int32_t* per_cell_accepted)
    {
      const auto& m = *s.mech;
      const int64_t n = st.n_cells;
      const BeLayout T = MakeBeLayout(m.S, m.R, (int32_t)m.info_rxn.size(), m.nnz);
      int per_sm = 0;
      MICMB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_backward_euler_thread, kThreadsPerBlock, 0));
      if (per_sm < 1)
        throw Error(MICMB_ERR_UNSUPPORTED, "Backward Euler kernel cannot be resident");
      int64_t grid = (int64_t)per_sm * s.sm_count;
      grid = std::max<int64_t>(1, std::min<int64_t>(grid, (n + kThreadsPerBlock - 1) / kThreadsPerBlock));
      const int64_t doubles = grid * kThreadsPerBlock * (int64_t)T.per_slot;
      if (!st.thread_ws.p || st.thread_ws.bytes < (size_t)doubles * sizeof(double))
        st.thread_ws = DeviceMemory((size_t)doubles * sizeof(double));
      if (!st.status.p)
        st.status = DeviceMemory(sizeof(int32_t) * std::max<int64_t>(n, 1));
      if (!st.accepted.p)
        st.accepted = DeviceMemory(sizeof(int32_t) * std::max<int64_t>(n, 1));
      FusedArgs A{};
      A.n_cells = n;
      A.L = st.L;
      A.variables_in = st.variables.as<double>();
      A.variables_out = st.variables.as<double>();
      A.rate_constants = st.rate_constants.as<double>();
      A.atol = st.atol.as<double>();
      A.rtol = st.rtol;
      char* cbase = st.counters.as<char>();
      A.next_cell = reinterpret_cast<int32_t*>(cbase + 8);
      A.stats = reinterpret_cast<unsigned long long*>(cbase + 64);
      A.cell_status = st.status.as<int32_t>();
      A.cell_accepted = st.accepted.as<int32_t>();
      cudaStream_t stream = st.stream;
      MICMB_CUDA(cudaMemsetAsync(cbase, 0, 128, stream));
      if (n > 0)
      {
        k_backward_euler_thread<<<(unsigned)grid, kThreadsPerBlock, 0, stream>>>(s.dev, P, dt, A,
                                                                                  st.thread_ws.as<double>(), T);
        MICMB_CUDA(cudaGetLastError());
      }
      unsigned long long hs[8];
      MICMB_CUDA(cudaMemcpyAsync(hs, A.stats, sizeof(hs), cudaMemcpyDeviceToHost, stream));
      if (per_cell_status && n > 0)
        MICMB_CUDA(cudaMemcpyAsync(per_cell_status, A.cell_status, sizeof(int32_t) * n, cudaMemcpyDeviceToHost,
                                   stream));
      if (per_cell_accepted && n > 0)
        MICMB_CUDA(cudaMemcpyAsync(per_cell_accepted, A.cell_accepted, sizeof(int32_t) * n, cudaMemcpyDeviceToHost,
                                   stream));
      MICMB_CUDA(cudaStreamSynchronize(stream));
      if (stats)
      {
        int32_t worst = MICMB_SOLVER_CONVERGED;
        if (hs[7])
        {
          std::vector<int32_t> stv(n);
          MICMB_CUDA(cudaMemcpy(stv.data(), A.cell_status, sizeof(int32_t) * n, cudaMemcpyDeviceToHost));
          for (auto v : stv)
            if (v != MICMB_SOLVER_CONVERGED)
            {
              worst = v;
              break;
            }
        }
        FillStats(stats, hs, worst, (int32_t)hs[7], dt);
      }
    }
  }  // namespace

  void DefaultBackwardEulerParams(micmb_backward_euler_params* p)
  {
    *p = micmb_backward_euler_params{};
    p->small = 1.0e-40;
    p->h_start = 0.0;
    p->max_number_of_steps = 11;
    p->n_time_step_reductions = 5;
    const double red[5] = { 0.5, 0.5, 0.5, 0.5, 0.1 };
    for (int i = 0; i < 5; ++i)
      p->time_step_reductions[i] = red[i];
  }

  void SolveBackwardEuler(micmb_solver& s, micmb_state& st, double dt, const micmb_backward_euler_params& params,
                          int32_t step_control, micmb_solver_stats* stats, int32_t* per_cell_status,
                          int32_t* per_cell_accepted)
  {
    if (params.max_number_of_steps < 1 || params.n_time_step_reductions < 0 || params.n_time_step_reductions > 8 ||
        !(params.small >= 0.0) || !(params.h_start >= 0.0))
      throw Error(MICMB_ERR_INVALID_ARGUMENT,
                  "Backward Euler parameters: max_number_of_steps >= 1, 0..8 reductions, small and h_start >= 0");
    if (!s.mech->constraints.empty())
      throw Error(MICMB_ERR_UNSUPPORTED, "Backward Euler takes no algebraic constraints (micm's applies none)");
    const BeParams P = ToDevice(params);
    if (step_control == MICMB_STEP_GLOBAL)
      SolveBackwardEulerGlobal(s, st, dt, P, stats, per_cell_status, per_cell_accepted);
    else
      SolveBackwardEulerPerCell(s, st, dt, P, stats, per_cell_status, per_cell_accepted);
  }
}  // namespace micmb
