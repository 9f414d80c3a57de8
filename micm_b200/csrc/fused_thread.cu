// fused_thread.cu -- the persistent fused solve with one grid cell per thread.
//
// Every thread of a resident grid owns a private working set (state, stages,
// rate constants, rates and the LU factor) in global memory, laid out so that
// the 32 threads of a warp touch 32 consecutive doubles for the same entry:
// every access of the sparse kernels is a full 256-byte line.  A warp runs
// attempts in lockstep -- forcing (only where a step starts), -J, the LU in
// micm's update order, the stages and the error norm -- so all its threads
// follow the same instruction stream over the mechanism's tables, and a
// thread whose cell finishes takes the next unsolved cell from a global atomic
// counter between two attempts.  Per-cell results are bit-identical to the
// plain per-stage kernels: the same routines in the same order.
#include "runtime.hpp"

#include <algorithm>

namespace micmb
{
  namespace
  {
    // 128-thread blocks.  The kernel is compiled for four residencies (the
    // minimum-blocks hint of __launch_bounds__): 16 blocks per SM (32
    // registers, 64 warps: every warp slot, with spills), 12 (40 registers),
    // 8 (64 registers) and 5 (96 registers, no spills, 20 warps).  More
    // resident warps hide more HBM latency, fewer registers spill more; on the
    // 210- and 600-species mechanisms and TS1 the full-occupancy build measured
    // fastest (11-34 % over the 96-register one).  micmb_fused_config.ctas_per_sm
    // selects the build; the autotuner times them.
    constexpr int kThreadsPerBlock = 128;

    __device__ __forceinline__ size_t cell_base(int64_t c, int32_t L, int32_t ncol)
    {
      return (size_t)(c / L) * (size_t)L * (size_t)ncol + (size_t)(c % L);
    }

    static_assert(sizeof(CellCtl) == 8 * sizeof(double), "a lane's CellCtl record is 8 doubles");

    // entry offsets (each entry = 32 doubles, one per lane) of a thread's working set
    struct ThreadLayout
    {
      int32_t oY, oYn, oF0, oFc, oK, oLU, oInv, oKk, oScr, oCj, oKeq, oCtl, per_slot;
    };

    // oCj / oKeq: constraint Jacobian terms and K_eq values (DAE mechanisms only);
    // oCtl: 32 CellCtl records (8 doubles each), one per lane
    ThreadLayout MakeThreadLayout(int32_t S, int32_t R, int32_t stages, int32_t n_info, int32_t nnz,
                                  int32_t n_cterms = 0, int32_t n_eq = 0)
    {
      ThreadLayout t;
      int32_t o = 0;
      t.oY = o;
      o += S;
      t.oYn = o;
      o += S;
      t.oF0 = o;
      o += S;
      t.oFc = o;
      o += S;
      t.oK = o;
      o += stages * S;
      t.oLU = o;
      o += nnz;
      t.oInv = o;
      o += S;
      t.oKk = o;
      o += R;
      t.oScr = o;
      o += (R > n_info ? R : n_info);
      t.oCj = o;
      o += n_cterms;
      t.oKeq = o;
      o += n_eq;
      t.oCtl = o;
      o += 8;  // the lanes' CellCtl records, 64 bytes each
      t.per_slot = o;
      return t;
    }

    __device__ __forceinline__ void count_attempt(CellCtl& cc, const DevParams& P)
    {
      cc.decompositions += 1;
      cc.solves += P.stages;
      for (int32_t s = 1; s < P.stages; ++s)
        cc.function_calls += P.new_f[s] ? 1 : 0;
    }

    // DAE: the mechanism has algebraic constraints (a separate instantiation,
    // so the constraint code costs the ODE kernels no registers)
    template<bool DAE>
    __device__ __forceinline__ void fused_thread_body(const DevMech& M, const DevParams& P, const StepBounds& B,
                                                      const FusedArgs& A, double* ws, const ThreadLayout& T)
    {
      const int lane = threadIdx.x & 31;
      const int64_t wslot = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
      double* w = ws + (size_t)wslot * (size_t)T.per_slot * 32 + lane;
      const int32_t S = M.S, R = M.R, L = A.L;
      Strided Y{ w + (size_t)T.oY * 32, 32 };
      Strided Yn{ w + (size_t)T.oYn * 32, 32 };
      Strided F0{ w + (size_t)T.oF0 * 32, 32 };
      Strided Fc{ w + (size_t)T.oFc * 32, 32 };
      double* Kb = w + (size_t)T.oK * 32;
      Strided LU{ w + (size_t)T.oLU * 32, 32 };
      Strided inv{ w + (size_t)T.oInv * 32, 32 };
      Strided kk{ w + (size_t)T.oKk * 32, 32 };
      Strided scr{ w + (size_t)T.oScr * 32, 32 };
      Strided cj{ w + (size_t)T.oCj * 32, 32 };
      Strided kq{ w + (size_t)T.oKeq * 32, 32 };
      auto Kv = [&](int32_t st) { return Strided{ Kb + (size_t)st * S * 32, 32 }; };

      // solver statistics of the block's finished cells (one global atomic per block and counter)
      __shared__ unsigned long long block_stats[9];
      if (threadIdx.x < 9)
        block_stats[threadIdx.x] = 0;
      __syncthreads();
      // The cell's step-control record stays in the warp's working-set slot
      // (64 bytes per lane), not in registers: it is read a few times per
      // attempt, and out of the register budget it no longer pushes the LU
      // and solve loops' values into spills (+5 % at 1M cells, 210 species).
      CellCtl& c = *reinterpret_cast<CellCtl*>(ws + (size_t)wslot * (size_t)T.per_slot * 32 + (size_t)T.oCtl * 32 +
                                               (size_t)lane * 8);
      ctl_init(c, B);
      int64_t cell = 0;
      int32_t n_ckpt = 0;
      bool have = false, need_f0 = false, need_init = false;

      auto write_out = [&]() {
        const size_t by = cell_base(cell, L, S);
        for (int32_t i = 0; i < S; ++i)
        {
          A.variables_out[by + (size_t)i * L] = post_clamp(M, i, Y[i]);
        }
        if (A.cell_status)
          A.cell_status[cell] = c.state;
        if (A.cell_accepted)
          A.cell_accepted[cell] = A.ckpt_y ? n_ckpt : c.accepted;
        atomicAdd(block_stats + 0, (unsigned long long)c.function_calls);
        atomicAdd(block_stats + 1, (unsigned long long)c.jacobian_updates);
        atomicAdd(block_stats + 2, (unsigned long long)c.number_of_steps);
        atomicAdd(block_stats + 3, (unsigned long long)c.accepted);
        atomicAdd(block_stats + 4, (unsigned long long)c.rejected);
        atomicAdd(block_stats + 5, (unsigned long long)c.decompositions);
        atomicAdd(block_stats + 6, (unsigned long long)c.solves);
        if (c.state != MICMB_SOLVER_CONVERGED)
          atomicAdd(block_stats + 7, 1ull);
        if (c.init_iterations)
          atomicAdd(block_stats + 8, (unsigned long long)c.init_iterations);
      };
      // take cells until one needs an attempt (or none are left)
      auto claim = [&]() {
        for (;;)
        {
          cell = atomicAdd(A.next_cell, 1);
          if (cell >= A.n_cells)
          {
            have = false;
            return;
          }
          const size_t by = cell_base(cell, L, S);
          const size_t bk = cell_base(cell, L, R);
          for (int32_t i = 0; i < S; ++i)
            Y[i] = A.variables_in[by + (size_t)i * L];
          for (int32_t r = 0; r < R; ++r)
            kk[r] = A.rate_constants[bk + (size_t)r * L];
          ctl_init(c, B);
          n_ckpt = 0;
          if constexpr (DAE)
          {
            // K_eq values; the constraint initialisation runs in the attempt
            // loop, outside this lambda, so that the lambda stays inlined
            const size_t bq = cell_base(cell, L, M.n_eq);
            for (int32_t q = 0; q < M.n_eq; ++q)
              kq[q] = A.keq[bq + (size_t)q * L];
            need_init = true;
            have = true;
            return;
          }
          if (ctl_begin_step(c, P, B))
          {
            c.function_calls += 1;
            c.jacobian_updates += 1;
            need_f0 = true;
            have = true;
            return;
          }
          write_out();
        }
      };

      claim();
      while (__any_sync(0xffffffffu, have))
      {
        if (!have)
          continue;
        if (need_init)
        {
          // micm's constraint initialisation of the algebraic variables, then the first step
          need_init = false;
          const int32_t st = constraint_init_cell(M, P, kq, Y, Fc, LU, inv, cj, c);
          if (st != MICMB_SOLVER_CONVERGED)
            c.state = st;
          else if (ctl_begin_step(c, P, B))
          {
            c.function_calls += 1;
            c.jacobian_updates += 1;
            need_f0 = true;
          }
          if (c.state != MICMB_SOLVER_RUNNING)
          {
            write_out();
            claim();
            continue;
          }
        }
        if (need_f0)
        {
          reaction_rates<1>(M, kk, Y, scr, 0);
          forcing_gather<1>(M, scr, F0, 0);
          if constexpr (DAE)
            constraint_forcing(M, kq, Y, F0);
        }
        const double H = c.H;
        const double alpha = 1.0 / (H * P.gamma0);
        jacobian_rates<1>(M, kk, Y, scr, 0);
        if constexpr (DAE)
          constraint_jacobian(M, kq, Y, cj);
        if constexpr (DAE)
          thread_lu_gathered(M, scr, alpha, LU, inv, cj);  // -J + alpha M, then LU
        else
          thread_lu_gathered(M, scr, alpha, LU, inv);  // -J + alpha I, then LU
        bool fc_is_src = false;
        for (int32_t st = 0; st < P.stages; ++st)
        {
          const int32_t sc = st * (st - 1) / 2;
          if (st > 0 && P.new_f[st])
          {
            for (int32_t i = 0; i < S; ++i)
            {
              double v = Y[i];
              for (int32_t j = 0; j < st; ++j)
                v += P.a[sc + j] * Kv(j)[i];
              Yn[i] = v;
            }
            reaction_rates<1>(M, kk, Yn, scr, 0);
            forcing_gather<1>(M, scr, Fc, 0);
            if constexpr (DAE)
              constraint_forcing(M, kq, Yn, Fc);
            fc_is_src = true;
          }
          double coh[6];
          for (int32_t j = 0; j < st; ++j)
            coh[j] = P.c[sc + j] / H;
          Strided Ks = Kv(st);
          for (int32_t i = 0; i < S; ++i)
          {
            double v = fc_is_src ? Fc[i] : F0[i];
            if (!DAE || M.mass[i] != 0.0)  // algebraic rows have no mass coupling
              for (int32_t j = 0; j < st; ++j)
                v += coh[j] * Kv(j)[i];
            Ks[i] = v;
          }
          thread_solve(M, LU, Ks);
        }
        // Ynew, and the error norm summed in species order (micm's order)
        double sum = 0.0;
        for (int32_t i = 0; i < S; ++i)
        {
          double v = Y[i];
          double e = 0.0;
          for (int32_t st = 0; st < P.stages; ++st)
          {
            const double kv = Kv(st)[i];
            v += P.m[st] * kv;
            e += P.e[st] * kv;
          }
          Yn[i] = v;
          if (DAE && M.mass[i] == 0.0)
            e = v - Y[i];  // SetAlgebraicErrors: the step change
          sum += scaled_sq(Y[i], v, e, A.atol[i], A.rtol);
        }
        const double error = error_from_sum(sum, (double)S);
        count_attempt(c, P);
        const double h_used = c.H;
        const int res = ctl_after_error(c, P, B, error);
        if (res == 1)
        {
          if (A.ckpt_y)
          {
            double* dst = A.ckpt_y + ((size_t)cell * A.max_ckpt + n_ckpt) * S;
            for (int32_t i = 0; i < S; ++i)
              dst[i] = Y[i];
            if (A.ckpt_k)
            {
              double* kd = A.ckpt_k + ((size_t)cell * A.max_ckpt + n_ckpt) * (size_t)P.stages * S;
              for (int32_t st = 0; st < P.stages; ++st)
                for (int32_t i = 0; i < S; ++i)
                  kd[(size_t)st * S + i] = Kv(st)[i];
            }
            A.ckpt_h[(size_t)cell * A.max_ckpt + n_ckpt] = h_used;
            ++n_ckpt;
          }
          for (int32_t i = 0; i < S; ++i)
            Y[i] = Yn[i];
          bool more = ctl_begin_step(c, P, B);
          if (more && A.ckpt_y && n_ckpt >= A.max_ckpt)
          {
            c.state = MICMB_SOLVER_CONVERGENCE_EXCEEDED_MAX_STEPS;
            more = false;
          }
          if (more)
          {
            c.function_calls += 1;
            c.jacobian_updates += 1;
            need_f0 = true;
          }
          else
          {
            write_out();
            claim();
          }
        }
        else if (res == 0)
          need_f0 = false;
        else
        {
          write_out();
          claim();
        }
      }
      __syncthreads();
      if (threadIdx.x < 9 && block_stats[threadIdx.x])
        atomicAdd(A.stats + threadIdx.x, block_stats[threadIdx.x]);
    }

    template<bool DAE>
    __global__ void __launch_bounds__(kThreadsPerBlock, 5)
        k_fused_thread_r96(DevMech M, DevParams P, StepBounds B, FusedArgs A, double* ws, ThreadLayout T)
    {
      fused_thread_body<DAE>(M, P, B, A, ws, T);
    }

    template<bool DAE>
    __global__ void __launch_bounds__(kThreadsPerBlock, 8)
        k_fused_thread_r64(DevMech M, DevParams P, StepBounds B, FusedArgs A, double* ws, ThreadLayout T)
    {
      fused_thread_body<DAE>(M, P, B, A, ws, T);
    }

    template<bool DAE>
    __global__ void __launch_bounds__(kThreadsPerBlock, 12)
        k_fused_thread_r40(DevMech M, DevParams P, StepBounds B, FusedArgs A, double* ws, ThreadLayout T)
    {
      fused_thread_body<DAE>(M, P, B, A, ws, T);
    }

    template<bool DAE>
    __global__ void __launch_bounds__(kThreadsPerBlock, 16)
        k_fused_thread(DevMech M, DevParams P, StepBounds B, FusedArgs A, double* ws, ThreadLayout T)
    {
      fused_thread_body<DAE>(M, P, B, A, ws, T);
    }

    using ThreadKernel = void (*)(DevMech, DevParams, StepBounds, FusedArgs, double*, ThreadLayout);

    // the build a configuration asks for (ctas_per_sm; 0 = full occupancy)
    template<bool DAE>
    ThreadKernel ThreadKernelBuild(const micmb_fused_config& cfg)
    {
      if (cfg.ctas_per_sm == 0 || cfg.ctas_per_sm > 12)
        return k_fused_thread<DAE>;
      if (cfg.ctas_per_sm > 8)
        return k_fused_thread_r40<DAE>;
      if (cfg.ctas_per_sm > 5)
        return k_fused_thread_r64<DAE>;
      return k_fused_thread_r96<DAE>;
    }

    ThreadKernel ThreadKernelFor(const micmb_solver& s)
    {
      return s.mech->constraints.empty() ? ThreadKernelBuild<false>(s.fused) : ThreadKernelBuild<true>(s.fused);
    }

    int ThreadBlocksPerSm(const micmb_solver& s)
    {
      int per_sm = 0;
      MICMB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, ThreadKernelFor(s), kThreadsPerBlock, 0));
      if (s.fused.variant == 2 && s.fused.ctas_per_sm > 0)
        per_sm = std::min(per_sm, s.fused.ctas_per_sm);
      return per_sm;
    }
  }  // namespace

  int64_t FusedThreadResidentCells(const micmb_solver& s)
  {
    return (int64_t)std::max(ThreadBlocksPerSm(s), 1) * s.sm_count * kThreadsPerBlock;
  }

  int64_t FusedThreadWorkspaceDoubles(const micmb_solver& s, int64_t n_cells)
  {
    const auto& m = *s.mech;
    const ThreadLayout T = MakeThreadLayout(m.S, m.R, s.params.stages, (int32_t)m.info_rxn.size(), m.nnz,
                                            (int32_t)m.c_term_col.size(), m.n_eq);
    const int64_t threads = std::min<int64_t>(FusedThreadResidentCells(s),
                                              (n_cells + kThreadsPerBlock - 1) / kThreadsPerBlock * kThreadsPerBlock);
    return std::max<int64_t>(threads, kThreadsPerBlock) * (int64_t)T.per_slot;
  }

  bool SolveFusedThread(micmb_solver& s, micmb_state& st, const FusedArgs& A_in, double dt)
  {
    const auto& m = *s.mech;
    const ThreadLayout T = MakeThreadLayout(m.S, m.R, s.params.stages, (int32_t)m.info_rxn.size(), m.nnz,
                                            (int32_t)m.c_term_col.size(), m.n_eq);
    const ThreadKernel kernel = ThreadKernelFor(s);
    const int per_sm = ThreadBlocksPerSm(s);
    if (per_sm < 1)
      return false;
    int64_t grid = (int64_t)per_sm * s.sm_count;
    grid = std::max<int64_t>(1, std::min<int64_t>(grid, (A_in.n_cells + kThreadsPerBlock - 1) / kThreadsPerBlock));
    const int64_t doubles = grid * kThreadsPerBlock * (int64_t)T.per_slot;
    if (!st.thread_ws.p || st.thread_ws.bytes < (size_t)doubles * sizeof(double))
      st.thread_ws = DeviceMemory((size_t)doubles * sizeof(double));
    const StepBounds B = step_bounds(s.params, dt);
    kernel<<<(unsigned)grid, kThreadsPerBlock, 0, st.stream>>>(s.dev, s.params, B, A_in, st.thread_ws.as<double>(),
                                                               T);
    MICMB_CUDA(cudaGetLastError());
    return true;
  }
}  // namespace micmb
