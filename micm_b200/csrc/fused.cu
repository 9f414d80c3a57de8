// fused.cu -- the whole adaptive Rosenbrock solve of a cell in one persistent
// kernel.  Each warp owns one grid cell at a time: the cell's state, stage
// vectors, rate constants and (when it fits) its LU factor live in the warp's
// slice of shared memory for the entire solve, and the 32 lanes split every
// stage (forcing, -J assembly, LU, triangular solves, error norm) by the level
// schedules of the mechanism compiler.  When a warp finishes its cell it takes
// the next unsolved cell from a global atomic counter, so cells with uneven
// step counts balance across the GPU without any host involvement.
#include "runtime.hpp"

#include <algorithm>

namespace micmb
{
  namespace
  {
    constexpr int kWarp = 32;

    __device__ __forceinline__ size_t cell_base(int64_t c, int32_t L, int32_t ncol)
    {
      return (size_t)(c / L) * (size_t)L * (size_t)ncol + (size_t)(c % L);
    }

    // per-warp shared-memory layout (doubles); every vector has one extra zero
    // slot (index S) that padded table terms read
    struct WarpLayout
    {
      int32_t S, R, stages, scratch_cols, nnz;
      int32_t VS;        // vector stride = S + 1 rounded to even
      int32_t KS;        // rate-constant block
      int32_t SC;        // scratch block = scratch_cols + 1 rounded to even
      int32_t LUS;       // LU block = nnz + 1 rounded to even
      int32_t per_warp;  // doubles per warp
    };

    __host__ __device__ inline int32_t RoundUp2(int32_t v)
    {
      return (v + 1) & ~1;
    }

    __host__ __device__ inline WarpLayout MakeLayout(int32_t S, int32_t R, int32_t stages, int32_t n_info, int32_t nnz,
                                                     bool lu_shared)
    {
      WarpLayout w;
      w.S = S;
      w.R = R;
      w.stages = stages;
      w.scratch_cols = R > n_info ? R : n_info;
      w.nnz = nnz;
      w.VS = RoundUp2(S + 1);
      w.KS = RoundUp2(R > 0 ? R : 1);
      w.SC = RoundUp2(w.scratch_cols + 1);
      w.LUS = RoundUp2(nnz + 1);
      w.per_warp = w.VS * (5 + stages) + w.KS + w.SC + (lu_shared ? w.LUS : 0);
      return w;
    }

    __device__ __forceinline__ void count_attempt(CellCtl& cc, const DevParams& P)
    {
      cc.decompositions += 1;
      cc.solves += P.stages;
      for (int32_t s = 1; s < P.stages; ++s)
        cc.function_calls += P.new_f[s] ? 1 : 0;
    }

    template<bool LU_SHARED>
    __global__ void __launch_bounds__(256) k_fused(DevMech M, DevParams P, StepBounds B, FusedArgs A, WarpLayout W)
    {
      extern __shared__ __align__(16) double smem[];
      const int warp = threadIdx.x >> 5;
      const int lane = threadIdx.x & 31;
      const int warps = blockDim.x >> 5;
      const int32_t S = M.S, R = M.R, L = A.L;
      double* base = smem + (size_t)warp * W.per_warp;
      const int32_t VS = W.VS;
      double* Y = base;
      double* Yn = Y + VS;
      double* F0 = Yn + VS;
      double* Fc = F0 + VS;
      double* inv = Fc + VS;
      double* K = inv + VS;
      double* kk = K + (size_t)P.stages * VS;
      double* scr = kk + W.KS;
      double* LU = LU_SHARED ? (scr + W.SC)
                             : A.lu_global + ((size_t)blockIdx.x * warps + warp) * (size_t)A.lu_slot_stride;
      // zero slots read by padded table terms (never written afterwards)
      if (lane == 0)
      {
        for (int32_t st = 0; st < P.stages; ++st)
          K[(size_t)st * VS + S] = 0.0;
        Y[S] = 0.0;
        Yn[S] = 0.0;
        scr[M.scratch_zero] = 0.0;
        LU[M.nnz] = 0.0;
      }
      __syncwarp();
      long long acc[8] = { 0 };

      for (;;)
      {
        int cell = 0;
        if (lane == 0)
          cell = atomicAdd(A.next_cell, 1);
        cell = __shfl_sync(0xffffffffu, cell, 0);
        if (cell >= A.n_cells)
          break;
        const size_t by = cell_base(cell, L, S);
        const size_t bk = cell_base(cell, L, R);
        for (int32_t i = lane; i < S; i += kWarp)
          Y[i] = A.variables_in[by + (size_t)i * L];
        for (int32_t r = lane; r < R; r += kWarp)
          kk[r] = A.rate_constants[bk + (size_t)r * L];
        __syncwarp();

        CellCtl c;
        ctl_init(c, B);
        int32_t n_ckpt = 0;
        while (ctl_begin_step(c, P, B))
        {
          c.function_calls += 1;
          c.jacobian_updates += 1;
          if (A.ckpt_y)
          {
            if (n_ckpt >= A.max_ckpt)
            {
              c.state = MICMB_SOLVER_CONVERGENCE_EXCEEDED_MAX_STEPS;
              break;
            }
          }
          reaction_rates<kWarp>(M, Unit{ kk }, Unit{ Y }, Unit{ scr }, lane);
          __syncwarp();
          warp_gather(M.w_forcing, scr, F0, 0.0, lane);
          __syncwarp();
          for (;;)
          {
            const double alpha = 1.0 / (c.H * P.gamma0);
            jacobian_rates<kWarp>(M, Unit{ kk }, Unit{ Y }, Unit{ scr }, lane);
            __syncwarp();
            warp_gather(M.w_jacobian, scr, LU, alpha, lane);
            __syncwarp();
            warp_lu(M.w_lu, LU, inv, lane);
            const double* Fsrc = F0;
            for (int32_t st = 0; st < P.stages; ++st)
            {
              const int32_t sc = st * (st - 1) / 2;
              if (st > 0 && P.new_f[st])
              {
                for (int32_t i = lane; i < S; i += kWarp)
                {
                  double v = Y[i];
                  for (int32_t j = 0; j < st; ++j)
                    v += P.a[sc + j] * K[(size_t)j * VS + i];
                  Yn[i] = v;
                }
                __syncwarp();
                reaction_rates<kWarp>(M, Unit{ kk }, Unit{ Yn }, Unit{ scr }, lane);
                __syncwarp();
                warp_gather(M.w_forcing, scr, Fc, 0.0, lane);
                __syncwarp();
                Fsrc = Fc;
              }
              double* Ks = K + (size_t)st * VS;
              for (int32_t i = lane; i < S; i += kWarp)
              {
                double v = Fsrc[i];
                for (int32_t j = 0; j < st; ++j)
                {
                  const double c_over_h = P.c[sc + j] / c.H;
                  v += c_over_h * K[(size_t)j * VS + i];
                }
                Ks[i] = v;
              }
              __syncwarp();
              warp_solve(M.w_fwd, LU, Ks, lane);
              warp_solve(M.w_bwd, LU, Ks, lane);
            }
            // error norm in species order (micm's order): stripe by stripe, the
            // lanes' terms added in lane order
            double sum = 0.0;
            for (int32_t base = 0; base < S; base += kWarp)
            {
              const int32_t i = base + lane;
              double q = 0.0;
              if (i < S)
              {
                double v = Y[i];
                double e = 0.0;
                for (int32_t st = 0; st < P.stages; ++st)
                {
                  const double kv = K[(size_t)st * VS + i];
                  v += P.m[st] * kv;
                  e += P.e[st] * kv;
                }
                Yn[i] = v;
                q = scaled_sq(Y[i], v, e, A.atol[i], A.rtol);
              }
              sum = warp_seq_add(sum, q, (S - base < kWarp) ? S - base : kWarp);
            }
            const double error = error_from_sum(sum, (double)S);
            count_attempt(c, P);
            const double h_used = c.H;
            const int res = ctl_after_error(c, P, B, error);
            __syncwarp();
            if (res == 1)
            {
              if (A.ckpt_y)
              {
                // checkpoint the accepted step: its starting state and step size
                double* dst = A.ckpt_y + ((size_t)cell * A.max_ckpt + n_ckpt) * S;
                for (int32_t i = lane; i < S; i += kWarp)
                  dst[i] = Y[i];
                if (lane == 0)
                  A.ckpt_h[(size_t)cell * A.max_ckpt + n_ckpt] = h_used;
                ++n_ckpt;
              }
              for (int32_t i = lane; i < S; i += kWarp)
                Y[i] = Yn[i];
              __syncwarp();
              break;
            }
            if (res < 0)
              break;
          }
          if (c.state != MICMB_SOLVER_RUNNING)
            break;
        }
        for (int32_t i = lane; i < S; i += kWarp)
        {
          const double v = Y[i];
          A.variables_out[by + (size_t)i * L] = (v < 0.0) ? 0.0 : v;
        }
        if (lane == 0)
        {
          if (A.cell_status)
            A.cell_status[cell] = c.state;
          if (A.cell_accepted)
            A.cell_accepted[cell] = A.ckpt_y ? n_ckpt : c.accepted;
          acc[0] += c.function_calls;
          acc[1] += c.jacobian_updates;
          acc[2] += c.number_of_steps;
          acc[3] += c.accepted;
          acc[4] += c.rejected;
          acc[5] += c.decompositions;
          acc[6] += c.solves;
          acc[7] += (c.state == MICMB_SOLVER_CONVERGED) ? 0 : 1;
        }
        __syncwarp();
      }
      if (lane == 0)
        for (int q = 0; q < 8; ++q)
          if (acc[q])
            atomicAdd(A.stats + q, (unsigned long long)acc[q]);
    }
  }  // namespace

  size_t FusedSharedBytes(const micmb_solver& s, bool lu_in_shared)
  {
    const auto& m = *s.mech;
    WarpLayout w = MakeLayout(m.S, m.R, s.params.stages, (int32_t)m.info_rxn.size(), m.nnz, lu_in_shared);
    return (size_t)w.per_warp * sizeof(double);
  }

  int FusedWarpsPerCta(const micmb_solver& s, const micmb_fused_config& cfg)
  {
    const size_t per = FusedSharedBytes(s, cfg.lu_in_shared != 0);
    int w = per == 0 ? 8 : (int)std::min<size_t>(8, s.smem_optin / per);
    if (cfg.cells_per_cta > 0)
      w = std::min(w, cfg.cells_per_cta);
    return w;
  }

  void SolveFused(micmb_solver& s, micmb_state& st, double dt, micmb_solver_stats* stats, int32_t* per_cell_status,
                  int32_t* per_cell_accepted, const FusedArgs* adj)
  {
    const auto& m = *s.mech;
    micmb_fused_config cfg = s.fused;
    if (cfg.lu_in_shared && FusedWarpsPerCta(s, cfg) < 1)
      cfg.lu_in_shared = 0;
    const int warps = FusedWarpsPerCta(s, cfg);
    if (warps < 1)
      throw Error(MICMB_ERR_UNSUPPORTED, "mechanism too large for the fused kernel's shared-memory working set");
    if (!s.dev.has_warp)
      throw Error(MICMB_ERR_UNSUPPORTED, "mechanism exceeds the fused kernel's 16-bit table positions (nnz <= 65534)");
    const bool lu_shared = cfg.lu_in_shared != 0;
    WarpLayout W = MakeLayout(m.S, m.R, s.params.stages, (int32_t)m.info_rxn.size(), m.nnz, lu_shared);
    const size_t smem = (size_t)W.per_warp * sizeof(double) * warps;
    const int threads = warps * kWarp;
    auto kernel = lu_shared ? k_fused<true> : k_fused<false>;
    MICMB_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int per_sm = 0;
    MICMB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem));
    if (per_sm < 1)
      throw Error(MICMB_ERR_UNSUPPORTED, "fused kernel cannot be resident with this configuration");
    if (cfg.ctas_per_sm > 0)
      per_sm = std::min(per_sm, cfg.ctas_per_sm);
    int64_t grid = (int64_t)per_sm * s.sm_count;
    // an adjoint chunk brings its own cell range (n_cells > 0, pointers already offset)
    const int64_t n = (adj && adj->n_cells > 0)
                          ? adj->n_cells
                          : (st.solve_limit > 0 ? std::min<int64_t>(st.solve_limit, st.n_cells) : st.n_cells);
    grid = std::max<int64_t>(1, std::min<int64_t>(grid, (n + warps - 1) / warps));

    FusedArgs A{};
    if (adj)
      A = *adj;
    A.n_cells = n;
    A.L = st.L;
    if (!adj)
    {
      A.variables_in = st.variables.as<double>();
      A.variables_out = st.variables.as<double>();
    }
    if (!A.rate_constants)
      A.rate_constants = st.rate_constants.as<double>();
    A.keq = st.keq.as<double>();
    A.atol = st.atol.as<double>();
    A.rtol = st.rtol;
    char* cbase = st.counters.as<char>();
    A.next_cell = reinterpret_cast<int32_t*>(cbase + 8);
    A.stats = reinterpret_cast<unsigned long long*>(cbase + 64);
    // per-cell outputs cover the whole state, whatever prefix this call solves
    if (!st.status.p)
      st.status = DeviceMemory(sizeof(int32_t) * std::max<int64_t>(st.n_cells, 1));
    if (!st.accepted.p)
      st.accepted = DeviceMemory(sizeof(int32_t) * std::max<int64_t>(st.n_cells, 1));
    if (!A.cell_status)
      A.cell_status = st.status.as<int32_t>();
    if (!A.cell_accepted)
      A.cell_accepted = st.accepted.as<int32_t>();
    if (!lu_shared)
    {
      const int64_t slots = grid * warps;
      const int64_t stride = ((int64_t)m.nnz + 1 + 31) & ~31ll;
      if (st.lu_slot_count < slots * stride || !st.lu_slots.p)
      {
        st.lu_slots = DeviceMemory(sizeof(double) * (size_t)(slots * stride));
        st.lu_slot_count = slots * stride;
      }
      A.lu_global = st.lu_slots.as<double>();
      A.lu_slot_stride = stride;
    }
    MICMB_CUDA(cudaMemsetAsync(cbase, 0, 160, st.stream));
    if (n > 0 && !m.constraints.empty())
    {
      // algebraic constraints: the one-cell-per-thread kernel is the fused form that has them
      if (adj)
        throw Error(MICMB_ERR_UNSUPPORTED, "the adjoint does not cover algebraic constraints");
      if (!SolveFusedThread(s, st, A, dt))
        throw Error(MICMB_ERR_UNSUPPORTED, "one-cell-per-thread kernel cannot be resident");
    }
    else if (n > 0)
    {
      bool done = false;
      if (s.fused.variant == 0)
        done = SolveFusedStream(s, st, dt, A);
      else if (s.fused.variant == 2)
        done = SolveFusedThread(s, st, A, dt);
      if (!done)
      {
        if (A.ckpt_k)
          throw Error(MICMB_ERR_INTERNAL, "the direct fused kernel stores no stage vectors");
        const StepBounds B = step_bounds(s.params, dt);
        kernel<<<(unsigned)grid, threads, smem, st.stream>>>(s.dev, s.params, B, A, W);
        MICMB_CUDA(cudaGetLastError());
      }
    }
    if (stats || per_cell_status || per_cell_accepted)
    {
      unsigned long long hs[9];
      MICMB_CUDA(cudaMemcpyAsync(hs, A.stats, sizeof(hs), cudaMemcpyDeviceToHost, st.stream));
      if (per_cell_status)
        MICMB_CUDA(cudaMemcpyAsync(per_cell_status, A.cell_status, sizeof(int32_t) * n, cudaMemcpyDeviceToHost,
                                   st.stream));
      if (per_cell_accepted)
        MICMB_CUDA(cudaMemcpyAsync(per_cell_accepted, A.cell_accepted, sizeof(int32_t) * n, cudaMemcpyDeviceToHost,
                                   st.stream));
      MICMB_CUDA(cudaStreamSynchronize(st.stream));
      int32_t err_flag = 0;
      MICMB_CUDA(cudaMemcpy(&err_flag, cbase + 16, sizeof(int32_t), cudaMemcpyDeviceToHost));
      if (err_flag)
        throw Error(MICMB_ERR_TIMEOUT, "fused kernel: a pipeline wait timed out");
      if (stats)
      {
        stats->function_calls = (int64_t)hs[0];
        stats->jacobian_updates = (int64_t)hs[1];
        stats->number_of_steps = (int64_t)hs[2];
        stats->accepted = (int64_t)hs[3];
        stats->rejected = (int64_t)hs[4];
        stats->decompositions = (int64_t)hs[5];
        stats->solves = (int64_t)hs[6];
        stats->cells_not_converged = (int32_t)hs[7];
        stats->constraint_init_iterations = (int64_t)hs[8];
        stats->final_time = dt;
        stats->state = hs[7] ? MICMB_SOLVER_CONVERGENCE_EXCEEDED_MAX_STEPS : MICMB_SOLVER_CONVERGED;
        if (hs[7])
        {
          std::vector<int32_t> stv(n);
          MICMB_CUDA(cudaMemcpy(stv.data(), A.cell_status, sizeof(int32_t) * n, cudaMemcpyDeviceToHost));
          for (auto v : stv)
            if (v != MICMB_SOLVER_CONVERGED)
            {
              stats->state = v;
              break;
            }
        }
      }
    }
  }
}  // namespace micmb
