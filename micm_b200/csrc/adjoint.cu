// adjoint.cu -- discrete adjoint of the accepted Rosenbrock steps of a
// per-cell fused solve (no counterpart in micm).
//
// The forward solve (SolveFused with checkpointing) stores, for every accepted
// step n of every cell, the starting state y_n, the step size H_n and (where
// memory allows) the stage vectors K_s.  The backward sweep, one cell per
// thread, then walks each cell's steps backwards.  For step n it rebuilds
// alpha I - J(y_n) and its LU factor, takes the stored stages or recomputes
// them exactly as the forward pass did (same routines, so the same bits), and
// applies the transposed step with the step size held fixed:
//
//   y_{n+1} = y_n + sum_s m_s K_s,   M K_s = F(Y_s) + sum_{j<s} (c_sj / H) K_j,
//   M = 1/(H gamma_0) I - J(y_n),    Y_s = y_n + sum_{j<s} a_sj K_j
//
//   Kbar_s = m_s ybar;  for s = S-1..0: Rbar_s = M^-T Kbar_s, Gbar_s += Rbar_s,
//   Kbar_j += (c_sj / H) Rbar_s, and the chain rule through Y_s (new function
//   evaluation: ybar += J(Y_s)^T Gbar_s, Kbar_j += a_sj J(Y_s)^T Gbar_s) or
//   through the reused evaluation (Gbar_{s-1} += Gbar_s);
//   finally ybar += J(y_n)^T Gbar_0 + sum_s H_r-terms of M's dependence on y_n.
//
// Rate-parameter gradients are taken with respect to log k_r (w_r = k_r prod y,
// so d w_r / d log k_r = w_r).  The same recurrences, in the same order, are
// restated on the CPU by the test oracle (om_adjoint_per_cell).
#include "runtime.hpp"

#include <algorithm>
#include <vector>

namespace micmb
{
  namespace
  {
    constexpr int kMaxAdjStages = 6;

    __device__ __forceinline__ size_t cell_base(int64_t c, int32_t L, int32_t ncol)
    {
      return (size_t)(c / L) * (size_t)L * (size_t)ncol + (size_t)(c % L);
    }

    struct AdjArgs
    {
      int64_t n_cells;
      int32_t L;
      int32_t max_ckpt;
      const double* rate_constants;  // vector layout [R]
      const double* y0;              // vector layout [S]: initial state (clamp derivative when no step)
      const double* ybar_final;      // vector layout [S]
      const double* ckpt_y;          // [cell][max_ckpt][S]
      const double* ckpt_h;          // [cell][max_ckpt]
      const double* ckpt_k;          // [cell][max_ckpt][stages][S] stored stage vectors, or null
      const int32_t* n_ckpt;         // [cell]
      double* ybar0;                 // vector layout [S]
      double* kbar;                  // [cell][R]
      int32_t* next_cell;
      const int32_t* order;          // cells in decreasing step count (thread kernel), or null
    };

    // ---- one cell per thread, private working sets in global memory ----

    // entry offsets of a thread's working set (each entry is 32 doubles, one per lane)
    struct AdjThreadLayout
    {
      int32_t oy, oF0, oFc, oInv, oYb, oTmp, oYs, oK, oKb, oGb, oRb, oKk, oKbar, oScr, oLU, per_slot;
    };

    AdjThreadLayout MakeAdjThreadLayout(int32_t S, int32_t R, int32_t ns, int32_t n_info, int32_t nnz)
    {
      AdjThreadLayout t;
      int32_t o = 0;
      auto take = [&](int32_t n) {
        const int32_t at = o;
        o += n;
        return at;
      };
      t.oy = take(S);
      t.oF0 = take(S);
      t.oFc = take(S);
      t.oInv = take(S);
      t.oYb = take(S);
      t.oTmp = take(S);
      t.oYs = take(ns * S);
      t.oK = take(ns * S);
      t.oKb = take(ns * S);
      t.oGb = take(ns * S);
      t.oRb = take(ns * S);
      t.oKk = take(R);
      t.oKbar = take(R);
      t.oScr = take(R > n_info ? R : n_info);
      t.oLU = take(nnz);
      t.per_slot = o;
      return t;
    }

    template<class V>
    __device__ __forceinline__ double nu_dot_t(const DevMech& M, int32_t r, V v)
    {
      double s = 0.0;
      for (int32_t i = M.prod_start[r]; i < M.prod_start[r + 1]; ++i)
        s += M.prod_yield[i] * v[M.prod_ids[i]];
      for (int32_t i = M.react_start[r]; i < M.react_start[r + 1]; ++i)
        s -= v[M.react_ids[i]];
      return s;
    }

    template<class V>
    __device__ __forceinline__ double prod_except_t(const DevMech& M, int32_t r, V y, int32_t a, int32_t b)
    {
      double v = 1.0;
      for (int32_t i = M.react_start[r]; i < M.react_start[r + 1]; ++i)
        if (i != a && i != b)
          v *= y[M.react_ids[i]];
      return v;
    }

    // yb += J(y)^T g ; kb[r] += (nu_r . g) w_r(y)  (reactions in order, as the oracle)
    template<class V>
    __device__ void vjp_f_t(const DevMech& M, V kk, V y, V g, V yb, V kb)
    {
      for (int32_t r = 0; r < M.R; ++r)
      {
        const double c = nu_dot_t(M, r, g);
        if (c == 0.0)
          continue;
        kb[r] += c * (kk[r] * prod_except_t(M, r, y, -1, -1));
        for (int32_t i = M.react_start[r]; i < M.react_start[r + 1]; ++i)
          yb[M.react_ids[i]] += c * kk[r] * prod_except_t(M, r, y, i, -1);
      }
    }

    template<class V>
    __device__ void jacobian_term_t(const DevMech& M, V kk, V y, V Rb, V Kv, V yb, V kb)
    {
      for (int32_t r = 0; r < M.R; ++r)
      {
        const double rho = nu_dot_t(M, r, Rb);
        if (rho == 0.0)
          continue;
        const int32_t r0 = M.react_start[r], r1 = M.react_start[r + 1];
        double gk = 0.0;
        for (int32_t i = r0; i < r1; ++i)
          gk += kk[r] * prod_except_t(M, r, y, i, -1) * Kv[M.react_ids[i]];
        kb[r] += rho * gk;
        for (int32_t i = r0; i < r1; ++i)
          for (int32_t j = r0; j < r1; ++j)
            if (i != j)
              yb[M.react_ids[j]] += rho * kk[r] * prod_except_t(M, r, y, i, j) * Kv[M.react_ids[i]];
      }
    }

    // vjp_f_t over fixed-width reactant lists (rate_desc)
    template<class V>
    __device__ void vjp_narrow(const DevMech& M, V kk, V y, V g, V yb, V kb)
    {
      const int32_t S = M.S;
      for (int32_t r = 0; r < M.R; ++r)
      {
        const double c = nu_dot_t(M, r, g);
        if (c == 0.0)
          continue;
        const int4 d = M.rate_desc[r];
        const int32_t id[3] = { d.x, d.y, d.z };
        double yv[3];
        int32_t nr = 0;
#pragma unroll
        for (int q = 0; q < 3; ++q)
        {
          yv[q] = id[q] < S ? y[id[q]] : 1.0;
          nr += id[q] < S ? 1 : 0;
        }
        const double k = kk[r];
        kb[r] += c * (k * (((1.0 * yv[0]) * yv[1]) * yv[2]));
        for (int q = 0; q < nr; ++q)
        {
          double v = 1.0;
          for (int o = 0; o < nr; ++o)
            if (o != q)
              v *= yv[o];
          yb[id[q]] += c * k * v;
        }
      }
    }

    // Reactions with at most three reactants (rate_desc): one pass over the
    // reactions at the step's starting state applies J(y)^T Gbar_0 and the
    // second-order terms of every stage, with w_r's partial derivatives formed
    // once per reaction instead of once per use.
    template<class V>
    __device__ void step_terms_narrow(const DevMech& M, int32_t ns, V kk, V y, V Gb0, const V* Rb, const V* K, V yb,
                                      V kb)
    {
      const int32_t S = M.S;
      for (int32_t r = 0; r < M.R; ++r)
      {
        const int4 d = M.rate_desc[r];
        const int32_t id[3] = { d.x, d.y, d.z };
        int32_t nr = 0;
        double yv[3];
#pragma unroll
        for (int q = 0; q < 3; ++q)
        {
          yv[q] = id[q] < S ? y[id[q]] : 1.0;
          nr += id[q] < S ? 1 : 0;
        }
        const double k = kk[r];
        // first derivatives k * prod of the other reactants (in reactant order)
        double P1[3];
#pragma unroll
        for (int q = 0; q < 3; ++q)
        {
          double v = 1.0;
#pragma unroll
          for (int o = 0; o < 3; ++o)
            if (o != q && o < nr)
              v *= yv[o];
          P1[q] = v;
        }
        // J(y)^T Gbar_0
        const double c = nu_dot_t(M, r, Gb0);
        if (c != 0.0)
        {
          kb[r] += c * (k * (((1.0 * (nr > 0 ? yv[0] : 1.0)) * (nr > 1 ? yv[1] : 1.0)) * (nr > 2 ? yv[2] : 1.0)));
          for (int q = 0; q < nr; ++q)
            yb[id[q]] += c * k * P1[q];
        }
        // second-order terms of every stage
        for (int32_t st = 0; st < ns; ++st)
        {
          const double rho = nu_dot_t(M, r, Rb[st]);
          if (rho == 0.0)
            continue;
          double kv[3];
          for (int q = 0; q < nr; ++q)
            kv[q] = K[st][id[q]];
          double gk = 0.0;
          for (int q = 0; q < nr; ++q)
            gk += k * P1[q] * kv[q];
          kb[r] += rho * gk;
          for (int q = 0; q < nr; ++q)
            for (int o = 0; o < nr; ++o)
              if (q != o)
              {
                double v = 1.0;  // product of the reactants other than q and o
                for (int z = 0; z < nr; ++z)
                  if (z != q && z != o)
                    v *= yv[z];
                yb[id[o]] += rho * k * v * kv[q];
              }
        }
      }
    }

    __device__ __forceinline__ void adjoint_thread_body(const DevMech& M, const DevParams& P, const AdjArgs& A,
                                                        const AdjThreadLayout& T, double* ws)
    {
      const int lane = threadIdx.x & 31;
      const int64_t wslot = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
      double* w = ws + (size_t)wslot * (size_t)T.per_slot * 32 + lane;
      const int32_t S = M.S, R = M.R, L = A.L, ns = P.stages;
      auto at = [&](int32_t entry) { return Strided{ w + (size_t)entry * 32, 32 }; };
      Strided y = at(T.oy), F0 = at(T.oF0), Fc = at(T.oFc), inv = at(T.oInv), yb = at(T.oYb), tmp = at(T.oTmp);
      Strided kk = at(T.oKk), kb = at(T.oKbar), scr = at(T.oScr), LU = at(T.oLU);
      auto Ys = [&](int32_t s) { return at(T.oYs + s * S); };
      auto K = [&](int32_t s) { return at(T.oK + s * S); };
      auto Kb = [&](int32_t s) { return at(T.oKb + s * S); };
      auto Gb = [&](int32_t s) { return at(T.oGb + s * S); };
      auto Rb = [&](int32_t s) { return at(T.oRb + s * S); };

      int64_t cell = 0;
      int32_t n = -1;  // checkpoint being processed; -1: no cell
      auto finish = [&]() {
        const size_t by = cell_base(cell, L, S);
        for (int32_t i = 0; i < S; ++i)
          A.ybar0[by + (size_t)i * L] = yb[i];
        for (int32_t r = 0; r < R; ++r)
          A.kbar[(size_t)cell * R + r] = kb[r];
      };
      auto claim = [&]() {
        for (;;)
        {
          const int64_t k = atomicAdd(A.next_cell, 1);
          if (k >= A.n_cells)
          {
            n = -1;
            return;
          }
          cell = A.order ? A.order[k] : k;
          const size_t by = cell_base(cell, L, S);
          const size_t bk = cell_base(cell, L, R);
          for (int32_t r = 0; r < R; ++r)
          {
            kk[r] = A.rate_constants[bk + (size_t)r * L];
            kb[r] = 0.0;
          }
          const int32_t n_ck = A.n_ckpt[cell];
          if (n_ck > 0)
          {
            n = n_ck - 1;
            return;
          }
          for (int32_t i = 0; i < S; ++i)
            yb[i] = (A.y0[by + (size_t)i * L] < 0.0) ? 0.0 : A.ybar_final[by + (size_t)i * L];
          finish();
        }
      };

      claim();
      while (__any_sync(0xffffffffu, n >= 0))
      {
        if (n < 0)
          continue;
        const size_t by = cell_base(cell, L, S);
        const double* yc = A.ckpt_y + ((size_t)cell * A.max_ckpt + n) * S;
        const double H = A.ckpt_h[(size_t)cell * A.max_ckpt + n];
        for (int32_t i = 0; i < S; ++i)
          y[i] = yc[i];
        // ---- the accepted step's factor, stages and stage inputs ----
        const double alpha = 1.0 / (H * P.gamma0);
        jacobian_rates<1>(M, kk, y, scr, 0);
        thread_lu_gathered(M, scr, alpha, LU, inv);  // -J + alpha I, then LU
        if (A.ckpt_k)
        {
          // stages stored by the forward pass; stage inputs rebuilt from them
          const double* kc = A.ckpt_k + ((size_t)cell * A.max_ckpt + n) * (size_t)ns * S;
          for (int32_t st = 0; st < ns; ++st)
          {
            Strided Ks = K(st);
            for (int32_t i = 0; i < S; ++i)
              Ks[i] = kc[(size_t)st * S + i];
          }
          for (int32_t st = 0; st < ns; ++st)
          {
            const int32_t sc = st * (st - 1) / 2;
            Strided Yst = Ys(st);
            if (st > 0 && P.new_f[st])
              for (int32_t i = 0; i < S; ++i)
              {
                double v = y[i];
                for (int32_t j = 0; j < st; ++j)
                  v += P.a[sc + j] * K(j)[i];
                Yst[i] = v;
              }
            else
              for (int32_t i = 0; i < S; ++i)
                Yst[i] = y[i];
          }
        }
        else
        {
          reaction_rates<1>(M, kk, y, scr, 0);
          forcing_gather<1>(M, scr, F0, 0);
          bool fc_is_src = false;
          for (int32_t st = 0; st < ns; ++st)
          {
            const int32_t sc = st * (st - 1) / 2;
            Strided Yst = Ys(st);
            if (st > 0 && P.new_f[st])
            {
              for (int32_t i = 0; i < S; ++i)
              {
                double v = y[i];
                for (int32_t j = 0; j < st; ++j)
                  v += P.a[sc + j] * K(j)[i];
                Yst[i] = v;
              }
              reaction_rates<1>(M, kk, Yst, scr, 0);
              forcing_gather<1>(M, scr, Fc, 0);
              fc_is_src = true;
            }
            else
              for (int32_t i = 0; i < S; ++i)
                Yst[i] = y[i];
            double coh[kMaxAdjStages];
            for (int32_t j = 0; j < st; ++j)
              coh[j] = P.c[sc + j] / H;
            Strided Ks = K(st);
            for (int32_t i = 0; i < S; ++i)
            {
              double v = fc_is_src ? Fc[i] : F0[i];
              for (int32_t j = 0; j < st; ++j)
                v += coh[j] * K(j)[i];
              Ks[i] = v;
            }
            thread_solve(M, LU, Ks);
          }
        }
        if (n == A.n_ckpt[cell] - 1)
          for (int32_t i = 0; i < S; ++i)
          {
            double v = y[i];
            for (int32_t st = 0; st < ns; ++st)
              v += P.m[st] * K(st)[i];
            yb[i] = (v < 0.0) ? 0.0 : A.ybar_final[by + (size_t)i * L];
          }
        // ---- reverse sweep ----
        for (int32_t i = 0; i < S; ++i)
        {
          const double g = yb[i];
          for (int32_t st = 0; st < ns; ++st)
          {
            Kb(st)[i] = P.m[st] * g;
            Gb(st)[i] = 0.0;
          }
        }
        for (int32_t st = ns - 1; st >= 0; --st)
        {
          const int32_t sc = st * (st - 1) / 2;
          Strided rb = Rb(st);
          for (int32_t i = 0; i < S; ++i)
            rb[i] = Kb(st)[i];
          solve_upper<1>(M.fwd_t_s, LU, rb, 0);  // U^T w = Kbar (divides by u_ii)
          solve_lower<1>(M.bwd_t_s, LU, rb, 0);  // L^T z = w
          double coh[kMaxAdjStages];
          for (int32_t j = 0; j < st; ++j)
            coh[j] = P.c[sc + j] / H;
          for (int32_t i = 0; i < S; ++i)
          {
            const double v = rb[i];
            Gb(st)[i] += v;
            for (int32_t j = 0; j < st; ++j)
              Kb(j)[i] += coh[j] * v;
          }
          if (st == 0)
            continue;
          if (P.new_f[st])
          {
            for (int32_t i = 0; i < S; ++i)
              tmp[i] = 0.0;
            if (M.rate_desc)
              vjp_narrow(M, kk, Ys(st), Gb(st), tmp, kb);
            else
              vjp_f_t(M, kk, Ys(st), Gb(st), tmp, kb);
            for (int32_t i = 0; i < S; ++i)
            {
              const double t = tmp[i];
              yb[i] += t;
              for (int32_t j = 0; j < st; ++j)
                Kb(j)[i] += P.a[sc + j] * t;
            }
          }
          else
            for (int32_t i = 0; i < S; ++i)
              Gb(st - 1)[i] += Gb(st)[i];
        }
        if (M.rate_desc)
        {
          Strided rbs[kMaxAdjStages], ks[kMaxAdjStages];
          for (int32_t st = 0; st < ns; ++st)
          {
            rbs[st] = Rb(st);
            ks[st] = K(st);
          }
          step_terms_narrow(M, ns, kk, y, Gb(0), rbs, ks, yb, kb);
        }
        else
        {
          vjp_f_t(M, kk, y, Gb(0), yb, kb);
          for (int32_t st = 0; st < ns; ++st)
            jacobian_term_t(M, kk, y, Rb(st), K(st), yb, kb);
        }
        if (--n < 0)
        {
          finish();
          claim();
        }
      }
    }

    // 96 registers, 5 blocks of 128 per SM, no spills.  A full-occupancy build
    // (32 registers, as the forward kernel's fastest) measured slower here:
    // 1.38 s against 1.16 s on 131,072 cells of the 60-species mechanism, and
    // 67.6 s against 52.5 s on 262,144 cells of the 600-species one, where its
    // larger working-set footprint also leaves less memory for checkpoints.
    __global__ void __launch_bounds__(128, 5)
        k_adjoint_thread(DevMech M, DevParams P, AdjArgs A, AdjThreadLayout T, double* ws)
    {
      adjoint_thread_body(M, P, A, T, ws);
    }

    using AdjThreadKernel = void (*)(DevMech, DevParams, AdjArgs, AdjThreadLayout, double*);

    AdjThreadKernel AdjointThreadKernelFor(const micmb_solver&)
    {
      return k_adjoint_thread;
    }

    // Cells in decreasing order of accepted steps (counting sort on the step
    // count): the backward sweep takes the longest cells first, so the last
    // cells finish together, and the 32 cells of a warp have similar counts.
    __global__ void k_step_histogram(const int32_t* n_ckpt, int64_t n, int32_t max_ckpt, int32_t* bins)
    {
      const int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
      if (c < n)
        atomicAdd(bins + (max_ckpt - min(max(n_ckpt[c], 0), max_ckpt)), 1);
    }

    __global__ void k_step_offsets(int32_t* bins, int32_t n_bins)
    {
      int32_t run = 0;
      for (int32_t b = 0; b < n_bins; ++b)
      {
        const int32_t v = bins[b];
        bins[b] = run;
        run += v;
      }
    }

    __global__ void k_step_scatter(const int32_t* n_ckpt, int64_t n, int32_t max_ckpt, int32_t* cursor,
                                   int32_t* order)
    {
      const int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
      if (c < n)
        order[atomicAdd(cursor + (max_ckpt - min(max(n_ckpt[c], 0), max_ckpt)), 1)] = (int32_t)c;
    }

    // out[r] = sum over cells of kbar[cell][r], in a fixed order (deterministic)
    __global__ void k_sum_cells(const double* kbar, int64_t n_cells, int32_t R, double* out)
    {
      __shared__ double part[256];
      const int32_t r = blockIdx.x;
      double s = 0.0;
      for (int64_t c = threadIdx.x; c < n_cells; c += blockDim.x)
        s += kbar[(size_t)c * R + r];
      part[threadIdx.x] = s;
      __syncthreads();
      for (int w = blockDim.x / 2; w > 0; w >>= 1)
      {
        if ((int)threadIdx.x < w)
          part[threadIdx.x] += part[threadIdx.x + w];
        __syncthreads();
      }
      if (threadIdx.x == 0)
        out[r] = part[0];
    }
  }  // namespace

  namespace
  {
    // arguments for cells [begin, begin + count) of the state; begin is a
    // multiple of L, so every vector-layout array of the chunk starts at
    // begin * columns and is laid out like a state of `count` cells.  The
    // checkpoints hold the chunk's cells only.
    AdjArgs ChunkArgs(micmb_solver& s, micmb_state& st, int32_t max_ckpt, int64_t begin, int64_t count)
    {
      const auto& m = *s.mech;
      AdjArgs A{};
      A.n_cells = count;
      A.L = st.L;
      A.max_ckpt = max_ckpt;
      A.rate_constants = st.rate_constants.as<double>() + (size_t)begin * m.R;
      A.y0 = st.adj_y0.as<double>() + (size_t)begin * m.S;
      A.ybar_final = st.adj_ybar.as<double>() + (size_t)begin * m.S;
      A.ckpt_y = st.adj_ckpt_y.as<double>();
      A.ckpt_h = st.adj_ckpt_h.as<double>();
      A.ckpt_k = st.adj_ckpt_k.p ? st.adj_ckpt_k.as<double>() : nullptr;
      A.n_ckpt = st.accepted.as<int32_t>() + begin;
      A.ybar0 = st.adj_ybar.as<double>() + (size_t)begin * m.S;  // overwritten cell by cell after its last read
      A.kbar = st.adj_kbar_cells.as<double>() + (size_t)begin * m.R;
      char* cbase = st.counters.as<char>();
      A.next_cell = reinterpret_cast<int32_t*>(cbase + 8);
      return A;
    }
  }  // namespace

  // one cell per thread: per-thread working sets in global memory, no atomics
  void LaunchAdjointThread(micmb_solver& s, micmb_state& st, int32_t max_ckpt, int64_t begin, int64_t count)
  {
    const auto& m = *s.mech;
    if (s.params.stages > kMaxAdjStages)
      throw Error(MICMB_ERR_UNSUPPORTED, "too many stages for the adjoint kernel");
    const AdjThreadLayout T = MakeAdjThreadLayout(m.S, m.R, s.params.stages, (int32_t)m.info_rxn.size(), m.nnz);
    const AdjThreadKernel kernel = AdjointThreadKernelFor(s);
    int per_sm = 0;
    MICMB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, 128, 0));
    if (per_sm < 1)
      throw Error(MICMB_ERR_UNSUPPORTED, "adjoint kernel cannot be resident");
    const int64_t n = count;
    int64_t grid = (int64_t)per_sm * s.sm_count;
    grid = std::max<int64_t>(1, std::min<int64_t>(grid, (n + 127) / 128));
    const int64_t doubles = grid * 128 * (int64_t)T.per_slot;
    if (!st.thread_ws.p || st.thread_ws.bytes < (size_t)doubles * sizeof(double))
      st.thread_ws = DeviceMemory((size_t)doubles * sizeof(double));
    AdjArgs A = ChunkArgs(s, st, max_ckpt, begin, count);
    MICMB_CUDA(cudaMemsetAsync(A.next_cell, 0, 8, st.stream));
    if (n > 0)
    {
      const int32_t n_bins = max_ckpt + 1;
      const size_t need = sizeof(int32_t) * ((size_t)n + (size_t)n_bins);
      if (!st.adj_order.p || st.adj_order.bytes < need)
        st.adj_order = DeviceMemory(need);
      int32_t* order = st.adj_order.as<int32_t>();
      int32_t* bins = order + n;
      const unsigned blocks = (unsigned)((n + 255) / 256);
      MICMB_CUDA(cudaMemsetAsync(bins, 0, sizeof(int32_t) * n_bins, st.stream));
      k_step_histogram<<<blocks, 256, 0, st.stream>>>(A.n_ckpt, n, max_ckpt, bins);
      k_step_offsets<<<1, 1, 0, st.stream>>>(bins, n_bins);
      k_step_scatter<<<blocks, 256, 0, st.stream>>>(A.n_ckpt, n, max_ckpt, bins, order);
      MICMB_CUDA(cudaGetLastError());
      A.order = order;
      kernel<<<(unsigned)grid, 128, 0, st.stream>>>(s.dev, s.params, A, T, st.thread_ws.as<double>());
      MICMB_CUDA(cudaGetLastError());
    }
  }

  int64_t AdjointThreadWorkspaceDoubles(const micmb_solver& s, int64_t n_cells)
  {
    const auto& m = *s.mech;
    const AdjThreadLayout T = MakeAdjThreadLayout(m.S, m.R, s.params.stages, (int32_t)m.info_rxn.size(), m.nnz);
    int per_sm = 0;
    MICMB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, AdjointThreadKernelFor(s), 128, 0));
    const int64_t grid = std::max<int64_t>(1, std::min<int64_t>((int64_t)per_sm * s.sm_count, (n_cells + 127) / 128));
    return grid * 128 * (int64_t)T.per_slot;
  }

  void ReduceAdjointParameters(micmb_solver& s, micmb_state& st)
  {
    const auto& m = *s.mech;
    if (m.R > 0)
    {
      k_sum_cells<<<(unsigned)m.R, 256, 0, st.stream>>>(st.adj_kbar_cells.as<double>(), st.n_cells, m.R,
                                                         st.adj_kbar.as<double>());
      MICMB_CUDA(cudaGetLastError());
    }
  }

  void LaunchAdjoint(micmb_solver& s, micmb_state& st, int32_t max_ckpt, int64_t begin, int64_t count)
  {
    LaunchAdjointThread(s, st, max_ckpt, begin, count);
  }
}  // namespace micmb
