// plain.cu -- the per-stage method: one kernel per Rosenbrock stage over all
// grid cells, one thread per cell, data in HBM in micm's vector layout
// (groups of L cells, column-major inside a group, so a warp of consecutive
// cells reads 32 consecutive doubles of a column).  Step control lives on the
// device: per cell (independent adaptive solves) or global (micm's single
// step size, rosenbrock.inl:353-402), so no attempt needs a host round trip.
#include "runtime.hpp"

#include <algorithm>
#include <cmath>
#include <vector>

namespace micmb
{
  namespace
  {
    constexpr int kBlock = 256;

    __device__ __forceinline__ size_t cell_base(int64_t c, int32_t L, int32_t ncol)
    {
      return (size_t)(c / L) * (size_t)L * (size_t)ncol + (size_t)(c % L);
    }

    inline unsigned Blocks(int64_t n, int block = kBlock)
    {
      return (unsigned)std::max<int64_t>(1, (n + block - 1) / block);
    }

    // buffers of the plain path, passed by value
    struct PlainArgs
    {
      int64_t n;
      int32_t L;
      int32_t global;  // 1: one CellCtl for all cells
      double* y;
      double* k;
      double* jac;
      double* f0;
      double* fcur;
      double* ynew;
      double* K;        // stages * S columns
      double* scratch;  // max(R, n_info) columns
      double* inv;      // S columns
      double* err_cell; // [n]
      const double* atol;
      double rtol;
      CellCtl* ctl;
      int32_t* status;  // [n] (per-cell) or [1]
      int32_t scratch_cols;
      const double* keq;  // K_eq per cell (equilibrium constraints)
      double* cjac;       // constraint Jacobian terms per cell
    };

    __device__ __forceinline__ Strided keq_of(const DevMech& M, const PlainArgs& a, int64_t c)
    {
      return Strided{ const_cast<double*>(a.keq) + cell_base(c, a.L, M.n_eq), a.L };
    }
    __device__ __forceinline__ Strided cjac_of(const DevMech& M, const PlainArgs& a, int64_t c)
    {
      return Strided{ a.cjac + cell_base(c, a.L, M.n_cterms), a.L };
    }

    __device__ __forceinline__ CellCtl* ctl_of(const PlainArgs& a, int64_t c)
    {
      return a.global ? a.ctl : a.ctl + c;
    }

    __device__ __forceinline__ bool running(const PlainArgs& a, int64_t c)
    {
      return a.status[a.global ? 0 : c] == MICMB_SOLVER_RUNNING;
    }

    __global__ void k_rate_constants(DevMech M, const double* __restrict__ cond, const double* __restrict__ params,
                                     double* __restrict__ k, int64_t n_pad, int32_t L)
    {
      const int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
      const int64_t per_group = (int64_t)M.R * L;
      if (idx >= n_pad * M.R)
        return;
      const int64_t g = idx / per_group;
      const int64_t rem = idx - g * per_group;
      const int32_t r = (int32_t)(rem / L);
      const int32_t l = (int32_t)(rem - (int64_t)r * L);
      const double* cb = cond + (size_t)g * 3 * L + l;
      const double* pb = params + (size_t)g * (size_t)M.P * L + l;
      auto param = [&](int32_t col) { return pb[(size_t)col * L]; };
      k[idx] = rate_constant(M, r, cb[0], cb[L], cb[2 * L], param);
    }

    // K_eq(T) per cell and equilibrium constraint (equilibrium_constraint.hpp:290-309;
    // micm computes it in UpdateStateParameters)
    __global__ void k_constraint_keq(DevMech M, const double* __restrict__ cond, double* __restrict__ keq,
                                     int64_t n_pad, int32_t L)
    {
      const int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
      const int64_t per_group = (int64_t)M.n_eq * L;
      if (idx >= n_pad * M.n_eq)
        return;
      const int64_t g = idx / per_group;
      const int64_t rem = idx - g * per_group;
      const int32_t q = (int32_t)(rem / L);
      const int32_t l = (int32_t)(rem - (int64_t)q * L);
      const double T = cond[(size_t)g * 3 * L + l];
      for (int32_t c = 0; c < M.n_constraints; ++c)
        if (M.con[c].x == MICMB_CONSTRAINT_EQUILIBRIUM && M.con_eq[c].y == q)
          keq[idx] = constraint_keq(M, c, T);
    }

    __global__ void k_init_ctl(CellCtl* ctl, int32_t* status, int64_t n, StepBounds b)
    {
      const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
      if (i >= n)
        return;
      CellCtl c;
      ctl_init(c, b);
      ctl[i] = c;
      status[i] = MICMB_SOLVER_RUNNING;
    }

    // top of the outer step loop for cells that just accepted (or start)
    __global__ void k_step_begin(PlainArgs a, DevParams P, StepBounds b, int64_t n_ctl)
    {
      const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
      if (i >= n_ctl || a.status[i] != MICMB_SOLVER_RUNNING)
        return;
      CellCtl c = a.ctl[i];
      if (!c.new_step)
        return;
      if (!ctl_begin_step(c, P, b))
      {
        a.status[i] = c.state;
        c.new_step = 0;
      }
      else
      {
        c.function_calls += 1;    // initial forcing
        c.jacobian_updates += 1;  // Jacobian at the start of the step
      }
      a.ctl[i] = c;
    }

    // F0 = f(Y) for cells starting a step
    template<bool DAE>
    __global__ void k_forcing0(DevMech M, PlainArgs a)
    {
      const int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
      if (c >= a.n || !running(a, c) || !ctl_of(a, c)->new_step)
        return;
      const int32_t L = a.L;
      Strided y{ a.y + cell_base(c, L, M.S), L };
      Strided k{ a.k + cell_base(c, L, M.R), L };
      Strided rate{ a.scratch + cell_base(c, L, a.scratch_cols), L };
      Strided f{ a.f0 + cell_base(c, L, M.S), L };
      reaction_rates<1>(M, k, y, rate, 0);
      forcing_gather<1>(M, rate, f, 0);
      if constexpr (DAE)
        constraint_forcing(M, keq_of(M, a, c), y, f);
    }

    // alpha I - J at Y for every running cell (micm re-assembles after a rejection)
    template<bool DAE>
    __global__ void k_jacobian(DevMech M, PlainArgs a, double gamma0)
    {
      const int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
      if (c >= a.n || !running(a, c))
        return;
      const int32_t L = a.L;
      const double H = ctl_of(a, c)->H;
      const double alpha = 1.0 / (H * gamma0);
      Strided y{ a.y + cell_base(c, L, M.S), L };
      Strided k{ a.k + cell_base(c, L, M.R), L };
      Strided dr{ a.scratch + cell_base(c, L, a.scratch_cols), L };
      Strided J{ a.jac + cell_base(c, L, M.nnz), L };
      jacobian_rates<1>(M, k, y, dr, 0);
      if constexpr (DAE)
      {
        const Strided cj = cjac_of(M, a, c);
        constraint_jacobian(M, keq_of(M, a, c), y, cj);
        jacobian_gather<1>(M, dr, J, alpha, true, 0, cj);
      }
      else
        jacobian_gather<1>(M, dr, J, alpha, true, 0);
    }

    __global__ void k_decompose(DevMech M, PlainArgs a)
    {
      const int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
      if (c >= a.n || !running(a, c))
        return;
      const int32_t L = a.L;
      Strided J{ a.jac + cell_base(c, L, M.nnz), L };
      Strided inv{ a.inv + cell_base(c, L, M.S), L };
      thread_lu(M, J, inv);
    }

    // Ynew = Y + sum_j a_sj K_j ; Fcur = f(Ynew)
    template<bool DAE>
    __global__ void k_stage_forcing(DevMech M, PlainArgs a, DevParams P, int32_t s)
    {
      const int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
      if (c >= a.n || !running(a, c))
        return;
      const int32_t L = a.L, S = M.S;
      const size_t bs = cell_base(c, L, S);
      Strided y{ a.y + bs, L };
      Strided yn{ a.ynew + bs, L };
      const int32_t sc = s * (s - 1) / 2;
      for (int32_t i = 0; i < S; ++i)
      {
        double v = y[i];
        for (int32_t j = 0; j < s; ++j)
          v += P.a[sc + j] * a.K[cell_base(c, L, P.stages * S) + (size_t)(j * S + i) * L];
        yn[i] = v;
      }
      Strided k{ a.k + cell_base(c, L, M.R), L };
      Strided rate{ a.scratch + cell_base(c, L, a.scratch_cols), L };
      Strided f{ a.fcur + bs, L };
      reaction_rates<1>(M, k, yn, rate, 0);
      forcing_gather<1>(M, rate, f, 0);
      if constexpr (DAE)
        constraint_forcing(M, keq_of(M, a, c), yn, f);
    }

    // K_s = F + sum_j (c_sj / H) K_j ; K_s = (LU)^-1 K_s
    template<bool DAE>
    __global__ void k_stage_solve(DevMech M, PlainArgs a, DevParams P, int32_t s, int32_t src_is_f0)
    {
      const int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
      if (c >= a.n || !running(a, c))
        return;
      const int32_t L = a.L, S = M.S;
      const double H = ctl_of(a, c)->H;
      const size_t bs = cell_base(c, L, S);
      const size_t bk = cell_base(c, L, P.stages * S);
      Strided F{ (src_is_f0 ? a.f0 : a.fcur) + bs, L };
      Strided Ks{ a.K + bk + (size_t)s * S * L, L };
      const int32_t sc = s * (s - 1) / 2;
      double coh[6];
      for (int32_t j = 0; j < s; ++j)
        coh[j] = P.c[sc + j] / H;
      for (int32_t i = 0; i < S; ++i)
      {
        double v = F[i];
        if (!DAE || M.mass[i] != 0.0)  // algebraic rows have no mass coupling
          for (int32_t j = 0; j < s; ++j)
            v += coh[j] * a.K[bk + (size_t)(j * S + i) * L];
        Ks[i] = v;
      }
      Strided J{ a.jac + cell_base(c, L, M.nnz), L };
      thread_solve(M, J, Ks);
    }

    // Ynew = Y + sum m_s K_s ; Yerr = sum e_s K_s ; the cell's sum of scaled
    // squared errors in species order (micm's order).
    template<bool DAE>
    __device__ double finish_cell(const DevMech& M, const PlainArgs& a, const DevParams& P, int64_t c)
    {
      const int32_t L = a.L, S = M.S;
      const size_t bs = cell_base(c, L, S);
      const size_t bk = cell_base(c, L, P.stages * S);
      Strided y{ a.y + bs, L };
      Strided yn{ a.ynew + bs, L };
      double sum = 0.0;
      for (int32_t i = 0; i < S; ++i)
      {
        double v = y[i];
        double e = 0.0;
        for (int32_t st = 0; st < P.stages; ++st)
        {
          const double kv = a.K[bk + (size_t)(st * S + i) * L];
          v += P.m[st] * kv;
          e += P.e[st] * kv;
        }
        yn[i] = v;
        if (DAE && M.mass[i] == 0.0)
          e = v - y[i];  // SetAlgebraicErrors: the step change
        sum += scaled_sq(y[i], v, e, a.atol[i], a.rtol);
      }
      return sum;
    }

    // per-cell step control with constraints: micm's constraint initialisation of each cell
    __global__ void k_constraint_init_per_cell(DevMech M, PlainArgs a, DevParams P)
    {
      const int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
      if (c >= a.n)
        return;
      const int32_t L = a.L;
      Strided y{ a.y + cell_base(c, L, M.S), L };
      Strided delta{ a.f0 + cell_base(c, L, M.S), L };
      Strided J{ a.jac + cell_base(c, L, M.nnz), L };
      Strided inv{ a.inv + cell_base(c, L, M.S), L };
      CellCtl cc = a.ctl[c];
      const int32_t st = constraint_init_cell(M, P, keq_of(M, a, c), y, delta, J, inv, cjac_of(M, a, c), cc);
      if (st != MICMB_SOLVER_CONVERGED)
      {
        cc.state = st;
        cc.new_step = 0;
        a.status[c] = st;
      }
      a.ctl[c] = cc;
    }

    // Global step control with constraints: micm's InitializeConstraints on an
    // n-cell State (rosenbrock.inl:407-576).  Iteration `it` has three words
    // in `slots` (zeroed before the first): [3it] the largest finite |G| over
    // every cell's algebraic rows (the bits of a non-negative double, so an
    // integer atomicMax orders them), [3it+1] the residual's NaN (1) / Inf (2)
    // flags, [3it+2] the Newton update's flags.  Every kernel replays the
    // decisions of the iterations before its own from these words, so the
    // grid agrees without a host round trip.
    __device__ __forceinline__ bool cinit_continues(const unsigned long long* slots, int32_t it, double tol)
    {
      for (int32_t j = 0; j < it; ++j)
        if (slots[3 * j + 1] || __longlong_as_double((long long)slots[3 * j]) < tol || slots[3 * j + 2])
          return false;
      return true;
    }

    __device__ __forceinline__ void warp_flags_max(unsigned long long* slot_max, unsigned long long* slot_flags,
                                                   double v, unsigned flags)
    {
      for (int off = 16; off > 0; off >>= 1)
      {
        const double o = __shfl_xor_sync(0xffffffffu, v, off);
        v = o > v ? o : v;
        flags |= __shfl_xor_sync(0xffffffffu, flags, off);
      }
      if ((threadIdx.x & 31) == 0)
      {
        if (slot_max && v > 0.0)
          atomicMax(slot_max, (unsigned long long)__double_as_longlong(v));
        if (flags)
          atomicOr(slot_flags, (unsigned long long)flags);
      }
    }

    // G(y) per cell into f0; the grid's largest finite |G| and flags
    __global__ void k_cinit_residual(DevMech M, PlainArgs a, DevParams P, unsigned long long* slots, int32_t it)
    {
      if (!cinit_continues(slots, it, P.cinit_tol))
        return;  // uniform over the grid
      const int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
      double max_res = 0.0;
      unsigned flags = 0;
      if (c < a.n)
      {
        const int32_t L = a.L;
        Strided y{ a.y + cell_base(c, L, M.S), L };
        Strided delta{ a.f0 + cell_base(c, L, M.S), L };
        for (int32_t i = 0; i < M.S; ++i)
          delta[i] = 0.0;
        constraint_forcing(M, keq_of(M, a, c), y, delta);
        for (int32_t i = 0; i < M.S; ++i)
          if (M.mass[i] == 0.0)
          {
            const double v = delta[i];
            flags |= isnan(v) ? 1u : (isinf(v) ? 2u : 0u);
            const double av = fabs(v);
            if (!isnan(av) && !isinf(av))
              max_res = (max_res > av ? max_res : av);
          }
      }
      warp_flags_max(slots + 3 * it, slots + 3 * it + 1, max_res, flags);
    }

    // the Newton update of every cell when iteration `it` neither stopped nor converged
    __global__ void k_cinit_update(DevMech M, PlainArgs a, DevParams P, unsigned long long* slots, int32_t it)
    {
      if (!cinit_continues(slots, it, P.cinit_tol) || slots[3 * it + 1] ||
          __longlong_as_double((long long)slots[3 * it]) < P.cinit_tol)
        return;  // uniform over the grid
      const int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
      unsigned flags = 0;
      if (c < a.n)
      {
        const int32_t L = a.L;
        Strided y{ a.y + cell_base(c, L, M.S), L };
        Strided delta{ a.f0 + cell_base(c, L, M.S), L };
        Strided A{ a.jac + cell_base(c, L, M.nnz), L };
        Strided inv{ a.inv + cell_base(c, L, M.S), L };
        const Strided cj = cjac_of(M, a, c);
        constraint_jacobian(M, keq_of(M, a, c), y, cj);
        lu_decompose_gathered<false>(M, M.lu_s, M.diag_row_of, cj, 1.0, A, inv, cj);
        solve_lower<1>(M.fwd_s, A, delta, 0);
        solve_upper<1>(M.bwd_s, A, delta, 0);
        for (int32_t i = 0; i < M.S; ++i)
          if (M.mass[i] == 0.0)
          {
            const double d = delta[i];
            flags |= isnan(d) ? 1u : (isinf(d) ? 2u : 0u);
            if (!isnan(d) && !isinf(d))
              y[i] = y[i] + d;
          }
      }
      warp_flags_max(nullptr, slots + 3 * it + 2, 0.0, flags);
    }

    // Several ranks: word `w` of iteration `it` encoded for the all-gather (NaN,
    // +Inf, else the maximum; the update's word carries flags only) ...
    __global__ void k_cinit_encode(const unsigned long long* slots, int32_t it, int32_t w, double* out)
    {
      const unsigned long long f = slots[3 * it + w];
      const double mx = (w == 1) ? __longlong_as_double((long long)slots[3 * it]) : 0.0;
      *out = (f & 1u) ? __longlong_as_double(0x7ff8000000000000LL)
                      : ((f & 2u) ? __longlong_as_double(0x7ff0000000000000LL) : mx);
    }

    // ... and the ranks' values combined in rank order (NaN first, then +Inf,
    // else the largest) back into the words, so every rank decides alike.
    __global__ void k_cinit_decode(unsigned long long* slots, int32_t it, int32_t w, const double* gathered,
                                   int32_t world)
    {
      double v = 0.0;
      for (int32_t r = 0; r < world; ++r)
      {
        const double g = gathered[r];
        if (isnan(v) || isnan(g))
          v = __longlong_as_double(0x7ff8000000000000LL);
        else if (isinf(v) || isinf(g))
          v = __longlong_as_double(0x7ff0000000000000LL);
        else
          v = g > v ? g : v;
      }
      slots[3 * it + w] = isnan(v) ? 1ull : (isinf(v) ? 2ull : 0ull);
      if (w == 1)
        slots[3 * it] = (isnan(v) || isinf(v)) ? 0ull : (unsigned long long)__double_as_longlong(v);
    }

    // the State's outcome and counts from the words (one thread)
    __global__ void k_cinit_finish(PlainArgs a, DevParams P, const unsigned long long* slots)
    {
      CellCtl cc = a.ctl[0];
      int32_t state = MICMB_SOLVER_CONSTRAINT_INITIALIZATION_FAILED;
      for (int32_t it = 0; it < P.cinit_max_iter; ++it)
      {
        const unsigned long long f = slots[3 * it + 1], u = slots[3 * it + 2];
        if (f & 1u)
        {
          state = MICMB_SOLVER_NAN_DETECTED;
          break;
        }
        if (f & 2u)
        {
          state = MICMB_SOLVER_INF_DETECTED;
          break;
        }
        cc.init_iterations = it + 1;
        if (__longlong_as_double((long long)slots[3 * it]) < P.cinit_tol)
        {
          state = MICMB_SOLVER_CONVERGED;
          break;
        }
        cc.jacobian_updates += 1;
        cc.decompositions += 1;
        cc.solves += 1;
        if (u & 1u)
        {
          state = MICMB_SOLVER_NAN_DETECTED;
          break;
        }
        if (u & 2u)
        {
          state = MICMB_SOLVER_INF_DETECTED;
          break;
        }
      }
      if (state != MICMB_SOLVER_CONVERGED)
      {
        cc.state = state;
        cc.new_step = 0;
        a.status[0] = state;
      }
      a.ctl[0] = cc;
    }

    __device__ __forceinline__ void count_attempt(CellCtl& cc, const DevParams& P)
    {
      cc.decompositions += 1;
      cc.solves += P.stages;
      for (int32_t s = 1; s < P.stages; ++s)
        cc.function_calls += P.new_f[s] ? 1 : 0;
    }

    template<bool DAE>
    __global__ void k_finish_per_cell(DevMech M, PlainArgs a, DevParams P, StepBounds b)
    {
      const int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
      if (c >= a.n || !running(a, c))
        return;
      const double error = error_from_sum(finish_cell<DAE>(M, a, P, c), (double)M.S);
      CellCtl cc = a.ctl[c];
      count_attempt(cc, P);
      const int res = ctl_after_error(cc, P, b, error);
      if (res == 1)
      {
        const int32_t L = a.L;
        const size_t bs = cell_base(c, L, M.S);
        for (int32_t i = 0; i < M.S; ++i)
          a.y[bs + (size_t)i * L] = a.ynew[bs + (size_t)i * L];
      }
      a.status[c] = cc.state;
      a.ctl[c] = cc;
    }

    // Fixed-shape tree over the kBlock values of a block (thread 0 returns the total).
    __device__ __forceinline__ double block_tree_sum(double v, double* red)
    {
      red[threadIdx.x] = v;
      __syncthreads();
      for (int w = kBlock / 2; w > 0; w >>= 1)
      {
        if ((int)threadIdx.x < w)
          red[threadIdx.x] += red[threadIdx.x + w];
        __syncthreads();
      }
      return red[0];
    }

    // Global mode, first level: each cell's sum in species order, then one
    // partial per block (fixed tree over its kBlock cells) in blk_err[block].
    // A single cell's error therefore equals micm's bit for bit.
    template<bool DAE>
    __global__ void k_finish_partial(DevMech M, PlainArgs a, DevParams P, double* blk_err)
    {
      __shared__ double red[kBlock];
      const int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
      if (a.status[0] != MICMB_SOLVER_RUNNING)
        return;  // uniform over the grid in global mode
      const double v = (c < a.n) ? finish_cell<DAE>(M, a, P, c) : 0.0;
      const double t = block_tree_sum(v, red);
      if (threadIdx.x == 0)
        blk_err[blockIdx.x] = t;
    }

    // The block partials reduced in a fixed order by one block: each thread a
    // strided sequential sum, then a fixed tree.  Deterministic for a given
    // cell count.
    __device__ __forceinline__ double reduce_blocks(const double* blk_err, int64_t n_blk, double* red)
    {
      double acc = 0.0;
      for (int64_t i = threadIdx.x; i < n_blk; i += kBlock)
        acc += blk_err[i];
      return block_tree_sum(acc, red);
    }

    // micm's step control from the job's sum of squared scaled errors
    __device__ __forceinline__ void global_decide(const PlainArgs& a, const DevParams& P, const StepBounds& b,
                                                  double total, double n_values, int32_t* last_accept)
    {
      const double error = error_from_sum(total, n_values > 0.0 ? n_values : 1.0);
      CellCtl cc = a.ctl[0];
      count_attempt(cc, P);
      const int res = ctl_after_error(cc, P, b, error);
      *last_accept = (res == 1);
      a.status[0] = cc.state;
      a.ctl[0] = cc;
    }

    // Global decision on one GPU: all cells' partials, then the step control.
    __global__ void k_global_decide(PlainArgs a, DevParams P, StepBounds b, int32_t S, const double* blk_err,
                                    int64_t n_blk, int32_t* last_accept)
    {
      __shared__ double red[kBlock];
      if (a.status[0] != MICMB_SOLVER_RUNNING)
        return;
      const double total = reduce_blocks(blk_err, n_blk, red);
      if (threadIdx.x == 0)
        global_decide(a, P, b, total, (double)(a.n * (int64_t)S), last_accept);
    }

    // Several ranks, first half: this shard's sum (the same reduction), for the exchange.
    __global__ void k_shard_sum(PlainArgs a, const double* blk_err, int64_t n_blk, double* shard_sum)
    {
      __shared__ double red[kBlock];
      if (a.status[0] != MICMB_SOLVER_RUNNING)
        return;
      const double total = reduce_blocks(blk_err, n_blk, red);
      if (threadIdx.x == 0)
        *shard_sum = total;
    }

    // Several ranks, second half: the gathered shard sums added in rank order.
    __global__ void k_global_decide_gathered(PlainArgs a, DevParams P, StepBounds b, const double* gathered,
                                             int32_t world, double n_values, int32_t* last_accept)
    {
      if (a.status[0] != MICMB_SOLVER_RUNNING)
        return;
      double total = 0.0;
      for (int32_t r = 0; r < world; ++r)
        total += gathered[r];
      global_decide(a, P, b, total, n_values, last_accept);
    }

    __global__ void k_global_apply(DevMech M, PlainArgs a, const int32_t* last_accept)
    {
      const int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
      if (c >= a.n || !*last_accept)
        return;
      const int32_t L = a.L;
      const size_t bs = cell_base(c, L, M.S);
      for (int32_t i = 0; i < M.S; ++i)
        a.y[bs + (size_t)i * L] = a.ynew[bs + (size_t)i * L];
    }

    __global__ void k_count_running(const int32_t* status, int64_t n, int32_t* count)
    {
      const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
      const bool r = i < n && status[i] == MICMB_SOLVER_RUNNING;
      const unsigned ballot = __ballot_sync(0xffffffffu, r);
      if ((threadIdx.x & 31) == 0 && ballot)
        atomicAdd(count, __popc(ballot));
    }

    // Solver::PostSolveClamp (solver.hpp:275-297) over real cells
    __global__ void k_clamp(DevMech M, double* y, int64_t n, int32_t L)
    {
      const int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
      const int64_t per_group = (int64_t)M.S * L;
      const int64_t g = idx / per_group;
      const int32_t l = (int32_t)(idx % L);
      if (g * L + l >= n)
        return;
      const int32_t i = (int32_t)((idx - g * per_group) / L);
      y[idx] = post_clamp(M, i, y[idx]);
    }

    // stats reduction over per-cell controls
    __global__ void k_reduce_stats(const CellCtl* ctl, const int32_t* status, int64_t n,
                                   unsigned long long* acc, int32_t* cell_status, int32_t* cell_accepted)
    {
      const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
      long long v[9] = { 0 };
      if (i < n)
      {
        const CellCtl c = ctl[i];
        v[0] = c.function_calls;
        v[1] = c.jacobian_updates;
        v[2] = c.number_of_steps;
        v[3] = c.accepted;
        v[4] = c.rejected;
        v[5] = c.decompositions;
        v[6] = c.solves;
        v[7] = (status[i] == MICMB_SOLVER_CONVERGED) ? 0 : 1;
        v[8] = c.init_iterations;
        if (cell_status)
          cell_status[i] = status[i];
        if (cell_accepted)
          cell_accepted[i] = c.accepted;
      }
#pragma unroll
      for (int q = 0; q < 9; ++q)
      {
        long long s = v[q];
        for (int off = 16; off > 0; off >>= 1)
          s += __shfl_xor_sync(0xffffffffu, s, off);
        if ((threadIdx.x & 31) == 0 && s)
          atomicAdd(acc + q, (unsigned long long)s);
      }
    }

    PlainArgs MakeArgs(micmb_solver& s, micmb_state& st, int32_t global)
    {
      const auto& m = *s.mech;
      PlainArgs a{};
      a.n = st.n_cells;
      a.L = st.L;
      a.global = global;
      a.y = st.variables.as<double>();
      a.k = st.rate_constants.as<double>();
      a.jac = st.jacobian.as<double>();
      a.f0 = st.forcing0.as<double>();
      a.fcur = st.fcur.as<double>();
      a.ynew = st.ynew.as<double>();
      a.K = st.stages.as<double>();
      a.scratch = st.scratch.as<double>();
      a.inv = st.inv_diag.as<double>();
      a.err_cell = st.err_cell.as<double>();
      a.atol = st.atol.as<double>();
      a.rtol = st.rtol;
      a.ctl = st.ctl.as<CellCtl>();
      a.status = st.status.as<int32_t>();
      a.scratch_cols = std::max<int32_t>(m.R, (int32_t)m.info_rxn.size());
      a.keq = st.keq.as<double>();
      a.cjac = st.cjac.as<double>();
      return a;
    }
  }  // namespace

  void EnsurePlainBuffers(micmb_state& st)
  {
    const auto& m = *st.solver->mech;
    const int32_t S = m.S;
    if (!st.jacobian.p)
    {
      st.jacobian = DeviceMemory(st.dense_bytes(m.nnz));
      st.forcing0 = DeviceMemory(st.dense_bytes(S));
      st.fcur = DeviceMemory(st.dense_bytes(S));
      st.ynew = DeviceMemory(st.dense_bytes(S));
      st.stages = DeviceMemory(st.dense_bytes(6 * S));
      st.scratch = DeviceMemory(st.dense_bytes(std::max<int32_t>(std::max<int32_t>(m.R, (int32_t)m.info_rxn.size()), 1)));
      st.inv_diag = DeviceMemory(st.dense_bytes(S));
      st.err_cell = DeviceMemory(sizeof(double) * std::max<int64_t>(st.n_cells, 1));
      if (!m.c_term_col.empty())
        st.cjac = DeviceMemory(st.dense_bytes((int32_t)m.c_term_col.size()));
      MICMB_CUDA(cudaMemsetAsync(st.jacobian.p, 0, st.jacobian.bytes, st.stream));
      MICMB_CUDA(cudaMemsetAsync(st.forcing0.p, 0, st.forcing0.bytes, st.stream));
      MICMB_CUDA(cudaMemsetAsync(st.ynew.p, 0, st.ynew.bytes, st.stream));
    }
    if (!st.ctl.p)
    {
      st.ctl = DeviceMemory(sizeof(CellCtl) * std::max<int64_t>(st.n_cells, 1));
      st.status = DeviceMemory(sizeof(int32_t) * std::max<int64_t>(st.n_cells, 1));
    }
  }

  void LaunchRateConstants(micmb_solver& s, micmb_state& st)
  {
    const int64_t total = st.n_pad * s.mech->R;
    if (total > 0)
    {
      k_rate_constants<<<Blocks(total), kBlock, 0, st.stream>>>(s.dev, st.conditions.as<double>(),
                                                                st.custom_params.as<double>(),
                                                                st.rate_constants.as<double>(), st.n_pad, st.L);
      MICMB_CUDA(cudaGetLastError());
    }
    const int64_t n_keq = st.n_pad * s.mech->n_eq;
    if (n_keq > 0)
    {
      k_constraint_keq<<<Blocks(n_keq), kBlock, 0, st.stream>>>(s.dev, st.conditions.as<double>(),
                                                                st.keq.as<double>(), st.n_pad, st.L);
      MICMB_CUDA(cudaGetLastError());
    }
  }

  namespace
  {
    // one word of a constraint-initialisation iteration through the state's all-gather hook
    void ExchangeInitWord(micmb_state& st, unsigned long long* slots, int32_t it, int32_t w, cudaStream_t stream)
    {
      double* gx = st.gx_buf.as<double>();
      k_cinit_encode<<<1, 1, 0, stream>>>(slots, it, w, gx);
      MICMB_CUDA(cudaGetLastError());
      if (st.gx_fn(gx, gx + 1, st.gx_world, stream, st.gx_user) != 0)
        throw Error(MICMB_ERR_INTERNAL, "global step control: the all-gather of the constraint residuals failed");
      k_cinit_decode<<<1, 1, 0, stream>>>(slots, it, w, gx + 1, st.gx_world);
      MICMB_CUDA(cudaGetLastError());
    }
  }  // namespace

  void SolvePlain(micmb_solver& s, micmb_state& st, double dt, int32_t step_control, micmb_solver_stats* stats,
                  int32_t* per_cell_status, int32_t* per_cell_accepted)
  {
    EnsurePlainBuffers(st);
    const auto& m = *s.mech;
    const DevParams P = s.params;
    const StepBounds b = step_bounds(P, dt);
    const int32_t global = step_control == MICMB_STEP_GLOBAL ? 1 : 0;
    const int64_t n = st.n_cells;
    const int64_t n_ctl = global ? 1 : n;
    PlainArgs a = MakeArgs(s, st, global);
    cudaStream_t stream = st.stream;
    int32_t* dcount = st.counters.as<int32_t>();
    int32_t* last_accept = dcount + 1;
    unsigned long long* dstats = reinterpret_cast<unsigned long long*>(st.counters.as<char>() + 64);

    k_init_ctl<<<Blocks(n_ctl), kBlock, 0, stream>>>(a.ctl, a.status, n_ctl, b);
    MICMB_CUDA(cudaGetLastError());
    if (n == 0)
      return;
    if (!m.constraints.empty() && !global)
    {
      k_constraint_init_per_cell<<<Blocks(n), kBlock, 0, stream>>>(s.dev, a, P);
      MICMB_CUDA(cudaGetLastError());
    }
    else if (!m.constraints.empty())
    {
      const int32_t iters = std::max<int32_t>(P.cinit_max_iter, 0);
      const size_t slot_bytes = sizeof(unsigned long long) * 3 * (size_t)std::max<int32_t>(iters, 1);
      if (!st.cinit_slots.p || st.cinit_slots.bytes < slot_bytes)
        st.cinit_slots = DeviceMemory(slot_bytes);
      auto* slots = st.cinit_slots.as<unsigned long long>();
      MICMB_CUDA(cudaMemsetAsync(slots, 0, slot_bytes, stream));
      for (int32_t it = 0; it < iters; ++it)
      {
        k_cinit_residual<<<Blocks(n), kBlock, 0, stream>>>(s.dev, a, P, slots, it);
        MICMB_CUDA(cudaGetLastError());
        if (st.gx_fn)
          ExchangeInitWord(st, slots, it, 1, stream);
        k_cinit_update<<<Blocks(n), kBlock, 0, stream>>>(s.dev, a, P, slots, it);
        MICMB_CUDA(cudaGetLastError());
        if (st.gx_fn)
          ExchangeInitWord(st, slots, it, 2, stream);
      }
      k_cinit_finish<<<1, 1, 0, stream>>>(a, P, slots);
      MICMB_CUDA(cudaGetLastError());
    }
    // which forcing each stage's right-hand side reads (rosenbrock.inl:140-195)
    std::vector<int32_t> src_is_f0(P.stages, 1);
    {
      bool have_fcur = false;
      for (int32_t st_i = 1; st_i < P.stages; ++st_i)
      {
        if (P.new_f[st_i])
          have_fcur = true;
        src_is_f0[st_i] = have_fcur ? 0 : 1;
      }
    }
    const unsigned grid = Blocks(n);
    // mechanisms with constraints run their own instantiations of the stage
    // kernels, so the constraint code costs the ODE kernels no registers
    const bool dae = !m.constraints.empty();
    int64_t attempts = 0;
    int64_t batch = 8;
    const int64_t max_attempts = (int64_t)(P.max_steps + 2) * 2000;
    for (;;)
    {
      for (int64_t it = 0; it < batch; ++it)
      {
        k_step_begin<<<Blocks(n_ctl), kBlock, 0, stream>>>(a, P, b, n_ctl);
        (dae ? k_forcing0<true> : k_forcing0<false>)<<<grid, kBlock, 0, stream>>>(s.dev, a);
        (dae ? k_jacobian<true> : k_jacobian<false>)<<<grid, kBlock, 0, stream>>>(s.dev, a, P.gamma0);
        k_decompose<<<grid, kBlock, 0, stream>>>(s.dev, a);
        for (int32_t stg = 0; stg < P.stages; ++stg)
        {
          if (stg > 0 && P.new_f[stg])
            (dae ? k_stage_forcing<true> : k_stage_forcing<false>)<<<grid, kBlock, 0, stream>>>(s.dev, a, P, stg);
          (dae ? k_stage_solve<true> : k_stage_solve<false>)<<<grid, kBlock, 0, stream>>>(s.dev, a, P, stg,
                                                                                          src_is_f0[stg]);
        }
        if (global)
        {
          (dae ? k_finish_partial<true> : k_finish_partial<false>)<<<grid, kBlock, 0, stream>>>(s.dev, a, P,
                                                                                                a.err_cell);
          if (st.gx_fn)
          {
            double* gx = st.gx_buf.as<double>();
            k_shard_sum<<<1, kBlock, 0, stream>>>(a, a.err_cell, (int64_t)grid, gx);
            MICMB_CUDA(cudaGetLastError());
            if (st.gx_fn(gx, gx + 1, st.gx_world, stream, st.gx_user) != 0)
              throw Error(MICMB_ERR_INTERNAL, "global step control: the all-gather of the error sums failed");
            k_global_decide_gathered<<<1, 1, 0, stream>>>(a, P, b, gx + 1, st.gx_world,
                                                          (double)st.gx_total_cells * (double)m.S, last_accept);
          }
          else
            k_global_decide<<<1, kBlock, 0, stream>>>(a, P, b, m.S, a.err_cell, (int64_t)grid, last_accept);
          k_global_apply<<<grid, kBlock, 0, stream>>>(s.dev, a, last_accept);
        }
        else
          (dae ? k_finish_per_cell<true> : k_finish_per_cell<false>)<<<grid, kBlock, 0, stream>>>(s.dev, a, P, b);
        MICMB_CUDA(cudaGetLastError());
      }
      attempts += batch;
      // one host round trip per batch: stop when no cell is running
      MICMB_CUDA(cudaMemsetAsync(dcount, 0, sizeof(int32_t), stream));
      k_count_running<<<Blocks(n_ctl), kBlock, 0, stream>>>(a.status, n_ctl, dcount);
      MICMB_CUDA(cudaMemcpyAsync(st.host_counters, dcount, sizeof(int32_t), cudaMemcpyDeviceToHost, stream));
      MICMB_CUDA(cudaStreamSynchronize(stream));
      if (st.host_counters[0] == 0)
        break;
      if (attempts > max_attempts)
        throw Error(MICMB_ERR_INTERNAL, "plain solve did not terminate");
      batch = std::min<int64_t>(batch * 2, 64);
    }
    const int64_t total = st.n_pad * m.S;
    k_clamp<<<Blocks(total), kBlock, 0, stream>>>(s.dev, a.y, n, st.L);
    MICMB_CUDA(cudaMemsetAsync(dstats, 0, 9 * sizeof(unsigned long long), stream));
    k_reduce_stats<<<Blocks(n_ctl), kBlock, 0, stream>>>(a.ctl, a.status, n_ctl, dstats, nullptr, nullptr);
    MICMB_CUDA(cudaGetLastError());
    unsigned long long hs[9];
    MICMB_CUDA(cudaMemcpyAsync(hs, dstats, sizeof(hs), cudaMemcpyDeviceToHost, stream));
    CellCtl c0{};
    if (global)
      MICMB_CUDA(cudaMemcpyAsync(&c0, a.ctl, sizeof(CellCtl), cudaMemcpyDeviceToHost, stream));
    MICMB_CUDA(cudaStreamSynchronize(stream));
    if (per_cell_status || per_cell_accepted)
    {
      std::vector<int32_t> stv(n_ctl);
      std::vector<CellCtl> cv(n_ctl);
      MICMB_CUDA(cudaMemcpy(stv.data(), a.status, sizeof(int32_t) * n_ctl, cudaMemcpyDeviceToHost));
      MICMB_CUDA(cudaMemcpy(cv.data(), a.ctl, sizeof(CellCtl) * n_ctl, cudaMemcpyDeviceToHost));
      for (int64_t c = 0; c < n; ++c)
      {
        const int64_t i = global ? 0 : c;
        if (per_cell_status)
          per_cell_status[c] = stv[i];
        if (per_cell_accepted)
          per_cell_accepted[c] = cv[i].accepted;
      }
    }
    if (stats)
    {
      stats->function_calls = (int64_t)hs[0];
      stats->jacobian_updates = (int64_t)hs[1];
      stats->number_of_steps = (int64_t)hs[2];
      stats->accepted = (int64_t)hs[3];
      stats->rejected = (int64_t)hs[4];
      stats->decompositions = (int64_t)hs[5];
      stats->solves = (int64_t)hs[6];
      stats->cells_not_converged = global ? (hs[7] ? (int32_t)n : 0) : (int32_t)hs[7];
      stats->constraint_init_iterations = (int64_t)hs[8];
      stats->final_time = global ? c0.t : dt;
      int32_t worst = MICMB_SOLVER_CONVERGED;
      if (global)
        worst = c0.state;
      else if (hs[7])
      {
        std::vector<int32_t> stv(n);
        MICMB_CUDA(cudaMemcpy(stv.data(), a.status, sizeof(int32_t) * n, cudaMemcpyDeviceToHost));
        for (auto v : stv)
          if (v != MICMB_SOLVER_CONVERGED)
          {
            worst = v;
            break;
          }
      }
      stats->state = worst;
    }
  }

  // ---------------------------------------------------------------------
  // single-stage entry points (one call = one kernel over all cells)
  // ---------------------------------------------------------------------
  namespace
  {
    __global__ void k_add_forcing(DevMech M, PlainArgs a)
    {
      const int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
      if (c >= a.n)
        return;
      const int32_t L = a.L;
      Strided y{ a.y + cell_base(c, L, M.S), L };
      Strided k{ a.k + cell_base(c, L, M.R), L };
      Strided rate{ a.scratch + cell_base(c, L, a.scratch_cols), L };
      Strided f{ a.fcur + cell_base(c, L, M.S), L };
      Strided out{ a.f0 + cell_base(c, L, M.S), L };
      reaction_rates<1>(M, k, y, rate, 0);
      forcing_gather<1>(M, rate, f, 0);
      for (int32_t i = 0; i < M.S; ++i)
        out[i] = out[i] + f[i];
    }

    __global__ void k_subtract_jacobian(DevMech M, PlainArgs a)
    {
      const int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
      if (c >= a.n)
        return;
      const int32_t L = a.L;
      Strided y{ a.y + cell_base(c, L, M.S), L };
      Strided k{ a.k + cell_base(c, L, M.R), L };
      Strided dr{ a.scratch + cell_base(c, L, a.scratch_cols), L };
      Strided J{ a.jac + cell_base(c, L, M.nnz), L };
      jacobian_rates<1>(M, k, y, dr, 0);
      // add the assembled -J to the existing values, term by term as micm does
      for (int32_t e = 0; e < M.nnz; ++e)
      {
        double acc = J[e];
        for (int32_t t = M.j_start[e]; t < M.j_start[e + 1]; ++t)
          acc += M.j_coef[t] * dr[M.j_info[t]];
        J[e] = acc;
      }
    }

    __global__ void k_alpha_minus_jacobian(DevMech M, PlainArgs a, double alpha)
    {
      const int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
      if (c >= a.n)
        return;
      const int32_t L = a.L;
      Strided J{ a.jac + cell_base(c, L, M.nnz), L };
      for (int32_t i = 0; i < M.S; ++i)
        J[M.diag_pos[i]] = J[M.diag_pos[i]] + alpha;
    }

    __global__ void k_decompose_all(DevMech M, PlainArgs a)
    {
      const int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
      if (c >= a.n)
        return;
      const int32_t L = a.L;
      Strided J{ a.jac + cell_base(c, L, M.nnz), L };
      Strided inv{ a.inv + cell_base(c, L, M.S), L };
      thread_lu(M, J, inv);
    }

    __global__ void k_linear_solve_all(DevMech M, PlainArgs a)
    {
      const int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
      if (c >= a.n)
        return;
      const int32_t L = a.L;
      Strided J{ a.jac + cell_base(c, L, M.nnz), L };
      Strided x{ a.f0 + cell_base(c, L, M.S), L };
      thread_solve(M, J, x);
    }

    // errors are in f0, y in variables, ynew in the ynew buffer
    __global__ void k_error_cells(DevMech M, PlainArgs a)
    {
      const int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
      if (c >= a.n)
        return;
      const int32_t L = a.L;
      const size_t bs = cell_base(c, L, M.S);
      double sum = 0.0;
      for (int32_t i = 0; i < M.S; ++i)
        sum += scaled_sq(a.y[bs + (size_t)i * L], a.ynew[bs + (size_t)i * L], a.f0[bs + (size_t)i * L], a.atol[i],
                         a.rtol);
      a.err_cell[c] = sum;
    }
  }  // namespace

  void LaunchAddForcing(micmb_solver& s, micmb_state& st)
  {
    EnsurePlainBuffers(st);
    PlainArgs a = MakeArgs(s, st, 0);
    k_add_forcing<<<Blocks(st.n_cells), kBlock, 0, st.stream>>>(s.dev, a);
    MICMB_CUDA(cudaGetLastError());
  }
  void LaunchSubtractJacobian(micmb_solver& s, micmb_state& st)
  {
    EnsurePlainBuffers(st);
    PlainArgs a = MakeArgs(s, st, 0);
    k_subtract_jacobian<<<Blocks(st.n_cells), kBlock, 0, st.stream>>>(s.dev, a);
    MICMB_CUDA(cudaGetLastError());
  }
  void LaunchAlphaMinusJacobian(micmb_solver& s, micmb_state& st, double alpha)
  {
    EnsurePlainBuffers(st);
    PlainArgs a = MakeArgs(s, st, 0);
    k_alpha_minus_jacobian<<<Blocks(st.n_cells), kBlock, 0, st.stream>>>(s.dev, a, alpha);
    MICMB_CUDA(cudaGetLastError());
  }
  void LaunchDecompose(micmb_solver& s, micmb_state& st)
  {
    EnsurePlainBuffers(st);
    PlainArgs a = MakeArgs(s, st, 0);
    k_decompose_all<<<Blocks(st.n_cells), kBlock, 0, st.stream>>>(s.dev, a);
    MICMB_CUDA(cudaGetLastError());
  }
  void LaunchLinearSolve(micmb_solver& s, micmb_state& st)
  {
    EnsurePlainBuffers(st);
    PlainArgs a = MakeArgs(s, st, 0);
    k_linear_solve_all<<<Blocks(st.n_cells), kBlock, 0, st.stream>>>(s.dev, a);
    MICMB_CUDA(cudaGetLastError());
  }
  void NormalizedError(micmb_solver& s, micmb_state& st, double* global_out, double* per_cell_out)
  {
    EnsurePlainBuffers(st);
    PlainArgs a = MakeArgs(s, st, 0);
    const int64_t n = st.n_cells;
    k_error_cells<<<Blocks(n), kBlock, 0, st.stream>>>(s.dev, a);
    MICMB_CUDA(cudaGetLastError());
    std::vector<double> cells(n);
    MICMB_CUDA(cudaMemcpyAsync(cells.data(), a.err_cell, sizeof(double) * n, cudaMemcpyDeviceToHost, st.stream));
    MICMB_CUDA(cudaStreamSynchronize(st.stream));
    const int32_t S = s.mech->S;
    if (per_cell_out)
      for (int64_t c = 0; c < n; ++c)
      {
        const double rms = std::sqrt(cells[c] / (double)S);
        per_cell_out[c] = rms < 1.0e-10 ? 1.0e-10 : rms;
      }
    if (global_out)
    {
      double sum = 0.0;
      for (int64_t c = 0; c < n; ++c)
        sum += cells[c];
      const double rms = std::sqrt(sum / (double)std::max<int64_t>(1, n * S));
      *global_out = rms < 1.0e-10 ? 1.0e-10 : rms;
    }
  }
}  // namespace micmb
