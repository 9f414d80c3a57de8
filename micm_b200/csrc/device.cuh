// device.cuh -- per-cell building blocks of the Rosenbrock solve, shared by the
// per-stage ("plain") kernels and the persistent fused kernel.
//
// Every function works on one grid cell with `nl` cooperating lanes (`lane` in
// [0, nl)): the plain kernels call them with nl = 1 and data in global memory
// in micm's vector layout (stride L between columns), the fused kernel with a
// warp (nl = 32) and data staged in shared memory (stride 1).  Each output
// value is produced by exactly one lane, summing its terms in the order micm's
// scatter loops apply them (process_set.hpp:524-670,
// lu_decomposition_mozart_in_place.inl:171-210, linear_solver_in_place.inl:113-167),
// so results do not depend on nl.  The library is compiled with -fmad=false:
// each multiply and add rounds separately, as micm's CPU build does.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/micmb.h"
#include "crmath.cuh"

namespace micmb
{
  // ---------------------------------------------------------------------
  // device tables
  // ---------------------------------------------------------------------
  struct DevSchedule
  {
    int32_t n_levels;
    const int32_t* level_start;
    const int32_t* target;
    const int32_t* aux;
    const int32_t* term_start;
    const int32_t* ta;
    const int32_t* tb;
    const int2* tab;  // (ta, tb) of each term in one 8-byte load
    // per item in one 16-byte load: {target, first term, end of terms, aux}
    const int4* item;
    // serial LU schedule only (else nullptr): per item {diag row of the
    // target or -1, first Jacobian gather term, end of them, diag row of aux}
    const int4* item_j;
  };

  // one Jacobian gather term (coefficient and Jacobian-info index) in one 16-byte load
  struct alignas(16) JTerm
  {
    double coef;
    int32_t info;
    int32_t pad;
  };

  // register-blocked serial schedule (mechanism.hpp BlockedSchedule)
  struct DevBlocked
  {
    int32_t n_blocks;
    const int4* block;   // {first op, n ops, n slots | kind << 4 | (diag slot + 1) << 8, pivot row}
    const int4* target;  // slot targets (-1 unused)
    const int4* aux;     // backward solve: diagonal positions of the slot rows
    const uint4* op;     // {shared index, slot mask, slot 0 | slot 1 << 16, slot 2 | slot 3 << 16}
  };

  // lane-interleaved level schedule (mechanism.hpp WarpTable)
  struct DevWarpTable
  {
    int32_t n_levels;
    const int32_t* level_chunk_start;  // [n_levels + 1]
    const int4* chunk;                 // term base, T, first item, n items
    const uint32_t* item;
    const uint32_t* term;
    const double* coef;
  };

  struct DevMech
  {
    int32_t S, R, P, nnz, n_info;
    // rate constants by rate column
    const int32_t* rate_kind;
    const double* rate_p;      // [R][MICMB_RATE_PARAM_STRIDE]
    const int32_t* rate_param_col;
    const int32_t* rate_n_mult;
    const double* rate_mult;   // [R][MICMB_MAX_PARAMETERIZED][4]
    const double* rate_scale;  // [R] multiplicative scale (1.0 by default)
    // reactants and products by rate column
    const int32_t* react_start;
    const int32_t* react_ids;
    const int32_t* prod_start;
    const int32_t* prod_ids;
    const double* prod_yield;
    // forcing gather by species
    const int32_t* f_start;
    const int32_t* f_rxn;
    const double* f_coef;
    // jacobian infos and gather by nonzero
    const int32_t* info_rxn;
    const int32_t* info_dep_start;
    const int32_t* info_dep_ids;
    const int32_t* j_start;
    const int32_t* j_info;
    const double* j_coef;
    const JTerm* jterm;  // j_coef and j_info together
    const int32_t* diag_pos;     // [S] storage position of a_ii
    const int32_t* diag_row_of;  // [nnz] row i if the position holds a_ii, else -1
    DevSchedule lu, fwd, bwd, fwd_t, bwd_t;
    DevSchedule lu_s, fwd_s, bwd_s, fwd_t_s, bwd_t_s;  // serial forms (one thread per cell)
    int32_t has_blocked;                                // register-blocked serial forms present
    DevBlocked lu_b, fwd_b, bwd_b;
    // algebraic constraints (n_constraints = 0 for an ODE mechanism)
    int32_t n_constraints, n_eq, n_cterms;
    const int4* con;           // {kind, row, t0, t1}
    const int2* con_eq;        // {n_react, K_eq index}
    const double* con_p;       // [n_constraints * 4]
    const int32_t* ct_col;     // term state columns
    const double* ct_coef;     // coefficient / stoichiometry
    const double* mass;        // [S] mass-matrix diagonal
    const int32_t* cj_start;   // [nnz + 1] constraint terms received by each LU position
    const int32_t* cj_term;
    // warp-interleaved tables (fused kernel); dummy slots: LU[nnz], x[S], scratch[scratch_zero]
    int32_t has_warp;
    int32_t scratch_zero;
    DevWarpTable w_lu, w_fwd, w_bwd, w_fwd_t, w_bwd_t, w_forcing, w_jacobian;
    // fixed-width product lists (nullptr when a reaction has more than three reactants)
    const int4* rate_desc;   // [R]
    const int4* drate_desc;  // [n_info]
  };

  // Rosenbrock tableau in device-friendly form
  struct DevParams
  {
    int32_t stages;
    int32_t max_steps;
    double round_off, factor_min, factor_max, rejection_factor_decrease, safety_factor;
    double h_min_param, h_max_param, h_start_param;
    int32_t new_f[6];
    double inv_order;  // 1 / estimator_of_local_order
    double a[15], c[15], m[6], e[6], gamma0;
    int32_t cinit_max_iter;  // DAE constraint initialisation
    double cinit_tol;
  };

  // column accessor with a runtime stride (global vector layout) or unit stride (shared)
  struct Strided
  {
    double* p;
    int32_t s;
    __device__ __forceinline__ double& operator[](int32_t i) const
    {
      return p[(size_t)i * (size_t)s];
    }
  };
  struct Unit
  {
    double* p;
    __device__ __forceinline__ double& operator[](int32_t i) const
    {
      return p[i];
    }
  };

  template<int NL>
  __device__ __forceinline__ void lane_sync()
  {
    if constexpr (NL > 1)
      __syncwarp();
  }

  // ---------------------------------------------------------------------
  // rate constants (rate_constant_functions.hpp:52-136), with the C library's
  // correctly rounded exp, pow and log10 (crmath.cuh)
  // ---------------------------------------------------------------------
  __device__ __forceinline__ double falloff(const double* p, double T, double rho, double numerator_scale)
  {
    const double k0 = p[0] * cr_exp(p[2] / T) * cr_pow(T / 300.0, p[1]);
    const double kinf = p[3] * cr_exp(p[5] / T) * cr_pow(T / 300.0, p[4]);
    const double ratio = k0 * rho / kinf;
    return k0 * numerator_scale / (1.0 + ratio) * cr_pow(p[6], p[7] / (p[7] + cr_pow(cr_log10(ratio), 2.0)));
  }

  // k for rate column r given the cell's conditions and custom-parameter column reader
  template<class ParamFn>
  __device__ __forceinline__ double rate_constant(const DevMech& M, int32_t r, double T, double Pr, double rho,
                                                  ParamFn param)
  {
    const double* p = M.rate_p + (size_t)r * MICMB_RATE_PARAM_STRIDE;
    double k;
    switch (M.rate_kind[r])
    {
      case MICMB_RATE_ARRHENIUS: k = p[0] * cr_exp(p[2] / T) * cr_pow(T / p[3], p[1]) * (1.0 + p[4] * Pr); break;
      case MICMB_RATE_TROE: k = falloff(p, T, rho, rho); break;
      case MICMB_RATE_TERNARY_CHEMICAL_ACTIVATION: k = falloff(p, T, rho, 1.0); break;
      case MICMB_RATE_BRANCHED:
      {
        const double a = p[5] * rho;
        const double b = 0.43 * cr_pow(T / 298.0, -8.0);
        const double A_val = a / (1.0 + a / b) * cr_pow(0.41, 1.0 / (1.0 + cr_pow(cr_log10(a / b), 2.0)));
        const double pre = p[1] * cr_exp(-p[2] / T);
        k = (p[0] == 0.0) ? pre * (p[6] / (p[6] + A_val)) : pre * (A_val / (A_val + p[6]));
        break;
      }
      case MICMB_RATE_TUNNELING: k = p[0] * cr_exp(-p[1] / T + p[2] / (T * T * T)); break;
      case MICMB_RATE_TAYLOR_SERIES:
      {
        double poly = 0.0, t_pow = 1.0;
        const int32_t n = (int32_t)p[5];
        for (int32_t j = 0; j < n; ++j, t_pow *= T)
          poly += p[6 + j] * t_pow;
        k = poly * p[0] * cr_exp(p[2] / T) * cr_pow(T / p[3], p[1]) * (1.0 + p[4] * Pr);
        break;
      }
      case MICMB_RATE_REVERSIBLE: k = p[0] * cr_exp(p[1] / T) * p[2]; break;
      case MICMB_RATE_USER_DEFINED: k = param(M.rate_param_col[r]) * p[0]; break;
      case MICMB_RATE_SURFACE:
      {
        const double radius = param(M.rate_param_col[r]);
        const double num_conc = param(M.rate_param_col[r] + 1);
        const double mean_free_speed = sqrt(p[1] * T);
        k = 4.0 * num_conc * 3.14159265358979323846 * radius * radius /
            (radius / p[0] + 4.0 / (mean_free_speed * p[2]));
        break;
      }
      default: k = 0.0;
    }
    const int32_t nm = M.rate_n_mult[r];
    if (nm > 0)
    {
      double v = 1.0;
      const double* c = M.rate_mult + (size_t)r * MICMB_MAX_PARAMETERIZED * 4;
      for (int32_t i = 0; i < nm; ++i)
        v *= c[4 * i + 0] + c[4 * i + 1] * T + c[4 * i + 2] * Pr + c[4 * i + 3] * rho;
      k *= v;
    }
    const double scale = M.rate_scale[r];
    if (scale != 1.0)
      k *= scale;
    return k;
  }

  // ---------------------------------------------------------------------
  // forcing: rate_r = k_r * prod(y reactants); f_s = sum_terms coef * rate
  // ---------------------------------------------------------------------
  template<int NL, class KV, class YV, class RV>
  __device__ __forceinline__ void reaction_rates(const DevMech& M, KV k, YV y, RV rate, int lane)
  {
    for (int32_t r = lane; r < M.R; r += NL)
    {
      double v = k[r];
      for (int32_t i = M.react_start[r]; i < M.react_start[r + 1]; ++i)
        v *= y[M.react_ids[i]];
      rate[r] = v;
    }
  }

  // reaction_rates / jacobian_rates over fixed-width product lists; y[S + 1]
  // must hold 1.0.  Same products in the same order as the loops above.
  template<int NL, class KV, class YV, class RV>
  __device__ __forceinline__ void reaction_rates_narrow(const DevMech& M, KV k, YV y, RV rate, int lane)
  {
#pragma unroll 4
    for (int32_t r = lane; r < M.R; r += NL)
    {
      const int4 d = M.rate_desc[r];
      double v = k[r];
      v *= y[d.x];
      v *= y[d.y];
      v *= y[d.z];
      rate[r] = v;
    }
  }

  template<int NL, class KV, class YV, class DV>
  __device__ __forceinline__ void jacobian_rates_narrow(const DevMech& M, KV k, YV y, DV drate, int lane)
  {
#pragma unroll 4
    for (int32_t i = lane; i < M.n_info; i += NL)
    {
      const int4 d = M.drate_desc[i];
      double v = k[d.x];
      v *= y[d.y];
      v *= y[d.z];
      v *= y[d.w];
      drate[i] = v;
    }
  }

  template<int NL, class RV, class FV>
  __device__ __forceinline__ void forcing_gather(const DevMech& M, RV rate, FV f, int lane)
  {
    for (int32_t s = lane; s < M.S; s += NL)
    {
      double acc = 0.0;
#pragma unroll 2
      for (int32_t t = M.f_start[s]; t < M.f_start[s + 1]; ++t)
        acc += M.f_coef[t] * rate[M.f_rxn[t]];
      f[s] = acc;
    }
  }

  // ---------------------------------------------------------------------
  // algebraic constraints, one cell (linear_constraint.hpp:216-290,
  // equilibrium_constraint.hpp:290-580): keq holds the cell's K_eq values
  // ---------------------------------------------------------------------
  __device__ __forceinline__ double con_pow(double c, double e)
  {
    return cr_pow(c > 0.0 ? c : 0.0, e);
  }

  // f[row] = G(y) for every constraint: the residual overwrites the algebraic row
  template<class KV, class YV, class FV>
  __device__ __forceinline__ void constraint_forcing(const DevMech& M, KV keq, YV y, FV f)
  {
    for (int32_t c = 0; c < M.n_constraints; ++c)
    {
      const int4 cd = M.con[c];
      if (cd.x == MICMB_CONSTRAINT_LINEAR)
      {
        double sum = 0.0;
        for (int32_t t = cd.z; t < cd.w; ++t)
          sum += M.ct_coef[t] * y[M.ct_col[t]];
        f[cd.y] = sum - M.con_p[4 * c];
      }
      else
      {
        const int2 eq = M.con_eq[c];
        double rp = keq[eq.y], pp = 1.0;
        const int32_t tr = cd.z + eq.x;
        for (int32_t t = cd.z; t < tr; ++t)
          rp *= con_pow(y[M.ct_col[t]], M.ct_coef[t]);
        for (int32_t t = tr; t < cd.w; ++t)
          pp *= con_pow(y[M.ct_col[t]], M.ct_coef[t]);
        f[cd.y] = rp - pp;
      }
    }
  }

  // cj[t] = what the Jacobian entry of constraint term t loses (jac -= cj[t]):
  // the coefficient (linear), dG/dy (equilibrium reactant) or -dG/dy
  // (equilibrium product, which micm adds: jac - (-p) == jac + p exactly)
  template<class KV, class YV, class CV>
  __device__ __forceinline__ void constraint_jacobian(const DevMech& M, KV keq, YV y, CV cj)
  {
    for (int32_t c = 0; c < M.n_constraints; ++c)
    {
      const int4 cd = M.con[c];
      if (cd.x == MICMB_CONSTRAINT_LINEAR)
      {
        for (int32_t t = cd.z; t < cd.w; ++t)
          cj[t] = M.ct_coef[t];
        continue;
      }
      const int2 eq = M.con_eq[c];
      const int32_t tr = cd.z + eq.x;
      const double K = keq[eq.y];
      for (int side = 0; side < 2; ++side)
      {
        const int32_t a = side ? tr : cd.z, b = side ? cd.w : tr;
        for (int32_t i = a; i < b; ++i)
        {
          double prod = side ? 1.0 : K;
          for (int32_t j = a; j < b; ++j)
            if (j != i)
              prod *= con_pow(y[M.ct_col[j]], M.ct_coef[j]);
          const double conc = y[M.ct_col[i]], st = M.ct_coef[i];
          double partial;
          if (st == 1.0)
            partial = prod;
          else if (conc > 0.0)
            partial = st * prod * cr_pow(conc, st - 1.0);
          else
            partial = 0.0;
          cj[i] = side ? -partial : partial;
        }
      }
    }
  }

  // K_eq(T) of every equilibrium constraint (Van't Hoff), in constraint order
  __device__ __forceinline__ double constraint_keq(const DevMech& M, int32_t c, double T)
  {
    const double* q = M.con_p + 4 * c;
    return q[0] * cr_exp((q[1] / q[2]) * (1.0 / T - 1.0 / q[3]));
  }

  // ---------------------------------------------------------------------
  // -J + alpha I: d_rate per info, then gather per nonzero
  // ---------------------------------------------------------------------
  template<int NL, class KV, class YV, class DV>
  __device__ __forceinline__ void jacobian_rates(const DevMech& M, KV k, YV y, DV drate, int lane)
  {
    for (int32_t i = lane; i < M.n_info; i += NL)
    {
      double v = k[M.info_rxn[i]];
      for (int32_t d = M.info_dep_start[i]; d < M.info_dep_start[i + 1]; ++d)
        v *= y[M.info_dep_ids[d]];
      drate[i] = v;
    }
  }

  // jac[e] = sum_terms coef * drate, minus its constraint terms cj (algebraic
  // rows), plus alpha times the mass-matrix diagonal when add_alpha
  template<int NL, class DV, class JV, class CV>
  __device__ __forceinline__ void jacobian_gather(const DevMech& M, DV drate, JV jac, double alpha, bool add_alpha,
                                                  int lane, CV cj)
  {
    for (int32_t e = lane; e < M.nnz; e += NL)
    {
      double acc = 0.0;
#pragma unroll 2
      for (int32_t t = M.j_start[e]; t < M.j_start[e + 1]; ++t)
      {
        const JTerm jt = M.jterm[t];
        acc += jt.coef * drate[jt.info];
      }
      if (M.n_constraints)
        for (int32_t t = M.cj_start[e]; t < M.cj_start[e + 1]; ++t)
          acc -= cj[M.cj_term[t]];
      const int32_t dr = M.diag_row_of[e];
      if (add_alpha && dr >= 0)
        acc += M.n_constraints ? alpha * M.mass[dr] : alpha;
      jac[e] = acc;
    }
  }
  template<int NL, class DV, class JV>
  __device__ __forceinline__ void jacobian_gather(const DevMech& M, DV drate, JV jac, double alpha, bool add_alpha,
                                                  int lane)
  {
    jacobian_gather<NL>(M, drate, jac, alpha, add_alpha, lane, drate);
  }

  // ---------------------------------------------------------------------
  // in-place LU (Crout order of micm's Mozart updates); inv = 1/a_kk scratch [S]
  // ---------------------------------------------------------------------
  template<int NL, class AV, class IV>
  __device__ __forceinline__ void lu_decompose(const DevSchedule& sch, const int32_t* diag_row, AV A, IV inv,
                                               int lane)
  {
    for (int32_t l = 0; l < sch.n_levels; ++l)
    {
      const int32_t end = sch.level_start[l + 1];
      for (int32_t it = sch.level_start[l] + lane; it < end; it += NL)
      {
        const int4 rec = sch.item[it];
        const int32_t e = rec.x;
        double v = A[e];
#pragma unroll 2
        for (int32_t t = rec.y; t < rec.z; ++t)
        {
          const int2 ab = sch.tab[t];
          v -= A[ab.x] * A[ab.y];
        }
        const int32_t aux = rec.w;  // -2: partial sum (stored, finalised by a later unit)
        if (aux >= 0)
          v *= inv[diag_row[aux]];
        A[e] = v;
        const int32_t dr = diag_row[e];
        if (aux != -2 && dr >= 0)
          inv[dr] = 1.0 / v;
      }
      lane_sync<NL>();
    }
  }

  // jacobian_gather (add_alpha) followed by lu_decompose on a serial schedule
  // (every entry is one item, visited once, after the items it reads): each
  // item starts from the value jacobian_gather would store for its entry --
  // the gathered sum, then + alpha on the diagonal -- instead of reading it
  // back, so the Jacobian never makes a round trip through memory.  Same
  // operations in the same order as the two passes.
  // With constraints, each entry also loses its constraint terms cj (micm
  // subtracts the constraints' derivatives after the processes'), and the
  // diagonal gains alpha times the mass-matrix diagonal.  PROCESS = false
  // leaves the process gather out (the constraint initialisation's matrix).
  template<bool PROCESS = true, class DV, class AV, class IV, class CV>
  __device__ __forceinline__ void lu_decompose_gathered(const DevMech& M, const DevSchedule& sch,
                                                        const int32_t* diag_row, DV drate, double alpha, AV A, IV inv,
                                                        CV cj)
  {
    // sch is the serial LU schedule (item_j present); diag_row is folded into item_j
    (void)diag_row;
    const int32_t n_items = sch.level_start[sch.n_levels];
    for (int32_t it = 0; it < n_items; ++it)
    {
      const int4 rec = sch.item[it];
      const int4 rj = sch.item_j[it];
      const int32_t e = rec.x;
      double v = 0.0;
      if constexpr (PROCESS)
#pragma unroll 2
        for (int32_t t = rj.y; t < rj.z; ++t)
        {
          const JTerm jt = M.jterm[t];
          v += jt.coef * drate[jt.info];
        }
      if (M.n_constraints)
        for (int32_t t = M.cj_start[e]; t < M.cj_start[e + 1]; ++t)
          v -= cj[M.cj_term[t]];
      const int32_t dr = rj.x;
      if (dr >= 0)
        v += M.n_constraints ? alpha * M.mass[dr] : alpha;
      // two terms per iteration: their four operand loads issue together
#pragma unroll 2
      for (int32_t t = rec.y; t < rec.z; ++t)
      {
        const int2 ab = sch.tab[t];
        v -= A[ab.x] * A[ab.y];
      }
      const int32_t aux = rec.w;
      if (aux >= 0)
        v *= inv[rj.w];
      A[e] = v;
      if (aux != -2 && dr >= 0)
        inv[dr] = 1.0 / v;
    }
  }

  // ---------------------------------------------------------------------
  // register-blocked serial LU and solves (one thread per cell): up to four
  // entries of a block in registers; each op loads its shared operand once
  // and updates the entries that use it.  Every entry receives its terms in
  // the serial schedule's order, so results are bit-identical to
  // lu_decompose / lu_decompose_gathered / solve_lower / solve_upper.
  // ---------------------------------------------------------------------
  __device__ __forceinline__ uint32_t blk_lo(uint32_t v)
  {
    return v & 0xFFFFu;
  }
  __device__ __forceinline__ uint32_t blk_hi(uint32_t v)
  {
    return v >> 16;
  }

  // GATHER: each entry starts from its -J gather (+ alpha on the diagonal),
  // as lu_decompose_gathered; otherwise from the stored value, as lu_decompose.
  template<bool GATHER, class DV, class AV, class IV>
  __device__ __forceinline__ void lu_blocked(const DevMech& M, const DevBlocked& T, DV drate, double alpha, AV A,
                                             IV inv)
  {
    auto init = [&](int32_t e) -> double {
      if constexpr (GATHER)
      {
        double v = 0.0;
        for (int32_t t = M.j_start[e]; t < M.j_start[e + 1]; ++t)
          v += M.j_coef[t] * drate[M.j_info[t]];
        if (M.diag_row_of[e] >= 0)
          v += alpha;
        return v;
      }
      else
        return A[e];
    };
    for (int32_t k = 0; k < T.n_blocks; ++k)
    {
      const int4 bk = __ldg(T.block + k);
      const int4 tg = __ldg(T.target + k);
      const int32_t n = bk.z & 0xF, kind = (bk.z >> 4) & 0xF, diag = (bk.z >> 8) - 1;
      double a0 = init(tg.x), a1 = 0.0, a2 = 0.0, a3 = 0.0;
      if (n > 1)
        a1 = init(tg.y);
      if (n > 2)
        a2 = init(tg.z);
      if (n > 3)
        a3 = init(tg.w);
      for (int32_t o = bk.x; o < bk.x + bk.y; ++o)
      {
        const uint4 op = __ldg(T.op + o);
        const double sh = A[op.x];
        if (op.y & 1u)
          a0 -= sh * A[blk_lo(op.z)];
        if (op.y & 2u)
          a1 -= sh * A[blk_hi(op.z)];
        if (op.y & 4u)
          a2 -= sh * A[blk_lo(op.w)];
        if (op.y & 8u)
          a3 -= sh * A[blk_hi(op.w)];
      }
      if (kind == 1)  // L column: times 1/a_kk of the pivot
      {
        const double iv = inv[bk.w];
        a0 *= iv;
        a1 *= iv;
        a2 *= iv;
        a3 *= iv;
      }
      A[tg.x] = a0;
      if (n > 1)
        A[tg.y] = a1;
      if (n > 2)
        A[tg.z] = a2;
      if (n > 3)
        A[tg.w] = a3;
      if (diag >= 0)
        inv[bk.w] = 1.0 / (diag == 0 ? a0 : (diag == 1 ? a1 : (diag == 2 ? a2 : a3)));
    }
  }

  // UPPER: U x = b with the division by the diagonal (solve_upper); else the
  // unit-lower L y = b (solve_lower).  In place.
  template<bool UPPER, class AV, class XV>
  __device__ __forceinline__ void solve_blocked(const DevBlocked& T, AV A, XV x)
  {
    for (int32_t k = 0; k < T.n_blocks; ++k)
    {
      const int4 bk = __ldg(T.block + k);
      const int4 tg = __ldg(T.target + k);
      const int32_t n = bk.z & 0xF;
      double a0 = x[tg.x], a1 = 0.0, a2 = 0.0, a3 = 0.0;
      if (n > 1)
        a1 = x[tg.y];
      if (n > 2)
        a2 = x[tg.z];
      if (n > 3)
        a3 = x[tg.w];
      for (int32_t o = bk.x; o < bk.x + bk.y; ++o)
      {
        const uint4 op = __ldg(T.op + o);
        const double sh = x[op.x];
        if (op.y & 1u)
          a0 -= A[blk_lo(op.z)] * sh;
        if (op.y & 2u)
          a1 -= A[blk_hi(op.z)] * sh;
        if (op.y & 4u)
          a2 -= A[blk_lo(op.w)] * sh;
        if (op.y & 8u)
          a3 -= A[blk_hi(op.w)] * sh;
      }
      if constexpr (UPPER)
      {
        const int4 ax = __ldg(T.aux + k);
        x[tg.x] = a0 / A[ax.x];
        if (n > 1)
          x[tg.y] = a1 / A[ax.y];
        if (n > 2)
          x[tg.z] = a2 / A[ax.z];
        if (n > 3)
          x[tg.w] = a3 / A[ax.w];
      }
      else
      {
        x[tg.x] = a0;
        if (n > 1)
          x[tg.y] = a1;
        if (n > 2)
          x[tg.z] = a2;
        if (n > 3)
          x[tg.w] = a3;
      }
    }
  }

  // The one-thread-per-cell LU and solves: blocked when the mechanism has
  // the blocked forms, else the serial schedules.
  template<class DV, class AV, class IV, class CV>
  __device__ __forceinline__ void thread_lu_gathered(const DevMech& M, DV drate, double alpha, AV A, IV inv, CV cj);
  template<class AV, class XV>
  __device__ __forceinline__ void thread_solve(const DevMech& M, AV A, XV x);

  // L y = b (unit diagonal), in place
  template<int NL, class AV, class XV>
  __device__ __forceinline__ void solve_lower(const DevSchedule& sch, AV A, XV x, int lane)
  {
    for (int32_t l = 0; l < sch.n_levels; ++l)
    {
      const int32_t end = sch.level_start[l + 1];
      for (int32_t it = sch.level_start[l] + lane; it < end; it += NL)
      {
        const int4 rec = sch.item[it];
        const int32_t i = rec.x;
        double v = x[i];
#pragma unroll 2
        for (int32_t t = rec.y; t < rec.z; ++t)
        {
          const int2 ab = sch.tab[t];
          v -= A[ab.x] * x[ab.y];
        }
        x[i] = v;
      }
      lane_sync<NL>();
    }
  }

  // upper solve with division by the diagonal (aux), in place
  template<int NL, class AV, class XV>
  __device__ __forceinline__ void solve_upper(const DevSchedule& sch, AV A, XV x, int lane)
  {
    for (int32_t l = 0; l < sch.n_levels; ++l)
    {
      const int32_t end = sch.level_start[l + 1];
      for (int32_t it = sch.level_start[l] + lane; it < end; it += NL)
      {
        const int4 rec = sch.item[it];
        const int32_t i = rec.x;
        double v = x[i];
#pragma unroll 2
        for (int32_t t = rec.y; t < rec.z; ++t)
        {
          const int2 ab = sch.tab[t];
          v -= A[ab.x] * x[ab.y];
        }
        const int32_t aux = rec.w;  // -2: partial sum
        x[i] = aux >= 0 ? v / A[aux] : v;
      }
      lane_sync<NL>();
    }
  }

  template<class DV, class AV, class IV, class CV>
  __device__ __forceinline__ void thread_lu_gathered(const DevMech& M, DV drate, double alpha, AV A, IV inv, CV cj)
  {
    if (M.has_blocked && !M.n_constraints)
      lu_blocked<true>(M, M.lu_b, drate, alpha, A, inv);
    else
      lu_decompose_gathered(M, M.lu_s, M.diag_row_of, drate, alpha, A, inv, cj);
  }
  template<class DV, class AV, class IV>
  __device__ __forceinline__ void thread_lu_gathered(const DevMech& M, DV drate, double alpha, AV A, IV inv)
  {
    thread_lu_gathered(M, drate, alpha, A, inv, drate);
  }

  template<class AV, class IV>
  __device__ __forceinline__ void thread_lu(const DevMech& M, AV A, IV inv)
  {
    if (M.has_blocked)
      lu_blocked<false>(M, M.lu_b, A, 0.0, A, inv);
    else
      lu_decompose<1>(M.lu_s, M.diag_row_of, A, inv, 0);
  }

  // x = (LU)^-1 x: forward then backward substitution
  template<class AV, class XV>
  __device__ __forceinline__ void thread_solve(const DevMech& M, AV A, XV x)
  {
    if (M.has_blocked)
    {
      solve_blocked<false>(M.fwd_b, A, x);
      solve_blocked<true>(M.bwd_b, A, x);
    }
    else
    {
      solve_lower<1>(M.fwd_s, A, x, 0);
      solve_upper<1>(M.bwd_s, A, x, 0);
    }
  }

  // ---------------------------------------------------------------------
  // warp-interleaved versions (32 lanes, one cell, shared-memory operands)
  // ---------------------------------------------------------------------
  __device__ __forceinline__ int4 load_chunk(const int4* p)
  {
    return __ldg(p);
  }

  // in-place LU; A[nnz] must be 0; inv[S] receives 1/a_ii
  __device__ __forceinline__ void warp_lu(const DevWarpTable& W, double* A, double* inv, int lane)
  {
    for (int32_t l = 0; l < W.n_levels; ++l)
    {
      const int32_t c1 = __ldg(W.level_chunk_start + l + 1);
      for (int32_t ch = __ldg(W.level_chunk_start + l); ch < c1; ++ch)
      {
        const int4 c = load_chunk(W.chunk + ch);
        if (lane < c.w)
        {
          const uint32_t it = __ldg(W.item + c.z + lane);
          const uint32_t e = it & 0xFFFFu, hi = it >> 16;
          double v = A[e];
          const uint32_t* tp = W.term + c.x + lane;
          int32_t t = 0;
          for (; t + 4 <= c.y; t += 4)
          {
            const uint32_t q0 = __ldg(tp + (t + 0) * 32), q1 = __ldg(tp + (t + 1) * 32);
            const uint32_t q2 = __ldg(tp + (t + 2) * 32), q3 = __ldg(tp + (t + 3) * 32);
            const double a0 = A[q0 & 0xFFFFu], b0 = A[q0 >> 16], a1 = A[q1 & 0xFFFFu], b1 = A[q1 >> 16];
            const double a2 = A[q2 & 0xFFFFu], b2 = A[q2 >> 16], a3 = A[q3 & 0xFFFFu], b3 = A[q3 >> 16];
            v -= a0 * b0;
            v -= a1 * b1;
            v -= a2 * b2;
            v -= a3 * b3;
          }
          for (; t < c.y; ++t)
          {
            const uint32_t q = __ldg(tp + t * 32);
            v -= A[q & 0xFFFFu] * A[q >> 16];
          }
          if (hi >= 0xFFFEu)  // U entry, or a partial sum
            A[e] = v;
          else if (hi & 0x8000u)
          {
            A[e] = v;
            inv[hi & 0x7FFFu] = 1.0 / v;
          }
          else
            A[e] = v * inv[hi];
        }
      }
      __syncwarp();
    }
  }

  // x_i = (x_i - sum A[a] x[b]) [/ A[aux]]; x[S] and A[nnz] must be 0
  __device__ __forceinline__ void warp_solve(const DevWarpTable& W, const double* A, double* x, int lane)
  {
    for (int32_t l = 0; l < W.n_levels; ++l)
    {
      const int32_t c1 = __ldg(W.level_chunk_start + l + 1);
      for (int32_t ch = __ldg(W.level_chunk_start + l); ch < c1; ++ch)
      {
        const int4 c = load_chunk(W.chunk + ch);
        if (lane < c.w)
        {
          const uint32_t it = __ldg(W.item + c.z + lane);
          const uint32_t i = it & 0xFFFFu, hi = it >> 16;
          double v = x[i];
          const uint32_t* tp = W.term + c.x + lane;
          int32_t t = 0;
          for (; t + 4 <= c.y; t += 4)
          {
            const uint32_t q0 = __ldg(tp + (t + 0) * 32), q1 = __ldg(tp + (t + 1) * 32);
            const uint32_t q2 = __ldg(tp + (t + 2) * 32), q3 = __ldg(tp + (t + 3) * 32);
            const double a0 = A[q0 & 0xFFFFu], b0 = x[q0 >> 16], a1 = A[q1 & 0xFFFFu], b1 = x[q1 >> 16];
            const double a2 = A[q2 & 0xFFFFu], b2 = x[q2 >> 16], a3 = A[q3 & 0xFFFFu], b3 = x[q3 >> 16];
            v -= a0 * b0;
            v -= a1 * b1;
            v -= a2 * b2;
            v -= a3 * b3;
          }
          for (; t < c.y; ++t)
          {
            const uint32_t q = __ldg(tp + t * 32);
            v -= A[q & 0xFFFFu] * x[q >> 16];
          }
          x[i] = (hi >= 0xFFFEu) ? v : v / A[hi];
        }
      }
      __syncwarp();
    }
  }

  // out[target] = sum coef * src[term] (+ alpha on flagged items); src[scratch_zero] must be 0
  __device__ __forceinline__ void warp_gather(const DevWarpTable& W, const double* src, double* out, double alpha,
                                              int lane)
  {
    const int32_t c1 = __ldg(W.level_chunk_start + 1);
    for (int32_t ch = 0; ch < c1; ++ch)
    {
      const int4 c = load_chunk(W.chunk + ch);
      if (lane < c.w)
      {
        const uint32_t it = __ldg(W.item + c.z + lane);
        double acc = 0.0;
        const uint32_t* tp = W.term + c.x + lane;
        const double* cp = W.coef + c.x + lane;
        int32_t t = 0;
        for (; t + 4 <= c.y; t += 4)
        {
          const uint32_t q0 = __ldg(tp + (t + 0) * 32), q1 = __ldg(tp + (t + 1) * 32);
          const uint32_t q2 = __ldg(tp + (t + 2) * 32), q3 = __ldg(tp + (t + 3) * 32);
          const double f0 = __ldg(cp + (t + 0) * 32), f1 = __ldg(cp + (t + 1) * 32);
          const double f2 = __ldg(cp + (t + 2) * 32), f3 = __ldg(cp + (t + 3) * 32);
          const double s0 = src[q0], s1 = src[q1], s2 = src[q2], s3 = src[q3];
          acc += f0 * s0;
          acc += f1 * s1;
          acc += f2 * s2;
          acc += f3 * s3;
        }
        for (; t < c.y; ++t)
          acc += __ldg(cp + t * 32) * src[__ldg(tp + t * 32)];
        if ((it >> 16) != 0xFFFFu)
          acc += alpha;
        out[it & 0xFFFFu] = acc;
      }
    }
  }

  // ---------------------------------------------------------------------
  // normalized error (rosenbrock.inl:353-402).  micm adds the scaled squares
  // of one cell in species order with one accumulator (ReduceStrict,
  // vector_matrix.hpp:858-866); every per-cell sum here is formed in that
  // order, so a cell's error equals micm's bit for bit.
  // ---------------------------------------------------------------------
  __host__ __device__ __forceinline__ double scaled_sq(double y, double ynew, double err, double atol, double rtol)
  {
    const double ay = fabs(y), an = fabs(ynew);
    const double ymax = ay > an ? ay : an;
    const double q = err / (atol + rtol * ymax);
    return q * q;
  }

  // Sequential sum of the 32-lane stripe values q (lane l holds the term of
  // species base + l) added to acc in species order; every lane returns the
  // same total.  `count` is the number of valid lanes of this stripe.
  __device__ __forceinline__ double warp_seq_add(double acc, double q, int32_t count)
  {
    for (int l = 0; l < count; ++l)
      acc += __shfl_sync(0xffffffffu, q, l);
    return acc;
  }

  // The scaled error (max(sqrt(sum / n), 1e-10)) from a sum of squares.
  __host__ __device__ __forceinline__ double error_from_sum(double sum, double n)
  {
    const double rms = sqrt(sum / n);
    return (rms < 1.0e-10) ? 1.0e-10 : rms;
  }

  // ---------------------------------------------------------------------
  // step control (rosenbrock.inl:80-293)
  // ---------------------------------------------------------------------
  struct CellCtl
  {
    double t;
    double H;
    int32_t reject_last;
    int32_t reject_more;
    int32_t state;  // MICMB_SOLVER_*
    int32_t new_step;
    int32_t function_calls, jacobian_updates, number_of_steps, accepted, rejected, decompositions, solves;
    int32_t init_iterations;  // DAE constraint initialisation
  };

  struct StepBounds
  {
    double dt, h_min, h_max, h_start;
  };

  __host__ __device__ inline StepBounds step_bounds(const DevParams& p, double dt)
  {
    StepBounds b;
    b.dt = dt;
    // rosenbrock.inl:33-36, with std::min(a,b) = (b<a)?b:a and std::max(a,b) = (a<b)?b:a
    b.h_min = p.h_min_param == 0.0 ? 1.0e-15 * dt : p.h_min_param;
    b.h_max = p.h_max_param == 0.0 ? dt : ((p.h_max_param < dt) ? p.h_max_param : dt);
    const double hs = p.h_start_param == 0.0 ? 1.0e-6 * dt : ((p.h_start_param < b.h_max) ? p.h_start_param : b.h_max);
    const double ahs = fabs(hs), ahm = fabs(b.h_max);
    const double lo = (b.h_min < ahs) ? ahs : b.h_min;
    b.h_start = (ahm < lo) ? ahm : lo;
    return b;
  }

  __host__ __device__ inline void ctl_init(CellCtl& c, const StepBounds& b)
  {
    c.t = 0.0;
    c.H = b.h_start;
    c.reject_last = 0;
    c.reject_more = 0;
    c.state = MICMB_SOLVER_RUNNING;
    c.new_step = 1;
    c.function_calls = c.jacobian_updates = c.number_of_steps = 0;
    c.accepted = c.rejected = c.decompositions = c.solves = 0;
    c.init_iterations = 0;
  }

  // Top of micm's outer loop: returns false (and sets state) when the cell is done.
  __host__ __device__ inline bool ctl_begin_step(CellCtl& c, const DevParams& p, const StepBounds& b)
  {
    if (!((c.t - b.dt + p.round_off) <= 0))
    {
      if (c.state == MICMB_SOLVER_RUNNING)
        c.state = MICMB_SOLVER_CONVERGED;
      return false;
    }
    if (c.number_of_steps > p.max_steps)
    {
      c.state = MICMB_SOLVER_CONVERGENCE_EXCEEDED_MAX_STEPS;
      return false;
    }
    if (((c.t + 0.1 * c.H) == c.t) || (c.H <= p.round_off))
    {
      c.state = MICMB_SOLVER_STEP_SIZE_TOO_SMALL;
      return false;
    }
    const double rem = fabs(b.dt - c.t);
    c.H = (rem < c.H) ? rem : c.H;  // std::min(H, |dt - t|)
    return true;
  }

  // Accept/reject after the error norm. Returns 1 accepted, 0 rejected, -1 stopped (NaN/Inf).
  __host__ __device__ inline int ctl_after_error(CellCtl& c, const DevParams& p, const StepBounds& b, double error)
  {
    // std::min(factor_max, std::max(factor_min, safety / pow(error, 1/order))),
    // with micm's (the C library's) correctly rounded pow
    const double x = p.safety_factor / cr_pow(error, p.inv_order);
    const double lo = (p.factor_min < x) ? x : p.factor_min;
    const double fac = (lo < p.factor_max) ? lo : p.factor_max;
    double Hnew = c.H * fac;
    c.number_of_steps += 1;
    if (isnan(error))
    {
      c.state = MICMB_SOLVER_NAN_DETECTED;
      return -1;
    }
    if (isinf(error))
    {
      c.state = MICMB_SOLVER_INF_DETECTED;
      return -1;
    }
    if ((error < 1) || (c.H < b.h_min))
    {
      c.accepted += 1;
      c.t = c.t + c.H;
      Hnew = (b.h_max < Hnew) ? b.h_max : Hnew;  // std::max(h_min, std::min(Hnew, h_max))
      Hnew = (b.h_min < Hnew) ? Hnew : b.h_min;
      if (c.reject_last)
        Hnew = (c.H < Hnew) ? c.H : Hnew;        // std::min(Hnew, H)
      c.reject_last = 0;
      c.reject_more = 0;
      c.H = Hnew;
      c.new_step = 1;
      return 1;
    }
    if (c.reject_more)
      Hnew = c.H * p.rejection_factor_decrease;
    c.reject_more = c.reject_last;
    c.reject_last = 1;
    c.H = Hnew;
    if (c.accepted >= 1)
      c.rejected += 1;
    c.jacobian_updates += 1;
    c.new_step = 0;
    return 0;
  }

  // Solver::PostSolveClamp (solver.hpp:275-297): std::max(y, 0) on every
  // variable; with constraints only the ODE variables, by (y > 0 ? y : 0), and
  // the algebraic ones are left as solved.
  __device__ __forceinline__ double post_clamp(const DevMech& M, int32_t i, double v)
  {
    if (!M.n_constraints)
      return (v < 0.0) ? 0.0 : v;
    return M.mass[i] > 0.0 ? (v > 0.0 ? v : 0.0) : v;
  }

  // ---------------------------------------------------------------------
  // InitializeConstraints for one cell (rosenbrock.inl:407-576): Newton on the
  // algebraic variables until max |G| over the algebraic rows is below the
  // tolerance.  delta (S), A (the LU), inv (S) and cj (constraint terms) are
  // the cell's scratch.  Returns MICMB_SOLVER_CONVERGED or the failure state
  // and counts into the cell's statistics.
  // ---------------------------------------------------------------------
  template<class KV, class YV, class DV, class AV, class IV, class CV>
  __device__ __forceinline__ int32_t constraint_init_cell(const DevMech& M, const DevParams& P, KV keq, YV y,
                                                          DV delta, AV A, IV inv, CV cj, CellCtl& c)
  {
    const int32_t S = M.S;
    for (int32_t iter = 0; iter < P.cinit_max_iter; ++iter)
    {
      for (int32_t i = 0; i < S; ++i)
        delta[i] = 0.0;
      constraint_forcing(M, keq, y, delta);
      double max_res = 0.0;
      bool any_nan = false, any_inf = false;
      for (int32_t i = 0; i < S; ++i)
        if (M.mass[i] == 0.0)
        {
          const double v = delta[i];
          any_nan = any_nan || isnan(v);
          any_inf = any_inf || isinf(v);
          const double a = fabs(v);
          if (!isnan(a) && !isinf(a))
            max_res = (max_res > a ? max_res : a);
        }
      if (any_nan)
        return MICMB_SOLVER_NAN_DETECTED;
      if (any_inf)
        return MICMB_SOLVER_INF_DETECTED;
      c.init_iterations = iter + 1;
      if (max_res < P.cinit_tol)
        return MICMB_SOLVER_CONVERGED;
      // the constraints' -dG/dy, then alpha = 1 times the mass diagonal, then the LU
      constraint_jacobian(M, keq, y, cj);
      c.jacobian_updates += 1;
      lu_decompose_gathered<false>(M, M.lu_s, M.diag_row_of, cj, 1.0, A, inv, cj);
      c.decompositions += 1;
      solve_lower<1>(M.fwd_s, A, delta, 0);
      solve_upper<1>(M.bwd_s, A, delta, 0);
      c.solves += 1;
      for (int32_t i = 0; i < S; ++i)
        if (M.mass[i] == 0.0)
        {
          const double d = delta[i];
          any_nan = any_nan || isnan(d);
          any_inf = any_inf || isinf(d);
          if (!isnan(d) && !isinf(d))
            y[i] = y[i] + d;
        }
      if (any_nan)
        return MICMB_SOLVER_NAN_DETECTED;
      if (any_inf)
        return MICMB_SOLVER_INF_DETECTED;
    }
    return MICMB_SOLVER_CONSTRAINT_INITIALIZATION_FAILED;
  }
}  // namespace micmb
