/*
 * oracle.c -- TEST INFRASTRUCTURE ONLY: plain-C restatement of micm's
 * Rosenbrock path and its discrete adjoint.  See oracle.h for the reference
 * locations each part restates.  Dense n x n maps are used for the symbolic
 * steps (fine for the test sizes, n <= a few thousand).
 */
#define _GNU_SOURCE
#include "oracle.h"

#include <math.h>
#include <quadmath.h>
#include <pthread.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

static __thread char g_err[256];

const char* om_last_error(void)
{
  return g_err;
}

struct om_mech
{
  int S, R, P, nnz, n_info;
  int* species_col;  /* [S] system species -> column */
  int* reaction_col; /* [R] input reaction -> rate column */
  int* kind;         /* by rate column */
  double* rp;        /* [R][MICMB_RATE_PARAM_STRIDE] */
  int* pcol;
  int* nmult;
  double* mult; /* [R][4][4] */
  int *rs, *rid;  /* reactants by rate column (state columns) */
  int *ps, *pid;  /* products */
  double* py;
  int *info_ind, *info_rxn, *info_ds, *info_dep;
  int* pos; /* [S*S] storage position or -1 */
  int *nz_row, *nz_col;
  int cr; /* 0: the C library's exp/pow/log10 (micm's); 1: correctly rounded (quad precision) */
  /* algebraic constraints (DAE form, constraint_set.hpp): each replaces the
   * ODE row of its algebraic species (mass-matrix diagonal 0 there) */
  int nc, n_eq, n_cterms;
  int *c_kind, *c_row, *c_t0, *c_t1, *c_nreact, *c_keq;
  double* c_par;   /* [nc][4] */
  int* ct_col;     /* term state columns */
  double* ct_coef; /* coefficient / stoichiometry */
  int* ct_pos;     /* LU position of (row, term column) */
  double* mass;    /* [S] 1 ODE row, 0 algebraic row */
  char* alg;       /* [S] algebraic row */
};

#define NA 6.02214076e23
#define KB 1.380649e-23
#define RGAS (KB * NA)
#define PI 3.14159265358979323846

static void* xcalloc(size_t n, size_t s)
{
  void* p = calloc(n ? n : 1, s ? s : 1);
  if (!p)
  {
    fprintf(stderr, "oracle: out of memory\n");
    abort();
  }
  return p;
}

void om_destroy(om_mech* m)
{
  if (!m)
    return;
  free(m->species_col);
  free(m->reaction_col);
  free(m->kind);
  free(m->rp);
  free(m->pcol);
  free(m->nmult);
  free(m->mult);
  free(m->rs);
  free(m->rid);
  free(m->ps);
  free(m->pid);
  free(m->py);
  free(m->info_ind);
  free(m->info_rxn);
  free(m->info_ds);
  free(m->info_dep);
  free(m->pos);
  free(m->nz_row);
  free(m->nz_col);
  free(m->c_kind);
  free(m->c_row);
  free(m->c_t0);
  free(m->c_t1);
  free(m->c_nreact);
  free(m->c_keq);
  free(m->c_par);
  free(m->ct_col);
  free(m->ct_coef);
  free(m->ct_pos);
  free(m->mass);
  free(m->alg);
  free(m);
}

/* Markowitz (linear_solver.inl:30-124) on a dense 0/1 pattern; perm[new] = old. */
static void markowitz(int n, unsigned char* M, int* perm)
{
  uint64_t* rd = xcalloc(n, sizeof(uint64_t));
  uint64_t* cd = xcalloc(n, sizeof(uint64_t));
  unsigned char* alive = xcalloc(n, 1);
  int* cols = xcalloc(n, sizeof(int));
  int* ins = xcalloc(n, sizeof(int));
  for (int i = 0; i < n; ++i)
  {
    alive[i] = 1;
    for (int j = 0; j < n; ++j)
      if (M[(size_t)i * n + j])
      {
        rd[i]++;
        cd[j]++;
      }
  }
  for (int step = 0; step < n; ++step)
  {
    int pivot = n;
    uint64_t best = UINT64_MAX;
    for (int v = 0; v < n; ++v)
    {
      if (!alive[v])
        continue;
      uint64_t cost = (rd[v] - 1u) * (cd[v] - 1u);
      if (pivot == n || cost < best)
      {
        best = cost;
        pivot = v;
      }
    }
    perm[step] = pivot;
    alive[pivot] = 0;
    int nc = 0, ni = 0;
    for (int c = 0; c < n; ++c)
      if (c != pivot && alive[c] && M[(size_t)pivot * n + c])
        cols[nc++] = c;
    for (int i = 0; i < n; ++i)
      if (i != pivot && alive[i] && M[(size_t)i * n + pivot])
        ins[ni++] = i;
    for (int a = 0; a < ni; ++a)
      for (int b = 0; b < nc; ++b)
        if (!M[(size_t)ins[a] * n + cols[b]])
        {
          M[(size_t)ins[a] * n + cols[b]] = 1;
          rd[ins[a]]++;
          cd[cols[b]]++;
        }
    for (int b = 0; b < nc; ++b)
    {
      M[(size_t)pivot * n + cols[b]] = 0;
      cd[cols[b]]--;
    }
    for (int a = 0; a < ni; ++a)
    {
      M[(size_t)ins[a] * n + pivot] = 0;
      rd[ins[a]]--;
    }
  }
  free(rd);
  free(cd);
  free(alive);
  free(cols);
  free(ins);
}

om_mech* om_create(const micmb_mechanism_desc* d)
{
  const int S = d->n_species, R = d->n_reactions;
  if (S <= 0 || R < 0)
  {
    snprintf(g_err, sizeof g_err, "bad sizes");
    return NULL;
  }
  om_mech* m = xcalloc(1, sizeof(om_mech));
  m->S = S;
  m->R = R;
  /* 1. stable counting sort by kind (solver_builder.inl:274-329) */
  int* order = xcalloc(R, sizeof(int));
  {
    int k = 0;
    for (int kind = 0; kind <= MICMB_RATE_SURFACE; ++kind)
      for (int r = 0; r < R; ++r)
        if (d->rate_type[r] == kind)
          order[k++] = r;
    if (k != R)
    {
      snprintf(g_err, sizeof g_err, "unsupported rate kind");
      free(order);
      om_destroy(m);
      return NULL;
    }
  }
  m->reaction_col = xcalloc(R, sizeof(int));
  for (int i = 0; i < R; ++i)
    m->reaction_col[order[i]] = i;
  /* 2. species columns */
  m->species_col = xcalloc(S, sizeof(int));
  unsigned char* M = xcalloc((size_t)S * S, 1);
  for (int r = 0; r < R; ++r)
    for (int i = d->reactant_start[r]; i < d->reactant_start[r + 1]; ++i)
    {
      int ind = d->reactant_species[i];
      if (ind < 0)
        continue;
      for (int j = d->reactant_start[r]; j < d->reactant_start[r + 1]; ++j)
        if (d->reactant_species[j] >= 0)
          M[(size_t)d->reactant_species[j] * S + ind] = 1;
      for (int j = d->product_start[r]; j < d->product_start[r + 1]; ++j)
        M[(size_t)d->product_species[j] * S + ind] = 1;
    }
  if (d->reorder_state)
  {
    int* perm = xcalloc(S, sizeof(int));
    markowitz(S, M, perm);
    for (int i = 0; i < S; ++i)
      m->species_col[perm[i]] = i;
    free(perm);
  }
  else
    for (int i = 0; i < S; ++i)
      m->species_col[i] = i;
  /* 2b. constraints: algebraic rows (solver_builder.inl:345-393) */
  m->mass = xcalloc(S, sizeof(double));
  m->alg = xcalloc(S, 1);
  for (int i = 0; i < S; ++i)
    m->mass[i] = 1.0;
  m->nc = d->n_constraints > 0 ? d->n_constraints : 0;
  if (m->nc)
  {
    const int nt = d->constraint_term_start[m->nc];
    m->n_cterms = nt;
    m->c_kind = xcalloc(m->nc, sizeof(int));
    m->c_row = xcalloc(m->nc, sizeof(int));
    m->c_t0 = xcalloc(m->nc, sizeof(int));
    m->c_t1 = xcalloc(m->nc, sizeof(int));
    m->c_nreact = xcalloc(m->nc, sizeof(int));
    m->c_keq = xcalloc(m->nc, sizeof(int));
    m->c_par = xcalloc((size_t)m->nc * 4, sizeof(double));
    m->ct_col = xcalloc(nt + 1, sizeof(int));
    m->ct_coef = xcalloc(nt + 1, sizeof(double));
    m->ct_pos = xcalloc(nt + 1, sizeof(int));
    for (int c = 0; c < m->nc; ++c)
    {
      const int row = m->species_col[d->constraint_species[c]];
      if (m->alg[row])
      {
        snprintf(g_err, sizeof g_err, "a species is the algebraic variable of two constraints");
        free(order);
        om_destroy(m);
        return NULL;
      }
      m->alg[row] = 1;
      m->mass[row] = 0.0;
      m->c_kind[c] = d->constraint_type[c];
      m->c_row[c] = row;
      m->c_t0[c] = d->constraint_term_start[c];
      m->c_t1[c] = d->constraint_term_start[c + 1];
      m->c_nreact[c] = m->c_kind[c] == MICMB_CONSTRAINT_EQUILIBRIUM ? d->constraint_n_reactants[c] : 0;
      m->c_keq[c] = m->c_kind[c] == MICMB_CONSTRAINT_EQUILIBRIUM ? m->n_eq++ : -1;
      memcpy(m->c_par + 4 * (size_t)c, d->constraint_params + 4 * (size_t)c, 4 * sizeof(double));
      for (int t = m->c_t0[c]; t < m->c_t1[c]; ++t)
      {
        m->ct_col[t] = m->species_col[d->constraint_term_species[t]];
        m->ct_coef[t] = d->constraint_term_coef[t];
      }
    }
  }
  /* 3. tables by rate column */
  m->kind = xcalloc(R, sizeof(int));
  m->rp = xcalloc((size_t)R * MICMB_RATE_PARAM_STRIDE, sizeof(double));
  m->pcol = xcalloc(R, sizeof(int));
  m->nmult = xcalloc(R, sizeof(int));
  m->mult = xcalloc((size_t)R * 16, sizeof(double));
  m->rs = xcalloc(R + 1, sizeof(int));
  m->ps = xcalloc(R + 1, sizeof(int));
  const int nre = d->reactant_start[R], npr = d->product_start[R];
  m->rid = xcalloc(nre, sizeof(int));
  m->pid = xcalloc(npr, sizeof(int));
  m->py = xcalloc(npr, sizeof(double));
  int next_param = 0, nr = 0, np = 0;
  for (int rc = 0; rc < R; ++rc)
  {
    const int r = order[rc];
    const double* p = d->rate_params + (size_t)r * MICMB_RATE_PARAM_STRIDE;
    double* q = m->rp + (size_t)rc * MICMB_RATE_PARAM_STRIDE;
    memcpy(q, p, sizeof(double) * MICMB_RATE_PARAM_STRIDE);
    m->kind[rc] = d->rate_type[r];
    m->pcol[rc] = -1;
    if (m->kind[rc] == MICMB_RATE_BRANCHED)
    {
      /* reaction_rate_store.hpp:268-281 */
      double n = floor(p[4]);
      double k0 = 2.0e-22 * NA * 1.0e-6 * exp(n);
      double air_ref = 2.45e19 / NA * 1.0e6;
      double a = k0 * air_ref;
      double b = 0.43 * pow(293.0 / 298.0, -8.0);
      double A_val = a / (1.0 + a / b) * pow(0.41, 1.0 / (1.0 + pow(log10(a / b), 2.0)));
      q[5] = k0;
      q[6] = A_val * (1.0 - p[3]) / p[3];
    }
    else if (m->kind[rc] == MICMB_RATE_USER_DEFINED)
    {
      m->pcol[rc] = next_param;
      next_param += 1;
    }
    else if (m->kind[rc] == MICMB_RATE_SURFACE)
    {
      q[1] = 8.0 * RGAS / (PI * p[1]);
      m->pcol[rc] = next_param;
      next_param += 2;
    }
    for (int i = d->reactant_start[r]; i < d->reactant_start[r + 1]; ++i)
    {
      int s = d->reactant_species[i];
      if (s >= 0)
        m->rid[nr++] = m->species_col[s];
      else
      {
        const double* c = d->parameterized_coef + 4 * (size_t)(-s - 1);
        memcpy(m->mult + ((size_t)rc * 4 + m->nmult[rc]) * 4, c, 4 * sizeof(double));
        m->nmult[rc]++;
      }
    }
    m->rs[rc + 1] = nr;
    for (int i = d->product_start[r]; i < d->product_start[r + 1]; ++i)
    {
      m->pid[np] = m->species_col[d->product_species[i]];
      m->py[np] = d->product_yield[i];
      np++;
    }
    m->ps[rc + 1] = np;
  }
  m->P = next_param;
  /* 4. jacobian infos (process_set.hpp:329-391): stable by independent column */
  m->info_ind = xcalloc(nr, sizeof(int));
  m->info_rxn = xcalloc(nr, sizeof(int));
  m->info_ds = xcalloc(nr + 1, sizeof(int));
  m->info_dep = xcalloc(nr * 3 + 1, sizeof(int));
  {
    int ni = 0, nd = 0;
    for (int ind = 0; ind < S; ++ind)
      for (int rc = 0; rc < R; ++rc)
        for (int i = m->rs[rc]; i < m->rs[rc + 1]; ++i)
          if (m->rid[i] == ind)
          {
            m->info_ind[ni] = ind;
            m->info_rxn[ni] = rc;
            int found = 0;
            for (int j = m->rs[rc]; j < m->rs[rc + 1]; ++j)
            {
              if (m->rid[j] == ind && !found)
              {
                found = 1;
                continue;
              }
              m->info_dep[nd++] = m->rid[j];
            }
            ni++;
            m->info_ds[ni] = nd;
          }
    m->n_info = ni;
  }
  /* 5. sparsity + diagonal, LU fill, storage positions */
  memset(M, 0, (size_t)S * S);
  for (int rc = 0; rc < R; ++rc)
    for (int i = m->rs[rc]; i < m->rs[rc + 1]; ++i)
    {
      int ind = m->rid[i];
      for (int j = m->rs[rc]; j < m->rs[rc + 1]; ++j)
        M[(size_t)m->rid[j] * S + ind] = 1;
      for (int j = m->ps[rc]; j < m->ps[rc + 1]; ++j)
        M[(size_t)m->pid[j] * S + ind] = 1;
    }
  for (int i = 0; i < S; ++i)
    M[(size_t)i * S + i] = 1;
  /* algebraic rows: kinetic entries out, the constraint's entries and diagonal in */
  for (int i = 0; i < S; ++i)
    if (m->alg[i])
      memset(M + (size_t)i * S, 0, S);
  for (int c = 0; c < m->nc; ++c)
  {
    M[(size_t)m->c_row[c] * S + m->c_row[c]] = 1;
    for (int t = m->c_t0[c]; t < m->c_t1[c]; ++t)
      M[(size_t)m->c_row[c] * S + m->ct_col[t]] = 1;
  }
  for (int i = 0; i < S; ++i)
    for (int k = i + 1; k < S; ++k)
      if (M[(size_t)i * S + k])
        for (int j = i + 1; j < S; ++j)
          if (M[(size_t)j * S + i])
            M[(size_t)j * S + k] = 1;
  m->pos = xcalloc((size_t)S * S, sizeof(int));
  int nnz = 0;
  for (size_t i = 0; i < (size_t)S * S; ++i)
    nnz += M[i];
  m->nz_row = xcalloc(nnz, sizeof(int));
  m->nz_col = xcalloc(nnz, sizeof(int));
  nnz = 0;
  for (int i = 0; i < S; ++i)
    for (int j = 0; j < S; ++j)
    {
      if (M[(size_t)i * S + j])
      {
        m->pos[(size_t)i * S + j] = nnz;
        m->nz_row[nnz] = i;
        m->nz_col[nnz] = j;
        nnz++;
      }
      else
        m->pos[(size_t)i * S + j] = -1;
    }
  m->nnz = nnz;
  for (int c = 0; c < m->nc; ++c)
    for (int t = m->c_t0[c]; t < m->c_t1[c]; ++t)
      m->ct_pos[t] = m->pos[(size_t)m->c_row[c] * S + m->ct_col[t]];
  free(M);
  free(order);
  return m;
}

int om_n_params(const om_mech* m)
{
  return m->P;
}
int om_nnz(const om_mech* m)
{
  return m->nnz;
}
void om_species_columns(const om_mech* m, int32_t* out)
{
  for (int i = 0; i < m->S; ++i)
    out[i] = m->species_col[i];
}
void om_reaction_columns(const om_mech* m, int32_t* out)
{
  for (int i = 0; i < m->R; ++i)
    out[i] = m->reaction_col[i];
}
void om_jacobian_pattern(const om_mech* m, int32_t* rows, int32_t* cols)
{
  for (int e = 0; e < m->nnz; ++e)
  {
    rows[e] = m->nz_row[e];
    cols[e] = m->nz_col[e];
  }
}

/* ---------------------------------------------------------------- */
/* rate constants (rate_constant_functions.hpp:52-136)               */
/* ---------------------------------------------------------------- */
/* The transcendental functions of the rate constants and the step-size
 * factor: the C library's (what micm calls), or correctly rounded results
 * (evaluated in quad precision by libquadmath, then rounded once to double;
 * wrong only when the exact value lies within about 2^-60 ulp of a rounding
 * boundary).  The second mode is an independent check of the GPU library's
 * own correctly rounded functions. */
static double o_exp(const om_mech* m, double x)
{
  return m->cr ? (double)expq((__float128)x) : exp(x);
}
static double o_pow(const om_mech* m, double x, double y)
{
  return m->cr ? (double)powq((__float128)x, (__float128)y) : pow(x, y);
}
static double o_log10(const om_mech* m, double x)
{
  return m->cr ? (double)log10q((__float128)x) : log10(x);
}

void om_set_correctly_rounded(om_mech* m, int on)
{
  m->cr = on ? 1 : 0;
}

/* exp (fn 0), log10 (1) or pow (2) with the mode's functions, element-wise
 * (for tests of both modes) */
void om_math_eval(const om_mech* m, int fn, const double* x, const double* y, double* out, int64_t n)
{
  for (int64_t i = 0; i < n; ++i)
    out[i] = fn == 0 ? o_exp(m, x[i]) : (fn == 1 ? o_log10(m, x[i]) : o_pow(m, x[i], y[i]));
}

static double falloff(const om_mech* m, const double* p, double T, double rho, double scale)
{
  double k0 = p[0] * o_exp(m, p[2] / T) * o_pow(m, T / 300.0, p[1]);
  double kinf = p[3] * o_exp(m, p[5] / T) * o_pow(m, T / 300.0, p[4]);
  double ratio = k0 * rho / kinf;
  return k0 * scale / (1.0 + ratio) * o_pow(m, p[6], p[7] / (p[7] + o_pow(m, o_log10(m, ratio), 2.0)));
}

static double rate_constant(const om_mech* m, int r, double T, double Pr, double rho, const double* prm)
{
  const double* p = m->rp + (size_t)r * MICMB_RATE_PARAM_STRIDE;
  double k = 0.0;
  switch (m->kind[r])
  {
    case MICMB_RATE_ARRHENIUS: k = p[0] * o_exp(m, p[2] / T) * o_pow(m, T / p[3], p[1]) * (1.0 + p[4] * Pr); break;
    case MICMB_RATE_TROE: k = falloff(m, p, T, rho, rho); break;
    case MICMB_RATE_TERNARY_CHEMICAL_ACTIVATION: k = falloff(m, p, T, rho, 1.0); break;
    case MICMB_RATE_BRANCHED:
    {
      double a = p[5] * rho;
      double b = 0.43 * o_pow(m, T / 298.0, -8.0);
      double A_val = a / (1.0 + a / b) * o_pow(m, 0.41, 1.0 / (1.0 + o_pow(m, o_log10(m, a / b), 2.0)));
      double pre = p[1] * o_exp(m, -p[2] / T);
      k = (p[0] == 0.0) ? pre * (p[6] / (p[6] + A_val)) : pre * (A_val / (A_val + p[6]));
      break;
    }
    case MICMB_RATE_TUNNELING: k = p[0] * o_exp(m, -p[1] / T + p[2] / (T * T * T)); break;
    case MICMB_RATE_TAYLOR_SERIES:
    {
      double poly = 0.0, tp = 1.0;
      int n = (int)p[5];
      for (int j = 0; j < n; ++j, tp *= T)
        poly += p[6 + j] * tp;
      k = poly * p[0] * o_exp(m, p[2] / T) * o_pow(m, T / p[3], p[1]) * (1.0 + p[4] * Pr);
      break;
    }
    case MICMB_RATE_REVERSIBLE: k = p[0] * o_exp(m, p[1] / T) * p[2]; break;
    case MICMB_RATE_USER_DEFINED: k = prm[m->pcol[r]] * p[0]; break;
    case MICMB_RATE_SURFACE:
    {
      double radius = prm[m->pcol[r]], num = prm[m->pcol[r] + 1];
      double mfs = sqrt(p[1] * T);
      k = 4.0 * num * PI * radius * radius / (radius / p[0] + 4.0 / (mfs * p[2]));
      break;
    }
  }
  if (m->nmult[r] > 0)
  {
    double v = 1.0;
    for (int i = 0; i < m->nmult[r]; ++i)
    {
      const double* c = m->mult + ((size_t)r * 4 + i) * 4;
      v *= c[0] + c[1] * T + c[2] * Pr + c[3] * rho;
    }
    k *= v;
  }
  return k;
}

void om_rate_constants(const om_mech* m, int n, const double* T, const double* P, const double* rho,
                       const double* params, double* k_out)
{
  for (int c = 0; c < n; ++c)
    for (int r = 0; r < m->R; ++r)
      k_out[(size_t)c * m->R + r] = rate_constant(m, r, T[c], P[c], rho[c], params + (size_t)c * m->P);
}

/* ---------------------------------------------------------------- */
/* per-cell numerics in micm's scatter order                         */
/* ---------------------------------------------------------------- */
static void forcing(const om_mech* m, const double* k, const double* y, double* f)
{
  for (int s = 0; s < m->S; ++s)
    f[s] = 0.0;
  for (int r = 0; r < m->R; ++r)
  {
    double rate = k[r];
    for (int i = m->rs[r]; i < m->rs[r + 1]; ++i)
      rate *= y[m->rid[i]];
    for (int i = m->rs[r]; i < m->rs[r + 1]; ++i)
      if (!m->alg[m->rid[i]])
        f[m->rid[i]] -= rate;
    for (int i = m->ps[r]; i < m->ps[r + 1]; ++i)
      if (!m->alg[m->pid[i]])
        f[m->pid[i]] += m->py[i] * rate;
  }
}

/* jac = -J (process_set.hpp:594-670) */
static void neg_jacobian(const om_mech* m, const double* k, const double* y, double* jac)
{
  const int S = m->S;
  for (int e = 0; e < m->nnz; ++e)
    jac[e] = 0.0;
  for (int q = 0; q < m->n_info; ++q)
  {
    int rc = m->info_rxn[q], ind = m->info_ind[q];
    double d = k[rc];
    for (int i = m->info_ds[q]; i < m->info_ds[q + 1]; ++i)
      d *= y[m->info_dep[i]];
    /* process terms of algebraic rows are skipped (process_set.hpp:623-660) */
    for (int i = m->info_ds[q]; i < m->info_ds[q + 1]; ++i)
      if (!m->alg[m->info_dep[i]])
        jac[m->pos[(size_t)m->info_dep[i] * S + ind]] += d;
    if (!m->alg[ind])
      jac[m->pos[(size_t)ind * S + ind]] += d;
    for (int i = m->ps[rc]; i < m->ps[rc + 1]; ++i)
      if (!m->alg[m->pid[i]])
        jac[m->pos[(size_t)m->pid[i] * S + ind]] -= m->py[i] * d;
  }
}

/* max(c, 0)^e, as the equilibrium constraint raises concentrations */
static double cpow_clamped(const om_mech* m, double c, double e)
{
  return o_pow(m, (c > 0.0 ? c : 0.0), e);
}

/* constraint residuals overwrite the algebraic rows of f
 * (linear_constraint.hpp:216-259, equilibrium_constraint.hpp:367-424) */
static void constraint_forcing(const om_mech* m, const double* keq, const double* y, double* f)
{
  for (int c = 0; c < m->nc; ++c)
  {
    if (m->c_kind[c] == MICMB_CONSTRAINT_LINEAR)
    {
      double sum = 0.0;
      for (int t = m->c_t0[c]; t < m->c_t1[c]; ++t)
        sum += m->ct_coef[t] * y[m->ct_col[t]];
      f[m->c_row[c]] = sum - m->c_par[4 * c];
    }
    else
    {
      double rp = keq[m->c_keq[c]], pp = 1.0;
      const int tr = m->c_t0[c] + m->c_nreact[c];
      for (int t = m->c_t0[c]; t < tr; ++t)
        rp *= cpow_clamped(m, y[m->ct_col[t]], m->ct_coef[t]);
      for (int t = tr; t < m->c_t1[c]; ++t)
        pp *= cpow_clamped(m, y[m->ct_col[t]], m->ct_coef[t]);
      f[m->c_row[c]] = rp - pp;
    }
  }
}

/* jac -= dG/dy for every constraint (linear_constraint.hpp:264-290,
 * equilibrium_constraint.hpp:432-580) */
static void constraint_neg_jacobian(const om_mech* m, const double* keq, const double* y, double* jac)
{
  for (int c = 0; c < m->nc; ++c)
  {
    if (m->c_kind[c] == MICMB_CONSTRAINT_LINEAR)
    {
      for (int t = m->c_t0[c]; t < m->c_t1[c]; ++t)
        jac[m->ct_pos[t]] -= m->ct_coef[t];
      continue;
    }
    const int t0 = m->c_t0[c], tr = t0 + m->c_nreact[c], t1 = m->c_t1[c];
    const double K = keq[m->c_keq[c]];
    for (int side = 0; side < 2; ++side)
    {
      const int a = side ? tr : t0, b = side ? t1 : tr;
      for (int i = a; i < b; ++i)
      {
        double prod = side ? 1.0 : K;
        for (int j = a; j < b; ++j)
          if (j != i)
            prod *= cpow_clamped(m, y[m->ct_col[j]], m->ct_coef[j]);
        const double conc = y[m->ct_col[i]], st = m->ct_coef[i];
        double partial;
        if (st == 1.0)
          partial = prod;
        else if (conc > 0.0)
          partial = st * prod * o_pow(m, conc, st - 1.0);
        else
          partial = 0.0;
        if (side)
          jac[m->ct_pos[i]] += partial;
        else
          jac[m->ct_pos[i]] -= partial;
      }
    }
  }
}

/* K_eq(T) per equilibrium constraint (equilibrium_constraint.hpp:290-309) */
void om_constraint_params(const om_mech* m, int n, const double* T, double* keq)
{
  for (int c0 = 0; c0 < n; ++c0)
    for (int c = 0; c < m->nc; ++c)
      if (m->c_kind[c] == MICMB_CONSTRAINT_EQUILIBRIUM)
      {
        const double* q = m->c_par + 4 * c;
        keq[(size_t)c0 * m->n_eq + m->c_keq[c]] = q[0] * o_exp(m, (q[1] / q[2]) * (1.0 / T[c0] - 1.0 / q[3]));
      }
}

int om_n_eq(const om_mech* m)
{
  return m->n_eq;
}

static void decompose(const om_mech* m, double* A)
{
  const int S = m->S;
  for (int i = 0; i < S; ++i)
  {
    double inv = 1.0 / A[m->pos[(size_t)i * S + i]];
    for (int j = i + 1; j < S; ++j)
    {
      int pji = m->pos[(size_t)j * S + i];
      if (pji >= 0)
        A[pji] *= inv;
    }
    for (int k = i + 1; k < S; ++k)
    {
      int pik = m->pos[(size_t)i * S + k];
      if (pik < 0)
        continue;
      for (int j = i + 1; j < S; ++j)
      {
        int pji = m->pos[(size_t)j * S + i];
        if (pji < 0)
          continue;
        A[m->pos[(size_t)j * S + k]] -= A[pji] * A[pik];
      }
    }
  }
}

static void lu_solve(const om_mech* m, const double* A, double* x)
{
  const int S = m->S;
  for (int i = 0; i < S; ++i)
    for (int j = 0; j < i; ++j)
    {
      int p = m->pos[(size_t)i * S + j];
      if (p >= 0)
        x[i] -= A[p] * x[j];
    }
  for (int i = S - 1; i >= 0; --i)
  {
    for (int j = i + 1; j < S; ++j)
    {
      int p = m->pos[(size_t)i * S + j];
      if (p >= 0)
        x[i] -= A[p] * x[j];
    }
    x[i] /= A[m->pos[(size_t)i * S + i]];
  }
}

/* (LU)^T z = g : U^T w = g, then L^T z = w */
static void lu_solve_transposed(const om_mech* m, const double* A, double* x)
{
  const int S = m->S;
  for (int i = 0; i < S; ++i)
  {
    for (int j = 0; j < i; ++j)
    {
      int p = m->pos[(size_t)j * S + i];
      if (p >= 0)
        x[i] -= A[p] * x[j];
    }
    x[i] /= A[m->pos[(size_t)i * S + i]];
  }
  for (int i = S - 1; i >= 0; --i)
    for (int j = i + 1; j < S; ++j)
    {
      int p = m->pos[(size_t)j * S + i];
      if (p >= 0)
        x[i] -= A[p] * x[j];
    }
}

/* ---------------------------------------------------------------- */
/* Rosenbrock (rosenbrock.inl:12-402) for one cell                   */
/* ---------------------------------------------------------------- */
typedef struct
{
  double* Y;
  double* Ynew;
  double* F0;
  double* K;
  double* Yerr;
  double* J;
  double* scratch; /* adjoint workspace */
} work_t;

static void work_alloc(work_t* w, const om_mech* m, int stages)
{
  const int S = m->S;
  w->Y = xcalloc(S, sizeof(double));
  w->Ynew = xcalloc(S, sizeof(double));
  w->F0 = xcalloc(S, sizeof(double));
  w->K = xcalloc((size_t)stages * S, sizeof(double));
  w->Yerr = xcalloc(S, sizeof(double));
  w->J = xcalloc(m->nnz, sizeof(double));
  w->scratch = xcalloc((size_t)(4 * stages + 8) * S + m->R, sizeof(double));
}

static void work_free(work_t* w)
{
  free(w->Y);
  free(w->Ynew);
  free(w->F0);
  free(w->K);
  free(w->Yerr);
  free(w->J);
  free(w->scratch);
}

static double dmin(double a, double b)
{
  return (b < a) ? b : a; /* std::min */
}
static double dmax(double a, double b)
{
  return (a < b) ? b : a; /* std::max */
}

/* Solver::PostSolveClamp (solver.hpp:275-297): std::max(y, 0) on every
 * variable; with constraints only the ODE variables are clamped, by
 * (y > 0 ? y : 0), and the algebraic ones are left as solved. */
static double post_clamp(const om_mech* m, int i, double v)
{
  if (!m->nc)
    return (v < 0.0) ? 0.0 : v;
  return m->mass[i] > 0.0 ? (v > 0.0 ? v : 0.0) : v;
}

/* returns state; stats[0..6]; optionally records accepted (y_n, H_n) */
/* micm's InitializeConstraints (rosenbrock.inl:407-576) for one cell: Newton
 * iterations on the algebraic variables until max |G| over algebraic rows is
 * below the tolerance.  Returns the solver state; counts its Jacobian
 * updates, decompositions and solves, and the iterations in *iters. */
static int initialize_constraints(const om_mech* m, const micmb_rosenbrock_params* p, const double* keq, double* Y,
                                  work_t* w, int64_t* ju, int64_t* dec, int64_t* sol, int64_t* iters)
{
  const int S = m->S;
  double* delta = w->F0;
  for (int iter = 0; iter < p->constraint_init_max_iterations; ++iter)
  {
    for (int i = 0; i < S; ++i)
      delta[i] = 0.0;
    constraint_forcing(m, keq, Y, delta);
    double max_res = 0.0;
    int any_nan = 0, any_inf = 0;
    for (int i = 0; i < S; ++i)
      if (m->mass[i] == 0.0)
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
    *iters = iter + 1;
    if (max_res < p->constraint_init_tolerance)
      return MICMB_SOLVER_CONVERGED;
    for (int e = 0; e < m->nnz; ++e)
      w->J[e] = 0.0;
    constraint_neg_jacobian(m, keq, Y, w->J);
    (*ju)++;
    for (int i = 0; i < S; ++i)
      w->J[m->pos[(size_t)i * S + i]] += 1.0 * m->mass[i];
    decompose(m, w->J);
    (*dec)++;
    lu_solve(m, w->J, delta);
    (*sol)++;
    for (int i = 0; i < S; ++i)
      if (m->mass[i] == 0.0)
      {
        const double d = delta[i];
        any_nan = any_nan || isnan(d);
        any_inf = any_inf || isinf(d);
        if (!isnan(d) && !isinf(d))
          Y[i] += d;
      }
    if (any_nan)
      return MICMB_SOLVER_NAN_DETECTED;
    if (any_inf)
      return MICMB_SOLVER_INF_DETECTED;
  }
  return MICMB_SOLVER_CONSTRAINT_INITIALIZATION_FAILED;
}

static int rosenbrock_cell(const om_mech* m, const micmb_rosenbrock_params* p, double dt, const double* k,
                           const double* keq, const double* atol, double rtol, work_t* w, int64_t* stats, double* ck_y,
                           double* ck_h, int max_ck, int* n_ck)
{
  const int S = m->S, ns = p->stages;
  double* Y = w->Y;
  const double h_min = p->h_min == 0.0 ? 1.0e-15 * dt : p->h_min;
  const double h_max = p->h_max == 0.0 ? dt : dmin(dt, p->h_max);
  const double h_start = p->h_start == 0.0 ? 1.0e-6 * dt : dmin(h_max, p->h_start);
  double H = dmin(dmax(h_min, fabs(h_start)), fabs(h_max));
  double t = 0.0;
  int reject_last = 0, reject_more = 0, state = MICMB_SOLVER_RUNNING;
  int64_t fc = 0, ju = 0, nst = 0, acc = 0, rej = 0, dec = 0, sol = 0, init_iters = 0;
  if (n_ck)
    *n_ck = 0;
  if (m->nc)
  {
    const int st = initialize_constraints(m, p, keq, Y, w, &ju, &dec, &sol, &init_iters);
    if (st != MICMB_SOLVER_CONVERGED)
      state = st;
  }
  while (state == MICMB_SOLVER_RUNNING && (t - dt + p->round_off) <= 0)
  {
    if (nst > p->max_number_of_steps)
    {
      state = MICMB_SOLVER_CONVERGENCE_EXCEEDED_MAX_STEPS;
      break;
    }
    if (((t + 0.1 * H) == t) || (H <= p->round_off))
    {
      state = MICMB_SOLVER_STEP_SIZE_TOO_SMALL;
      break;
    }
    H = dmin(H, fabs(dt - t));
    forcing(m, k, Y, w->F0);
    if (m->nc)
      constraint_forcing(m, keq, Y, w->F0);
    fc++;
    neg_jacobian(m, k, Y, w->J);
    if (m->nc)
      constraint_neg_jacobian(m, keq, Y, w->J);
    ju++;
    int accepted = 0;
    while (!accepted)
    {
      double alpha = 1.0 / (H * p->gamma[0]);
      for (int i = 0; i < S; ++i)
        w->J[m->pos[(size_t)i * S + i]] += alpha * m->mass[i]; /* alpha M - J */
      decompose(m, w->J);
      dec++;
      for (int s = 0; s < ns; ++s)
      {
        const int sc = s * (s - 1) / 2;
        double* Ks = w->K + (size_t)s * S;
        if (s == 0)
          memcpy(Ks, w->F0, sizeof(double) * S);
        else if (p->new_function_evaluation[s])
        {
          memcpy(w->Ynew, Y, sizeof(double) * S);
          for (int j = 0; j < s; ++j)
            for (int i = 0; i < S; ++i)
              w->Ynew[i] += p->a[sc + j] * w->K[(size_t)j * S + i];
          forcing(m, k, w->Ynew, Ks);
          if (m->nc)
            constraint_forcing(m, keq, w->Ynew, Ks);
          fc++;
        }
        if (s + 1 < ns && !p->new_function_evaluation[s + 1])
          memcpy(w->K + (size_t)(s + 1) * S, Ks, sizeof(double) * S);
        for (int j = 0; j < s; ++j)
        {
          double coh = p->c[sc + j] / H;
          for (int i = 0; i < S; ++i)
            if (m->mass[i] != 0.0) /* algebraic rows have no mass coupling */
              Ks[i] += coh * w->K[(size_t)j * S + i];
        }
        lu_solve(m, w->J, Ks);
        sol++;
      }
      memcpy(w->Ynew, Y, sizeof(double) * S);
      for (int s = 0; s < ns; ++s)
        for (int i = 0; i < S; ++i)
          w->Ynew[i] += p->m[s] * w->K[(size_t)s * S + i];
      for (int i = 0; i < S; ++i)
        w->Yerr[i] = 0.0;
      for (int s = 0; s < ns; ++s)
        for (int i = 0; i < S; ++i)
          w->Yerr[i] += p->e[s] * w->K[(size_t)s * S + i];
      for (int c = 0; c < m->nc; ++c) /* SetAlgebraicErrors: the step change */
        w->Yerr[m->c_row[c]] = w->Ynew[m->c_row[c]] - Y[m->c_row[c]];
      double sum = 0.0;
      for (int i = 0; i < S; ++i)
      {
        double ay = fabs(Y[i]), an = fabs(w->Ynew[i]);
        double ymax = ay > an ? ay : an;
        double q = w->Yerr[i] / (atol[i] + rtol * ymax);
        sum += q * q;
      }
      double error = dmax(sqrt(sum / (double)(S > 0 ? S : 1)), 1.0e-10);
      double fac = dmin(p->factor_max,
                        dmax(p->factor_min, p->safety_factor / o_pow(m, error, 1 / p->estimator_of_local_order)));
      double Hnew = H * fac;
      nst++;
      if (isnan(error))
      {
        state = MICMB_SOLVER_NAN_DETECTED;
        break;
      }
      if (isinf(error))
      {
        state = MICMB_SOLVER_INF_DETECTED;
        break;
      }
      if ((error < 1) || (H < h_min))
      {
        acc++;
        if (ck_y && n_ck)
        {
          if (*n_ck >= max_ck)
          {
            state = MICMB_SOLVER_CONVERGENCE_EXCEEDED_MAX_STEPS;
            break;
          }
          memcpy(ck_y + (size_t)(*n_ck) * S, Y, sizeof(double) * S);
          ck_h[*n_ck] = H;
          (*n_ck)++;
        }
        t = t + H;
        memcpy(Y, w->Ynew, sizeof(double) * S);
        Hnew = dmax(h_min, dmin(Hnew, h_max));
        if (reject_last)
          Hnew = dmin(Hnew, H);
        reject_last = 0;
        reject_more = 0;
        H = Hnew;
        accepted = 1;
      }
      else
      {
        if (reject_more)
          Hnew = H * p->rejection_factor_decrease;
        reject_more = reject_last;
        reject_last = 1;
        H = Hnew;
        if (acc >= 1)
          rej++;
        neg_jacobian(m, k, Y, w->J);
        if (m->nc)
          constraint_neg_jacobian(m, keq, Y, w->J);
        ju++;
      }
    }
  }
  if (state == MICMB_SOLVER_RUNNING)
    state = MICMB_SOLVER_CONVERGED;
  if (stats)
  {
    stats[0] = fc;
    stats[1] = ju;
    stats[2] = nst;
    stats[3] = acc;
    stats[4] = rej;
    stats[5] = dec;
    stats[6] = sol;
    stats[7] = state;
    memcpy(&stats[8], &t, sizeof(double));
    stats[9] = init_iters;
  }
  return state;
}

/* ---------------------------------------------------------------- */
/* adjoint building blocks: f = sum_r nu_r w_r(y), w_r = k_r prod y  */
/* ---------------------------------------------------------------- */
static double nu_dot(const om_mech* m, int r, const double* v)
{
  double s = 0.0;
  for (int i = m->ps[r]; i < m->ps[r + 1]; ++i)
    s += m->py[i] * v[m->pid[i]];
  for (int i = m->rs[r]; i < m->rs[r + 1]; ++i)
    s -= v[m->rid[i]];
  return s;
}

/* product of reactant concentrations skipping occurrences a and b (-1 = none) */
static double prod_except(const om_mech* m, int r, const double* y, int a, int b)
{
  double v = 1.0;
  for (int i = m->rs[r]; i < m->rs[r + 1]; ++i)
    if (i != a && i != b)
      v *= y[m->rid[i]];
  return v;
}

/* ybar += J(y)^T g ; kbar[r] += (nu_r . g) w_r(y) */
static void vjp_f(const om_mech* m, const double* k, const double* y, const double* g, double* ybar, double* kbar)
{
  for (int r = 0; r < m->R; ++r)
  {
    double c = nu_dot(m, r, g);
    if (c == 0.0)
      continue;
    kbar[r] += c * k[r] * prod_except(m, r, y, -1, -1);
    for (int i = m->rs[r]; i < m->rs[r + 1]; ++i)
      ybar[m->rid[i]] += c * k[r] * prod_except(m, r, y, i, -1);
  }
}

/* second-order term of the Jacobian: for rho = nu_r . Rbar and direction K,
 * ybar += rho * H_r K ; kbar[r] += rho * (grad w_r . K) */
static void jacobian_term(const om_mech* m, const double* k, const double* y, const double* Rbar, const double* K,
                          double* ybar, double* kbar)
{
  for (int r = 0; r < m->R; ++r)
  {
    double rho = nu_dot(m, r, Rbar);
    if (rho == 0.0)
      continue;
    double gk = 0.0;
    for (int i = m->rs[r]; i < m->rs[r + 1]; ++i)
      gk += k[r] * prod_except(m, r, y, i, -1) * K[m->rid[i]];
    kbar[r] += rho * gk;
    for (int i = m->rs[r]; i < m->rs[r + 1]; ++i)
      for (int j = m->rs[r]; j < m->rs[r + 1]; ++j)
        if (i != j)
          ybar[m->rid[j]] += rho * k[r] * prod_except(m, r, y, i, j) * K[m->rid[i]];
  }
}

static void adjoint_cell(const om_mech* m, const micmb_rosenbrock_params* p, const double* k, const double* ck_y,
                         const double* ck_h, int n_ck, double* ybar, double* kbar, work_t* w)
{
  const int S = m->S, ns = p->stages;
  double* Ys = w->scratch;                      /* [ns][S] stage inputs */
  double* Kb = Ys + (size_t)ns * S;             /* [ns][S] */
  double* Gb = Kb + (size_t)ns * S;             /* [ns][S] */
  double* Rb = Gb + (size_t)ns * S;             /* [ns][S] */
  double* yb = Rb + (size_t)ns * S;             /* [S] */
  double* tmp = yb + S;                         /* [S] */
  for (int n = n_ck - 1; n >= 0; --n)
  {
    const double* y = ck_y + (size_t)n * S;
    const double H = ck_h[n];
    /* recompute the accepted step */
    forcing(m, k, y, w->F0);
    neg_jacobian(m, k, y, w->J);
    const double alpha = 1.0 / (H * p->gamma[0]);
    for (int i = 0; i < S; ++i)
      w->J[m->pos[(size_t)i * S + i]] += alpha;
    decompose(m, w->J);
    for (int s = 0; s < ns; ++s)
    {
      const int sc = s * (s - 1) / 2;
      double* Ks = w->K + (size_t)s * S;
      memcpy(Ys + (size_t)s * S, y, sizeof(double) * S);
      if (s == 0)
        memcpy(Ks, w->F0, sizeof(double) * S);
      else if (p->new_function_evaluation[s])
      {
        for (int j = 0; j < s; ++j)
          for (int i = 0; i < S; ++i)
            Ys[(size_t)s * S + i] += p->a[sc + j] * w->K[(size_t)j * S + i];
        forcing(m, k, Ys + (size_t)s * S, Ks);
      }
      if (s + 1 < ns && !p->new_function_evaluation[s + 1])
        memcpy(w->K + (size_t)(s + 1) * S, Ks, sizeof(double) * S);
      for (int j = 0; j < s; ++j)
      {
        double coh = p->c[sc + j] / H;
        for (int i = 0; i < S; ++i)
          Ks[i] += coh * w->K[(size_t)j * S + i];
      }
      lu_solve(m, w->J, Ks);
    }
    /* reverse sweep */
    memcpy(yb, ybar, sizeof(double) * S);
    for (int s = 0; s < ns; ++s)
      for (int i = 0; i < S; ++i)
      {
        Kb[(size_t)s * S + i] = p->m[s] * ybar[i];
        Gb[(size_t)s * S + i] = 0.0;
      }
    for (int s = ns - 1; s >= 0; --s)
    {
      const int sc = s * (s - 1) / 2;
      double* rb = Rb + (size_t)s * S;
      memcpy(rb, Kb + (size_t)s * S, sizeof(double) * S);
      lu_solve_transposed(m, w->J, rb);
      for (int i = 0; i < S; ++i)
        Gb[(size_t)s * S + i] += rb[i];
      for (int j = 0; j < s; ++j)
      {
        double coh = p->c[sc + j] / H;
        for (int i = 0; i < S; ++i)
          Kb[(size_t)j * S + i] += coh * rb[i];
      }
      if (s == 0)
        continue;
      if (p->new_function_evaluation[s])
      {
        for (int i = 0; i < S; ++i)
          tmp[i] = 0.0;
        vjp_f(m, k, Ys + (size_t)s * S, Gb + (size_t)s * S, tmp, kbar);
        for (int i = 0; i < S; ++i)
          yb[i] += tmp[i];
        for (int j = 0; j < s; ++j)
          for (int i = 0; i < S; ++i)
            Kb[(size_t)j * S + i] += p->a[sc + j] * tmp[i];
      }
      else
        for (int i = 0; i < S; ++i)
          Gb[(size_t)(s - 1) * S + i] += Gb[(size_t)s * S + i];
    }
    vjp_f(m, k, y, Gb, yb, kbar);
    for (int s = 0; s < ns; ++s)
      jacobian_term(m, k, y, Rb + (size_t)s * S, w->K + (size_t)s * S, yb, kbar);
    memcpy(ybar, yb, sizeof(double) * S);
  }
}

/* ---------------------------------------------------------------- */
/* threaded drivers                                                  */
/* ---------------------------------------------------------------- */
typedef struct
{
  const om_mech* m;
  const micmb_rosenbrock_params* p;
  int n;
  double dt;
  const double *k, *atol;
  const double* keq; /* [cell][n_eq] or NULL */
  double rtol;
  double* y;
  int64_t* stats;
  const double *y0, *ybar_final;
  double *y_final, *ybar0, *kbar;
  int max_ck;
  int next;
  pthread_mutex_t lock;
  int adjoint;
  int failed;
} job_t;

static int take(job_t* j)
{
  pthread_mutex_lock(&j->lock);
  int c = j->next++;
  pthread_mutex_unlock(&j->lock);
  return c;
}

static void* worker(void* arg)
{
  job_t* j = arg;
  const om_mech* m = j->m;
  const int S = m->S;
  work_t w;
  work_alloc(&w, m, j->p->stages);
  double* ck_y = NULL;
  double* ck_h = NULL;
  if (j->adjoint)
  {
    ck_y = xcalloc((size_t)j->max_ck * S, sizeof(double));
    ck_h = xcalloc(j->max_ck, sizeof(double));
  }
  for (;;)
  {
    int c = take(j);
    if (c >= j->n)
      break;
    const double* k = j->k + (size_t)c * m->R;
    if (!j->adjoint)
    {
      memcpy(w.Y, j->y + (size_t)c * S, sizeof(double) * S);
      rosenbrock_cell(m, j->p, j->dt, k, j->keq ? j->keq + (size_t)c * m->n_eq : NULL, j->atol, j->rtol, &w,
                      j->stats ? j->stats + (size_t)c * 10 : NULL, NULL, NULL, 0, NULL);
      for (int i = 0; i < S; ++i)
        j->y[(size_t)c * S + i] = post_clamp(m, i, w.Y[i]);
    }
    else
    {
      int n_ck = 0;
      memcpy(w.Y, j->y0 + (size_t)c * S, sizeof(double) * S);
      int st = rosenbrock_cell(m, j->p, j->dt, k, NULL, j->atol, j->rtol, &w, NULL, ck_y, ck_h, j->max_ck, &n_ck);
      if (st != MICMB_SOLVER_CONVERGED)
        j->failed = 1;
      double* yb = j->ybar0 + (size_t)c * S;
      for (int i = 0; i < S; ++i)
      {
        double v = w.Y[i];
        j->y_final[(size_t)c * S + i] = v < 0.0 ? 0.0 : v;
        yb[i] = v < 0.0 ? 0.0 : j->ybar_final[(size_t)c * S + i]; /* d max(y,0)/dy */
      }
      double* kb = j->kbar + (size_t)c * m->R;
      for (int r = 0; r < m->R; ++r)
        kb[r] = 0.0;
      adjoint_cell(m, j->p, k, ck_y, ck_h, n_ck, yb, kb, &w);
    }
  }
  free(ck_y);
  free(ck_h);
  work_free(&w);
  return NULL;
}

static int run(job_t* j, int n_threads)
{
  if (n_threads < 1)
    n_threads = 1;
  pthread_mutex_init(&j->lock, NULL);
  pthread_t* th = xcalloc(n_threads, sizeof(pthread_t));
  for (int t = 1; t < n_threads; ++t)
    pthread_create(&th[t], NULL, worker, j);
  worker(j);
  for (int t = 1; t < n_threads; ++t)
    pthread_join(th[t], NULL);
  free(th);
  pthread_mutex_destroy(&j->lock);
  return j->failed ? -1 : 0;
}

int om_solve_per_cell_keq(const om_mech* m, const micmb_rosenbrock_params* p, int n, double dt, const double* k,
                          const double* keq, const double* atol, double rtol, double* y, int64_t* stats_out,
                          int n_threads)
{
  if (m->nc && m->n_eq && !keq)
  {
    snprintf(g_err, sizeof g_err, "equilibrium constraints need K_eq values");
    return -1;
  }
  job_t j;
  memset(&j, 0, sizeof j);
  j.m = m;
  j.p = p;
  j.n = n;
  j.dt = dt;
  j.k = k;
  j.keq = m->nc ? keq : NULL;
  j.atol = atol;
  j.rtol = rtol;
  j.y = y;
  j.stats = stats_out;
  return run(&j, n_threads);
}

int om_solve_per_cell(const om_mech* m, const micmb_rosenbrock_params* p, int n, double dt, const double* k,
                      const double* atol, double rtol, double* y, int64_t* stats_out, int n_threads)
{
  return om_solve_per_cell_keq(m, p, n, dt, k, NULL, atol, rtol, y, stats_out, n_threads);
}

/* ---------------------------------------------------------------- */
/* Backward Euler on one cell (backward_euler.inl:12-193: Newton     */
/* iterations on forcing, -J + I/H, the in-place LU and a solve,     */
/* clamped at zero; IsConverged :195-246; default parameters of      */
/* backward_euler_solver_parameters.hpp: small 1e-40, 11 iterations, */
/* step reductions 0.5, 0.5, 0.5, 0.5, 0.1)                          */
/* ---------------------------------------------------------------- */
#define OM_SOLVER_ACCEPTING_UNCONVERGED 8 /* micm's SolverState::AcceptingUnconvergedIntegration */

static int backward_euler_cell(const om_mech* m, double dt, const double* k, const double* atol, double rtol,
                               double* Yn1, double* Yn, double* f, double* J, int64_t* stats)
{
  const int S = m->S;
  const double small = 1.0e-40;
  const int max_iter = 11;
  const double reductions[5] = { 0.5, 0.5, 0.5, 0.5, 0.1 };
  int64_t st[7] = { 0 }; /* function_calls, jacobian_updates, number_of_steps, accepted, rejected,
                            decompositions, solves */
  double H = dt, t = 0.0;
  int n_ok = 0, n_fail = 0, state = MICMB_SOLVER_NOT_YET_CALLED;
  memcpy(Yn, Yn1, sizeof(double) * S);
  while (t < dt)
  {
    state = MICMB_SOLVER_RUNNING;
    int converged = 0, iterations = 0;
    do
    {
      st[2]++;
      forcing(m, k, Yn1, f);
      st[0]++;
      neg_jacobian(m, k, Yn1, J);
      st[1]++;
      for (int i = 0; i < S; ++i)
        J[m->pos[(size_t)i * S + i]] += 1 / H;
      decompose(m, J);
      st[5]++;
      for (int i = 0; i < S; ++i)
        f[i] -= (Yn1[i] - Yn[i]) / H;
      lu_solve(m, J, f);
      st[6]++;
      for (int i = 0; i < S; ++i)
      {
        const double v = Yn1[i] + f[i];
        Yn1[i] = (0.0 > v) ? 0.0 : v;
      }
      if (iterations++ == 0)
        continue;
      converged = 1;
      for (int i = 0; i < S; ++i)
      {
        const double r = f[i];
        if (!isfinite(r))
          converged = 0;
        else if (fabs(r) > small && fabs(r) > atol[i] && fabs(r) > rtol * fabs(Yn1[i]))
          converged = 0;
      }
    } while (!converged && iterations < max_iter);
    if (!converged)
    {
      st[4]++;
      n_ok = 0;
      if (n_fail >= 5)
      {
        t += H;
        state = OM_SOLVER_ACCEPTING_UNCONVERGED;
        int any_nan = 0, any_inf = 0;
        for (int i = 0; i < S; ++i)
        {
          any_nan = any_nan || isnan(Yn1[i]);
          any_inf = any_inf || isinf(Yn1[i]);
        }
        if (any_nan)
          state = MICMB_SOLVER_NAN_DETECTED;
        else if (any_inf)
          state = MICMB_SOLVER_INF_DETECTED;
        break;
      }
      memcpy(Yn1, Yn, sizeof(double) * S);
      H *= reductions[n_fail++];
    }
    else
    {
      st[3]++;
      state = MICMB_SOLVER_CONVERGED;
      t += H;
      memcpy(Yn, Yn1, sizeof(double) * S);
      if (++n_ok >= 2)
      {
        n_ok = 0;
        H *= 2.0;
      }
    }
    H = dmin(H, dt - t);
  }
  if (stats)
  {
    for (int q = 0; q < 7; ++q)
      stats[q] = st[q];
    stats[7] = state;
    memcpy(&stats[8], &t, sizeof(double));
    stats[9] = 0;
  }
  return state;
}

/* Backward Euler per cell (a 1-cell State per cell), one Solve(dt) each.
 * y [cell][column] in/out; stats_out [cell][10] as om_solve_per_cell's. */
int om_backward_euler_per_cell(const om_mech* m, int n, double dt, const double* k, const double* atol, double rtol,
                               double* y, int64_t* stats_out)
{
  const int S = m->S;
  double* Yn = xcalloc(S, sizeof(double));
  double* f = xcalloc(S, sizeof(double));
  double* J = xcalloc(m->nnz, sizeof(double));
  for (int c = 0; c < n; ++c)
    backward_euler_cell(m, dt, k + (size_t)c * m->R, atol, rtol, y + (size_t)c * S, Yn, f, J,
                        stats_out ? stats_out + (size_t)c * 10 : NULL);
  free(Yn);
  free(f);
  free(J);
  return 0;
}

/* ---------------------------------------------------------------- */
/* global step control (one step size for all cells), micm's          */
/* AbstractRosenbrockSolver::Solve on a multi-cell State               */
/* (rosenbrock.inl:12-304), with the error norm's sum over cells       */
/* formed in a fixed order that a GPU reproduces: per cell in species  */
/* order, per block of 256 cells a pairwise tree, per shard each of    */
/* 256 lanes adds the blocks b = lane, lane + 256, ... in order and a  */
/* tree joins the lanes, and the shards' sums are added in rank order. */
/* micm itself adds all values with one accumulator, so the two agree  */
/* to rounding (exactly for one cell).                                 */
/* ---------------------------------------------------------------- */
static double tree256(double* red)
{
  for (int w = 128; w > 0; w >>= 1)
    for (int t = 0; t < w; ++t)
      red[t] += red[t + w];
  return red[0];
}

static double shard_error_sum(const double* cell_sum, int n)
{
  const int n_blk = (n + 255) / 256;
  double* blk = xcalloc(n_blk > 0 ? n_blk : 1, sizeof(double));
  double red[256];
  for (int b = 0; b < n_blk; ++b)
  {
    for (int t = 0; t < 256; ++t)
    {
      const int c = b * 256 + t;
      red[t] = c < n ? cell_sum[c] : 0.0;
    }
    blk[b] = tree256(red);
  }
  for (int t = 0; t < 256; ++t)
  {
    double acc = 0.0;
    for (int b = t; b < n_blk; b += 256)
      acc += blk[b];
    red[t] = acc;
  }
  free(blk);
  return tree256(red);
}

/* A shard's flags and maximum as one value for the exchange: NaN when any
 * value was NaN, +Inf when any was infinite, else the maximum.  Combining
 * encoded values by om_max_combine keeps micm's order of checks (NaN first). */
static double encode_max(int any_nan, int any_inf, double max_value)
{
  if (any_nan)
    return NAN;
  if (any_inf)
    return INFINITY;
  return max_value;
}

double om_max_combine(double a, double b)
{
  if (isnan(a) || isnan(b))
    return NAN;
  if (isinf(a) || isinf(b))
    return INFINITY;
  return a > b ? a : b;
}

/* micm's InitializeConstraints (rosenbrock.inl:407-576) on an n-cell State:
 * the largest |G| over every cell's algebraic rows decides convergence, and
 * while it is not met every cell takes the Newton update (one Jacobian
 * update, decomposition and solve counted per iteration for the State).
 * With `exchange`, the shard's encoded maximum goes through exchange(v,
 * OM_EXCHANGE_MAX, user) and the job's comes back. */
static int initialize_constraints_global(const om_mech* m, const micmb_rosenbrock_params* p, int n,
                                         const double* keq, double* y, double* delta, double* J,
                                         om_exchange_fn exchange, void* user, int64_t* ju, int64_t* dec,
                                         int64_t* sol, int64_t* iters)
{
  const int S = m->S;
  for (int iter = 0; iter < p->constraint_init_max_iterations; ++iter)
  {
    int any_nan = 0, any_inf = 0;
    double max_res = 0.0;
    for (int c = 0; c < n; ++c)
    {
      double* d = delta + (size_t)c * S;
      for (int i = 0; i < S; ++i)
        d[i] = 0.0;
      constraint_forcing(m, keq + (size_t)c * m->n_eq, y + (size_t)c * S, d);
      for (int i = 0; i < S; ++i)
        if (m->mass[i] == 0.0)
        {
          const double v = d[i];
          any_nan = any_nan || isnan(v);
          any_inf = any_inf || isinf(v);
          const double a = fabs(v);
          if (!isnan(a) && !isinf(a))
            max_res = (max_res > a ? max_res : a);
        }
    }
    double v = encode_max(any_nan, any_inf, max_res);
    if (exchange)
      v = exchange(v, OM_EXCHANGE_MAX, user);
    if (isnan(v))
      return MICMB_SOLVER_NAN_DETECTED;
    if (isinf(v))
      return MICMB_SOLVER_INF_DETECTED;
    *iters = iter + 1;
    if (v < p->constraint_init_tolerance)
      return MICMB_SOLVER_CONVERGED;
    for (int c = 0; c < n; ++c)
    {
      double* Jc = J + (size_t)c * m->nnz;
      double* d = delta + (size_t)c * S;
      for (int e = 0; e < m->nnz; ++e)
        Jc[e] = 0.0;
      constraint_neg_jacobian(m, keq + (size_t)c * m->n_eq, y + (size_t)c * S, Jc);
      for (int i = 0; i < S; ++i)
        Jc[m->pos[(size_t)i * S + i]] += 1.0 * m->mass[i];
      decompose(m, Jc);
      lu_solve(m, Jc, d);
    }
    (*ju)++;
    (*dec)++;
    (*sol)++;
    any_nan = any_inf = 0;
    for (int c = 0; c < n; ++c)
    {
      const double* d = delta + (size_t)c * S;
      double* yc = y + (size_t)c * S;
      for (int i = 0; i < S; ++i)
        if (m->mass[i] == 0.0)
        {
          any_nan = any_nan || isnan(d[i]);
          any_inf = any_inf || isinf(d[i]);
          if (!isnan(d[i]) && !isinf(d[i]))
            yc[i] += d[i];
        }
    }
    v = encode_max(any_nan, any_inf, 0.0);
    if (exchange)
      v = exchange(v, OM_EXCHANGE_MAX, user);
    if (isnan(v))
      return MICMB_SOLVER_NAN_DETECTED;
    if (isinf(v))
      return MICMB_SOLVER_INF_DETECTED;
  }
  return MICMB_SOLVER_CONSTRAINT_INITIALIZATION_FAILED;
}

/* y [cell][column] in/out, k [cell][R]; stats_out [10] as one row of
 * om_solve_per_cell's.  n_shards / shard_start: the cells split into shards
 * (shard_start[0] = 0, shard_start[n_shards] = n), the job's sum is the
 * shards' sums in shard order.  With `exchange` set, the n cells are this
 * rank's shard only: exchange(this shard's sum, OM_EXCHANGE_SUM, user) returns the job's sum,
 * and total_cells counts every rank's cells. */
int om_solve_global(const om_mech* m, const micmb_rosenbrock_params* p, int n, double dt, const double* k,
                    const double* keq, const double* atol, double rtol, double* y, int64_t* stats_out, int n_shards,
                    const int* shard_start, om_exchange_fn exchange, void* user, int64_t total_cells)
{
  const int S = m->S, ns = p->stages;
  if (m->nc && m->n_eq && !keq)
  {
    snprintf(g_err, sizeof g_err, "equilibrium constraints need K_eq values");
    return -1;
  }
  const double* kq = keq;
  double kq_none = 0.0;
  if (!kq)
    kq = &kq_none;
  const size_t nS = (size_t)n * S;
  double* F0 = xcalloc(nS + 1, sizeof(double));
  double* Ynew = xcalloc(nS + 1, sizeof(double));
  double* Yerr = xcalloc(nS + 1, sizeof(double));
  double* K = xcalloc((size_t)ns * nS + 1, sizeof(double));
  double* J = xcalloc((size_t)n * m->nnz + 1, sizeof(double));
  double* cell_sum = xcalloc((size_t)n + 1, sizeof(double));
  const double h_min = p->h_min == 0.0 ? 1.0e-15 * dt : p->h_min;
  const double h_max = p->h_max == 0.0 ? dt : dmin(dt, p->h_max);
  const double h_start = p->h_start == 0.0 ? 1.0e-6 * dt : dmin(h_max, p->h_start);
  double H = dmin(dmax(h_min, fabs(h_start)), fabs(h_max));
  double t = 0.0;
  int reject_last = 0, reject_more = 0, state = MICMB_SOLVER_RUNNING;
  int64_t fc = 0, ju = 0, nst = 0, acc = 0, rej = 0, dec = 0, sol = 0, init_iters = 0;
  const double n_values = (double)(exchange ? total_cells : n) * (double)S;
  if (m->nc)
  {
    const int st = initialize_constraints_global(m, p, n, kq, y, F0, J, exchange, user, &ju, &dec, &sol,
                                                 &init_iters);
    if (st != MICMB_SOLVER_CONVERGED)
      state = st;
  }
  while ((t - dt + p->round_off) <= 0 && state == MICMB_SOLVER_RUNNING)
  {
    if (nst > p->max_number_of_steps)
    {
      state = MICMB_SOLVER_CONVERGENCE_EXCEEDED_MAX_STEPS;
      break;
    }
    if (((t + 0.1 * H) == t) || (H <= p->round_off))
    {
      state = MICMB_SOLVER_STEP_SIZE_TOO_SMALL;
      break;
    }
    H = dmin(H, fabs(dt - t));
    for (int c = 0; c < n; ++c)
    {
      forcing(m, k + (size_t)c * m->R, y + (size_t)c * S, F0 + (size_t)c * S);
      if (m->nc)
        constraint_forcing(m, kq + (size_t)c * m->n_eq, y + (size_t)c * S, F0 + (size_t)c * S);
    }
    fc++;
    for (int c = 0; c < n; ++c)
      {
        neg_jacobian(m, k + (size_t)c * m->R, y + (size_t)c * S, J + (size_t)c * m->nnz);
        if (m->nc)
          constraint_neg_jacobian(m, kq + (size_t)c * m->n_eq, y + (size_t)c * S, J + (size_t)c * m->nnz);
      }
    ju++;
    int accepted = 0;
    while (!accepted)
    {
      const double alpha = 1.0 / (H * p->gamma[0]);
      for (int c = 0; c < n; ++c)
      {
        double* Jc = J + (size_t)c * m->nnz;
        for (int i = 0; i < S; ++i)
          Jc[m->pos[(size_t)i * S + i]] += alpha * m->mass[i]; /* alpha M - J */
        decompose(m, Jc);
      }
      dec++;
      for (int s = 0; s < ns; ++s)
      {
        const int sc = s * (s - 1) / 2;
        for (int c = 0; c < n; ++c)
        {
          const double* Yc = y + (size_t)c * S;
          double* Ks = K + ((size_t)s * n + c) * S;
          double* Yn = Ynew + (size_t)c * S;
          if (s == 0)
            memcpy(Ks, F0 + (size_t)c * S, sizeof(double) * S);
          else if (p->new_function_evaluation[s])
          {
            memcpy(Yn, Yc, sizeof(double) * S);
            for (int j = 0; j < s; ++j)
              for (int i = 0; i < S; ++i)
                Yn[i] += p->a[sc + j] * K[((size_t)j * n + c) * S + i];
            forcing(m, k + (size_t)c * m->R, Yn, Ks);
            if (m->nc)
              constraint_forcing(m, kq + (size_t)c * m->n_eq, Yn, Ks);
          }
          if (s + 1 < ns && !p->new_function_evaluation[s + 1])
            memcpy(K + ((size_t)(s + 1) * n + c) * S, Ks, sizeof(double) * S);
          for (int j = 0; j < s; ++j)
          {
            const double coh = p->c[sc + j] / H;
            for (int i = 0; i < S; ++i)
              if (m->mass[i] != 0.0) /* algebraic rows have no mass coupling */
                Ks[i] += coh * K[((size_t)j * n + c) * S + i];
          }
          lu_solve(m, J + (size_t)c * m->nnz, Ks);
        }
        if (s > 0 && p->new_function_evaluation[s])
          fc++;
        sol++;
      }
      for (int c = 0; c < n; ++c)
      {
        const double* Yc = y + (size_t)c * S;
        double* Yn = Ynew + (size_t)c * S;
        double* Ye = Yerr + (size_t)c * S;
        memcpy(Yn, Yc, sizeof(double) * S);
        for (int s = 0; s < ns; ++s)
          for (int i = 0; i < S; ++i)
            Yn[i] += p->m[s] * K[((size_t)s * n + c) * S + i];
        for (int i = 0; i < S; ++i)
          Ye[i] = 0.0;
        for (int s = 0; s < ns; ++s)
          for (int i = 0; i < S; ++i)
            Ye[i] += p->e[s] * K[((size_t)s * n + c) * S + i];
        for (int q = 0; q < m->nc; ++q) /* SetAlgebraicErrors: the step change */
          Ye[m->c_row[q]] = Yn[m->c_row[q]] - Yc[m->c_row[q]];
        double sum = 0.0;
        for (int i = 0; i < S; ++i)
        {
          const double ay = fabs(Yc[i]), an = fabs(Yn[i]);
          const double ymax = ay > an ? ay : an;
          const double q = Ye[i] / (atol[i] + rtol * ymax);
          sum += q * q;
        }
        cell_sum[c] = sum;
      }
      double total = 0.0;
      if (exchange)
        total = exchange(shard_error_sum(cell_sum, n), OM_EXCHANGE_SUM, user);
      else
        for (int r = 0; r < n_shards; ++r)
          total += shard_error_sum(cell_sum + shard_start[r], shard_start[r + 1] - shard_start[r]);
      const double error = dmax(sqrt(total / (n_values > 0.0 ? n_values : 1.0)), 1.0e-10);
      const double fac = dmin(p->factor_max,
                              dmax(p->factor_min, p->safety_factor / o_pow(m, error, 1 / p->estimator_of_local_order)));
      double Hnew = H * fac;
      nst++;
      if (isnan(error))
      {
        state = MICMB_SOLVER_NAN_DETECTED;
        break;
      }
      if (isinf(error))
      {
        state = MICMB_SOLVER_INF_DETECTED;
        break;
      }
      if ((error < 1) || (H < h_min))
      {
        acc++;
        t = t + H;
        memcpy(y, Ynew, sizeof(double) * nS);
        Hnew = dmax(h_min, dmin(Hnew, h_max));
        if (reject_last)
          Hnew = dmin(Hnew, H);
        reject_last = 0;
        reject_more = 0;
        H = Hnew;
        accepted = 1;
      }
      else
      {
        if (reject_more)
          Hnew = H * p->rejection_factor_decrease;
        reject_more = reject_last;
        reject_last = 1;
        H = Hnew;
        if (acc >= 1)
          rej++;
        for (int c = 0; c < n; ++c)
          {
        neg_jacobian(m, k + (size_t)c * m->R, y + (size_t)c * S, J + (size_t)c * m->nnz);
        if (m->nc)
          constraint_neg_jacobian(m, kq + (size_t)c * m->n_eq, y + (size_t)c * S, J + (size_t)c * m->nnz);
      }
        ju++;
      }
    }
  }
  if (state == MICMB_SOLVER_RUNNING)
    state = MICMB_SOLVER_CONVERGED;
  for (size_t e = 0; e < nS; ++e)
    y[e] = post_clamp(m, (int)(e % (size_t)(S > 0 ? S : 1)), y[e]);
  if (stats_out)
  {
    stats_out[0] = fc;
    stats_out[1] = ju;
    stats_out[2] = nst;
    stats_out[3] = acc;
    stats_out[4] = rej;
    stats_out[5] = dec;
    stats_out[6] = sol;
    stats_out[7] = state;
    memcpy(&stats_out[8], &t, sizeof(double));
    stats_out[9] = init_iters;
  }
  free(F0);
  free(Ynew);
  free(Yerr);
  free(K);
  free(J);
  free(cell_sum);
  return 0;
}

/* Backward Euler on one n-cell State (micm's multi-cell semantics,
 * backward_euler.inl:10-186): one step size, and an attempt converges only
 * when every cell's test passes (IsConverged :188-246, a logical AND over
 * cells and species).  y [cell][column] in/out, k [cell][R]; stats_out [10]
 * as one row of om_solve_per_cell's. */
int om_backward_euler_global(const om_mech* m, int n, double dt, const double* k, const double* atol, double rtol,
                             double* y, int64_t* stats_out)
{
  const int S = m->S;
  const double small = 1.0e-40;
  const int max_iter = 11;
  const double reductions[5] = { 0.5, 0.5, 0.5, 0.5, 0.1 };
  double* Yn = xcalloc((size_t)n * S, sizeof(double));
  double* f = xcalloc((size_t)n * S, sizeof(double));
  double* J = xcalloc((size_t)m->nnz, sizeof(double));
  int64_t st[7] = { 0 };
  double H = dt, t = 0.0;
  int n_ok = 0, n_fail = 0, state = MICMB_SOLVER_NOT_YET_CALLED;
  memcpy(Yn, y, sizeof(double) * (size_t)n * S);
  while (t < dt)
  {
    state = MICMB_SOLVER_RUNNING;
    int converged = 0, iterations = 0;
    do
    {
      st[2]++;
      st[0]++;
      st[1]++;
      st[5]++;
      st[6]++;
      for (int c = 0; c < n; ++c)
      {
        double* Yc = y + (size_t)c * S;
        double* fc = f + (size_t)c * S;
        const double* Ync = Yn + (size_t)c * S;
        forcing(m, k + (size_t)c * m->R, Yc, fc);
        neg_jacobian(m, k + (size_t)c * m->R, Yc, J);
        for (int i = 0; i < S; ++i)
          J[m->pos[(size_t)i * S + i]] += 1 / H;
        decompose(m, J);
        for (int i = 0; i < S; ++i)
          fc[i] -= (Yc[i] - Ync[i]) / H;
        lu_solve(m, J, fc);
        for (int i = 0; i < S; ++i)
        {
          const double v = Yc[i] + fc[i];
          Yc[i] = (0.0 > v) ? 0.0 : v;
        }
      }
      if (iterations++ == 0)
        continue;
      converged = 1;
      for (size_t e = 0; e < (size_t)n * S; ++e)
      {
        const double r = f[e];
        const int i = (int)(e % (size_t)S);
        if (!isfinite(r))
          converged = 0;
        else if (fabs(r) > small && fabs(r) > atol[i] && fabs(r) > rtol * fabs(y[e]))
          converged = 0;
      }
    } while (!converged && iterations < max_iter);
    if (!converged)
    {
      st[4]++;
      n_ok = 0;
      if (n_fail >= 5)
      {
        t += H;
        state = OM_SOLVER_ACCEPTING_UNCONVERGED;
        int any_nan = 0, any_inf = 0;
        for (size_t e = 0; e < (size_t)n * S; ++e)
        {
          any_nan = any_nan || isnan(y[e]);
          any_inf = any_inf || isinf(y[e]);
        }
        if (any_nan)
          state = MICMB_SOLVER_NAN_DETECTED;
        else if (any_inf)
          state = MICMB_SOLVER_INF_DETECTED;
        break;
      }
      memcpy(y, Yn, sizeof(double) * (size_t)n * S);
      H *= reductions[n_fail++];
    }
    else
    {
      st[3]++;
      state = MICMB_SOLVER_CONVERGED;
      t += H;
      memcpy(Yn, y, sizeof(double) * (size_t)n * S);
      if (++n_ok >= 2)
      {
        n_ok = 0;
        H *= 2.0;
      }
    }
    H = dmin(H, dt - t);
  }
  if (stats_out)
  {
    for (int q = 0; q < 7; ++q)
      stats_out[q] = st[q];
    stats_out[7] = state;
    memcpy(&stats_out[8], &t, sizeof(double));
    stats_out[9] = 0;
  }
  free(Yn);
  free(f);
  free(J);
  return 0;
}

/* One Rosenbrock step of size H from Y (no error estimate), Y <- Y + sum m_s K_s;
 * the stage recurrences of adjoint_cell's recomputation. */
static void fixed_step(const om_mech* m, const micmb_rosenbrock_params* p, const double* k, double H, double* Y,
                       work_t* w)
{
  const int S = m->S, ns = p->stages;
  double* Ys = w->scratch;
  forcing(m, k, Y, w->F0);
  neg_jacobian(m, k, Y, w->J);
  const double alpha = 1.0 / (H * p->gamma[0]);
  for (int i = 0; i < S; ++i)
    w->J[m->pos[(size_t)i * S + i]] += alpha;
  decompose(m, w->J);
  for (int s = 0; s < ns; ++s)
  {
    const int sc = s * (s - 1) / 2;
    double* Ks = w->K + (size_t)s * S;
    if (s == 0)
      memcpy(Ks, w->F0, sizeof(double) * S);
    else if (p->new_function_evaluation[s])
    {
      memcpy(Ys, Y, sizeof(double) * S);
      for (int j = 0; j < s; ++j)
        for (int i = 0; i < S; ++i)
          Ys[i] += p->a[sc + j] * w->K[(size_t)j * S + i];
      forcing(m, k, Ys, Ks);
    }
    if (s + 1 < ns && !p->new_function_evaluation[s + 1])
      memcpy(w->K + (size_t)(s + 1) * S, Ks, sizeof(double) * S);
    for (int j = 0; j < s; ++j)
    {
      double coh = p->c[sc + j] / H;
      for (int i = 0; i < S; ++i)
        Ks[i] += coh * w->K[(size_t)j * S + i];
    }
    lu_solve(m, w->J, Ks);
  }
  for (int i = 0; i < S; ++i)
  {
    double v = Y[i];
    for (int s = 0; s < ns; ++s)
      v += p->m[s] * w->K[(size_t)s * S + i];
    Y[i] = v;
  }
}

int om_replay_per_cell(const om_mech* m, const micmb_rosenbrock_params* p, int n, const double* k, const double* h,
                       const int32_t* n_steps, int max_steps, double* y)
{
  const int S = m->S;
  work_t w;
  work_alloc(&w, m, p->stages);
  for (int c = 0; c < n; ++c)
  {
    double* Y = y + (size_t)c * S;
    for (int q = 0; q < n_steps[c] && q < max_steps; ++q)
      fixed_step(m, p, k + (size_t)c * m->R, h[(size_t)c * max_steps + q], Y, &w);
    for (int i = 0; i < S; ++i)
      Y[i] = Y[i] < 0.0 ? 0.0 : Y[i];
  }
  work_free(&w);
  return 0;
}

/* accepted step sizes of a per-cell solve: h [cell][max_steps], n_steps [cell] */
int om_step_sizes_per_cell(const om_mech* m, const micmb_rosenbrock_params* p, int n, double dt, const double* k,
                           const double* atol, double rtol, const double* y0, int max_steps, double* h,
                           int32_t* n_steps)
{
  const int S = m->S;
  work_t w;
  work_alloc(&w, m, p->stages);
  double* ck_y = xcalloc((size_t)max_steps * S, sizeof(double));
  for (int c = 0; c < n; ++c)
  {
    int nck = 0;
    memcpy(w.Y, y0 + (size_t)c * S, sizeof(double) * S);
    rosenbrock_cell(m, p, dt, k + (size_t)c * m->R, NULL, atol, rtol, &w, NULL, ck_y, h + (size_t)c * max_steps, max_steps,
                    &nck);
    n_steps[c] = nck;
  }
  free(ck_y);
  work_free(&w);
  return 0;
}

int om_adjoint_per_cell(const om_mech* m, const micmb_rosenbrock_params* p, int n, double dt, const double* k,
                        const double* atol, double rtol, const double* y0, const double* ybar_final,
                        double* y_final, double* ybar0, double* kbar, int max_steps_stored, int n_threads)
{
  job_t j;
  memset(&j, 0, sizeof j);
  j.m = m;
  j.p = p;
  j.n = n;
  j.dt = dt;
  j.k = k;
  j.atol = atol;
  j.rtol = rtol;
  j.y0 = y0;
  j.ybar_final = ybar_final;
  j.y_final = y_final;
  j.ybar0 = ybar0;
  j.kbar = kbar;
  j.max_ck = max_steps_stored;
  j.adjoint = 1;
  int rc = run(&j, n_threads);
  if (rc)
    snprintf(g_err, sizeof g_err, "a cell did not converge (or exceeded the checkpoint capacity)");
  return rc;
}
