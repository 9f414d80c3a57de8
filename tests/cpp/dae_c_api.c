/* A DAE mechanism through the plain C ABI (micmb.h): A -> B (Arrhenius,
 * A = 0.1) with the equilibrium constraint C = K_eq(T) B replacing C's row
 * (micm's test/integration/test_equilibrium_constraint.cpp system).  Compiles
 * the mechanism on the host and prints its LU-filled Jacobian pattern, one
 * "row col" pair per line, after the line "nnz <n>". */
#include "micmb.h"

#include <stdio.h>
#include <string.h>

int main(void)
{
  double rate_params[MICMB_RATE_PARAM_STRIDE];
  memset(rate_params, 0, sizeof rate_params);
  rate_params[0] = 0.1; /* A */
  rate_params[3] = 300.0; /* D, micm's default */
  const int32_t rate_type[1] = { MICMB_RATE_ARRHENIUS };
  const int32_t reactant_start[2] = { 0, 1 }, reactant_species[1] = { 0 };
  const int32_t product_start[2] = { 0, 1 }, product_species[1] = { 1 };
  const double product_yield[1] = { 1.0 };
  /* the constraint: algebraic species C (2); reactant B (1), product C (2) */
  const int32_t c_type[1] = { MICMB_CONSTRAINT_EQUILIBRIUM }, c_species[1] = { 2 };
  const int32_t c_term_start[2] = { 0, 2 }, c_term_species[2] = { 1, 2 }, c_n_reactants[1] = { 1 };
  const double c_term_coef[2] = { 1.0, 1.0 };
  const double c_params[4] = { 0.034, -2400.0, 1.380649e-23 * 6.02214076e23, 298.15 };

  micmb_mechanism_desc d;
  memset(&d, 0, sizeof d);
  d.n_species = 3;
  d.n_reactions = 1;
  d.rate_type = rate_type;
  d.rate_params = rate_params;
  d.reactant_start = reactant_start;
  d.reactant_species = reactant_species;
  d.product_start = product_start;
  d.product_species = product_species;
  d.product_yield = product_yield;
  d.reorder_state = 0;
  d.n_constraints = 1;
  d.constraint_type = c_type;
  d.constraint_species = c_species;
  d.constraint_term_start = c_term_start;
  d.constraint_term_species = c_term_species;
  d.constraint_term_coef = c_term_coef;
  d.constraint_n_reactants = c_n_reactants;
  d.constraint_params = c_params;

  micmb_mechanism* m = NULL;
  if (micmb_mechanism_create(&d, &m) != MICMB_OK)
  {
    fprintf(stderr, "create: %s\n", micmb_last_error());
    return 1;
  }
  micmb_mechanism_info info;
  if (micmb_mechanism_get_info(m, &info) != MICMB_OK)
    return 2;
  int32_t rows[64], cols[64];
  if (info.jacobian_nnz > 64 || micmb_mechanism_jacobian_pattern(m, rows, cols) != MICMB_OK)
    return 3;
  printf("nnz %d\n", info.jacobian_nnz);
  for (int32_t e = 0; e < info.jacobian_nnz; ++e)
    printf("%d %d\n", rows[e], cols[e]);
  micmb_mechanism_destroy(m);
  return 0;
}
