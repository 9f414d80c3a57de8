// The constraint classes of micm.hpp reject what micm's reject
// (constraint/types/linear_constraint.hpp:150-172,
// equilibrium_constraint.hpp:208-245) and the builder rejects constraints on
// species outside the system; all before any device call.  Prints one line
// per case: "<case> ok" when the expected MicmException was thrown.
#include <micm_b200/micm.hpp>

#include <cstdio>
#include <functional>

using namespace micm;

static int Expect(const char* name, const std::function<void()>& f)
{
  try
  {
    f();
  }
  catch (const MicmException&)
  {
    std::printf("%s ok\n", name);
    return 0;
  }
  std::printf("%s no exception\n", name);
  return 1;
}

int main()
{
  auto A = Species("A");
  auto B = Species("B");
  auto C = Species("C");
  auto X = Species("X");
  Phase gas_phase{ "gas", std::vector<PhaseSpecies>{ A, B, C } };
  using D = VectorMatrix<Real, 4>;
  int failures = 0;
  failures += Expect("linear_without_terms", [&] { LinearConstraint<D, D>("c", C, {}, 1.0); });
  failures += Expect("equilibrium_without_reactants", [&] {
    EquilibriumConstraint<D, D>("c", C, {}, { { C, 1.0 } }, { .K_HLC_ref_ = 1.0, .delta_H_ = 0.0 });
  });
  failures += Expect("equilibrium_without_products", [&] {
    EquilibriumConstraint<D, D>("c", C, { { B, 1.0 } }, {}, { .K_HLC_ref_ = 1.0, .delta_H_ = 0.0 });
  });
  failures += Expect("equilibrium_nonpositive_stoichiometry", [&] {
    EquilibriumConstraint<D, D>("c", C, { { B, 0.0 } }, { { C, 1.0 } }, { .K_HLC_ref_ = 1.0, .delta_H_ = 0.0 });
  });
  failures += Expect("equilibrium_nonpositive_constant", [&] {
    EquilibriumConstraint<D, D>("c", C, { { B, 1.0 } }, { { C, 1.0 } }, { .K_HLC_ref_ = 0.0, .delta_H_ = 0.0 });
  });
  failures += Expect("species_outside_the_system", [&] {
    Process rxn = ChemicalReactionBuilder()
                      .SetReactants({ A })
                      .SetProducts({ { B, 1 } })
                      .SetRateConstant(ArrheniusRateConstantParameters{ .A_ = 0.1 })
                      .SetPhase(gas_phase)
                      .Build();
    std::vector<Constraint<D, D>> constraints;
    constraints.emplace_back(LinearConstraint<D, D>("c", X, { { A, 1.0 }, { X, 1.0 } }, 1.0));
    auto solver = CudaSolverBuilderInPlace<CudaRosenbrockSolverParameters, 4>(
                      RosenbrockSolverParameters::FourStageDifferentialAlgebraicRosenbrockParameters())
                      .SetSystem(System(gas_phase))
                      .SetReactions({ rxn })
                      .SetConstraints(std::move(constraints))
                      .Build();
  });
  return failures;
}
