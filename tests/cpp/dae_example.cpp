// micm's equilibrium-constraint integration case (test/integration/
// test_equilibrium_constraint.cpp: A -> B, B <=> C held in equilibrium by a
// Van't Hoff constant, C algebraic) written against micm's API with
// SetConstraints, compiled against the B200 solver's micm.hpp.  Three cells at
// different temperatures, started off equilibrium so the constraint
// initialisation iterates.  Prints each output time's state of every cell at
// full precision.  Argument: "plain" (global step control) or "fused"
// (per-cell step control).
#include <micm_b200/micm.hpp>

#include <cstdio>
#include <cstring>
#include <iostream>

using namespace micm;

int main(int argc, char** argv)
{
  auto A = Species("A");
  auto B = Species("B");
  auto C = Species("C");
  Phase gas_phase{ "gas", std::vector<PhaseSpecies>{ A, B, C } };

  Process rxn = ChemicalReactionBuilder()
                    .SetReactants({ A })
                    .SetProducts({ { B, 1 } })
                    .SetRateConstant(ArrheniusRateConstantParameters{ .A_ = 0.1, .B_ = 0, .C_ = 0 })
                    .SetPhase(gas_phase)
                    .Build();

  std::vector<Constraint<VectorMatrix<Real, 4>, VectorMatrix<Real, 4>>> constraints;
  constraints.emplace_back(EquilibriumConstraint<VectorMatrix<Real, 4>, VectorMatrix<Real, 4>>(
      "B_C_eq", C, std::vector<StoichSpecies>{ { B, 1.0 } }, std::vector<StoichSpecies>{ { C, 1.0 } },
      { .K_HLC_ref_ = 0.034, .delta_H_ = -2400.0 }));

  try
  {
    auto solver = CudaSolverBuilderInPlace<CudaRosenbrockSolverParameters, 4>(
                      RosenbrockSolverParameters::FourStageDifferentialAlgebraicRosenbrockParameters())
                      .SetSystem(System(gas_phase))
                      .SetReactions({ rxn })
                      .SetConstraints(std::move(constraints))
                      .SetReorderState(false)
                      .Build();
    if (argc > 1 && std::strcmp(argv[1], "fused") == 0)
      solver.SetMethod(Method::Fused);
    const Index n = 3;
    auto state = solver.GetState(n);
    if (state.constraint_size_ != 1 || state.upper_left_identity_diagonal_[state.variable_map_.at("C")] != 0.0 ||
        state.upper_left_identity_diagonal_[state.variable_map_.at("A")] != 1.0)
      return 4;
    for (Index c = 0; c < n; ++c)
    {
      state.conditions_[c].temperature_ = 280.0 + 15.0 * c;
      state.conditions_[c].pressure_ = 101325.0;
      state.conditions_[c].CalculateIdealAirDensity();
      state.variables_[c][state.variable_map_.at("A")] = 1.0;
      state.variables_[c][state.variable_map_.at("B")] = 0.1;
      state.variables_[c][state.variable_map_.at("C")] = 0.0;
    }
    state.SyncInputsToDevice();
    solver.UpdateStateParameters(state);
    const double outputs[] = { 1.0, 5.0, 20.0, 60.0 };
    double t = 0.0;
    for (double target : outputs)
    {
      auto result = solver.Solve(target - t, state);
      state.SyncOutputsToHost();
      if (result.state_ != SolverState::Converged)
        return 2;
      std::printf("%.17g %lld", target, (long long)result.stats_.constraint_init_iterations_);
      for (Index c = 0; c < n; ++c)
        for (Index i = 0; i < 3; ++i)
          std::printf(" %.17g", (double)state.variables_[c][i]);
      std::printf("\n");
      t = target;
    }
  }
  catch (const MicmException& e)
  {
    std::cerr << "MicmException: " << e.what() << std::endl;
    return 3;
  }
  return 0;
}
