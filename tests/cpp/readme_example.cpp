// README example of micm (README.md:95-135) written against micm's CUDA-path
// API, compiled against the B200 solver's micm.hpp instead of micm's headers.
#include <micm_b200/micm.hpp>

#include <cstring>
#include <iomanip>
#include <iostream>

using namespace micm;

int main(int argc, char** argv)
{
  auto foo = Species{ "Foo" };
  auto bar = Species{ "Bar" };
  auto baz = Species{ "Baz" };

  Phase gas_phase{ "gas", std::vector<PhaseSpecies>{ foo, bar, baz } };
  System chemical_system{ gas_phase };

  Process r1 = ChemicalReactionBuilder()
                   .SetReactants({ foo })
                   .SetProducts({ StoichSpecies(bar, 0.8), StoichSpecies(baz, 0.2) })
                   .SetRateConstant(ArrheniusRateConstantParameters{ .A_ = 1.0e-3 })
                   .SetPhase(gas_phase)
                   .Build();
  Process r2 = ChemicalReactionBuilder()
                   .SetReactants({ foo, bar })
                   .SetProducts({ StoichSpecies(baz, 1) })
                   .SetRateConstant(ArrheniusRateConstantParameters{ .A_ = 1.0e-5, .C_ = 110.0 })
                   .SetPhase(gas_phase)
                   .Build();
  std::vector<Process> reactions{ r1, r2 };

  try
  {
    auto solver = CudaSolverBuilderInPlace<CudaRosenbrockSolverParameters, 1>(
                      RosenbrockSolverParameters::ThreeStageRosenbrockParameters())
                      .SetSystem(chemical_system)
                      .SetReactions(reactions)
                      .Build();
    if (argc > 1 && std::strcmp(argv[1], "fused") == 0)
      solver.SetMethod(Method::Fused);
    auto state = solver.GetState();
    state.conditions_[0].temperature_ = 287.45;  // K
    state.conditions_[0].pressure_ = 101319.9;   // Pa
    state.conditions_[0].CalculateIdealAirDensity();
    state[foo] = 20.0;  // mol m-3
    state.PrintHeader();
    for (int i = 0; i < 10; ++i)
    {
      state.SyncInputsToDevice();
      solver.UpdateStateParameters(state);
      auto result = solver.Solve(500.0, state);
      state.SyncOutputsToHost();
      if (result.state_ != SolverState::Converged)
        return 2;
      state.PrintState(i * 500);
    }
  }
  catch (const MicmException& e)
  {
    std::cerr << "MicmException: " << e.what() << std::endl;
    return 3;
  }
  return 0;
}
