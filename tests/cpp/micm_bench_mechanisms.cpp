// micm's own benchmark mechanisms (test/benchmark/ts1_mechanism.hpp,
// chapman_mechanism.hpp: bench::Ts1, bench::Chapman), compiled unchanged
// against this library's C++ API and driven the way micm_bench drives them
// (test/benchmark/bench_harness.hpp RunCase: three-stage Rosenbrock, Build,
// GetState, InitState, UpdateStateParameters, Solve(30 s)).  Prints, per
// mechanism, the solver state and accepted steps of one Solve and the first
// cell's concentrations.  Exit code 3 when no CUDA device is present.
#include <micm/GPU.hpp>

#include "chapman_mechanism.hpp"
#include "ts1_mechanism.hpp"

#include <iostream>

template<class Bench>
void Run(micm::Index cells)
{
  auto solver = Bench::Build(micm::CudaSolverBuilderInPlace<micm::CudaRosenbrockSolverParameters, 128>(
      micm::RosenbrockSolverParameters::ThreeStageRosenbrockParameters()));
  auto state = solver.GetState(cells);
  Bench::InitState(state, cells);
  state.SyncInputsToDevice();
  solver.UpdateStateParameters(state);
  auto result = solver.Solve(30.0, state);
  state.SyncOutputsToHost();
  std::cout << Bench::kName << " " << micm::SolverStateToString(result.state_) << " " << result.stats_.accepted_;
  const std::vector<micm::Real> first = state.variables_[0];
  for (auto v : first)
    std::cout << " " << v;
  std::cout << std::endl;
}

int main()
{
  try
  {
    Run<bench::Chapman>(1000);
    Run<bench::Ts1>(1000);
  }
  catch (const micm::MicmException& e)
  {
    std::cerr << "MicmException: " << e.what() << std::endl;
    return 3;
  }
  return 0;
}
