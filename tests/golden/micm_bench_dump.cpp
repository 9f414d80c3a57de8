// micm_bench_dump.cpp -- TEST FIXTURE GENERATOR (run by tests/golden/make_micm_bench.py).
//
// Builds one of micm_bench's mechanisms with micm's own code
// (test/benchmark/ts1_mechanism.hpp: bench::Ts1, MOZART-TS1;
// test/benchmark/chapman_mechanism.hpp: bench::Chapman) and prints, as one
// JSON document:
//   * the mechanism in this repository's description (species in gas-phase
//     order without parameterized species, third-body parameterizations,
//     reactions in input order with rate kind, parameters, reactants,
//     products, custom-parameter labels), recorded from what the benchmark's
//     Build() hands its solver builder;
//   * the benchmark's initial state as micm sets it (InitState) and micm's own
//     state columns for every species and custom parameter;
//   * micm's results on a 4-cell state built by micm_bench's recipe
//     (ThreeStageRosenbrockParameters, CpuSolverBuilderInPlace with vector
//     ordering L = 1, in-place Mozart LU, one State, so one step size for all
//     cells): rate constants after UpdateStateParameters and the variables and
//     statistics after each of 10 Solve(30 s) calls.  Cell c > 0 starts from
//     the InitState values with concentrations scaled by (1 + c/10) and the
//     temperature moved by kTemperatureShift[c] (air density recomputed).
// Usage: micm_bench_dump ts1|chapman.  Nothing here is linked by the product.
#include <micm/CPU.hpp>

#include "chapman_mechanism.hpp"
#include "ts1_mechanism.hpp"

#include <cstdio>
#include <iostream>
#include <map>
#include <sstream>
#include <string>
#include <type_traits>
#include <variant>
#include <vector>

namespace
{
  constexpr int kCells = 4;
  constexpr int kSolves = 10;
  constexpr double kDt = 30.0;
  constexpr double kTemperatureShift[kCells] = { 0.0, -15.0, 10.0, -30.0 };

  std::string Num(double v)
  {
    char b[40];
    std::snprintf(b, sizeof b, "%.17g", v);
    return b;
  }

  std::string Str(const std::string& s)
  {
    std::string o = "\"";
    for (char c : s)
    {
      if (c == '"' || c == '\\')
        o += '\\';
      o += c;
    }
    return o + "\"";
  }

  template<class M>
  std::string Rows(const M& m, std::size_t rows, std::size_t cols)
  {
    std::ostringstream o;
    o << "[";
    for (std::size_t r = 0; r < rows; ++r)
    {
      o << (r ? ",\n  [" : "[");
      for (std::size_t c = 0; c < cols; ++c)
        o << (c ? "," : "") << Num(m[r][c]);
      o << "]";
    }
    o << "]";
    return o.str();
  }

  std::string RateJson(const micm::RateConstantVariant& rc)
  {
    return std::visit(
        [](const auto& p) -> std::string
        {
          using T = std::decay_t<decltype(p)>;
          std::ostringstream o;
          if constexpr (std::is_same_v<T, micm::ArrheniusRateConstantParameters>)
            o << "\"kind\": \"arrhenius\", \"params\": [" << Num(p.A_) << "," << Num(p.B_) << "," << Num(p.C_) << ","
              << Num(p.D_) << "," << Num(p.E_) << "]";
          else if constexpr (std::is_same_v<T, micm::TroeRateConstantParameters>)
            o << "\"kind\": \"troe\", \"params\": [" << Num(p.k0_A_) << "," << Num(p.k0_B_) << "," << Num(p.k0_C_)
              << "," << Num(p.kinf_A_) << "," << Num(p.kinf_B_) << "," << Num(p.kinf_C_) << "," << Num(p.Fc_) << ","
              << Num(p.N_) << "]";
          else if constexpr (std::is_same_v<T, micm::UserDefinedRateConstantParameters>)
            o << "\"kind\": \"user_defined\", \"label\": " << Str(p.label_) << ", \"params\": ["
              << Num(p.scaling_factor_) << "]";
          else if constexpr (std::is_same_v<T, micm::SurfaceRateConstantParameters>)
            o << "\"kind\": \"surface\", \"label\": " << Str(p.label_) << ", \"params\": ["
              << Num(p.phase_species_.diffusion_coefficient_.value()) << ","
              << Num(p.phase_species_.species_.template GetProperty<micm::Real>(
                     micm::property_keys::MOLECULAR_WEIGHT))
              << "," << Num(p.reaction_probability_) << "]";
          else
            throw std::runtime_error("rate-constant kind not used by micm_bench's mechanisms");
          return o.str();
        },
        rc);
  }

  // Stands in for a solver builder: keeps what the benchmark's Build() sets.
  struct Recorder
  {
    micm::System system;
    std::vector<micm::Process> processes;
    Recorder& SetSystem(const micm::System& s)
    {
      system = s;
      return *this;
    }
    Recorder& SetReactions(const std::vector<micm::Process>& p)
    {
      processes = p;
      return *this;
    }
    Recorder& SetIgnoreUnusedSpecies(bool)
    {
      return *this;
    }
    Recorder Build()
    {
      return *this;
    }
  };

  template<class Bench>
  int Dump()
  {
    const Recorder rec = Bench::Build(Recorder{});
    const micm::Phase& gas = rec.system.gas_phase_;
    std::ostream& o = std::cout;

    std::vector<std::string> species;
    std::map<std::string, int> param_index;
    std::ostringstream params;
    for (const auto& ps : gas.phase_species_)
    {
      const auto& s = ps.species_;
      if (s.IsParameterized())
      {
        const auto& f = s.parameterize_;
        params << (param_index.empty() ? "" : ",\n  ") << "{\"name\": " << Str(s.name_) << ", \"coefficients\": ["
               << Num(f.c0_) << "," << Num(f.c_T_) << "," << Num(f.c_P_) << "," << Num(f.c_rho_) << "]}";
        const int at = (int)param_index.size();
        param_index[s.name_] = at;
      }
      else
        species.push_back(s.name_);
    }
    o << "{\n\"name\": " << Str(std::string(Bench::kName)) << ",\n\"source\": \"micm test/benchmark ("
      << Bench::kName << ")\",\n";
    o << "\"species\": [";
    for (std::size_t i = 0; i < species.size(); ++i)
      o << (i ? "," : "") << Str(species[i]);
    o << "],\n\"parameterized\": [" << params.str() << "],\n\"reactions\": [";
    for (std::size_t r = 0; r < rec.processes.size(); ++r)
    {
      const auto& rx = rec.processes[r].process_;
      o << (r ? ",\n  " : "\n  ") << "{" << RateJson(rx.rate_constant_) << ", \"reactants\": [";
      for (std::size_t i = 0; i < rx.reactants_.size(); ++i)
        o << (i ? "," : "") << Str(rx.reactants_[i].name_);
      o << "], \"products\": [";
      for (std::size_t i = 0; i < rx.products_.size(); ++i)
        o << (i ? "," : "") << "[" << Str(rx.products_[i].species_.name_) << ","
          << Num(rx.products_[i].coefficient_) << "]";
      o << "]}";
    }
    o << "],\n";

    // micm_bench's solver: three-stage Rosenbrock, vector ordering, in-place Mozart LU
    using Dense = micm::VectorMatrix<micm::Real, 1>;
    using Sparse = micm::SparseMatrix<micm::Real, micm::SparseMatrixVectorOrdering<1>>;
    using Builder = micm::CpuSolverBuilderInPlace<micm::RosenbrockSolverParameters, Dense, Sparse,
                                                  micm::LuDecompositionMozartInPlace<Sparse>>;
    auto solver = Bench::Build(Builder(micm::RosenbrockSolverParameters::ThreeStageRosenbrockParameters()));
    auto state = solver.GetState(kCells);
    Bench::InitState(state, kCells);

    o << "\"init\": {\"temperature\": " << Num(state.conditions_[0].temperature_)
      << ", \"pressure\": " << Num(state.conditions_[0].pressure_)
      << ", \"air_density\": " << Num(state.conditions_[0].air_density_) << ",\n \"concentrations\": {";
    bool first = true;
    for (const auto& name : species)
    {
      o << (first ? "" : ", ") << Str(name) << ": " << Num(state.variables_[0][state.variable_map_.at(name)]);
      first = false;
    }
    o << "},\n \"custom_parameters\": {";
    std::map<std::string, micm::Index> labels(state.custom_rate_parameter_map_.begin(),
                                              state.custom_rate_parameter_map_.end());
    first = true;
    for (const auto& [label, col] : labels)
    {
      o << (first ? "" : ", ") << Str(label) << ": " << Num(state.custom_rate_parameters_[0][col]);
      first = false;
    }
    o << "}},\n";
    o << "\"micm_columns\": {\"species\": {";
    first = true;
    for (const auto& name : species)
    {
      o << (first ? "" : ", ") << Str(name) << ": " << state.variable_map_.at(name);
      first = false;
    }
    o << "}, \"custom_parameters\": {";
    first = true;
    for (const auto& [label, col] : labels)
    {
      o << (first ? "" : ", ") << Str(label) << ": " << col;
      first = false;
    }
    o << "}},\n";

    // the 4-cell golden case
    const std::size_t S = state.variables_.NumColumns();
    for (int c = 1; c < kCells; ++c)
    {
      for (std::size_t j = 0; j < S; ++j)
        state.variables_[c][j] *= 1.0 + 0.1 * c;
      state.conditions_[c].temperature_ += kTemperatureShift[c];
      state.conditions_[c].CalculateIdealAirDensity();
    }
    o << "\"golden\": {\"cells\": " << kCells << ", \"dt\": " << Num(kDt) << ", \"tableau\": 3"
      << ", \"temperature\": [";
    for (int c = 0; c < kCells; ++c)
      o << (c ? "," : "") << Num(state.conditions_[c].temperature_);
    o << "], \"pressure\": [";
    for (int c = 0; c < kCells; ++c)
      o << (c ? "," : "") << Num(state.conditions_[c].pressure_);
    o << "], \"air_density\": [";
    for (int c = 0; c < kCells; ++c)
      o << (c ? "," : "") << Num(state.conditions_[c].air_density_);
    o << "],\n \"initial_variables\": " << Rows(state.variables_, kCells, S) << ",\n";
    o << " \"custom_parameters\": "
      << Rows(state.custom_rate_parameters_, kCells, state.custom_rate_parameters_.NumColumns()) << ",\n";
    solver.UpdateStateParameters(state);
    o << " \"rate_constants\": " << Rows(state.rate_constants_, kCells, state.rate_constants_.NumColumns())
      << ",\n";
    o << " \"solves\": [";
    for (int k = 0; k < kSolves; ++k)
    {
      const auto result = solver.Solve(kDt, state);
      const auto& st = result.stats_;
      o << (k ? ",\n  " : "\n  ") << "{\"state\": " << Str(micm::SolverStateToString(result.state_))
        << ", \"accepted\": " << st.accepted_ << ", \"rejected\": " << st.rejected_
        << ", \"number_of_steps\": " << st.number_of_steps_ << ", \"function_calls\": " << st.function_calls_
        << ", \"jacobian_updates\": " << st.jacobian_updates_ << ", \"decompositions\": " << st.decompositions_
        << ", \"solves\": " << st.solves_ << ",\n   \"variables\": " << Rows(state.variables_, kCells, S) << "}";
    }
    o << "]}\n}\n";
    return 0;
  }
}  // namespace

int main(int argc, char** argv)
{
  const std::string which = argc > 1 ? argv[1] : "";
  if (which == "ts1")
    return Dump<bench::Ts1>();
  if (which == "chapman")
    return Dump<bench::Chapman>();
  std::cerr << "usage: micm_bench_dump ts1|chapman\n";
  return 2;
}
