// ref_bridge.cpp -- TEST INFRASTRUCTURE ONLY.
//
// A C ABI over the reference implementation itself (NCAR/micm 3.13.0, header
// only), compiled from the reference's own headers by oracle/Makefile into
// oracle/_ref/libmicm_ref.so.  The product never links or loads this library;
// tests, smoke() and bench.py's CPU baseline use it as the checker.
//
// It builds a micm solver from the same flat mechanism description the
// product takes (include/micmb.h), with
//   CpuSolverBuilderInPlace<RosenbrockSolverParameters, VectorMatrix<double,L>,
//     SparseMatrix<double, SparseMatrixVectorOrdering<L>>,
//     LuDecompositionMozartInPlace<...>>
// (include/micm/solver/solver_builder.hpp:243-255) -- the same algorithm as
// micm's CUDA path (in-place Mozart LU, vector ordering).
//
// All per-cell arrays at this ABI are plain row-major [cell][column] in the
// reference's own column order (species after Markowitz reordering, reactions
// after the type sort); the permutation getters map system order to it.

#include <micm/CPU.hpp>
#include <micm/constraint/constraint.hpp>
#include <micm/constraint/types/equilibrium_constraint.hpp>
#include <micm/constraint/types/linear_constraint.hpp>
#include <micm/solver/solver_builder.hpp>

#include "../include/micmb.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <memory>
#include <string>
#include <thread>
#include <vector>

namespace
{
  template<std::size_t L>
  using DenseL = micm::VectorMatrix<double, L>;
  template<std::size_t L>
  using SparseL = micm::SparseMatrix<double, micm::SparseMatrixVectorOrdering<L>>;
  template<std::size_t L>
  using BuilderL = micm::CpuSolverBuilderInPlace<
      micm::RosenbrockSolverParameters,
      DenseL<L>,
      SparseL<L>,
      micm::LuDecompositionMozartInPlace<SparseL<L>>>;
  template<std::size_t L>
  using SolverL = decltype(std::declval<BuilderL<L>>().Build());
  // micm's Backward Euler on the same matrices and in-place Mozart LU
  using BuilderBE = micm::CpuSolverBuilderInPlace<
      micm::BackwardEulerSolverParameters,
      DenseL<1>,
      SparseL<1>,
      micm::LuDecompositionMozartInPlace<SparseL<1>>>;
  using SolverBE = decltype(std::declval<BuilderBE>().Build());

  thread_local std::string g_error;

  micm::RosenbrockSolverParameters TableauFor(int kind)
  {
    switch (kind)
    {
      case 2: return micm::RosenbrockSolverParameters::TwoStageRosenbrockParameters();
      case 3: return micm::RosenbrockSolverParameters::ThreeStageRosenbrockParameters();
      case 4: return micm::RosenbrockSolverParameters::FourStageRosenbrockParameters();
      case 40: return micm::RosenbrockSolverParameters::FourStageDifferentialAlgebraicRosenbrockParameters();
      case 60: return micm::RosenbrockSolverParameters::SixStageDifferentialAlgebraicRosenbrockParameters();
    }
    throw std::runtime_error("unknown tableau kind");
  }

  struct Built
  {
    micm::System system;
    std::vector<micm::Process> processes;
    std::vector<micm::Species> species;
    int n_species = 0;
    int n_reactions = 0;
    std::vector<int> sorted_position;  // input reaction -> rate column
    // algebraic constraints as the description gives them
    struct ConstraintSpec
    {
      int kind = 0, species = 0, n_react = 0;
      std::vector<std::pair<int, double>> terms;
      double p[4] = { 0, 0, 0, 0 };
    };
    std::vector<ConstraintSpec> constraints;
  };

  std::string SpeciesName(int i)
  {
    return "s" + std::to_string(i);
  }

  Built Build(const micmb_mechanism_desc* d, const double* atol)
  {
    Built b;
    b.n_species = d->n_species;
    b.n_reactions = d->n_reactions;
    std::vector<micm::PhaseSpecies> phase_species;
    for (int i = 0; i < d->n_species; ++i)
    {
      micm::Species s(SpeciesName(i));
      if (atol)
        s.SetProperty<double>("absolute tolerance", atol[i]);
      b.species.push_back(s);
      phase_species.emplace_back(s);
    }
    micm::Phase gas("gas", phase_species);
    b.system = micm::System(gas);
    std::vector<micm::Species> param_species;
    for (int p = 0; p < d->n_parameterized; ++p)
    {
      micm::Species s("param" + std::to_string(p));
      s.parameterize_ = { .c0_ = d->parameterized_coef[4 * p + 0],
                          .c_T_ = d->parameterized_coef[4 * p + 1],
                          .c_P_ = d->parameterized_coef[4 * p + 2],
                          .c_rho_ = d->parameterized_coef[4 * p + 3],
                          .has_value_ = static_cast<micm::Bool>(true) };
      param_species.push_back(s);
    }
    for (int r = 0; r < d->n_reactions; ++r)
    {
      std::vector<micm::Species> reactants;
      for (int i = d->reactant_start[r]; i < d->reactant_start[r + 1]; ++i)
      {
        int s = d->reactant_species[i];
        reactants.push_back(s >= 0 ? b.species[s] : param_species[-s - 1]);
      }
      std::vector<micm::StoichSpecies> products;
      for (int i = d->product_start[r]; i < d->product_start[r + 1]; ++i)
        products.push_back(micm::StoichSpecies{ b.species[d->product_species[i]], d->product_yield[i] });
      const double* p = d->rate_params + (size_t)r * MICMB_RATE_PARAM_STRIDE;
      micm::ChemicalReactionBuilder rb;
      rb.SetReactants(reactants).SetProducts(products).SetPhase(gas);
      std::string label = "r" + std::to_string(r);
      switch (d->rate_type[r])
      {
        case MICMB_RATE_ARRHENIUS:
          rb.SetRateConstant(
              micm::ArrheniusRateConstantParameters{ .A_ = p[0], .B_ = p[1], .C_ = p[2], .D_ = p[3], .E_ = p[4] });
          break;
        case MICMB_RATE_TROE:
          rb.SetRateConstant(micm::TroeRateConstantParameters{ .k0_A_ = p[0],
                                                               .k0_B_ = p[1],
                                                               .k0_C_ = p[2],
                                                               .kinf_A_ = p[3],
                                                               .kinf_B_ = p[4],
                                                               .kinf_C_ = p[5],
                                                               .Fc_ = p[6],
                                                               .N_ = p[7] });
          break;
        case MICMB_RATE_TERNARY_CHEMICAL_ACTIVATION:
          rb.SetRateConstant(micm::TernaryChemicalActivationRateConstantParameters{ .k0_A_ = p[0],
                                                                                    .k0_B_ = p[1],
                                                                                    .k0_C_ = p[2],
                                                                                    .kinf_A_ = p[3],
                                                                                    .kinf_B_ = p[4],
                                                                                    .kinf_C_ = p[5],
                                                                                    .Fc_ = p[6],
                                                                                    .N_ = p[7] });
          break;
        case MICMB_RATE_BRANCHED:
        {
          micm::BranchedRateConstantParameters bp{};
          bp.branch_ = p[0] == 0.0 ? micm::BranchedRateConstantParameters::Branch::Alkoxy
                                   : micm::BranchedRateConstantParameters::Branch::Nitrate;
          bp.X_ = p[1];
          bp.Y_ = p[2];
          bp.a0_ = p[3];
          bp.n_ = (micm::Index)p[4];
          rb.SetRateConstant(bp);
          break;
        }
        case MICMB_RATE_TUNNELING:
          rb.SetRateConstant(micm::TunnelingRateConstantParameters{ .A_ = p[0], .B_ = p[1], .C_ = p[2] });
          break;
        case MICMB_RATE_TAYLOR_SERIES:
        {
          micm::TaylorSeriesRateConstantParameters tp{};
          tp.A_ = p[0];
          tp.B_ = p[1];
          tp.C_ = p[2];
          tp.D_ = p[3];
          tp.E_ = p[4];
          tp.n_coefficients_ = (micm::Index)p[5];
          for (int j = 0; j < (int)tp.n_coefficients_; ++j)
            tp.coefficients_[j] = p[6 + j];
          rb.SetRateConstant(tp);
          break;
        }
        case MICMB_RATE_REVERSIBLE:
          rb.SetRateConstant(micm::ReversibleRateConstantParameters{ .A_ = p[0], .C_ = p[1], .k_r_ = p[2] });
          break;
        case MICMB_RATE_USER_DEFINED:
          rb.SetRateConstant(micm::UserDefinedRateConstantParameters{ .label_ = label, .scaling_factor_ = p[0] });
          break;
        case MICMB_RATE_SURFACE:
        {
          micm::Species ss("surf" + std::to_string(r));
          ss.SetProperty<double>(micm::property_keys::MOLECULAR_WEIGHT, p[1]);
          micm::PhaseSpecies ps(ss, p[0]);
          rb.SetRateConstant(
              micm::SurfaceRateConstantParameters{ .label_ = label, .phase_species_ = ps, .reaction_probability_ = p[2] });
          break;
        }
        default: throw std::runtime_error("unsupported rate constant type");
      }
      b.processes.push_back(rb.Build());
    }
    // stable sort by type, as SolverBuilder::Build does (solver_builder.inl:274-329)
    std::vector<int> order(d->n_reactions);
    for (int r = 0; r < d->n_reactions; ++r)
      order[r] = r;
    std::stable_sort(
        order.begin(), order.end(), [&](int a, int c) { return d->rate_type[a] < d->rate_type[c]; });
    b.sorted_position.assign(d->n_reactions, 0);
    for (int i = 0; i < d->n_reactions; ++i)
      b.sorted_position[order[i]] = i;
    for (int c = 0; c < d->n_constraints; ++c)
    {
      Built::ConstraintSpec cs;
      cs.kind = d->constraint_type[c];
      cs.species = d->constraint_species[c];
      cs.n_react = d->constraint_n_reactants ? d->constraint_n_reactants[c] : 0;
      for (int t = d->constraint_term_start[c]; t < d->constraint_term_start[c + 1]; ++t)
        cs.terms.push_back({ d->constraint_term_species[t], d->constraint_term_coef[t] });
      for (int i = 0; i < 4; ++i)
        cs.p[i] = d->constraint_params[4 * c + i];
      b.constraints.push_back(cs);
    }
    return b;
  }

  // micm's constraint objects (linear_constraint.hpp:150-160,
  // equilibrium_constraint.hpp:208-220) for matrices of vector length L
  template<std::size_t L>
  std::vector<micm::Constraint<DenseL<L>, SparseL<L>>> MakeConstraints(const Built& b)
  {
    std::vector<micm::Constraint<DenseL<L>, SparseL<L>>> out;
    for (std::size_t c = 0; c < b.constraints.size(); ++c)
    {
      const auto& cs = b.constraints[c];
      const std::string name = "c" + std::to_string(c);
      std::vector<micm::StoichSpecies> terms;
      for (const auto& t : cs.terms)
        terms.emplace_back(b.species[t.first], t.second);
      if (cs.kind == MICMB_CONSTRAINT_LINEAR)
        out.emplace_back(micm::LinearConstraint<DenseL<L>, SparseL<L>>(name, b.species[cs.species], terms, cs.p[0]));
      else
      {
        std::vector<micm::StoichSpecies> re(terms.begin(), terms.begin() + cs.n_react);
        std::vector<micm::StoichSpecies> pr(terms.begin() + cs.n_react, terms.end());
        typename micm::EquilibriumConstraint<DenseL<L>, SparseL<L>>::VantHoffParam vh{};
        vh.K_HLC_ref_ = cs.p[0];
        vh.delta_H_ = cs.p[1];
        vh.R_ = cs.p[2];
        vh.T_ref_ = cs.p[3];
        out.emplace_back(micm::EquilibriumConstraint<DenseL<L>, SparseL<L>>(name, b.species[cs.species], re, pr, vh));
      }
    }
    return out;
  }

  struct Handle
  {
    Built built;
    micm::RosenbrockSolverParameters params = micm::RosenbrockSolverParameters::ThreeStageRosenbrockParameters();
    double rtol = 1e-6;
    bool reorder = true;
    std::unique_ptr<SolverL<1>> solver1;
    std::unique_ptr<SolverL<128>> solver128;  // built on first use (mref_solve_groups_v128)
    std::vector<int> species_column;  // system species -> state column
    std::vector<int> param_column;    // input reaction -> custom param column or -1
    int n_params = 0;
  };

  template<std::size_t L>
  SolverL<L> MakeSolver(Handle& h)
  {
    auto builder = BuilderL<L>(h.params);
    builder.SetSystem(h.built.system).SetReactions(h.built.processes).SetReorderState(h.reorder).SetIgnoreUnusedSpecies(true);
    if (!h.built.constraints.empty())
      builder.SetConstraints(MakeConstraints<L>(h.built));
    return builder.Build();
  }

  template<class State>
  void LoadCell(State& state, int lane, int n_params, int S, const double* T, const double* P, const double* rho,
                const double* params, const double* y, int cell)
  {
    state.conditions_[lane].temperature_ = T[cell];
    state.conditions_[lane].pressure_ = P[cell];
    state.conditions_[lane].air_density_ = rho[cell];
    for (int j = 0; j < S; ++j)
      state.variables_[lane][j] = y[(size_t)cell * S + j];
    for (int j = 0; j < n_params; ++j)
      state.custom_rate_parameters_[lane][j] = params[(size_t)cell * n_params + j];
  }

  void StatsOut(const micm::SolverResult& r, int64_t* out)
  {
    out[0] = (int64_t)r.stats_.function_calls_;
    out[1] = (int64_t)r.stats_.jacobian_updates_;
    out[2] = (int64_t)r.stats_.number_of_steps_;
    out[3] = (int64_t)r.stats_.accepted_;
    out[4] = (int64_t)r.stats_.rejected_;
    out[5] = (int64_t)r.stats_.decompositions_;
    out[6] = (int64_t)r.stats_.solves_;
    out[7] = (int64_t)r.state_;
    double ft = r.stats_.final_time_;
    std::memcpy(&out[8], &ft, sizeof(double));
    out[9] = (int64_t)r.stats_.constraint_init_iterations_;
  }

#define GUARD_BEGIN \
  try           \
  {
#define GUARD_END                   \
  }                                 \
  catch (const std::exception& e)   \
  {                                 \
    g_error = e.what();             \
    return -1;                      \
  }                                 \
  catch (...)                       \
  {                                 \
    g_error = "unknown exception";  \
    return -1;                      \
  }
}  // namespace

extern "C"
{
  const char* mref_last_error()
  {
    return g_error.c_str();
  }

  // tableau_kind: 2, 3, 4, 40 (4-stage DA), 60 (6-stage DA)
  void* mref_create(const micmb_mechanism_desc* d, const double* atol, double rtol, int tableau_kind)
  {
    try
    {
      auto h = std::make_unique<Handle>();
      h->built = Build(d, atol);
      h->params = TableauFor(tableau_kind);
      h->rtol = rtol;
      h->reorder = d->reorder_state != 0;
      h->solver1 = std::make_unique<SolverL<1>>(MakeSolver<1>(*h));
      auto state = h->solver1->GetState(1);
      h->species_column.resize(d->n_species);
      for (int i = 0; i < d->n_species; ++i)
        h->species_column[i] = (int)state.variable_map_.at(SpeciesName(i));
      // user parameters only: micm appends one K_eq parameter per equilibrium
      // constraint, which UpdateStateParameters fills from the temperature
      int n_eq = 0;
      for (const auto& cs : h->built.constraints)
        n_eq += cs.kind == MICMB_CONSTRAINT_EQUILIBRIUM ? 1 : 0;
      h->n_params = (int)state.custom_rate_parameter_map_.size() - n_eq;
      h->param_column.assign(d->n_reactions, -1);
      for (int r = 0; r < d->n_reactions; ++r)
      {
        std::string label = "r" + std::to_string(r);
        auto it = state.custom_rate_parameter_map_.find(label);
        if (it != state.custom_rate_parameter_map_.end())
          h->param_column[r] = (int)it->second;
        auto it2 = state.custom_rate_parameter_map_.find(label + ".effective radius [m]");
        if (it2 != state.custom_rate_parameter_map_.end())
          h->param_column[r] = (int)it2->second;
      }
      return h.release();
    }
    catch (const std::exception& e)
    {
      g_error = e.what();
      return nullptr;
    }
  }

  void mref_destroy(void* p)
  {
    delete static_cast<Handle*>(p);
  }

  int mref_n_custom_params(void* p)
  {
    return static_cast<Handle*>(p)->n_params;
  }

  int mref_species_columns(void* p, int32_t* out)
  {
    auto* h = static_cast<Handle*>(p);
    for (size_t i = 0; i < h->species_column.size(); ++i)
      out[i] = h->species_column[i];
    return 0;
  }

  int mref_reaction_columns(void* p, int32_t* out)
  {
    auto* h = static_cast<Handle*>(p);
    for (size_t i = 0; i < h->built.sorted_position.size(); ++i)
      out[i] = h->built.sorted_position[i];
    return 0;
  }

  int mref_custom_param_columns(void* p, int32_t* out)
  {
    auto* h = static_cast<Handle*>(p);
    for (size_t i = 0; i < h->param_column.size(); ++i)
      out[i] = h->param_column[i];
    return 0;
  }

  // LU-filled sparsity of State::jacobian_ in storage order; returns nnz.
  int mref_jacobian_pattern(void* p, int32_t* rows, int32_t* cols)
  {
    GUARD_BEGIN
    auto* h = static_cast<Handle*>(p);
    auto state = h->solver1->GetState(1);
    const int S = h->built.n_species;
    std::vector<std::pair<size_t, std::pair<int, int>>> elems;
    for (int i = 0; i < S; ++i)
      for (int j = 0; j < S; ++j)
        if (!state.jacobian_.IsZero(i, j))
          elems.push_back({ state.jacobian_.VectorIndex(0, i, j), { i, j } });
    std::sort(elems.begin(), elems.end());
    if (rows)
      for (size_t e = 0; e < elems.size(); ++e)
      {
        rows[e] = elems[e].second.first;
        cols[e] = elems[e].second.second;
      }
    return (int)elems.size();
    GUARD_END
  }

  // rate constants [cell][rate column]; params [cell][param column]
  int mref_rate_constants(void* p, int n, const double* T, const double* P, const double* rho, const double* params,
                          double* k_out)
  {
    GUARD_BEGIN
    auto* h = static_cast<Handle*>(p);
    const int S = h->built.n_species, R = h->built.n_reactions;
    auto state = h->solver1->GetState(n);
    std::vector<double> y((size_t)n * S, 0.0);
    for (int c = 0; c < n; ++c)
      LoadCell(state, c, h->n_params, S, T, P, rho, params, y.data(), c);
    h->solver1->UpdateStateParameters(state);
    for (int c = 0; c < n; ++c)
      for (int r = 0; r < R; ++r)
        k_out[(size_t)c * R + r] = state.rate_constants_[c][r];
    return 0;
    GUARD_END
  }

  // f = AddForcingTerms(y) starting from zero
  int mref_forcing(void* p, int n, const double* k, const double* y, double* f_out)
  {
    GUARD_BEGIN
    auto* h = static_cast<Handle*>(p);
    const int S = h->built.n_species, R = h->built.n_reactions;
    auto state = h->solver1->GetState(n);
    DenseL<1> Y(n, S, 0.0), F(n, S, 0.0);
    for (int c = 0; c < n; ++c)
    {
      for (int r = 0; r < R; ++r)
        state.rate_constants_[c][r] = k[(size_t)c * R + r];
      for (int j = 0; j < S; ++j)
        Y[c][j] = y[(size_t)c * S + j];
    }
    h->solver1->solver_.rates_.AddForcingTerms(state, Y, F);
    for (int c = 0; c < n; ++c)
      for (int j = 0; j < S; ++j)
        f_out[(size_t)c * S + j] = F[c][j];
    return 0;
    GUARD_END
  }

  // jac = Fill(0) + SubtractJacobianTerms(y): the stored -J, [cell][nnz] in storage order
  int mref_jacobian(void* p, int n, const double* k, const double* y, double* jac_out)
  {
    GUARD_BEGIN
    auto* h = static_cast<Handle*>(p);
    const int S = h->built.n_species, R = h->built.n_reactions;
    auto state = h->solver1->GetState(n);
    DenseL<1> Y(n, S, 0.0);
    for (int c = 0; c < n; ++c)
    {
      for (int r = 0; r < R; ++r)
        state.rate_constants_[c][r] = k[(size_t)c * R + r];
      for (int j = 0; j < S; ++j)
        Y[c][j] = y[(size_t)c * S + j];
    }
    state.jacobian_.Fill(0.0);
    h->solver1->solver_.rates_.SubtractJacobianTerms(state, Y, state.jacobian_);
    const auto& data = state.jacobian_.AsVector();
    const size_t nnz = data.size() / (size_t)n;
    for (size_t i = 0; i < data.size(); ++i)
      jac_out[i] = data[i];
    (void)nnz;
    return 0;
    GUARD_END
  }

  // in-place Mozart LU of [cell][nnz]
  int mref_decompose(void* p, int n, double* lu_inout)
  {
    GUARD_BEGIN
    auto* h = static_cast<Handle*>(p);
    auto state = h->solver1->GetState(n);
    auto& data = state.jacobian_.AsVector();
    for (size_t i = 0; i < data.size(); ++i)
      data[i] = lu_inout[i];
    h->solver1->solver_.linear_solver_.Factor(state.jacobian_);
    for (size_t i = 0; i < data.size(); ++i)
      lu_inout[i] = data[i];
    return 0;
    GUARD_END
  }

  // x = (LU)^-1 x, LU [cell][nnz], x [cell][S]
  int mref_linear_solve(void* p, int n, const double* lu, double* x_inout)
  {
    GUARD_BEGIN
    auto* h = static_cast<Handle*>(p);
    const int S = h->built.n_species;
    auto state = h->solver1->GetState(n);
    auto& data = state.jacobian_.AsVector();
    for (size_t i = 0; i < data.size(); ++i)
      data[i] = lu[i];
    DenseL<1> X(n, S, 0.0);
    for (int c = 0; c < n; ++c)
      for (int j = 0; j < S; ++j)
        X[c][j] = x_inout[(size_t)c * S + j];
    h->solver1->solver_.linear_solver_.Solve(X, state.jacobian_);
    for (int c = 0; c < n; ++c)
      for (int j = 0; j < S; ++j)
        x_inout[(size_t)c * S + j] = X[c][j];
    return 0;
    GUARD_END
  }

  // AbstractRosenbrockSolver::NormalizedError over all n cells; atol per state column
  double mref_normalized_error(void* p, int n, const double* y, const double* ynew, const double* err,
                               const double* atol_cols, double rtol)
  {
    try
    {
      auto* h = static_cast<Handle*>(p);
      const int S = h->built.n_species;
      auto state = h->solver1->GetState(n);
      state.SetRelativeTolerance(rtol);
      state.SetAbsoluteTolerances(std::vector<double>(atol_cols, atol_cols + S));
      DenseL<1> Y(n, S, 0.0), Yn(n, S, 0.0), E(n, S, 0.0);
      for (int c = 0; c < n; ++c)
        for (int j = 0; j < S; ++j)
        {
          Y[c][j] = y[(size_t)c * S + j];
          Yn[c][j] = ynew[(size_t)c * S + j];
          E[c][j] = err[(size_t)c * S + j];
        }
      typename DenseL<1>::template ScalarType<double> e;
      h->solver1->solver_.NormalizedError(Y, Yn, E, state, e);
      return (double)e;
    }
    catch (const std::exception& e)
    {
      g_error = e.what();
      return -1.0;
    }
  }

  // Global step control: one n-cell State, n_solves x (UpdateStateParameters + Solve(dt)).
  // y_inout [cell][column]; stats_out [n_solves][10] (int64, final_time bit-cast at [8]).
  int mref_solve_global(void* p, int n, double dt, int n_solves, const double* T, const double* P, const double* rho,
                        const double* params, double* y_inout, int64_t* stats_out)
  {
    GUARD_BEGIN
    auto* h = static_cast<Handle*>(p);
    const int S = h->built.n_species;
    auto state = h->solver1->GetState(n);
    state.SetRelativeTolerance(h->rtol);
    for (int c = 0; c < n; ++c)
      LoadCell(state, c, h->n_params, S, T, P, rho, params, y_inout, c);
    for (int i = 0; i < n_solves; ++i)
    {
      h->solver1->UpdateStateParameters(state);
      auto r = h->solver1->Solve(dt, state);
      if (stats_out)
        StatsOut(r, stats_out + 10 * i);
    }
    for (int c = 0; c < n; ++c)
      for (int j = 0; j < S; ++j)
        y_inout[(size_t)c * S + j] = state.variables_[c][j];
    return 0;
    GUARD_END
  }

  // micm's vector ordering with L = 128 (micm_bench's fastest CPU layout,
  // test/benchmark/bench_harness.hpp VectorDense<128> / VectorSparse<128>):
  // cells in consecutive groups of `group` cells, one State per group with one
  // step size for the group, groups taken by n_threads host threads (one State
  // per thread at a time, test/tutorial/test_openmp.cpp:115-122).  For cells
  // that share their inputs this is the same solve as per-cell control.
  // stats_out [group][10] accumulates over solves.
  int mref_solve_groups_v128(void* p, int n, int group, double dt, int n_solves, const double* T, const double* P,
                             const double* rho, const double* params, double* y_inout, int64_t* stats_out,
                             int n_threads)
  {
    GUARD_BEGIN
    auto* h = static_cast<Handle*>(p);
    const int S = h->built.n_species;
    if (group < 1)
      throw std::runtime_error("group must be at least 1");
    if (!h->solver128)
      h->solver128 = std::make_unique<SolverL<128>>(MakeSolver<128>(*h));
    if (n_threads < 1)
      n_threads = 1;
    const int n_groups = (n + group - 1) / group;
    std::atomic<int> next{ 0 };
    std::string failure;
    auto work = [&]()
    {
      try
      {
        for (;;)
        {
          const int g = next.fetch_add(1);
          if (g >= n_groups)
            break;
          const int c0 = g * group, count = std::min(group, n - c0);
          auto state = h->solver128->GetState(count);
          state.SetRelativeTolerance(h->rtol);
          for (int c = 0; c < count; ++c)
            LoadCell(state, c, h->n_params, S, T, P, rho, params, y_inout, c0 + c);
          int64_t acc[10] = { 0 };
          for (int i = 0; i < n_solves; ++i)
          {
            h->solver128->UpdateStateParameters(state);
            auto r = h->solver128->Solve(dt, state);
            int64_t one[10];
            StatsOut(r, one);
            for (int q = 0; q < 7; ++q)
              acc[q] += one[q];
            acc[7] = one[7];
            acc[8] = one[8];
            acc[9] += one[9];
          }
          for (int c = 0; c < count; ++c)
            for (int j = 0; j < S; ++j)
              y_inout[(size_t)(c0 + c) * S + j] = state.variables_[c][j];
          if (stats_out)
            std::memcpy(stats_out + 10 * (size_t)g, acc, sizeof(acc));
        }
      }
      catch (const std::exception& e)
      {
        failure = e.what();
      }
    };
    std::vector<std::thread> pool;
    for (int t = 1; t < n_threads; ++t)
      pool.emplace_back(work);
    work();
    for (auto& t : pool)
      t.join();
    if (!failure.empty())
      throw std::runtime_error(failure);
    return 0;
    GUARD_END
  }

  // micm's Backward Euler (backward_euler.inl, default parameters), a 1-cell
  // State per cell, one Solve(dt) each.  y_inout [cell][column]; stats_out
  // [cell][10] as mref_solve_per_cell's.
  int mref_backward_euler_per_cell(void* p, int n, double dt, const double* T, const double* P, const double* rho,
                                   const double* params, double* y_inout, int64_t* stats_out)
  {
    GUARD_BEGIN
    auto* h = static_cast<Handle*>(p);
    const int S = h->built.n_species;
    auto solver = BuilderBE(micm::BackwardEulerSolverParameters{})
                      .SetSystem(h->built.system)
                      .SetReactions(h->built.processes)
                      .SetReorderState(h->reorder)
                      .SetIgnoreUnusedSpecies(true)
                      .Build();
    auto state = solver.GetState(1);
    state.SetRelativeTolerance(h->rtol);
    for (int c = 0; c < n; ++c)
    {
      LoadCell(state, 0, h->n_params, S, T, P, rho, params, y_inout, c);
      solver.UpdateStateParameters(state);
      auto r = solver.Solve(dt, state);
      for (int j = 0; j < S; ++j)
        y_inout[(size_t)c * S + j] = state.variables_[0][j];
      if (stats_out)
        StatsOut(r, stats_out + 10 * (size_t)c);
    }
    return 0;
    GUARD_END
  }

  // micm's Backward Euler on one n-cell State (one step size and one
  // convergence test for all cells), one Solve(dt).  y_inout [cell][column];
  // stats_out [10] as one row of mref_solve_per_cell's.
  int mref_backward_euler_global(void* p, int n, double dt, const double* T, const double* P, const double* rho,
                                 const double* params, double* y_inout, int64_t* stats_out)
  {
    GUARD_BEGIN
    auto* h = static_cast<Handle*>(p);
    const int S = h->built.n_species;
    auto solver = BuilderBE(micm::BackwardEulerSolverParameters{})
                      .SetSystem(h->built.system)
                      .SetReactions(h->built.processes)
                      .SetReorderState(h->reorder)
                      .SetIgnoreUnusedSpecies(true)
                      .Build();
    auto state = solver.GetState(n);
    state.SetRelativeTolerance(h->rtol);
    for (int c = 0; c < n; ++c)
      LoadCell(state, c, h->n_params, S, T, P, rho, params, y_inout, c);
    solver.UpdateStateParameters(state);
    auto r = solver.Solve(dt, state);
    for (int c = 0; c < n; ++c)
      for (int j = 0; j < S; ++j)
        y_inout[(size_t)c * S + j] = state.variables_[c][j];
    if (stats_out)
      StatsOut(r, stats_out);
    return 0;
    GUARD_END
  }

  // Per-cell step control: a 1-cell State per cell (the reference's own idiom
  // for independent cells, test/tutorial/test_openmp.cpp:115-122), cells split
  // over n_threads host threads.  stats_out [cell][10] accumulates over solves
  // (state field = last solve's state).
  int mref_solve_per_cell(void* p, int n, double dt, int n_solves, const double* T, const double* P,
                          const double* rho, const double* params, double* y_inout, int64_t* stats_out,
                          int n_threads)
  {
    GUARD_BEGIN
    auto* h = static_cast<Handle*>(p);
    const int S = h->built.n_species;
    if (n_threads < 1)
      n_threads = 1;
    std::atomic<int> next{ 0 };
    std::string failure;
    auto work = [&]()
    {
      try
      {
        auto state = h->solver1->GetState(1);
        state.SetRelativeTolerance(h->rtol);
        for (;;)
        {
          int c = next.fetch_add(1);
          if (c >= n)
            break;
          LoadCell(state, 0, h->n_params, S, T, P, rho, params, y_inout, c);
          int64_t acc[10] = { 0 };
          for (int i = 0; i < n_solves; ++i)
          {
            h->solver1->UpdateStateParameters(state);
            auto r = h->solver1->Solve(dt, state);
            int64_t one[10];
            StatsOut(r, one);
            for (int q = 0; q < 7; ++q)
              acc[q] += one[q];
            acc[7] = one[7];
            acc[8] = one[8];
            acc[9] += one[9];
          }
          for (int j = 0; j < S; ++j)
            y_inout[(size_t)c * S + j] = state.variables_[0][j];
          if (stats_out)
            std::memcpy(stats_out + 10 * (size_t)c, acc, sizeof(acc));
        }
      }
      catch (const std::exception& e)
      {
        failure = e.what();
      }
    };
    std::vector<std::thread> pool;
    for (int t = 1; t < n_threads; ++t)
      pool.emplace_back(work);
    work();
    for (auto& t : pool)
      t.join();
    if (!failure.empty())
      throw std::runtime_error(failure);
    return 0;
    GUARD_END
  }
}
