// micm.hpp -- micm's CUDA-path C++ API, backed by the B200 solver's C ABI.
//
// Drop-in for code written against NCAR/micm 3.13.0's GPU path: the same
// namespace (micm), class and member names as
//   include/micm/system/{species,phase,system,conditions,stoich_species}.hpp
//   include/micm/process/{chemical_reaction,chemical_reaction_builder,process}.hpp,
//   include/micm/process/rate_constant/*.hpp
//   include/micm/solver/{rosenbrock_solver_parameters,solver_result,solver}.hpp
//   include/micm/cuda/solver/{cuda_solver_builder,cuda_solver_parameters,cuda_state}.hpp
//   include/micm/GPU.hpp (aliases)
// so that `CudaSolverBuilderInPlace<CudaRosenbrockSolverParameters, L>(params)
// .SetSystem(s).SetReactions(r).Build()`, `solver.GetState(n)`,
// `state.SyncInputsToDevice()`, `solver.UpdateStateParameters(state)`,
// `solver.Solve(dt, state)` and `state.SyncOutputsToHost()` behave as in micm.
// Everything numeric runs in libmicmb.so (include/micmb.h).
//
// Extensions beyond micm: Solver::SetStepControl (Global = micm's single step
// size, PerCell = an independent adaptive solve per cell), Solver::SetMethod
// (Plain per-stage kernels or the Fused persistent kernel) and
// Solver::SolveAdjoint.
#pragma once

#include "../micmb.h"

#include <algorithm>
#include <array>
#include <cmath>
#include <concepts>
#include <cstddef>
#include <cstdint>
#include <iomanip>
#include <iostream>
#include <limits>
#include <tuple>
#include <map>
#include <memory>
#include <optional>
#include <set>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <unordered_map>
#include <utility>
#include <variant>
#include <vector>

#ifndef MICM_DEFAULT_VECTOR_SIZE
#define MICM_DEFAULT_VECTOR_SIZE 4
#endif

namespace micm
{
  using Real = double;
  using Index = std::size_t;

  // ---------------------------------------------------------------- errors
  struct MicmException : public std::runtime_error
  {
    const char* category_;
    int code_;
    MicmException(const char* category, int code, const std::string& message)
        : std::runtime_error(message),
          category_(category),
          code_(code)
    {
    }
    const char* Category() const noexcept
    {
      return category_;
    }
    int Code() const noexcept
    {
      return code_;
    }
  };

  namespace detail
  {
    inline void Check(int rc)
    {
      if (rc != MICMB_OK)
        throw MicmException("MICM Internal Error", rc, micmb_last_error());
    }
  }  // namespace detail

  namespace constants
  {
    static constexpr Real BOLTZMANN_CONSTANT = 1.380649e-23;
    static constexpr Real AVOGADRO_CONSTANT = 6.02214076e23;
    static constexpr Real GAS_CONSTANT = BOLTZMANN_CONSTANT * AVOGADRO_CONSTANT;
  }  // namespace constants

  namespace property_keys
  {
    static constexpr const char* MOLECULAR_WEIGHT = "molecular weight [kg mol-1]";
    static constexpr const char* ABSOLUTE_TOLERANCE = "absolute tolerance";
  }  // namespace property_keys

  // ---------------------------------------------------------------- system
  struct Conditions
  {
    Real temperature_{ 0.0 };
    Real pressure_{ 0.0 };
    Real air_density_{ 0.0 };
    void CalculateIdealAirDensity()
    {
      air_density_ = pressure_ / (constants::GAS_CONSTANT * temperature_);
    }
  };

  struct ParameterizedFunction
  {
    Real c0_ = 0.0;
    Real c_T_ = 0.0;
    Real c_P_ = 0.0;
    Real c_rho_ = 0.0;
    bool has_value_ = false;
    bool HasValue() const
    {
      return has_value_;
    }
  };

  class Species
  {
   public:
    std::string name_;
    std::map<std::string, std::string> properties_string_;
    std::map<std::string, Real> properties_double_;
    std::map<std::string, bool> properties_bool_;
    std::map<std::string, int> properties_int_;
    ParameterizedFunction parameterize_{};

    Species() = default;
    Species(std::string name)
        : name_(std::move(name))
    {
    }
    Species(std::string name, const std::map<std::string, Real>& properties)
        : name_(std::move(name)),
          properties_double_(properties)
    {
    }
    bool IsParameterized() const
    {
      return parameterize_.HasValue();
    }
    bool HasProperty(const std::string& key) const
    {
      return properties_double_.count(key) || properties_string_.count(key) || properties_bool_.count(key) ||
             properties_int_.count(key);
    }
    void SetThirdBody()
    {
      parameterize_ = ParameterizedFunction{ 0.0, 0.0, 0.0, 1.0, true };
    }
    template<class T>
    T GetProperty(const std::string& key) const
    {
      if constexpr (std::is_same_v<T, std::string>)
        return properties_string_.at(key);
      else if constexpr (std::is_same_v<T, bool>)
        return properties_bool_.at(key);
      else if constexpr (std::is_same_v<T, int>)
        return properties_int_.at(key);
      else
        return static_cast<T>(properties_double_.at(key));
    }
    template<class T>
    void SetProperty(const std::string& key, T value)
    {
      if constexpr (std::is_same_v<T, std::string> || std::is_same_v<T, const char*>)
        properties_string_[key] = value;
      else if constexpr (std::is_same_v<T, bool>)
        properties_bool_[key] = value;
      else if constexpr (std::is_same_v<T, int>)
        properties_int_[key] = value;
      else
        properties_double_[key] = static_cast<Real>(value);
    }
  };

  class PhaseSpecies
  {
   public:
    Species species_;
    std::optional<Real> diffusion_coefficient_;
    std::optional<Real> density_;
    PhaseSpecies(const Species& species)
        : species_(species)
    {
    }
    PhaseSpecies(const Species& species, Real diffusion_coefficient)
        : species_(species),
          diffusion_coefficient_(diffusion_coefficient)
    {
    }
    void SetDiffusionCoefficient(Real d)
    {
      diffusion_coefficient_ = d;
    }
  };

  class Phase
  {
   public:
    std::string name_;
    std::vector<PhaseSpecies> phase_species_;
    Phase() = default;
    Phase(std::string name, const std::vector<PhaseSpecies>& phase_species)
        : name_(std::move(name)),
          phase_species_(phase_species)
    {
    }
    Index StateSize() const
    {
      Index n = 0;
      for (const auto& p : phase_species_)
        n += p.species_.IsParameterized() ? 0 : 1;
      return n;
    }
    std::vector<std::string> SpeciesNames() const
    {
      std::vector<std::string> names;
      for (const auto& p : phase_species_)
        if (!p.species_.IsParameterized())
          names.push_back(p.species_.name_);
      return names;
    }
  };

  class System
  {
   public:
    Phase gas_phase_;
    System() = default;
    System(const Phase& gas_phase)
        : gas_phase_(gas_phase)
    {
    }
    Index StateSize() const
    {
      return gas_phase_.StateSize();
    }
    std::vector<std::string> UniqueNames() const
    {
      return gas_phase_.SpeciesNames();
    }
  };

  struct StoichSpecies
  {
    Species species_;
    Real coefficient_{ 1.0 };
  };

  // ---------------------------------------------------------------- rate constants
  struct ArrheniusRateConstantParameters
  {
    Real A_{ 1 };
    Real B_{ 0 };
    Real C_{ 0 };
    Real D_{ 300 };
    Real E_{ 0 };
  };
  struct TroeRateConstantParameters
  {
    Real k0_A_ = 1.0;
    Real k0_B_ = 0.0;
    Real k0_C_ = 0.0;
    Real kinf_A_ = 1.0;
    Real kinf_B_ = 0.0;
    Real kinf_C_ = 0.0;
    Real Fc_ = 0.6;
    Real N_ = 1.0;
  };
  struct TernaryChemicalActivationRateConstantParameters
  {
    Real k0_A_ = 1.0;
    Real k0_B_ = 0.0;
    Real k0_C_ = 0.0;
    Real kinf_A_ = 1.0;
    Real kinf_B_ = 0.0;
    Real kinf_C_ = 0.0;
    Real Fc_ = 0.6;
    Real N_ = 1.0;
  };
  struct BranchedRateConstantParameters
  {
    enum class Branch
    {
      Alkoxy,
      Nitrate
    };
    Branch branch_;
    Real X_;
    Real Y_;
    Real a0_;
    Index n_;
  };
  struct TunnelingRateConstantParameters
  {
    Real A_ = 1.0;
    Real B_ = 0.0;
    Real C_ = 0.0;
  };
  struct TaylorSeriesRateConstantParameters
  {
    static constexpr Index MAX_COEFFICIENTS = 16;
    Real A_{ 1 };
    Real B_{ 0 };
    Real C_{ 0 };
    Real D_{ 300 };
    Real E_{ 0 };
    Real coefficients_[MAX_COEFFICIENTS] = { 1.0 };
    Index n_coefficients_{ 1 };
  };
  struct ReversibleRateConstantParameters
  {
    Real A_{ 1 };
    Real C_{ 0 };
    Real k_r_{ 0 };
  };
  struct UserDefinedRateConstantParameters
  {
    std::string label_;
    Real scaling_factor_{ 1.0 };
  };
  struct SurfaceRateConstantParameters
  {
    std::string label_;
    PhaseSpecies phase_species_{ Species{} };
    Real reaction_probability_{ 1.0 };
  };

  using RateConstantVariant = std::variant<
      ArrheniusRateConstantParameters,
      TroeRateConstantParameters,
      TernaryChemicalActivationRateConstantParameters,
      BranchedRateConstantParameters,
      TunnelingRateConstantParameters,
      TaylorSeriesRateConstantParameters,
      ReversibleRateConstantParameters,
      UserDefinedRateConstantParameters,
      SurfaceRateConstantParameters>;

  class ChemicalReaction
  {
   public:
    std::vector<Species> reactants_;
    std::vector<StoichSpecies> products_;
    RateConstantVariant rate_constant_;
    Phase phase_;
  };

  class Process
  {
   public:
    ChemicalReaction process_;
    Process(const ChemicalReaction& p)
        : process_(p)
    {
    }
  };

  class ChemicalReactionBuilder
  {
    std::vector<Species> reactants_;
    std::vector<StoichSpecies> products_;
    std::optional<RateConstantVariant> rate_constant_;
    Phase phase_;

   public:
    ChemicalReactionBuilder& SetReactants(const std::vector<Species>& reactants)
    {
      reactants_ = reactants;
      return *this;
    }
    ChemicalReactionBuilder& SetProducts(const std::vector<StoichSpecies>& products)
    {
      products_ = products;
      return *this;
    }
    template<class T>
    ChemicalReactionBuilder& SetRateConstant(T&& rate_constant)
    {
      rate_constant_ = RateConstantVariant(std::forward<T>(rate_constant));
      return *this;
    }
    ChemicalReactionBuilder& SetPhase(const Phase& phase)
    {
      phase_ = Phase(phase.name_, {});
      return *this;
    }
    Process Build()
    {
      if (!rate_constant_)
        throw MicmException("MICM Process", 1, "Rate constant has not been set.");
      return Process(ChemicalReaction{ reactants_, products_, *rate_constant_, phase_ });
    }
  };

  // ---------------------------------------------------------------- solver parameters
  struct RosenbrockSolverParameters
  {
    Index stages_{};
    Index upper_limit_tolerance_{};
    Index max_number_of_steps_{ 1000 };
    Real round_off_{ std::numeric_limits<Real>::epsilon() };
    Real factor_min_{ 0.2 };
    Real factor_max_{ 6 };
    Real rejection_factor_decrease_{ 0.1 };
    Real safety_factor_{ 0.9 };
    Real h_min_{ 0.0 };
    Real h_max_{ 0.0 };
    Real h_start_{ 0.0 };
    std::array<bool, 6> new_function_evaluation_{};
    Real estimator_of_local_order_{};
    std::array<Real, 15> a_{};
    std::array<Real, 15> c_{};
    std::array<Real, 6> m_{};
    std::array<Real, 6> e_{};
    std::array<Real, 6> alpha_{};
    std::array<Real, 6> gamma_{};
    Index constraint_init_max_iterations_{ 10 };  // DAE constraint initialisation (rosenbrock_solver_parameters.hpp:43-44)
    Real constraint_init_tolerance_{ 1e-10 };

    static RosenbrockSolverParameters TwoStageRosenbrockParameters()
    {
      return FromKind(2);
    }
    static RosenbrockSolverParameters ThreeStageRosenbrockParameters()
    {
      return FromKind(3);
    }
    static RosenbrockSolverParameters FourStageRosenbrockParameters()
    {
      return FromKind(4);
    }
    static RosenbrockSolverParameters FourStageDifferentialAlgebraicRosenbrockParameters()
    {
      return FromKind(40);
    }
    static RosenbrockSolverParameters SixStageDifferentialAlgebraicRosenbrockParameters()
    {
      return FromKind(60);
    }

    micmb_rosenbrock_params ToC() const
    {
      micmb_rosenbrock_params p{};
      p.stages = (int32_t)stages_;
      p.max_number_of_steps = (int32_t)max_number_of_steps_;
      p.round_off = round_off_;
      p.factor_min = factor_min_;
      p.factor_max = factor_max_;
      p.rejection_factor_decrease = rejection_factor_decrease_;
      p.safety_factor = safety_factor_;
      p.h_min = h_min_;
      p.h_max = h_max_;
      p.h_start = h_start_;
      p.estimator_of_local_order = estimator_of_local_order_;
      p.constraint_init_max_iterations = (int32_t)constraint_init_max_iterations_;
      p.constraint_init_tolerance = constraint_init_tolerance_;
      for (int i = 0; i < 6; ++i)
      {
        p.new_function_evaluation[i] = new_function_evaluation_[i] ? 1 : 0;
        p.m[i] = m_[i];
        p.e[i] = e_[i];
        p.alpha[i] = alpha_[i];
        p.gamma[i] = gamma_[i];
      }
      for (int i = 0; i < 15; ++i)
      {
        p.a[i] = a_[i];
        p.c[i] = c_[i];
      }
      return p;
    }

   protected:
    static RosenbrockSolverParameters FromKind(int kind)
    {
      micmb_rosenbrock_params p{};
      detail::Check(micmb_rosenbrock_params_default(kind, &p));
      RosenbrockSolverParameters r;
      r.stages_ = (Index)p.stages;
      r.max_number_of_steps_ = (Index)p.max_number_of_steps;
      r.round_off_ = p.round_off;
      r.factor_min_ = p.factor_min;
      r.factor_max_ = p.factor_max;
      r.rejection_factor_decrease_ = p.rejection_factor_decrease;
      r.safety_factor_ = p.safety_factor;
      r.estimator_of_local_order_ = p.estimator_of_local_order;
      r.constraint_init_max_iterations_ = (Index)p.constraint_init_max_iterations;
      r.constraint_init_tolerance_ = p.constraint_init_tolerance;
      for (int i = 0; i < 6; ++i)
      {
        r.new_function_evaluation_[i] = p.new_function_evaluation[i] != 0;
        r.m_[i] = p.m[i];
        r.e_[i] = p.e[i];
        r.alpha_[i] = p.alpha[i];
        r.gamma_[i] = p.gamma[i];
      }
      for (int i = 0; i < 15; ++i)
      {
        r.a_[i] = p.a[i];
        r.c_[i] = p.c[i];
      }
      return r;
    }
  };

  struct CudaRosenbrockSolverParameters : public RosenbrockSolverParameters
  {
    CudaRosenbrockSolverParameters(const RosenbrockSolverParameters& base)
        : RosenbrockSolverParameters(base)
    {
    }
  };

  // ---------------------------------------------------------------- results
  enum class SolverState
  {
    NotYetCalled,
    Running,
    Converged,
    ConvergenceExceededMaxSteps,
    StepSizeTooSmall,
    RepeatedlySingularMatrix,
    NaNDetected,
    InfDetected,
    AcceptingUnconvergedIntegration,
    ConstraintInitializationFailed
  };

  struct SolverStats
  {
    Index function_calls_{};
    Index jacobian_updates_{};
    Index number_of_steps_{};
    Index accepted_{};
    Index rejected_{};
    Index decompositions_{};
    Index solves_{};
    Index constraint_init_iterations_{};
    Real final_time_{};
  };

  inline std::string SolverStateToString(const SolverState& state)
  {
    switch (state)
    {
      case SolverState::NotYetCalled: return "Not Yet Called";
      case SolverState::Running: return "Running";
      case SolverState::Converged: return "Converged";
      case SolverState::ConvergenceExceededMaxSteps: return "Convergence Exceeded Max Steps";
      case SolverState::StepSizeTooSmall: return "Step Size Too Small";
      case SolverState::RepeatedlySingularMatrix: return "Repeatedly Singular Matrix";
      case SolverState::NaNDetected: return "NaNDetected";
      case SolverState::InfDetected: return "InfDetected";
      case SolverState::AcceptingUnconvergedIntegration: return "AcceptingUnconvergedIntegration";
      case SolverState::ConstraintInitializationFailed: return "Constraint Initialization Failed";
      default: return "Unknown";
    }
  }

  struct [[nodiscard]] SolverResult
  {
    SolverState state_ = SolverState::NotYetCalled;
    SolverStats stats_{};
  };

  // ---------------------------------------------------------------- dense host matrix
  // micm::VectorMatrix<T, L> (include/micm/util/vector_matrix.hpp): rows = grid
  // cells, columns = variables, stored in groups of L cells, column-major
  // inside a group.
  template<class T, Index L = MICM_DEFAULT_VECTOR_SIZE>
  class VectorMatrix
  {
    Index x_dim_ = 0;
    Index y_dim_ = 0;
    std::vector<T> data_;

   public:
    class Row
    {
      VectorMatrix& m_;
      Index row_;

     public:
      Row(VectorMatrix& m, Index row)
          : m_(m),
            row_(row)
      {
      }
      T& operator[](Index col)
      {
        return m_.data_[(row_ / L) * L * m_.y_dim_ + col * L + row_ % L];
      }
      Index Size() const
      {
        return m_.y_dim_;
      }
      // a whole row at once, as micm's VectorMatrix row proxy allows
      // (state.variables_[cell] = {...} in micm_bench's InitState)
      Row& operator=(const std::vector<T>& values)
      {
        if (values.size() != m_.y_dim_)
          throw MicmException("MICM Matrix", 1, "Matrix row size mismatch in assignment from vector");
        for (Index c = 0; c < m_.y_dim_; ++c)
          (*this)[c] = values[c];
        return *this;
      }
      operator std::vector<T>() const
      {
        std::vector<T> out(m_.y_dim_);
        for (Index c = 0; c < m_.y_dim_; ++c)
          out[c] = m_.data_[(row_ / L) * L * m_.y_dim_ + c * L + row_ % L];
        return out;
      }
    };
    class ConstRow
    {
      const VectorMatrix& m_;
      Index row_;

     public:
      ConstRow(const VectorMatrix& m, Index row)
          : m_(m),
            row_(row)
      {
      }
      const T& operator[](Index col) const
      {
        return m_.data_[(row_ / L) * L * m_.y_dim_ + col * L + row_ % L];
      }
      Index Size() const
      {
        return m_.y_dim_;
      }
      operator std::vector<T>() const
      {
        std::vector<T> out(m_.y_dim_);
        for (Index c = 0; c < m_.y_dim_; ++c)
          out[c] = (*this)[c];
        return out;
      }
    };
    VectorMatrix() = default;
    VectorMatrix(Index x, Index y, T init = T{})
        : x_dim_(x),
          y_dim_(y),
          data_(((x + L - 1) / L) * L * y, init)
    {
    }
    Row operator[](Index row)
    {
      return Row(*this, row);
    }
    ConstRow operator[](Index row) const
    {
      return ConstRow(*this, row);
    }
    Index NumRows() const
    {
      return x_dim_;
    }
    Index NumColumns() const
    {
      return y_dim_;
    }
    static constexpr Index GroupVectorSize()
    {
      return L;
    }
    std::vector<T>& AsVector()
    {
      return data_;
    }
    const std::vector<T>& AsVector() const
    {
      return data_;
    }
  };

  enum class StepControl
  {
    Global,  // micm's semantics: one step size and one error norm for all cells
    PerCell  // each cell integrates with its own adaptive step size
  };
  enum class Method
  {
    Plain,  // one kernel per Rosenbrock stage over all cells
    Fused   // one persistent kernel per solve (per-cell step control only)
  };

  template<Index L>
  class Solver;

  // ---------------------------------------------------------------- constraints
  // micm's algebraic constraints (constraint/types/linear_constraint.hpp:150-172,
  // equilibrium_constraint.hpp:41-47 and :208-245, constraint.hpp:26-45).  The
  // matrix-policy parameters are kept so that micm code names the same types;
  // the library evaluates the constraints on the device, so they select nothing.
  template<class DenseMatrixPolicy = void, class SparseMatrixPolicy = void>
  class LinearConstraint
  {
   public:
    std::string name_;
    Species algebraic_species_;
    std::vector<StoichSpecies> terms_;
    Real constant_{};

    LinearConstraint(std::string name, const Species& algebraic_species, const std::vector<StoichSpecies>& terms,
                     Real constant)
        : name_(std::move(name)),
          algebraic_species_(algebraic_species),
          terms_(terms),
          constant_(constant)
    {
      if (terms_.empty())
        throw MicmException("MICM Constraint", 1, "Linear constraint requires at least one term");
    }
    const std::string& AlgebraicSpecies() const
    {
      return algebraic_species_.name_;
    }
  };

  template<class DenseMatrixPolicy = void, class SparseMatrixPolicy = void>
  class EquilibriumConstraint
  {
   public:
    // Van't Hoff: K_eq(T) = K_HLC_ref * exp((delta_H / R) * (1/T - 1/T_ref))
    struct VantHoffParam
    {
      Real K_HLC_ref_;
      Real delta_H_;
      Real R_ = constants::GAS_CONSTANT;
      Real T_ref_ = 298.15;
    };

    std::string name_;
    Species algebraic_species_;
    std::vector<StoichSpecies> reactants_;
    std::vector<StoichSpecies> products_;
    VantHoffParam vant_hoff_param_{};

    EquilibriumConstraint(const std::string& name, const Species& algebraic_species,
                          std::vector<StoichSpecies> reactants, std::vector<StoichSpecies> products,
                          VantHoffParam vant_hoff_param)
        : name_(name),
          algebraic_species_(algebraic_species),
          reactants_(std::move(reactants)),
          products_(std::move(products)),
          vant_hoff_param_(vant_hoff_param)
    {
      if (reactants_.empty())
        throw MicmException("MICM Constraint", 1, "Equilibrium constraint requires at least one reactant");
      if (products_.empty())
        throw MicmException("MICM Constraint", 1, "Equilibrium constraint requires at least one product");
      for (const auto& s : reactants_)
        if (s.coefficient_ <= 0)
          throw MicmException("MICM Constraint", 2, "Stoichiometric coefficients must be positive");
      for (const auto& s : products_)
        if (s.coefficient_ <= 0)
          throw MicmException("MICM Constraint", 2, "Stoichiometric coefficients must be positive");
      if (vant_hoff_param_.K_HLC_ref_ <= 0)
        throw MicmException("MICM Constraint", 3, "Equilibrium constant must be positive");
    }
    const std::string& AlgebraicSpecies() const
    {
      return algebraic_species_.name_;
    }
  };

  template<class DenseMatrixPolicy = void, class SparseMatrixPolicy = void>
  class Constraint
  {
   public:
    using ConstraintVariant = std::variant<EquilibriumConstraint<DenseMatrixPolicy, SparseMatrixPolicy>,
                                           LinearConstraint<DenseMatrixPolicy, SparseMatrixPolicy>>;
    ConstraintVariant constraint_;

    template<typename T>
      requires std::same_as<std::decay_t<T>, EquilibriumConstraint<DenseMatrixPolicy, SparseMatrixPolicy>> ||
               std::same_as<std::decay_t<T>, LinearConstraint<DenseMatrixPolicy, SparseMatrixPolicy>>
    Constraint(T&& constraint)
        : constraint_(std::forward<T>(constraint))
    {
    }
    std::string GetName() const
    {
      return std::visit([](const auto& c) { return c.name_; }, constraint_);
    }
    const std::string& AlgebraicSpecies() const
    {
      return std::visit([](const auto& c) -> const std::string& { return c.AlgebraicSpecies(); }, constraint_);
    }
  };

  // ---------------------------------------------------------------- state
  template<Index L = MICM_DEFAULT_VECTOR_SIZE>
  class CudaState
  {
    friend class Solver<L>;
    std::shared_ptr<micmb_state> handle_;

   public:
    using DenseMatrixPolicyType = VectorMatrix<Real, L>;
    Index number_of_grid_cells_{ 1 };
    VectorMatrix<Real, L> variables_;
    VectorMatrix<Real, L> custom_rate_parameters_;
    VectorMatrix<Real, L> rate_constants_;
    std::vector<Conditions> conditions_;
    std::unordered_map<std::string, Index> variable_map_;
    std::unordered_map<std::string, Index> custom_rate_parameter_map_;
    std::vector<std::string> variable_names_;
    Real relative_tolerance_{ 1e-6 };
    std::vector<Real> absolute_tolerance_;
    Index constraint_size_{ 0 };
    std::vector<Real> upper_left_identity_diagonal_;  // mass-matrix diagonal by variable: 1 ODE, 0 algebraic

    class VariableProxy
    {
      CudaState& state_;
      Index index_;

     public:
      VariableProxy(CudaState& state, Index index)
          : state_(state),
            index_(index)
      {
      }
      operator Real() const
      {
        if (state_.number_of_grid_cells_ != 1)
          throw MicmException("MICM State", 1, "Cannot convert multi-gridcell State variable to single Real value");
        return state_.variables_[0][index_];
      }
      VariableProxy& operator=(Real value)
      {
        if (state_.number_of_grid_cells_ != 1)
          throw MicmException("MICM State", 1, "Cannot assign single value to multi-gridcell State variable");
        state_.variables_[0][index_] = value;
        return *this;
      }
      VariableProxy& operator=(const std::vector<Real>& values)
      {
        if (values.size() != state_.number_of_grid_cells_)
          throw MicmException("MICM State", 1, "Number of values does not match number of grid cells in State");
        for (Index i = 0; i < values.size(); ++i)
          state_.variables_[i][index_] = values[i];
        return *this;
      }
      Real& operator[](Index cell)
      {
        if (cell >= state_.number_of_grid_cells_)
          throw std::out_of_range("Grid cell index out of range");
        return state_.variables_[cell][index_];
      }
    };

    CudaState() = default;

    Index NumberOfGridCells() const
    {
      return number_of_grid_cells_;
    }
    VariableProxy operator[](Index index)
    {
      if (index >= variable_names_.size())
        throw std::out_of_range("Variable index out of range");
      return VariableProxy(*this, index);
    }
    VariableProxy operator[](const std::string& name)
    {
      auto it = variable_map_.find(name);
      if (it == variable_map_.end())
        throw MicmException("MICM State", 2, "Unknown variable '" + name + "'");
      return VariableProxy(*this, it->second);
    }
    VariableProxy operator[](const Species& species)
    {
      return (*this)[species.name_];
    }
    void SetConcentration(const Species& species, Real value)
    {
      (*this)[species] = value;
    }
    void SetConcentration(const Species& species, const std::vector<Real>& values)
    {
      (*this)[species] = values;
    }
    void SetCustomRateParameter(const std::string& label, Real value)
    {
      SetCustomRateParameter(label, std::vector<Real>(number_of_grid_cells_, value));
    }
    void SetCustomRateParameter(const std::string& label, const std::vector<Real>& values)
    {
      auto it = custom_rate_parameter_map_.find(label);
      if (it == custom_rate_parameter_map_.end())
        throw MicmException("MICM State", 3, "Unknown custom rate parameter '" + label + "'");
      if (values.size() != number_of_grid_cells_)
        throw MicmException("MICM State", 1, "Number of values does not match number of grid cells in State");
      for (Index i = 0; i < values.size(); ++i)
        custom_rate_parameters_[i][it->second] = values[i];
    }
    void SetCustomRateParameters(const std::unordered_map<std::string, std::vector<Real>>& parameters)
    {
      for (const auto& p : parameters)
        SetCustomRateParameter(p.first, p.second);
    }
    void SetRelativeTolerance(Real rtol)
    {
      relative_tolerance_ = rtol;
    }
    void SetAbsoluteTolerances(const std::vector<Real>& atol)
    {
      if (atol.size() != variable_names_.size())
        throw MicmException("MICM State", 4, "Absolute tolerance size does not match the number of variables");
      absolute_tolerance_ = atol;
    }

    // CudaState::SyncInputsToDevice (cuda_state.hpp:132-136): concentrations
    // plus tolerances; conditions and custom parameters travel with
    // Solver::UpdateStateParameters as in micm's CUDA path.
    void SyncInputsToDevice()
    {
      detail::Check(micmb_state_upload(handle_.get(), MICMB_BUF_VARIABLES, variables_.AsVector().data()));
      detail::Check(micmb_state_upload(handle_.get(), MICMB_BUF_ABSOLUTE_TOLERANCE, absolute_tolerance_.data()));
      detail::Check(micmb_state_set_relative_tolerance(handle_.get(), relative_tolerance_));
    }
    // CudaState::SyncOutputsToHost (cuda_state.hpp:139-148)
    void SyncOutputsToHost()
    {
      detail::Check(micmb_state_download(handle_.get(), MICMB_BUF_VARIABLES, variables_.AsVector().data()));
      if (rate_constants_.NumColumns() > 0)
        detail::Check(
            micmb_state_download(handle_.get(), MICMB_BUF_RATE_CONSTANTS, rate_constants_.AsVector().data()));
    }

    void PrintHeader()
    {
      auto names = variable_names_;
      std::cout << std::setw(5) << "time";
      for (const auto& n : names)
        std::cout << "," << std::setw(11) << n;
      std::cout << std::endl;
    }
    void PrintState(Real time)
    {
      std::ios oldState(nullptr);
      oldState.copyfmt(std::cout);
      std::cout << std::setw(5) << time << std::flush;
      for (Index c = 0; c < number_of_grid_cells_; ++c)
        for (Index i = 0; i < variable_names_.size(); ++i)
          std::cout << std::scientific << std::setprecision(2) << "," << std::setw(11) << variables_[c][i];
      std::cout << std::endl;
      std::cout.copyfmt(oldState);
    }
  };

  // ---------------------------------------------------------------- solver
  template<Index L = MICM_DEFAULT_VECTOR_SIZE>
  class Solver
  {
    std::shared_ptr<micmb_mechanism> mech_;
    std::shared_ptr<micmb_solver> solver_;
    std::vector<std::string> variable_names_;
    std::vector<std::string> param_labels_;
    std::vector<Real> atol_;  // by state column
    Index n_rate_constants_ = 0;
    std::vector<Real> mass_;  // by state column: 1 ODE row, 0 algebraic row
    Index n_constraints_ = 0;
    StepControl step_control_ = StepControl::Global;
    Method method_ = Method::Plain;

   public:
    RosenbrockSolverParameters solver_parameters_;

    Solver(std::shared_ptr<micmb_mechanism> mech, RosenbrockSolverParameters params,
           std::vector<std::string> variable_names, std::vector<std::string> param_labels, std::vector<Real> atol,
           Index n_rate_constants)
        : mech_(std::move(mech)),
          variable_names_(std::move(variable_names)),
          param_labels_(std::move(param_labels)),
          atol_(std::move(atol)),
          n_rate_constants_(n_rate_constants),
          solver_parameters_(params)
    {
      const micmb_rosenbrock_params p = params.ToC();
      micmb_solver* s = nullptr;
      detail::Check(micmb_solver_create(mech_.get(), &p, &s));
      solver_ = std::shared_ptr<micmb_solver>(s, micmb_solver_destroy);
    }

    void SetStepControl(StepControl s)
    {
      step_control_ = s;
    }
    void SetMethod(Method m)
    {
      method_ = m;
      if (m == Method::Fused)
        step_control_ = StepControl::PerCell;
    }
    Index MaximumNumberOfGridCells() const
    {
      return L;
    }
    micmb_solver* Handle() const
    {
      return solver_.get();
    }

    CudaState<L> GetState(const Index number_of_grid_cells = 1) const
    {
      CudaState<L> st;
      micmb_state* h = nullptr;
      detail::Check(micmb_state_create(solver_.get(), (int64_t)number_of_grid_cells, (int32_t)L, &h));
      st.handle_ = std::shared_ptr<micmb_state>(h, micmb_state_destroy);
      st.number_of_grid_cells_ = number_of_grid_cells;
      st.variables_ = VectorMatrix<Real, L>(number_of_grid_cells, variable_names_.size(), 0.0);
      st.custom_rate_parameters_ = VectorMatrix<Real, L>(number_of_grid_cells, param_labels_.size(), 0.0);
      st.rate_constants_ = VectorMatrix<Real, L>(number_of_grid_cells, n_rate_constants_, 0.0);
      st.conditions_.assign(number_of_grid_cells, Conditions{});
      st.variable_names_ = variable_names_;
      for (Index i = 0; i < variable_names_.size(); ++i)
        st.variable_map_[variable_names_[i]] = i;
      for (Index i = 0; i < param_labels_.size(); ++i)
        st.custom_rate_parameter_map_[param_labels_[i]] = i;
      st.absolute_tolerance_ = atol_;
      st.relative_tolerance_ = 1e-6;
      st.constraint_size_ = n_constraints_;
      st.upper_left_identity_diagonal_ = mass_.empty() ? std::vector<Real>(variable_names_.size(), 1.0) : mass_;
      return st;
    }

    // Solver::UpdateStateParameters -> CudaProcessSet::GpuCalculateRateConstants:
    // conditions and custom parameters to the device, rate constants on the GPU.
    void UpdateStateParameters(CudaState<L>& state)
    {
      const Index n = state.number_of_grid_cells_;
      VectorMatrix<Real, L> cond(n, 3, 0.0);
      for (Index c = 0; c < n; ++c)
      {
        cond[c][0] = state.conditions_[c].temperature_;
        cond[c][1] = state.conditions_[c].pressure_;
        cond[c][2] = state.conditions_[c].air_density_;
      }
      detail::Check(micmb_state_upload(state.handle_.get(), MICMB_BUF_CONDITIONS, cond.AsVector().data()));
      if (!param_labels_.empty())
        detail::Check(micmb_state_upload(state.handle_.get(), MICMB_BUF_CUSTOM_PARAMS,
                                         state.custom_rate_parameters_.AsVector().data()));
      detail::Check(micmb_update_state_parameters(solver_.get(), state.handle_.get()));
    }

    // Solver::Solve(time_step, state): integrate the device-resident state by
    // time_step and clamp negative concentrations to zero.
    SolverResult Solve(Real time_step, CudaState<L>& state)
    {
      micmb_solver_stats st{};
      const int rc = micmb_solve(solver_.get(), state.handle_.get(), time_step,
                                 method_ == Method::Fused ? MICMB_METHOD_FUSED : MICMB_METHOD_PLAIN,
                                 step_control_ == StepControl::Global ? MICMB_STEP_GLOBAL : MICMB_STEP_PER_CELL, &st,
                                 nullptr, nullptr);
      detail::Check(rc);
      SolverResult r;
      r.state_ = static_cast<SolverState>(st.state);
      r.stats_.function_calls_ = (Index)st.function_calls;
      r.stats_.jacobian_updates_ = (Index)st.jacobian_updates;
      r.stats_.number_of_steps_ = (Index)st.number_of_steps;
      r.stats_.accepted_ = (Index)st.accepted;
      r.stats_.rejected_ = (Index)st.rejected;
      r.stats_.decompositions_ = (Index)st.decompositions;
      r.stats_.solves_ = (Index)st.solves;
      r.stats_.constraint_init_iterations_ = (Index)st.constraint_init_iterations;
      r.stats_.final_time_ = st.final_time;
      return r;
    }

    // algebraic constraints: which rows are algebraic (set by the builder)
    void SetConstraintRows(std::vector<Real> mass, Index n_constraints)
    {
      mass_ = std::move(mass);
      n_constraints_ = n_constraints;
    }

    SolverResult Solve(Real time_step, CudaState<L>& state, const RosenbrockSolverParameters& params)
    {
      solver_parameters_ = params;
      const micmb_rosenbrock_params p = params.ToC();
      detail::Check(micmb_solver_set_params(solver_.get(), &p));
      return Solve(time_step, state);
    }

    // Autotuner (no micm counterpart): time the fused-kernel configurations on
    // this state, keep the fastest for later fused solves; cached by mechanism
    // hash in `cache_path` when given.
    void Autotune(Real time_step, CudaState<L>& state, const char* cache_path = nullptr)
    {
      micmb_fused_config chosen{};
      detail::Check(micmb_autotune(solver_.get(), state.handle_.get(), time_step, cache_path, &chosen));
    }

    // n_repeats x (UpdateStateParameters + fused Solve) replayed from one CUDA
    // graph (no micm counterpart); conditions and custom parameters are read
    // from the device copies the last UpdateStateParameters uploaded.
    void SolveRepeated(Real time_step, CudaState<L>& state, int32_t n_repeats)
    {
      detail::Check(micmb_solve_graph(solver_.get(), state.handle_.get(), time_step, n_repeats));
    }

    // Device bytes SolveAdjoint may hold in checkpoints (0: 80 % of the free
    // device memory); cells are swept in chunks that fit.
    void SetAdjointMemoryLimit(std::int64_t bytes)
    {
      detail::Check(micmb_set_adjoint_memory_limit(solver_.get(), bytes));
    }

    // Discrete adjoint of the accepted steps of a per-cell solve (no micm
    // counterpart).  dloss_dy_final and dloss_dy0 are [cell][variable] in the
    // state's VectorMatrix layout; dloss_dlogk is per reaction in input order.
    SolverResult SolveAdjoint(Real time_step, CudaState<L>& state, const VectorMatrix<Real, L>& dloss_dy_final,
                              VectorMatrix<Real, L>& dloss_dy0, std::vector<Real>& dloss_dlogk,
                              int32_t max_checkpoints = 512)
    {
      micmb_solver_stats st{};
      dloss_dy0 = VectorMatrix<Real, L>(state.number_of_grid_cells_, variable_names_.size(), 0.0);
      dloss_dlogk.assign(n_rate_constants_, 0.0);
      detail::Check(micmb_solve_adjoint(solver_.get(), state.handle_.get(), time_step,
                                        dloss_dy_final.AsVector().data(), dloss_dy0.AsVector().data(),
                                        dloss_dlogk.data(), max_checkpoints, &st));
      SolverResult r;
      r.state_ = static_cast<SolverState>(st.state);
      r.stats_.accepted_ = (Index)st.accepted;
      r.stats_.number_of_steps_ = (Index)st.number_of_steps;
      return r;
    }
  };

  // ---------------------------------------------------------------- builder
  // micm::SolverBuilder (solver_builder.hpp:45-255) specialised for the CUDA path
  // (cuda_solver_builder.hpp:25-37).
  template<class SolverParametersPolicy, Index L = MICM_DEFAULT_VECTOR_SIZE>
  class CudaSolverBuilderInPlace
  {
    SolverParametersPolicy options_;
    System system_;
    std::vector<Process> reactions_;
    bool ignore_unused_species_ = true;
    bool reorder_state_ = true;
    bool valid_system_ = false;
    // constraints as the C description takes them (SetConstraints)
    struct ConstraintRow
    {
      int32_t type;
      std::string species;
      std::vector<StoichSpecies> terms;  // equilibrium: reactants, then products
      int32_t n_reactants;
      double params[4];
    };
    std::vector<ConstraintRow> constraints_;

   public:
    CudaSolverBuilderInPlace(const SolverParametersPolicy& options)
        : options_(options)
    {
    }
    CudaSolverBuilderInPlace& SetSystem(const System& system)
    {
      system_ = system;
      valid_system_ = true;
      return *this;
    }
    CudaSolverBuilderInPlace& SetReactions(const std::vector<Process>& reactions)
    {
      reactions_ = reactions;
      return *this;
    }
    // SolverBuilder::SetConstraints (solver_builder.hpp:104-108): algebraic
    // constraints, each replacing its algebraic species' ODE row.  micm's CUDA
    // builder rejects them (solver_builder.inl:251-266); this one solves them
    // on the device (plain and fused methods, both step controls).
    template<class D, class S>
    CudaSolverBuilderInPlace& SetConstraints(std::vector<Constraint<D, S>>&& constraints)
    {
      constraints_.clear();
      for (const auto& c : constraints)
        std::visit(
            [&](const auto& v) {
              using T = std::decay_t<decltype(v)>;
              ConstraintRow row{};
              row.species = v.AlgebraicSpecies();
              if constexpr (std::is_same_v<T, LinearConstraint<D, S>>)
              {
                row.type = MICMB_CONSTRAINT_LINEAR;
                row.terms = v.terms_;
                row.params[0] = v.constant_;
              }
              else
              {
                row.type = MICMB_CONSTRAINT_EQUILIBRIUM;
                row.terms = v.reactants_;
                row.terms.insert(row.terms.end(), v.products_.begin(), v.products_.end());
                row.n_reactants = (int32_t)v.reactants_.size();
                row.params[0] = v.vant_hoff_param_.K_HLC_ref_;
                row.params[1] = v.vant_hoff_param_.delta_H_;
                row.params[2] = v.vant_hoff_param_.R_;
                row.params[3] = v.vant_hoff_param_.T_ref_;
              }
              constraints_.push_back(std::move(row));
            },
            c.constraint_);
      return *this;
    }
    CudaSolverBuilderInPlace& SetIgnoreUnusedSpecies(bool ignore)
    {
      ignore_unused_species_ = ignore;
      return *this;
    }
    CudaSolverBuilderInPlace& SetReorderState(bool reorder)
    {
      reorder_state_ = reorder;
      return *this;
    }

    Solver<L> Build()
    {
      if (!valid_system_)
        throw MicmException("MICM Solver", 1, "Missing chemical system.");
      const auto names = system_.UniqueNames();
      if (names.empty())
        throw MicmException("MICM Solver", 2, "Provided chemical system contains no species.");
      std::unordered_map<std::string, int32_t> sys_index;
      for (Index i = 0; i < names.size(); ++i)
        sys_index[names[i]] = (int32_t)i;
      const Index R = reactions_.size();
      std::vector<int32_t> rate_type(R), rstart{ 0 }, rspecies, pstart{ 0 }, pspecies;
      std::vector<double> rate_params(R * MICMB_RATE_PARAM_STRIDE, 0.0), pyield, pcoef;
      std::map<std::tuple<double, double, double, double>, int32_t> param_ids;
      std::set<std::string> used;
      for (Index r = 0; r < R; ++r)
      {
        const ChemicalReaction& rx = reactions_[r].process_;
        double* p = rate_params.data() + r * MICMB_RATE_PARAM_STRIDE;
        std::visit(
            [&](const auto& v) {
              using T = std::decay_t<decltype(v)>;
              if constexpr (std::is_same_v<T, ArrheniusRateConstantParameters>)
              {
                rate_type[r] = MICMB_RATE_ARRHENIUS;
                p[0] = v.A_, p[1] = v.B_, p[2] = v.C_, p[3] = v.D_, p[4] = v.E_;
              }
              else if constexpr (std::is_same_v<T, TroeRateConstantParameters> ||
                                 std::is_same_v<T, TernaryChemicalActivationRateConstantParameters>)
              {
                rate_type[r] = std::is_same_v<T, TroeRateConstantParameters> ? MICMB_RATE_TROE
                                                                              : MICMB_RATE_TERNARY_CHEMICAL_ACTIVATION;
                p[0] = v.k0_A_, p[1] = v.k0_B_, p[2] = v.k0_C_, p[3] = v.kinf_A_, p[4] = v.kinf_B_,
                p[5] = v.kinf_C_, p[6] = v.Fc_, p[7] = v.N_;
              }
              else if constexpr (std::is_same_v<T, BranchedRateConstantParameters>)
              {
                rate_type[r] = MICMB_RATE_BRANCHED;
                p[0] = v.branch_ == BranchedRateConstantParameters::Branch::Alkoxy ? 0.0 : 1.0;
                p[1] = v.X_, p[2] = v.Y_, p[3] = v.a0_, p[4] = (double)v.n_;
              }
              else if constexpr (std::is_same_v<T, TunnelingRateConstantParameters>)
              {
                rate_type[r] = MICMB_RATE_TUNNELING;
                p[0] = v.A_, p[1] = v.B_, p[2] = v.C_;
              }
              else if constexpr (std::is_same_v<T, TaylorSeriesRateConstantParameters>)
              {
                rate_type[r] = MICMB_RATE_TAYLOR_SERIES;
                p[0] = v.A_, p[1] = v.B_, p[2] = v.C_, p[3] = v.D_, p[4] = v.E_, p[5] = (double)v.n_coefficients_;
                for (Index j = 0; j < v.n_coefficients_ && j < 16; ++j)
                  p[6 + j] = v.coefficients_[j];
              }
              else if constexpr (std::is_same_v<T, ReversibleRateConstantParameters>)
              {
                rate_type[r] = MICMB_RATE_REVERSIBLE;
                p[0] = v.A_, p[1] = v.C_, p[2] = v.k_r_;
              }
              else if constexpr (std::is_same_v<T, UserDefinedRateConstantParameters>)
              {
                rate_type[r] = MICMB_RATE_USER_DEFINED;
                p[0] = v.scaling_factor_;
              }
              else
              {
                rate_type[r] = MICMB_RATE_SURFACE;
                if (!v.phase_species_.diffusion_coefficient_)
                  throw MicmException("MICM Species", 1, "Diffusion coefficient for species '" +
                                                             v.phase_species_.species_.name_ + "' is not defined");
                p[0] = *v.phase_species_.diffusion_coefficient_;
                p[1] = v.phase_species_.species_.template GetProperty<Real>(property_keys::MOLECULAR_WEIGHT);
                p[2] = v.reaction_probability_;
              }
            },
            rx.rate_constant_);
        for (const auto& s : rx.reactants_)
        {
          used.insert(s.name_);
          if (s.IsParameterized())
          {
            const auto& f = s.parameterize_;
            auto key = std::make_tuple(f.c0_, f.c_T_, f.c_P_, f.c_rho_);
            auto it = param_ids.find(key);
            if (it == param_ids.end())
            {
              it = param_ids.emplace(key, (int32_t)param_ids.size()).first;
              pcoef.insert(pcoef.end(), { f.c0_, f.c_T_, f.c_P_, f.c_rho_ });
            }
            rspecies.push_back(-(it->second + 1));
          }
          else
          {
            auto it = sys_index.find(s.name_);
            if (it == sys_index.end())
              throw MicmException("MICM Process", 2, s.name_);
            rspecies.push_back(it->second);
          }
        }
        rstart.push_back((int32_t)rspecies.size());
        for (const auto& p2 : rx.products_)
        {
          used.insert(p2.species_.name_);
          if (p2.species_.IsParameterized())
            continue;
          auto it = sys_index.find(p2.species_.name_);
          if (it == sys_index.end())
            throw MicmException("MICM Process", 3, p2.species_.name_);
          pspecies.push_back(it->second);
          pyield.push_back(p2.coefficient_);
        }
        pstart.push_back((int32_t)pspecies.size());
      }
      std::vector<int32_t> c_type, c_species, c_start{ 0 }, c_term_species, c_nreact;
      std::vector<double> c_coef, c_params;
      for (const auto& c : constraints_)
      {
        auto species_index = [&](const std::string& name) {
          auto it = sys_index.find(name);
          if (it == sys_index.end())
            throw MicmException("MICM Constraint", 4, "Species '" + name + "' is not in the chemical system");
          used.insert(name);
          return it->second;
        };
        c_type.push_back(c.type);
        c_species.push_back(species_index(c.species));
        for (const auto& t : c.terms)
        {
          c_term_species.push_back(species_index(t.species_.name_));
          c_coef.push_back(t.coefficient_);
        }
        c_start.push_back((int32_t)c_term_species.size());
        c_nreact.push_back(c.n_reactants);
        c_params.insert(c_params.end(), c.params, c.params + 4);
      }
      if (!ignore_unused_species_)
        for (const auto& n : names)
          if (!used.count(n))
            throw MicmException("MICM Solver", 3, "Unused species in chemical system: '" + n + "'.");
      micmb_mechanism_desc d{};
      d.n_species = (int32_t)names.size();
      d.n_reactions = (int32_t)R;
      d.rate_type = rate_type.data();
      d.rate_params = rate_params.data();
      d.reactant_start = rstart.data();
      d.reactant_species = rspecies.data();
      d.product_start = pstart.data();
      d.product_species = pspecies.data();
      d.product_yield = pyield.data();
      d.n_parameterized = (int32_t)param_ids.size();
      d.parameterized_coef = pcoef.data();
      d.reorder_state = reorder_state_ ? 1 : 0;
      d.n_constraints = (int32_t)constraints_.size();
      if (!constraints_.empty())
      {
        d.constraint_type = c_type.data();
        d.constraint_species = c_species.data();
        d.constraint_term_start = c_start.data();
        d.constraint_term_species = c_term_species.data();
        d.constraint_term_coef = c_coef.data();
        d.constraint_n_reactants = c_nreact.data();
        d.constraint_params = c_params.data();
      }
      micmb_mechanism* m = nullptr;
      detail::Check(micmb_mechanism_create(&d, &m));
      auto mech = std::shared_ptr<micmb_mechanism>(m, micmb_mechanism_destroy);
      std::vector<int32_t> col(names.size()), pcol(R);
      detail::Check(micmb_mechanism_species_columns(m, col.data()));
      if (R)
        detail::Check(micmb_mechanism_custom_param_columns(m, pcol.data()));
      std::vector<std::string> variable_names(names.size());
      std::vector<Real> atol(names.size(), 1e-3);  // SolverBuilder default (solver_builder.inl:208)
      for (Index i = 0; i < names.size(); ++i)
        variable_names[col[i]] = names[i];
      for (const auto& ps : system_.gas_phase_.phase_species_)
        if (!ps.species_.IsParameterized() && ps.species_.HasProperty(property_keys::ABSOLUTE_TOLERANCE))
          atol[col[sys_index[ps.species_.name_]]] =
              ps.species_.template GetProperty<Real>(property_keys::ABSOLUTE_TOLERANCE);
      micmb_mechanism_info info{};
      detail::Check(micmb_mechanism_get_info(m, &info));
      std::vector<std::string> labels(info.n_custom_params);
      std::set<std::string> seen;
      for (Index r = 0; r < R; ++r)
      {
        const auto& rc = reactions_[r].process_.rate_constant_;
        if (const auto* ud = std::get_if<UserDefinedRateConstantParameters>(&rc))
        {
          if (!seen.insert(ud->label_).second)
            throw MicmException("MICM Solver", 4, "Duplicate parameter labels detected: " + ud->label_);
          labels[pcol[r]] = ud->label_;
        }
        else if (const auto* sf = std::get_if<SurfaceRateConstantParameters>(&rc))
        {
          const std::string a = sf->label_ + ".effective radius [m]";
          const std::string b = sf->label_ + ".particle number concentration [# m-3]";
          if (!seen.insert(a).second || !seen.insert(b).second)
            throw MicmException("MICM Solver", 4, "Duplicate parameter labels detected: " + sf->label_);
          labels[pcol[r]] = a;
          labels[pcol[r] + 1] = b;
        }
      }
      Solver<L> solver(mech, options_, variable_names, labels, atol, R);
      if (!constraints_.empty())
      {
        std::vector<Real> mass(names.size(), 1.0);
        for (const auto& c : constraints_)
          mass[col[sys_index[c.species]]] = 0.0;
        solver.SetConstraintRows(std::move(mass), constraints_.size());
      }
      return solver;
    }
  };

  // include/micm/GPU.hpp aliases
  using GpuState = CudaState<MICM_DEFAULT_VECTOR_SIZE>;
  using CudaRosenbrock = Solver<MICM_DEFAULT_VECTOR_SIZE>;
  using GpuRosenbrockThreeStageBuilder = CudaSolverBuilderInPlace<CudaRosenbrockSolverParameters>;
}  // namespace micm
