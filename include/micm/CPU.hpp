// micm/CPU.hpp -- micm's CPU umbrella header (include/micm/CPU.hpp in micm),
// served by this library for code that includes it for micm's system and
// process types (Species, Phase, PhaseSpecies, System, ChemicalReactionBuilder,
// Process, the rate-constant parameter structs), as micm's benchmark
// mechanisms do (test/benchmark/ts1_mechanism.hpp, chapman_mechanism.hpp).
// The solver builder it provides is micm's CUDA-path one,
// CudaSolverBuilderInPlace; micm's CPU builders are not part of this library.
#pragma once

#include "../micm_b200/micm.hpp"
