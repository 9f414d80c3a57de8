// micm/util/property_keys.hpp (micm's species property names), served by
// this library: micm::property_keys lives in micm_b200/micm.hpp.
#pragma once

#include "../../micm_b200/micm.hpp"
