// Umbrella header of the drop-in host layer (the reference's pomerol.hpp).
#pragma once

#include "pomerol/Core.hpp"
#include "pomerol/Operators.hpp"
#include "pomerol/ED.hpp"
#include "pomerol/Correlators.hpp"
