// FDTDEngineCPU.h -- the reference header of this name for code written against
// the reference (its main.cu builds unchanged with this directory in place of
// the reference's include/): the class of the C++ mirror over the C ABI of
// libvocalsim_b200 (cpp/vocalsim_b200.hpp), in the global namespace.
#pragma once

#include "SimulationUnits.h"
#include "../vocalsim_b200.hpp"

using vsb::FDTDEngineCPU;
using vsb::FDTDSolver;
