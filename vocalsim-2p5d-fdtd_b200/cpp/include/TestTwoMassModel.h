// TestTwoMassModel.h -- present so that code including the reference's header
// of this name compiles.  The reference's manual harness testTwoMassModel()
// (a standalone 1 s two-mass run written to a text file; its call is
// commented out in the reference's main.cu) is not part of the solver path
// and is not provided; the two-mass model itself runs inside the engines.
#pragma once

#include "SimulationUnits.h"
#include "../vocalsim_b200.hpp"
