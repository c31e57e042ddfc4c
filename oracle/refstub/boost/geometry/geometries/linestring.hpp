// Stand-in: see boost/geometry.hpp in this directory.
#pragma once
#include "../../geometry.hpp"
