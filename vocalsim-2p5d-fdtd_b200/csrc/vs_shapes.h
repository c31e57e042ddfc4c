// vs_shapes.h -- single-plane-symmetric cross-sections (vs_shapes.cpp).
#pragma once

#include <string>
#include <vector>

namespace vsb {

struct ShapePt {
    float y, z;
};

// Aligned full contour of a single-plane-symmetric section of `area` (m^2)
// and its diameter (m); empty with *err set when the construction fails.
std::vector<ShapePt> sps_shape(float area, float* diameter, std::string* err);

// Half the z extent of `shape` along the vertical line y (the segment from
// z_lo to z_hi); false when the line does not cross the contour.
bool sps_half_depth(const std::vector<ShapePt>& shape, float y, float z_lo, float z_hi, float* depth);

}  // namespace vsb
