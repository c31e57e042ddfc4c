/*
 * ref_stubs.cpp -- link-time stand-ins for the reference's Boost-based
 * shape code.  TEST INFRASTRUCTURE ONLY (oracle/Makefile.ref).
 *
 * The reference's TubeGeometry.cu and TubeDepth.cu call ShapeGenerator and
 * Utils only for the single-plane-symmetric cross-section
 * (cross_sectional_shape 3, TubeGeometry.cu:367-428, TubeDepth.cu:493-640).
 * Their sources (ShapeGenerator.cpp, Utils.cpp) need Boost.Geometry, which is
 * not installed, so they are not built; these definitions satisfy the linker
 * and stop the program if shape 3 is ever requested.  Circular and elliptical
 * sections never reach them.
 */
#include "ShapeGenerator.h"
#include "Utils.h"

#include <cstdio>
#include <cstdlib>

[[noreturn]] static void shape3_not_built(const char* what) {
    std::fprintf(stderr, "ref_engine: %s needs Boost.Geometry (cross_sectional_shape 3 is not built)\n", what);
    std::exit(3);
}

ShapeGenerator::ShapeGenerator(int, vector<float>& a, vector<float>& b, vector<float>& c, vector<float>& d,
                               vector<float>& e, vector<float>& f, vector<float>& g, float)
    : s1_semi_major_axis_len(a), s1_semi_minor_axis_len(b), s2_semi_major_axis_len(c),
      s2_semi_minor_axis_len(d), s1_s2_center_distance(e), yIntersect(f), zIntersect(g) {
    shape3_not_built("ShapeGenerator");
}

ShapeGenerator::~ShapeGenerator() {}

void ShapeGenerator::combineRegularShapes(int, int) { shape3_not_built("ShapeGenerator::combineRegularShapes"); }

void Utils::saveTubeSegmentCoords(vector<vector<ShapeCoordinates>>&, vector<float>&) {
    shape3_not_built("Utils::saveTubeSegmentCoords");
}

vector<float> Utils::linspace(float, float, int) { shape3_not_built("Utils::linspace"); }

vector<ShapeCoordinates> Utils::findShapeIntersections(const vector<ShapeCoordinates>&,
                                                       const vector<ShapeCoordinates>&) {
    shape3_not_built("Utils::findShapeIntersections");
}

float Utils::computeTotalArea(const vector<ShapeCoordinates>&) { shape3_not_built("Utils::computeTotalArea"); }
