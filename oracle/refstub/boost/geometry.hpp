// Header-only stand-in for the Boost.Geometry names that the reference's
// ShapeGenerator.h and Utils.h declare type aliases with.  TEST
// INFRASTRUCTURE ONLY: it lets oracle/Makefile.ref compile the reference's
// grid setup and CPU engine without Boost.  Only the single-plane-symmetric
// cross-section (cross_sectional_shape 3) calls into Boost, and that mode is
// not built (oracle/ref_stubs.cpp aborts if it is reached).
#pragma once

namespace boost {
namespace geometry {
namespace model {
namespace d2 {
template <class T>
struct point_xy {
    T x_, y_;
};
}  // namespace d2
template <class P>
struct ring {};
template <class P>
struct linestring {};
template <class P>
struct multi_point {};
}  // namespace model
}  // namespace geometry
}  // namespace boost
