// vs_shapes.cpp -- single-plane-symmetric cross-sections (cross_sectional_shape 3).
//
// Restates, on the host, the reference's construction of such a section and
// of its depths:
//   * ShapeGenerator::combineRegularShapes (ShapeGenerator.cpp:35-197): a
//     3:1 ellipse s1 and a circle s2 of areas 3/4 and 1/4 of the section,
//     s2's centre at s1's semi-major axis + 0.003 mm; the upper half-contour
//     runs along s1 to the arcs' intersection and along s2 from there; both
//     shapes grow by 0.01 mm on every axis until twice the half-contour's area
//     reaches the section area; the half-contour's end points are put on the
//     axis and it is mirrored into the full contour;
//   * ShapeAlignment (ShapeAlignment.cu:9-152): the contour's diameter (the
//     largest distance between two of its points, first pair in index order)
//     is rotated onto the y axis and the contour shifted into the first
//     quadrant + 0.05;
//   * TubeDepth::generateTubeDepthSinglePlaneSymmetricShape
//     (TubeDepth.cu:493-640): half the z extent of the contour along the line
//     y = minY + offset.
// The reference takes the arcs' intersection, the contour area and the line
// crossings from Boost.Geometry on float points; here they are computed in
// double from the same float points (segment crossings, and the ring area as
// the sum of (y1 + y2)(z1 - z2) / 2) and rounded to float.  The float
// arithmetic around them follows the reference's expressions and order.
#include "vs_shapes.h"

#include <algorithm>
#include <cmath>
#include <limits>

namespace vsb {
namespace {

const double kPi = 3.14159265358979323846;
const float kMillimeter = (float)(1e-3 * 1.0);

// Utils::linspace (Utils.cpp:59-75)
std::vector<float> linspace(float start, float end, int n) {
    std::vector<float> r;
    if (n == 0) return r;
    if (n == 1) { r.push_back(start); return r; }
    const float step = (end - start) / (n - 1);
    r.reserve(n);
    for (int i = 0; i < n; ++i) r.push_back(start + step * i);
    return r;
}

// ShapeGenerator::generateEllipseCoordinates (ShapeGenerator.cpp:222-262)
std::vector<ShapePt> ellipse_arc(float y0, float y1, float a, float b, int n, float yc) {
    std::vector<ShapePt> s(n);
    const std::vector<float> y = linspace(y0, y1, n);
    std::vector<float> d2(n);
    for (int i = 0; i < n; ++i) {
        const float t = y[i] - yc;
        d2[i] = t * t;
    }
    const float a2 = a * a, b2 = b * b;
    d2[0] = a2;
    for (int i = 0; i < n / 2; ++i) d2[n - i - 1] = d2[i];
    for (int i = 0; i < n; ++i) {
        s[i].y = y[i];
        s[i].z = sqrtf(std::max(0.0f, b2 * (1.0f - d2[i] / a2)));
    }
    return s;
}

// Crossing of segments p1-p2 and q1-q2 (in double); false when they do not meet.
bool segment_cross(const ShapePt& p1, const ShapePt& p2, const ShapePt& q1, const ShapePt& q2, ShapePt* out) {
    const double px = p1.y, py = p1.z, rx = (double)p2.y - px, ry = (double)p2.z - py;
    const double qx = q1.y, qy = q1.z, sx = (double)q2.y - qx, sy = (double)q2.z - qy;
    const double den = rx * sy - ry * sx;
    if (den == 0.0) return false;
    const double t = ((qx - px) * sy - (qy - py) * sx) / den;
    const double u = ((qx - px) * ry - (qy - py) * rx) / den;
    if (t < 0.0 || t > 1.0 || u < 0.0 || u > 1.0) return false;
    out->y = (float)(px + t * rx);
    out->z = (float)(py + t * ry);
    return true;
}

// First crossing along s1 of two polylines whose y increases along them.
bool first_crossing(const std::vector<ShapePt>& s1, const std::vector<ShapePt>& s2, ShapePt* out) {
    size_t j = 0;
    for (size_t i = 0; i + 1 < s1.size(); ++i) {
        const float lo = std::min(s1[i].y, s1[i + 1].y), hi = std::max(s1[i].y, s1[i + 1].y);
        while (j + 1 < s2.size() && std::max(s2[j].y, s2[j + 1].y) < lo) ++j;
        for (size_t k = j; k + 1 < s2.size() && std::min(s2[k].y, s2[k + 1].y) <= hi; ++k)
            if (segment_cross(s1[i], s1[i + 1], s2[k], s2[k + 1], out)) return true;
    }
    return false;
}

// |area| of the ring through the points (closed back to the first point).
float ring_area(const std::vector<ShapePt>& c) {
    double sum = 0.0;
    const size_t n = c.size();
    for (size_t i = 0; i < n; ++i) {
        const ShapePt& a = c[i];
        const ShapePt& b = c[(i + 1) % n];
        sum += ((double)a.y + (double)b.y) * ((double)a.z - (double)b.z);
    }
    return (float)std::abs(sum / 2.0);
}

// ShapeGenerator::finalContourCoordinates (ShapeGenerator.cpp:264-309)
std::vector<ShapePt> half_contour(const ShapePt& ip, float a1, float b1, float a2, float b2, float yc1, float yc2,
                                  float y_start1, float y_end2, int nhalf) {
    const int seg = nhalf - 1;
    const std::vector<float> y1 = linspace(y_start1, ip.y, seg);
    const std::vector<float> y2 = linspace(ip.y, y_end2, seg);
    std::vector<ShapePt> c(2 * nhalf - 1);
    int k = 0;
    for (int i = 0; i < seg; ++i, ++k) {
        const float d = y1[i] - yc1;
        c[k] = {y1[i], sqrtf(std::max(0.0f, (b1 * b1) * (1.0f - (d * d) / (a1 * a1))))};
    }
    c[k++] = ip;
    for (int i = 0; i < seg; ++i, ++k) {
        const float d = y2[i] - yc2;
        c[k] = {y2[i], sqrtf(std::max(0.0f, (b2 * b2) * (1.0f - (d * d) / (a2 * a2))))};
    }
    return c;
}

}  // namespace

std::vector<ShapePt> sps_shape(float area, float* diameter, std::string* err) {
    const int ncoord = 1999;                        // TubeGeometry.cu:373
    const int nhalf = (ncoord + 1) / 2;
    const float m = 3.0f;
    const float x = area / (m + 1.0f);
    const float A1 = m * x, A2 = 1.0f * x;
    const float l1 = sqrtf((float)((double)A1 / (kPi * 3.0f * 1.0f)));
    const float l2 = sqrtf((float)((double)A2 / (kPi * 1.0f * 1.0f)));
    float a1 = l1 * 3.0f, b1 = l1 * 1.0f, a2 = l2 * 1.0f, b2 = l2 * 1.0f;
    const float yc1 = 0.0f;
    const float yc2 = yc1 + a1 + 0.003f * kMillimeter;
    const float grow = kMillimeter * 0.01f;
    std::vector<ShapePt> half;
    float got = -1.0f;
    for (int it = 0; got < area; ++it) {
        if (it > 0) { a1 = a1 + grow; b1 = b1 + grow; a2 = a2 + grow; b2 = b2 + grow; }
        if (it > 100000) { *err = "single-plane-symmetric section does not reach its area"; return {}; }
        const float y0 = yc1 - a1, y1 = yc1 + a1, z0 = yc2 - a2, z1 = yc2 + a2;
        const std::vector<ShapePt> s1 = ellipse_arc(y0, y1, a1, b1, nhalf, yc1);
        const std::vector<ShapePt> s2 = ellipse_arc(z0, z1, a2, b2, nhalf, yc2);
        ShapePt ip;
        if (!first_crossing(s1, s2, &ip)) { *err = "single-plane-symmetric section: the shapes do not meet"; return {}; }
        half = half_contour(ip, a1, b1, a2, b2, yc1, yc2, y0, z1, nhalf);
        got = 2 * ring_area(half);
    }
    half.front().z = 0.0f;
    half.back().z = 0.0f;
    std::vector<ShapePt> full = half;
    for (int i = (int)full.size() - 2; i >= 0; --i) full.push_back({full[i].y, -1 * full[i].z});
    // ShapeAlignment::shapeDiameter: per point its farthest point (first in
    // index order), then the first point with the largest such distance
    // (a row whose distance to the farthest corner of the bounding box cannot
    // exceed the best distance so far cannot be chosen and is skipped)
    const int n = (int)full.size();
    double bylo = full[0].y, byhi = full[0].y, bzlo = full[0].z, bzhi = full[0].z;
    for (const ShapePt& p : full) {
        bylo = std::min(bylo, (double)p.y); byhi = std::max(byhi, (double)p.y);
        bzlo = std::min(bzlo, (double)p.z); bzhi = std::max(bzhi, (double)p.z);
    }
    float best = 0.0f;
    int bi = 0, bj = 0;
    for (int i = 0; i < n; ++i) {
        const double fy = std::max(std::abs(full[i].y - bylo), std::abs(full[i].y - byhi));
        const double fz = std::max(std::abs(full[i].z - bzlo), std::abs(full[i].z - bzhi));
        if (std::sqrt(fy * fy + fz * fz) * (1.0 + 1e-5) < (double)best) continue;
        float mx = 0.0f;
        int mj = 0;
        for (int j = 0; j < n; ++j) {
            const float dy = full[i].y - full[j].y, dz = full[i].z - full[j].z;
            const float d = sqrtf(dy * dy + dz * dz);
            if (d > mx) { mx = d; mj = j; }
        }
        if (mx > best) { best = mx; bi = i; bj = mj; }
    }
    *diameter = best;
    // ShapeAlignment::rotateShapeAboutOrigin
    const float dy = full[bj].y - full[bi].y, dz = full[bj].z - full[bi].z;
    const float th = std::atan2(dz, dy);
    const float c = std::cos(-1 * th), s = std::sin(-1 * th);
    for (ShapePt& p : full) {
        const float y = p.y, z = p.z;
        p.y = c * y - s * z;
        p.z = s * y + c * z;
    }
    float minY = full[0].y, minZ = full[0].z;
    for (const ShapePt& p : full) { minY = std::min(minY, p.y); minZ = std::min(minZ, p.z); }
    const float shY = (minY < 0.0f ? -minY : 0.0f) + 0.05f;
    const float shZ = (minZ < 0.0f ? -minZ : 0.0f) + 0.05f;
    for (ShapePt& p : full) { p.y += shY; p.z += shZ; }
    return full;
}

bool sps_half_depth(const std::vector<ShapePt>& shape, float y, float z_lo, float z_hi, float* depth) {
    const ShapePt q1{y, z_lo}, q2{y, z_hi};
    float zmin = std::numeric_limits<float>::infinity(), zmax = -std::numeric_limits<float>::infinity();
    bool any = false;
    for (size_t i = 0; i + 1 < shape.size(); ++i) {
        const float lo = std::min(shape[i].y, shape[i + 1].y), hi = std::max(shape[i].y, shape[i + 1].y);
        if (y < lo || y > hi) continue;
        ShapePt p;
        if (segment_cross(shape[i], shape[i + 1], q1, q2, &p)) {
            zmin = std::min(zmin, p.z);
            zmax = std::max(zmax, p.z);
            any = true;
        }
    }
    *depth = (zmax - zmin) / 2.0f;
    return any;
}

}  // namespace vsb
