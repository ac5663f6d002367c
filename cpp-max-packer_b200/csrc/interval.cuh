// Outward-rounded FP64 interval arithmetic shared by host and device.
//
// Restates the raster interval primitives of the reference
// (engine/pack_geometry/src/validation_kernel.cpp:291-324 widened/add/
// subtract/multiply/divide, :1942-1966 interval vector ops, :2038-2079
// triangle_box_disjoint, :2081-2100 grid_cell_interval) so that device and
// host results are bit-identical to it: every operation is one IEEE binary64
// round-to-nearest operation (device: __dadd_rn/__dmul_rn/... so nothing is
// contracted into an FMA), then each bound moves one ulp outward with an
// integer-bit nextafter; min/max keep std::min/std::max semantics.
#pragma once

#include <cstdint>
#include <cstring>

#include "common.cuh"

namespace spk {

SPK_HD double f_add(double a, double b)
{
#ifdef __CUDA_ARCH__
    return __dadd_rn(a, b);
#else
    return a + b;
#endif
}
SPK_HD double f_sub(double a, double b)
{
#ifdef __CUDA_ARCH__
    return __dsub_rn(a, b);
#else
    return a - b;
#endif
}
SPK_HD double f_mul(double a, double b)
{
#ifdef __CUDA_ARCH__
    return __dmul_rn(a, b);
#else
    return a * b;
#endif
}
SPK_HD double f_div(double a, double b)
{
#ifdef __CUDA_ARCH__
    return __ddiv_rn(a, b);
#else
    return a / b;
#endif
}

SPK_HD std::uint64_t f_bits(double v)
{
#ifdef __CUDA_ARCH__
    return static_cast<std::uint64_t>(__double_as_longlong(v));
#else
    std::uint64_t b;
    std::memcpy(&b, &v, 8);
    return b;
#endif
}
SPK_HD double f_from_bits(std::uint64_t b)
{
#ifdef __CUDA_ARCH__
    return __longlong_as_double(static_cast<long long>(b));
#else
    double v;
    std::memcpy(&v, &b, 8);
    return v;
#endif
}

SPK_HD bool f_finite(double v) { return (f_bits(v) & 0x7ff0000000000000ULL) != 0x7ff0000000000000ULL; }

// IEEE nextafter(v, -inf) / nextafter(v, +inf) for finite v, from the bit
// representation (the next representable binary64 value in that direction).
SPK_HD double next_down(double v)
{
    if (v != v) {
        return v;
    }
    const std::uint64_t b = f_bits(v);
    if ((b & 0x7fffffffffffffffULL) == 0) {
        return f_from_bits(0x8000000000000001ULL);  // -denorm_min
    }
    if (b >> 63) {
        return (b & 0x7fffffffffffffffULL) == 0x7ff0000000000000ULL ? v : f_from_bits(b + 1);
    }
    return f_from_bits(b - 1);
}
SPK_HD double next_up(double v)
{
    if (v != v) {
        return v;
    }
    const std::uint64_t b = f_bits(v);
    if ((b & 0x7fffffffffffffffULL) == 0) {
        return f_from_bits(0x0000000000000001ULL);  // +denorm_min
    }
    if (b >> 63) {
        return f_from_bits(b - 1);
    }
    return b == 0x7ff0000000000000ULL ? v : f_from_bits(b + 1);
}

// std::min / std::max semantics: min(a, b) = (b < a) ? b : a.
SPK_HD double f_min(double a, double b) { return (b < a) ? b : a; }
SPK_HD double f_max(double a, double b) { return (a < b) ? b : a; }

struct Interval {
    double low;
    double high;
    bool valid;
};

SPK_HD Interval point_interval(double v) { return { v, v, f_finite(v) }; }

SPK_HD Interval widened(double low, double high)
{
    if (!f_finite(low) || !f_finite(high)) {
        return { 0, 0, false };
    }
    low = next_down(low);
    high = next_up(high);
    return { low, high, f_finite(low) && f_finite(high) };
}

SPK_HD Interval add_interval(Interval a, Interval b)
{
    if (!a.valid || !b.valid) {
        return { 0, 0, false };
    }
    return widened(f_add(a.low, b.low), f_add(a.high, b.high));
}

SPK_HD Interval subtract_interval(Interval a, Interval b)
{
    if (!a.valid || !b.valid) {
        return { 0, 0, false };
    }
    return widened(f_sub(a.low, b.high), f_sub(a.high, b.low));
}

SPK_HD Interval multiply_interval(Interval a, Interval b)
{
    if (!a.valid || !b.valid) {
        return { 0, 0, false };
    }
    const double v0 = f_mul(a.low, b.low), v1 = f_mul(a.low, b.high), v2 = f_mul(a.high, b.low),
                 v3 = f_mul(a.high, b.high);
    if (!f_finite(v0) || !f_finite(v1) || !f_finite(v2) || !f_finite(v3)) {
        return { 0, 0, false };
    }
    // std::ranges::min_element / max_element: the first minimum / maximum.
    double lo = v0, hi = v0;
    if (v1 < lo) lo = v1;
    if (v2 < lo) lo = v2;
    if (v3 < lo) lo = v3;
    if (hi < v1) hi = v1;
    if (hi < v2) hi = v2;
    if (hi < v3) hi = v3;
    return widened(lo, hi);
}

// multiply_interval(a, point_interval(p)).  With a point operand the four
// products are two, each computed twice, and the first-minimum / first-maximum
// scan picks the same values from the pair, so the result is identical.
SPK_HD Interval multiply_by_point(const Interval& a, double p)
{
    if (!a.valid || !f_finite(p)) {
        return { 0, 0, false };
    }
    const double v0 = f_mul(a.low, p), v2 = f_mul(a.high, p);
    if (!f_finite(v0) || !f_finite(v2)) {
        return { 0, 0, false };
    }
    double lo = v0, hi = v0;
    if (v2 < lo) lo = v2;
    if (hi < v2) hi = v2;
    return widened(lo, hi);
}

// transformed_interval (validation_kernel.cpp:805-943): row `row` of the
// rotation intervals applied to a point, plus the translation, as intervals.
// Host and device run this same code.
SPK_HD Interval transformed_interval_at(const double* point, const double* translation, const Interval (*rotation)[3],
                                        int row)
{
    Interval value = point_interval(translation[row]);
    for (int column = 0; column < 3; ++column) {
        value = add_interval(value, multiply_by_point(rotation[row][column], point[column]));
    }
    return value;
}

SPK_HD Interval divide_interval(Interval n, Interval d)
{
    if (!n.valid || !d.valid || d.low <= 0.0) {
        return { 0, 0, false };
    }
    const Interval reciprocal = widened(f_div(1.0, d.high), f_div(1.0, d.low));
    return multiply_interval(n, reciprocal);
}

struct IVec3 {
    Interval v[3];
};

SPK_HD IVec3 ivec_sub(const IVec3& a, const IVec3& b)
{
    return { { subtract_interval(a.v[0], b.v[0]), subtract_interval(a.v[1], b.v[1]),
               subtract_interval(a.v[2], b.v[2]) } };
}

SPK_HD IVec3 ivec_cross(const IVec3& a, const IVec3& b)
{
    return { { subtract_interval(multiply_interval(a.v[1], b.v[2]), multiply_interval(a.v[2], b.v[1])),
               subtract_interval(multiply_interval(a.v[2], b.v[0]), multiply_interval(a.v[0], b.v[2])),
               subtract_interval(multiply_interval(a.v[0], b.v[1]), multiply_interval(a.v[1], b.v[0])) } };
}

SPK_HD Interval ivec_dot(const IVec3& a, const IVec3& b)
{
    Interval r = point_interval(0.0);
    for (int i = 0; i < 3; ++i) {
        r = add_interval(r, multiply_interval(a.v[i], b.v[i]));
    }
    return r;
}

SPK_HD bool projection_separates(const IVec3* tri, const IVec3& box, const IVec3& axis)
{
    Interval tp = ivec_dot(tri[0], axis);
#pragma unroll
    for (int k = 1; k < 3; ++k) {
        const Interval p = ivec_dot(tri[k], axis);
        if (!p.valid) {
            return false;
        }
        tp.low = f_min(tp.low, p.low);
        tp.high = f_max(tp.high, p.high);
    }
    const Interval bp = ivec_dot(box, axis);
    return tp.valid && bp.valid && (tp.high < bp.low || bp.high < tp.low);
}

// 13-axis separating-axis test of a triangle (vertex intervals) and a box.
SPK_HD bool triangle_box_disjoint(const IVec3* tri, const IVec3& box)
{
    // The axis loops are unrolled so that their array indices are constants
    // and the intervals stay in registers; the operations and their order are
    // as written.
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        double lo = tri[0].v[a].low, hi = tri[0].v[a].high;
#pragma unroll
        for (int k = 1; k < 3; ++k) {
            lo = f_min(lo, tri[k].v[a].low);
            hi = f_max(hi, tri[k].v[a].high);
        }
        if (hi < box.v[a].low || box.v[a].high < lo) {
            return true;
        }
    }
    const IVec3 first = ivec_sub(tri[1], tri[0]);
    const IVec3 second = ivec_sub(tri[2], tri[0]);
    if (projection_separates(tri, box, ivec_cross(first, second))) {
        return true;
    }
    const IVec3 edges[3] = { first, second, ivec_sub(tri[2], tri[1]) };
    // The edge loop stays rolled: nine unrolled axis tests made the raster
    // wait on instruction fetch (measured faster rolled, at six blocks per SM).
#pragma unroll 1
    for (int e = 0; e < 3; ++e) {
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            IVec3 axis = { { point_interval(0.0), point_interval(0.0), point_interval(0.0) } };
            axis.v[a] = point_interval(1.0);
            if (projection_separates(tri, box, ivec_cross(edges[e], axis))) {
                return true;
            }
        }
    }
    return false;
}

// The parts of triangle_box_disjoint that depend on the triangle alone, for
// rasterising one triangle against many cells: the triangle's bounds on the
// three box axes, the ten remaining axes (normal, then edge e x unit axis a
// for e, a = 0..2, the test order) and the triangle's projection on each.
// face_sat_disjoint(f, box) with f from face_sat(tri, f) returns exactly
// triangle_box_disjoint(tri, box): every value is the same expression
// computed once instead of once per cell.
struct FaceSat {
    double lo[3], hi[3];
    IVec3 axis[10];
    double tp_low[10], tp_high[10];
    unsigned char usable[10];  // axis i can separate (all three vertex projections valid)
};

// FaceSat's box-axis bounds.
SPK_HD void face_sat_bounds(const IVec3* tri, FaceSat& f)
{
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        double lo = tri[0].v[a].low, hi = tri[0].v[a].high;
#pragma unroll
        for (int k = 1; k < 3; ++k) {
            lo = f_min(lo, tri[k].v[a].low);
            hi = f_max(hi, tri[k].v[a].high);
        }
        f.lo[a] = lo;
        f.hi[a] = hi;
    }
}

// FaceSat's axis i (0: the normal first x second; 1 + 3 e + a: edge e x
// unit axis a, with edges first = v1 - v0, second = v2 - v0, v2 - v1) and the
// triangle's projection on it.  Each axis is independent of the others, so a
// device launch gives each its own thread.
SPK_HD void face_sat_axis(const IVec3* tri, int i, FaceSat& f)
{
    IVec3 axis;
    if (i == 0) {
        axis = ivec_cross(ivec_sub(tri[1], tri[0]), ivec_sub(tri[2], tri[0]));
    }
    else {
        const int e = (i - 1) / 3, a = (i - 1) % 3;
        const IVec3 edge = e == 0 ? ivec_sub(tri[1], tri[0]) : e == 1 ? ivec_sub(tri[2], tri[0])
                                                                       : ivec_sub(tri[2], tri[1]);
        IVec3 unit = { { point_interval(0.0), point_interval(0.0), point_interval(0.0) } };
        unit.v[a] = point_interval(1.0);
        axis = ivec_cross(edge, unit);
    }
    f.axis[i] = axis;
    // projection_separates' triangle side: false whenever a vertex
    // projection is invalid, whatever the box.
    Interval tp = ivec_dot(tri[0], axis);
    bool usable = tp.valid;
    for (int k = 1; k < 3 && usable; ++k) {
        const Interval p = ivec_dot(tri[k], axis);
        if (!p.valid) {
            usable = false;
            break;
        }
        tp.low = f_min(tp.low, p.low);
        tp.high = f_max(tp.high, p.high);
    }
    f.tp_low[i] = tp.low;
    f.tp_high[i] = tp.high;
    f.usable[i] = usable ? 1 : 0;
}

SPK_HD void face_sat(const IVec3* tri, FaceSat& f)
{
    face_sat_bounds(tri, f);
    for (int i = 0; i < 10; ++i) {
        face_sat_axis(tri, i, f);
    }
}

SPK_HD bool face_sat_disjoint(const FaceSat& f, const IVec3& box)
{
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        if (f.hi[a] < box.v[a].low || box.v[a].high < f.lo[a]) {
            return true;
        }
    }
#pragma unroll 1
    for (int i = 0; i < 10; ++i) {
        if (!f.usable[i]) {
            continue;
        }
        const Interval bp = ivec_dot(box, f.axis[i]);
        if (bp.valid && (f.tp_high[i] < bp.low || bp.high < f.tp_low[i])) {
            return true;
        }
    }
    return false;
}

// Outward enclosure of the closed cell `index` on the lattice; false when an
// index is not exactly representable (|index| >= 2^53) or arithmetic overflows.
SPK_HD bool grid_cell_interval(const double* origin, double pitch, const std::int64_t* index, IVec3& out)
{
    const std::int64_t limit = std::int64_t { 1 } << 53;
    for (int a = 0; a < 3; ++a) {
        if (index[a] < -limit || index[a] >= limit) {
            return false;
        }
        const Interval low = add_interval(point_interval(origin[a]),
                                          multiply_interval(point_interval(pitch),
                                                            point_interval(static_cast<double>(index[a]))));
        const Interval high = add_interval(point_interval(origin[a]),
                                           multiply_interval(point_interval(pitch),
                                                             point_interval(static_cast<double>(index[a] + 1))));
        if (!low.valid || !high.valid) {
            return false;
        }
        out.v[a] = { f_min(low.low, high.low), f_max(low.high, high.high), true };
    }
    return true;
}

}  // namespace spk
