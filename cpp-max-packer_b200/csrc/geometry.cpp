// Host geometry for the conservative fields (see geometry.hpp for the
// reference function each part restates).  Compiled with -ffp-contract=off so
// every binary64 operation rounds exactly as in the reference build.
#include "geometry.hpp"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <exception>
#include <limits>
#include <mutex>
#include <thread>
#include <vector>

#include "exact.hpp"

namespace spk::geo {

namespace {

constexpr std::int64_t kExactIndex = std::int64_t { 1 } << 53;

bool finite3(const Vec3& v) { return std::isfinite(v[0]) && std::isfinite(v[1]) && std::isfinite(v[2]); }

double midpoint(double a, double b)
{
    // std::midpoint for binary64 (C++20): (a + b) / 2 in the normal range.
    constexpr double lo = std::numeric_limits<double>::min() * 2;
    constexpr double hi = std::numeric_limits<double>::max() / 2;
    const double abs_a = a < 0 ? -a : a;
    const double abs_b = b < 0 ? -b : b;
    if (abs_a <= hi && abs_b <= hi) {
        return (a + b) / 2;
    }
    if (abs_a < lo) {
        return a + b / 2;
    }
    if (abs_b < lo) {
        return a / 2 + b;
    }
    return a / 2 + b / 2;
}

// Exact comparison of a.translation + a.sign*a.local with b (compare_coordinates, :260-273).
exact::Sign compare_coordinates(const AxisCoordinate& a, const AxisCoordinate& b)
{
    const double terms[4] = { a.translation, a.sign * a.local, -b.translation, -(b.sign * b.local) };
    return exact::sum_sign(terms, 4);
}

bool cardinal_rotation(const Quat& quaternion, int* source_axis, int* sign)
{
    double magnitude = 0;
    int nonzero = 0;
    int q[4] = { 0, 0, 0, 0 };
    for (int i = 0; i < 4; ++i) {
        if (quaternion[i] == 0.0) {
            continue;
        }
        const double current = std::fabs(quaternion[i]);
        if (nonzero == 0) {
            magnitude = current;
        }
        else if (std::memcmp(&current, &magnitude, 8) != 0) {
            return false;
        }
        q[i] = std::signbit(quaternion[i]) ? -1 : 1;
        ++nonzero;
    }
    if (nonzero != 1 && nonzero != 2 && nonzero != 4) {
        return false;
    }
    const int x = q[0], y = q[1], z = q[2], w = q[3];
    const int d = nonzero;
    const int h[3][3] = { { w * w + x * x - y * y - z * z, 2 * (x * y - z * w), 2 * (x * z + y * w) },
                          { 2 * (x * y + z * w), w * w - x * x + y * y - z * z, 2 * (y * z - x * w) },
                          { 2 * (x * z - y * w), 2 * (y * z + x * w), w * w - x * x - y * y + z * z } };
    bool used[3] = { false, false, false };
    for (int row = 0; row < 3; ++row) {
        int found = -1;
        for (int column = 0; column < 3; ++column) {
            if (h[row][column] == d || h[row][column] == -d) {
                if (found != -1) {
                    return false;
                }
                found = column;
                sign[row] = h[row][column] / d;
            }
            else if (h[row][column] != 0) {
                return false;
            }
        }
        if (found < 0 || used[found]) {
            return false;
        }
        used[found] = true;
        source_axis[row] = found;
    }
    return true;
}

Interval transformed_interval(const Vec3& point, const Vec3& translation, const Interval rotation[3][3], int row)
{
    return transformed_interval_at(point.data(), translation.data(), rotation, row);
}

bool finite_pose_in(const Vec3& translation, const Quat& q)
{
    return finite3(translation) && std::isfinite(q[0]) && std::isfinite(q[1]) && std::isfinite(q[2]) &&
           std::isfinite(q[3]) && (q[0] != 0.0 || q[1] != 0.0 || q[2] != 0.0 || q[3] != 0.0);
}

// exact_predicates.cpp segment_triangle_crossing (:1056-1111) and helpers (:238-298).
enum class Crossing { none, crossing, boundary, degenerate };

exact::Point2 project(const Vec3& p, int dropped)
{
    if (dropped == 0) {
        return { p[1], p[2] };
    }
    if (dropped == 1) {
        return { p[0], p[2] };
    }
    return { p[0], p[1] };
}

int projection_for(const std::array<Vec3, 3>& tri)
{
    for (int dropped = 0; dropped < 3; ++dropped) {
        if (exact::orient2d(project(tri[0], dropped), project(tri[1], dropped), project(tri[2], dropped)) !=
            exact::Sign::zero) {
            return dropped;
        }
    }
    return -1;
}

bool point_on_segment(const exact::Point2& p, const exact::Point2& a, const exact::Point2& b)
{
    if (exact::orient2d(a, b, p) != exact::Sign::zero) {
        return false;
    }
    return p[0] >= std::min(a[0], b[0]) && p[0] <= std::max(a[0], b[0]) && p[1] >= std::min(a[1], b[1]) &&
           p[1] <= std::max(a[1], b[1]);
}

bool segments_intersect(const exact::Point2& a, const exact::Point2& b, const exact::Point2& c,
                        const exact::Point2& d)
{
    using exact::Sign;
    const Sign ab_c = exact::orient2d(a, b, c), ab_d = exact::orient2d(a, b, d);
    const Sign cd_a = exact::orient2d(c, d, a), cd_b = exact::orient2d(c, d, b);
    if (ab_c != Sign::zero && ab_d != Sign::zero && ab_c != ab_d && cd_a != Sign::zero && cd_b != Sign::zero &&
        cd_a != cd_b) {
        return true;
    }
    return (ab_c == Sign::zero && point_on_segment(c, a, b)) || (ab_d == Sign::zero && point_on_segment(d, a, b)) ||
           (cd_a == Sign::zero && point_on_segment(a, c, d)) || (cd_b == Sign::zero && point_on_segment(b, c, d));
}

bool point_in_triangle(const exact::Point2& p, const std::array<exact::Point2, 3>& t)
{
    using exact::Sign;
    const Sign s0 = exact::orient2d(t[0], t[1], p), s1 = exact::orient2d(t[1], t[2], p),
               s2 = exact::orient2d(t[2], t[0], p);
    const auto nonneg = [](Sign s) { return s != Sign::negative; };
    const auto nonpos = [](Sign s) { return s != Sign::positive; };
    return (nonneg(s0) && nonneg(s1) && nonneg(s2)) || (nonpos(s0) && nonpos(s1) && nonpos(s2));
}

Crossing segment_triangle_crossing(const Vec3& first, const Vec3& second, const std::array<Vec3, 3>& tri)
{
    using exact::Sign;
    const Sign first_side = exact::orient3d(tri[0], tri[1], tri[2], first);
    const Sign second_side = exact::orient3d(tri[0], tri[1], tri[2], second);
    if (first_side == Sign::zero && second_side == Sign::zero) {
        const int dropped = projection_for(tri);
        if (dropped < 0) {
            return Crossing::degenerate;  // the reference reports uncertain: both retry
        }
        const std::array<exact::Point2, 3> p { project(tri[0], dropped), project(tri[1], dropped),
                                               project(tri[2], dropped) };
        const exact::Point2 a = project(first, dropped), b = project(second, dropped);
        if (point_in_triangle(a, p) || point_in_triangle(b, p)) {
            return Crossing::degenerate;
        }
        for (int e = 0; e < 3; ++e) {
            if (segments_intersect(a, b, p[e], p[(e + 1) % 3])) {
                return Crossing::degenerate;
            }
        }
        return Crossing::none;
    }
    if (first_side == Sign::zero) {
        const int dropped = projection_for(tri);
        if (dropped < 0) {
            return Crossing::degenerate;
        }
        const std::array<exact::Point2, 3> p { project(tri[0], dropped), project(tri[1], dropped),
                                               project(tri[2], dropped) };
        return point_in_triangle(project(first, dropped), p) ? Crossing::boundary : Crossing::none;
    }
    if (second_side == Sign::zero) {
        return Crossing::degenerate;
    }
    if (first_side == second_side) {
        return Crossing::none;
    }
    const Sign e0 = exact::orient3d(first, second, tri[0], tri[1]);
    const Sign e1 = exact::orient3d(first, second, tri[1], tri[2]);
    const Sign e2 = exact::orient3d(first, second, tri[2], tri[0]);
    if (e0 == Sign::zero || e1 == Sign::zero || e2 == Sign::zero) {
        return Crossing::degenerate;
    }
    const bool same = (e0 == Sign::positive && e1 == Sign::positive && e2 == Sign::positive) ||
                      (e0 == Sign::negative && e1 == Sign::negative && e2 == Sign::negative);
    return same ? Crossing::crossing : Crossing::none;
}

constexpr double kSlopes[12][2] = { { 0.137, 0.271 }, { 0.223, 0.419 }, { 0.347, 0.163 }, { 0.431, 0.593 },
                                    { 0.557, 0.317 }, { 0.619, 0.733 }, { 0.709, 0.467 }, { 0.823, 0.197 },
                                    { 0.911, 0.541 }, { 0.293, 0.887 }, { 0.487, 0.773 }, { 0.677, 0.929 } };

// Ray parity against a triangle list; `prefilter` skips triangles whose
// bounding box is strictly disjoint from the segment's (local variant only).
// `bounds`, when given, holds each triangle's coordinate bounds: the values
// the prefilter would otherwise recompute per ray.
Decision ray_parity(const Vec3& point, const Bounds& reach, const std::vector<std::array<Vec3, 3>>& triangles,
                    bool prefilter, const std::vector<Bounds>* bounds = nullptr)
{
    const double span = std::max({ reach.max[0] - reach.min[0], reach.max[1] - reach.min[1],
                                   reach.max[2] - reach.min[2], 1.0 });
    for (const auto& slope : kSlopes) {
        const Vec3 endpoint { std::max(point[0], reach.max[0]) + 2 * span + 1, point[1] + slope[0] * span,
                              point[2] + slope[1] * span };
        std::uint64_t crossings = 0;
        bool retry = false;
        for (std::size_t i = 0; i < triangles.size(); ++i) {
            const auto& tri = triangles[i];
            if (prefilter) {
                bool disjoint = false;
                for (int a = 0; a < 3; ++a) {
                    const double low = bounds ? (*bounds)[i].min[a] : std::min({ tri[0][a], tri[1][a], tri[2][a] });
                    const double high = bounds ? (*bounds)[i].max[a] : std::max({ tri[0][a], tri[1][a], tri[2][a] });
                    disjoint = disjoint || std::max(point[a], endpoint[a]) < low ||
                               std::min(point[a], endpoint[a]) > high;
                }
                if (disjoint) {
                    continue;
                }
            }
            const Crossing relation = segment_triangle_crossing(point, endpoint, tri);
            if (relation == Crossing::crossing) {
                ++crossings;
            }
            else if (relation != Crossing::none) {
                retry = true;
                break;
            }
        }
        if (!retry) {
            return crossings % 2 == 0 ? Decision::no : Decision::yes;
        }
    }
    return Decision::indeterminate;
}

Decision point_in_material(const Vec3& point, const Placed& target)
{
    if (target.prepared->is_cuboid && target.is_cardinal) {
        bool strict_inside = true;
        for (int a = 0; a < 3; ++a) {
            const AxisCoordinate represented { 0.0, point[a], 1 };
            const auto above_low = compare_coordinates(represented, target.cuboid_min[a]);
            const auto below_high = compare_coordinates(represented, target.cuboid_max[a]);
            if (above_low == exact::Sign::negative || below_high == exact::Sign::positive) {
                return Decision::no;
            }
            strict_inside = strict_inside && above_low == exact::Sign::positive && below_high == exact::Sign::negative;
        }
        return strict_inside ? Decision::yes : Decision::indeterminate;
    }
    if (!target.world_exact) {
        return Decision::indeterminate;
    }
    const auto& mesh = *target.prepared->mesh;
    std::vector<std::array<Vec3, 3>> triangles(mesh.triangles.size());
    for (std::size_t i = 0; i < mesh.triangles.size(); ++i) {
        for (int k = 0; k < 3; ++k) {
            triangles[i][k] = target.world[mesh.triangles[i][k]];
        }
    }
    return ray_parity(point, target.conservative, triangles, false);
}

Decision local_interval_point_in_material(const Placed& solid, const Bounds& wi)
{
    for (int a = 0; a < 3; ++a) {
        if (wi.max[a] < solid.conservative.min[a] || wi.min[a] > solid.conservative.max[a]) {
            return Decision::no;
        }
    }
    Interval shifted[3];
    for (int a = 0; a < 3; ++a) {
        shifted[a] = subtract_interval({ wi.min[a], wi.max[a], true }, point_interval(solid.translation[a]));
    }
    Interval rotation[3][3];
    rotation_intervals(solid.q, rotation);
    IVec3 local;
    for (int la = 0; la < 3; ++la) {
        local.v[la] = point_interval(0.0);
        for (int wa = 0; wa < 3; ++wa) {
            local.v[la] = add_interval(local.v[la], multiply_interval(rotation[wa][la], shifted[wa]));
        }
        if (!local.v[la].valid) {
            return Decision::indeterminate;
        }
    }
    const auto& mesh = *solid.prepared->mesh;
    const auto& triangles = solid.prepared->triangles;
    const auto& bounds = solid.prepared->triangle_bounds;
    for (std::size_t i = 0; i < triangles.size(); ++i) {
        // The first three axes of triangle_box_disjoint, from the kept bounds:
        // a triangle they separate is disjoint, and the full test is skipped.
        bool separated = false;
        for (int a = 0; a < 3; ++a) {
            separated = separated || bounds[i].max[a] < local.v[a].low || local.v[a].high < bounds[i].min[a];
        }
        if (separated) {
            continue;
        }
        IVec3 tri[3];
        for (int k = 0; k < 3; ++k) {
            const Vec3& v = triangles[i][k];
            tri[k] = { { point_interval(v[0]), point_interval(v[1]), point_interval(v[2]) } };
        }
        if (!triangle_box_disjoint(tri, local)) {
            return Decision::indeterminate;
        }
    }
    Vec3 witness;
    for (int a = 0; a < 3; ++a) {
        witness[a] = midpoint(local.v[a].low, local.v[a].high);
        if (!std::isfinite(witness[a])) {
            return Decision::indeterminate;
        }
    }
    return ray_parity(witness, mesh.bounds, triangles, true, &bounds);
}

}  // namespace

bool finite_pose(const Vec3& translation, const Quat& q) { return finite_pose_in(translation, q); }

Prepared prepare(const Mesh& mesh)
{
    Prepared p;
    p.mesh = &mesh;
    p.triangles.resize(mesh.triangles.size());
    p.triangle_bounds.resize(mesh.triangles.size());
    for (std::size_t i = 0; i < mesh.triangles.size(); ++i) {
        auto& tri = p.triangles[i];
        for (int k = 0; k < 3; ++k) {
            tri[k] = mesh.vertices[mesh.triangles[i][k]];
        }
        for (int a = 0; a < 3; ++a) {
            p.triangle_bounds[i].min[a] = std::min({ tri[0][a], tri[1][a], tri[2][a] });
            p.triangle_bounds[i].max[a] = std::max({ tri[0][a], tri[1][a], tri[2][a] });
        }
    }
    // certify_cuboid (:384-447)
    const auto& vs = mesh.vertices;
    if (vs.size() != 8 || mesh.triangles.size() != 12) {
        return p;
    }
    Bounds b { vs.front(), vs.front() };
    for (const auto& v : vs) {
        for (int a = 0; a < 3; ++a) {
            if (!std::isfinite(v[a])) {
                return p;
            }
            b.min[a] = std::min(b.min[a], v[a]);
            b.max[a] = std::max(b.max[a], v[a]);
        }
    }
    for (int a = 0; a < 3; ++a) {
        if (!(b.min[a] < b.max[a])) {
            return p;
        }
    }
    bool corners[8] = {};
    for (const auto& v : vs) {
        unsigned mask = 0;
        for (int a = 0; a < 3; ++a) {
            if (v[a] == b.max[a]) {
                mask |= 1U << a;
            }
            else if (v[a] != b.min[a]) {
                return p;
            }
        }
        if (corners[mask]) {
            return p;
        }
        corners[mask] = true;
    }
    struct FaceMasks {
        unsigned values[2] {};
        int size {};
    } faces[6];
    for (const auto& t : mesh.triangles) {
        bool assigned = false;
        for (int axis = 0; axis < 3 && !assigned; ++axis) {
            for (int side = 0; side < 2; ++side) {
                const double plane = side == 0 ? b.min[axis] : b.max[axis];
                if (vs[t[0]][axis] == plane && vs[t[1]][axis] == plane && vs[t[2]][axis] == plane) {
                    unsigned mask = 0;
                    for (const auto index : t) {
                        const auto& v = vs[index];
                        const int aa = (axis + 1) % 3, bb = (axis + 2) % 3;
                        const unsigned corner = (v[aa] == b.max[aa] ? 1U : 0U) | (v[bb] == b.max[bb] ? 2U : 0U);
                        mask |= 1U << corner;
                    }
                    auto& f = faces[axis * 2 + side];
                    if (f.size == 2) {
                        return p;
                    }
                    f.values[f.size++] = mask;
                    assigned = true;
                    break;
                }
            }
        }
        if (!assigned) {
            return p;
        }
    }
    for (const auto& f : faces) {
        if (f.size != 2 || (f.values[0] | f.values[1]) != 0xFU || __builtin_popcount(f.values[0] & f.values[1]) != 2) {
            return p;
        }
    }
    p.is_cuboid = true;
    p.cuboid = b;
    return p;
}

std::optional<RotationTransform> rotation_transform(Quat q)
{
    double scale = 0;
    for (const double c : q) {
        if (!std::isfinite(c)) {
            return std::nullopt;
        }
        scale = std::max(scale, std::fabs(c));
    }
    if (!(scale > 0.0)) {
        return std::nullopt;
    }
    RotationTransform r;
    if (cardinal_rotation(q, r.source_axis, r.sign)) {
        r.exact_cardinal = true;
        for (int row = 0; row < 3; ++row) {
            r.matrix[row][r.source_axis[row]] = r.sign[row];
        }
        return r;
    }
    for (double& c : q) {
        c /= scale;
    }
    const double x = q[0], y = q[1], z = q[2], w = q[3];
    const double den = x * x + y * y + z * z + w * w;
    if (!(den > 0.0) || !std::isfinite(den)) {
        return std::nullopt;
    }
    const double m[3][3] = { { (w * w + x * x - y * y - z * z) / den, 2.0 * (x * y - z * w) / den,
                               2.0 * (x * z + y * w) / den },
                             { 2.0 * (x * y + z * w) / den, (w * w - x * x + y * y - z * z) / den,
                               2.0 * (y * z - x * w) / den },
                             { 2.0 * (x * z - y * w) / den, 2.0 * (y * z + x * w) / den,
                               (w * w - x * x - y * y + z * z) / den } };
    for (int i = 0; i < 3; ++i) {
        for (int j = 0; j < 3; ++j) {
            if (!std::isfinite(m[i][j])) {
                return std::nullopt;
            }
            r.matrix[i][j] = m[i][j];
        }
    }
    return r;
}

void rotation_intervals(const Quat& q, Interval h[3][3])
{
    Interval v[4];
    for (int i = 0; i < 4; ++i) {
        v[i] = point_interval(q[i]);
    }
    const auto sq = [&](int i) { return multiply_interval(v[i], v[i]); };
    const auto twice = [](Interval value) { return multiply_interval(point_interval(2.0), value); };
    const Interval d = add_interval(add_interval(sq(0), sq(1)), add_interval(sq(2), sq(3)));
    h[0][0] = subtract_interval(add_interval(sq(3), sq(0)), add_interval(sq(1), sq(2)));
    h[0][1] = twice(subtract_interval(multiply_interval(v[0], v[1]), multiply_interval(v[2], v[3])));
    h[0][2] = twice(add_interval(multiply_interval(v[0], v[2]), multiply_interval(v[1], v[3])));
    h[1][0] = twice(add_interval(multiply_interval(v[0], v[1]), multiply_interval(v[2], v[3])));
    h[1][1] = subtract_interval(add_interval(sq(3), sq(1)), add_interval(sq(0), sq(2)));
    h[1][2] = twice(subtract_interval(multiply_interval(v[1], v[2]), multiply_interval(v[0], v[3])));
    h[2][0] = twice(subtract_interval(multiply_interval(v[0], v[2]), multiply_interval(v[1], v[3])));
    h[2][1] = twice(add_interval(multiply_interval(v[1], v[2]), multiply_interval(v[0], v[3])));
    h[2][2] = subtract_interval(add_interval(sq(3), sq(2)), add_interval(sq(0), sq(1)));
    for (int i = 0; i < 3; ++i) {
        for (int j = 0; j < 3; ++j) {
            h[i][j] = divide_interval(h[i][j], d);
        }
    }
}

namespace {

// One chunk of place()'s general branch: its vertices' world points and
// intervals, whether all intervals are valid and all cardinal world points
// exact, and the bounds of its intervals.
struct VertexChunk {
    bool valid { true };
    bool world_exact { true };
    bool any { false };
    Bounds conservative {};
};

VertexChunk place_vertices(const Mesh& mesh, const Vec3& translation, const RotationTransform& transform,
                           const Interval rotation[3][3], Placed& out, std::size_t begin, std::size_t end)
{
    VertexChunk c;
    for (std::size_t i = begin; i < end; ++i) {
        for (int a = 0; a < 3; ++a) {
            double w = translation[a];
            for (int s = 0; s < 3; ++s) {
                w += transform.matrix[a][s] * mesh.vertices[i][s];
            }
            out.world[i][a] = w;
            const Interval iv = transformed_interval(mesh.vertices[i], translation, rotation, a);
            out.intervals[i].v[a] = iv;
            if (!iv.valid) {
                c.valid = false;
                return c;
            }
            if (out.is_cardinal) {
                const int source = out.source_axis[a];
                const double ta = translation[a];
                const double b = out.sign[a] * mesh.vertices[i][source];
                const double sum = ta + b;
                out.world[i][a] = sum;
                c.world_exact = c.world_exact && compare_coordinates({ ta, mesh.vertices[i][source], out.sign[a] },
                                                                     { 0.0, sum, 1 }) == exact::Sign::zero;
            }
            if (!c.any) {
                c.conservative.min[a] = iv.low;
                c.conservative.max[a] = iv.high;
            }
            else {
                c.conservative.min[a] = std::min(c.conservative.min[a], iv.low);
                c.conservative.max[a] = std::max(c.conservative.max[a], iv.high);
            }
        }
        c.any = true;
    }
    return c;
}

// Chunks for n independent items: one below 2048, else up to four of at
// least 1024.
std::size_t chunk_count(std::size_t n)
{
    if (n < 2048) {
        return 1;
    }
    const std::size_t cores = std::max(1U, std::thread::hardware_concurrency());
    return std::min({ std::size_t { 4 }, cores, n / 1024 });
}

// Runs body(p, begin, end) on the `parts` contiguous chunks of [0, n): chunk 0
// on the calling thread, each other one on a thread of its own, or on the
// calling thread when no thread can be had.  Returns after every chunk is
// done, rethrowing the first exception a chunk raised.
template <class Body>
void run_chunks(std::size_t n, std::size_t parts, const Body& body)
{
    std::exception_ptr failure;
    std::mutex failure_lock;
    const auto run = [&](std::size_t p) noexcept {
        try {
            body(p, n * p / parts, n * (p + 1) / parts);
        }
        catch (...) {
            const std::lock_guard<std::mutex> hold(failure_lock);
            if (!failure) {
                failure = std::current_exception();
            }
        }
    };
    {
        std::vector<std::thread> workers;
        struct JoinAll {
            std::vector<std::thread>& threads;
            ~JoinAll()
            {
                for (auto& t : threads) {
                    if (t.joinable()) {
                        t.join();
                    }
                }
            }
        } join { workers };
        for (std::size_t p = 1; p < parts; ++p) {
            try {
                workers.emplace_back(run, p);
            }
            catch (...) {
                run(p);
            }
        }
        run(0);
    }
    if (failure) {
        std::rethrow_exception(failure);
    }
}

}  // namespace

bool place(const Prepared& prepared, const Vec3& translation, const Quat& q, Placed& out)
{
    if (!finite_pose_in(translation, q)) {
        return false;
    }
    const auto transform = rotation_transform(q);
    if (!transform) {
        return false;
    }
    out = Placed {};
    out.prepared = &prepared;
    out.translation = translation;
    out.q = q;
    out.is_cardinal = transform->exact_cardinal;
    for (int a = 0; a < 3; ++a) {
        out.source_axis[a] = transform->source_axis[a];
        out.sign[a] = transform->sign[a];
    }
    const auto& mesh = *prepared.mesh;
    const std::size_t nv = mesh.vertices.size();
    out.world.resize(nv);
    out.intervals.resize(nv);
    if (prepared.is_cuboid && out.is_cardinal) {
        for (int world = 0; world < 3; ++world) {
            const int local = out.source_axis[world];
            const int sign = out.sign[world];
            const double lo = sign > 0 ? prepared.cuboid.min[local] : prepared.cuboid.max[local];
            const double hi = sign > 0 ? prepared.cuboid.max[local] : prepared.cuboid.min[local];
            out.cuboid_min[world] = { translation[world], lo, sign };
            out.cuboid_max[world] = { translation[world], hi, sign };
            const double rounded_lo = translation[world] + sign * lo;
            const double rounded_hi = translation[world] + sign * hi;
            out.conservative.min[world] = std::nextafter(rounded_lo, -std::numeric_limits<double>::infinity());
            out.conservative.max[world] = std::nextafter(rounded_hi, std::numeric_limits<double>::infinity());
        }
        out.finite = finite3(out.conservative.min) && finite3(out.conservative.max);
        out.world_exact = true;
        for (std::size_t i = 0; i < nv; ++i) {
            for (int a = 0; a < 3; ++a) {
                const int source = out.source_axis[a];
                const double ta = translation[a];
                const double b = out.sign[a] * mesh.vertices[i][source];
                const double sum = ta + b;
                out.world[i][a] = sum;
                out.world_exact = out.world_exact && compare_coordinates({ ta, mesh.vertices[i][source], out.sign[a] },
                                                                         { 0.0, sum, 1 }) == exact::Sign::zero;
                out.intervals[i].v[a] = widened(sum, sum);
            }
        }
        return true;
    }
    Interval rotation[3][3];
    rotation_intervals(q, rotation);
    // Vertices are independent: contiguous chunks run on up to four host
    // threads, and their bounds combine in vertex order.  std::min / std::max
    // keep the earlier of equal values, so the combined bounds are the ones a
    // single pass over all vertices gives.
    const std::size_t parts = chunk_count(nv);
    std::vector<VertexChunk> chunks(parts);
    run_chunks(nv, parts, [&](std::size_t p, std::size_t begin, std::size_t end) {
        chunks[p] = place_vertices(mesh, translation, *transform, rotation, out, begin, end);
    });
    out.world_exact = out.is_cardinal;
    bool first = true;
    for (const auto& c : chunks) {
        if (!c.valid) {
            return false;
        }
        out.world_exact = out.world_exact && c.world_exact;
        if (!c.any) {
            continue;
        }
        for (int a = 0; a < 3; ++a) {
            if (first) {
                out.conservative.min[a] = c.conservative.min[a];
                out.conservative.max[a] = c.conservative.max[a];
            }
            else {
                out.conservative.min[a] = std::min(out.conservative.min[a], c.conservative.min[a]);
                out.conservative.max[a] = std::max(out.conservative.max[a], c.conservative.max[a]);
            }
        }
        first = false;
    }
    out.finite = !first;
    return true;
}

bool trim_index(double bound, double origin, double pitch, bool lower, std::int64_t& out)
{
    const long double ratio = (static_cast<long double>(bound) - origin) / pitch;
    if (!std::isfinite(ratio) || ratio <= static_cast<long double>(-kExactIndex + 1) ||
        ratio >= static_cast<long double>(kExactIndex)) {
        return false;
    }
    auto index = static_cast<std::int64_t>(std::floor(ratio));
    out = lower ? index - 1 : index + 1;
    return true;
}

bool object_window(const Placed& placed, const double* origin, double pitch, Window& out)
{
    if (!placed.finite) {
        return false;
    }
    for (int a = 0; a < 3; ++a) {
        std::int64_t first, last;
        if (!trim_index(placed.conservative.min[a], origin[a], pitch, true, first) ||
            !trim_index(placed.conservative.max[a], origin[a], pitch, false, last) || last < first ||
            static_cast<std::uint64_t>(last - first) + 1 > UINT32_MAX) {
            return false;
        }
        out.first[a] = first;
        out.shape[a] = static_cast<std::uint32_t>(last - first + 1);
    }
    return true;
}

bool environment_window(const Bounds& container, const double* origin, double pitch, Window& out)
{
    for (int a = 0; a < 3; ++a) {
        const double low = (container.min[a] - origin[a]) / pitch;
        const double high = (container.max[a] - origin[a]) / pitch;
        if (!std::isfinite(low) || !std::isfinite(high)) {
            return false;
        }
        const double floored = std::floor(low);
        const double ceiled = std::ceil(high);
        if (!(floored > -0x1p63) || !(floored < 0x1p63) || ceiled < -0x1p63 || !(ceiled < 0x1p63)) {
            return false;
        }
        const auto first = static_cast<std::int64_t>(floored) - 1;
        const auto last = static_cast<std::int64_t>(ceiled);
        if (last < first) {
            return false;
        }
        const auto delta = static_cast<std::uint64_t>(last) - static_cast<std::uint64_t>(first);
        if (delta >= UINT32_MAX) {
            return false;
        }
        out.first[a] = first;
        out.shape[a] = static_cast<std::uint32_t>(delta + 1);
    }
    return true;
}

bool outward_grid_cell(const double* origin, double pitch, const std::int64_t* index, Bounds& out)
{
    IVec3 cell;
    if (!grid_cell_interval(origin, pitch, index, cell)) {
        return false;
    }
    for (int a = 0; a < 3; ++a) {
        out.min[a] = cell.v[a].low;
        out.max[a] = cell.v[a].high;
    }
    return true;
}

PlanKind plan_placed_window(const Placed& placed, const Window& whole, const double* origin, double pitch,
                            Window& out)
{
    out = whole;
    if (!placed.finite) {
        return PlanKind::full_window;
    }
    const auto& b = placed.conservative;
    std::int64_t whole_last[3], candidate_last[3];
    Window candidate = whole;
    bool empty = false;
    for (int a = 0; a < 3; ++a) {
        if (!whole.shape[a] || whole.first[a] < -kExactIndex ||
            whole.first[a] > kExactIndex - static_cast<std::int64_t>(whole.shape[a])) {
            return PlanKind::full_window;
        }
        whole_last[a] = whole.first[a] + whole.shape[a] - 1;
        std::int64_t first, last;
        if (!trim_index(b.min[a], origin[a], pitch, true, first) || !trim_index(b.max[a], origin[a], pitch, false, last) ||
            first > last) {
            return PlanKind::full_window;
        }
        candidate.first[a] = std::max(whole.first[a], first);
        candidate_last[a] = std::min(whole_last[a], last);
        empty |= candidate.first[a] > candidate_last[a];
    }
    Bounds first_cell, last_cell;
    if (!outward_grid_cell(origin, pitch, whole.first, first_cell) ||
        !outward_grid_cell(origin, pitch, whole_last, last_cell)) {
        return PlanKind::full_window;
    }
    if (empty) {
        for (int a = 0; a < 3; ++a) {
            if (last_cell.max[a] < b.min[a] || first_cell.min[a] > b.max[a]) {
                return PlanKind::certified_empty;
            }
        }
        return PlanKind::full_window;
    }
    for (int a = 0; a < 3; ++a) {
        candidate.shape[a] = static_cast<std::uint32_t>(candidate_last[a] - candidate.first[a] + 1);
        for (const bool lower : { true, false }) {
            if (lower ? candidate.first[a] == whole.first[a] : candidate_last[a] == whole_last[a]) {
                continue;
            }
            std::int64_t index[3] = { whole.first[0], whole.first[1], whole.first[2] };
            index[a] = lower ? candidate.first[a] - 1 : candidate_last[a] + 1;
            Bounds cell;
            if (!outward_grid_cell(origin, pitch, index, cell) ||
                !(lower ? cell.max[a] < b.min[a] : cell.min[a] > b.max[a])) {
                return PlanKind::full_window;
            }
        }
    }
    out = candidate;
    const bool same = candidate.first[0] == whole.first[0] && candidate.first[1] == whole.first[1] &&
                      candidate.first[2] == whole.first[2] && candidate.shape[0] == whole.shape[0] &&
                      candidate.shape[1] == whole.shape[1] && candidate.shape[2] == whole.shape[2];
    return same ? PlanKind::full_window : PlanKind::cropped_window;
}

namespace {

// floor((v - origin) / pitch) with the quotient in long double, as
// rasterize_boundary forms it (validation_kernel.cpp:3282-3330).  The binary64
// quotient is within 2^-52 of the exact one, relative, and the long double
// quotient within 2^-62.  When the binary64 quotient lies farther than 2^-48
// (relative) from every integer, all three have the same floor, so the long
// double division is needed only near integers and for huge or non-finite
// quotients.  `lower` selects the reference's range check for a lower or an
// upper bound; false when it fails.
bool quotient_floor(double v, double origin, double pitch, bool lower, std::int64_t& out)
{
    const double q = (v - origin) / pitch;
    if (std::isfinite(q) && std::fabs(q) < 0x1p50) {
        const double f = std::floor(q);
        const double margin = std::fabs(q) * 0x1p-48 + 0x1p-60;
        if (q - f > margin && (f + 1.0) - q > margin) {
            out = static_cast<std::int64_t>(f);
            return true;
        }
    }
    const long double ratio = (static_cast<long double>(v) - origin) / pitch;
    if (!std::isfinite(ratio) ||
        (lower ? ratio <= static_cast<long double>(std::numeric_limits<std::int64_t>::min() + 1)
               : ratio >= static_cast<long double>(std::numeric_limits<std::int64_t>::max()))) {
        return false;
    }
    out = static_cast<std::int64_t>(std::floor(ratio));
    return true;
}

}  // namespace

bool face_ranges(const Placed& placed, const Window& window, const double* origin, double pitch,
                 std::vector<FaceRange>& out)
{
    const auto& mesh = *placed.prepared->mesh;
    out.resize(mesh.triangles.size());
    std::int64_t window_last[3];
    for (int a = 0; a < 3; ++a) {
        window_last[a] = window.first[a] + static_cast<std::int64_t>(window.shape[a] - 1);
    }
    // Faces are independent: contiguous chunks on up to four host threads.
    const std::size_t faces = mesh.triangles.size();
    const std::size_t parts = chunk_count(faces);
    std::vector<char> ok(parts, 1);
    run_chunks(faces, parts, [&](std::size_t p, std::size_t begin, std::size_t end) {
        for (std::size_t f = begin; f < end; ++f) {
            const auto& face = mesh.triangles[f];
            auto& r = out[f];
            r.outside = 0;
            r.pad = 0;
            for (int a = 0; a < 3; ++a) {
                double low = placed.intervals[face[0]].v[a].low, high = placed.intervals[face[0]].v[a].high;
                for (int k = 1; k < 3; ++k) {
                    low = std::min(low, placed.intervals[face[k]].v[a].low);
                    high = std::max(high, placed.intervals[face[k]].v[a].high);
                }
                std::int64_t lo, hi;
                if (!quotient_floor(low, origin[a], pitch, true, lo) ||
                    !quotient_floor(high, origin[a], pitch, false, hi)) {
                    ok[p] = 0;
                    return;
                }
                r.first[a] = lo - 1;
                r.last[a] = hi + 1;
                if (r.last[a] < window.first[a] || r.first[a] > window_last[a]) {
                    r.outside = 1;
                }
                r.first[a] = std::max(r.first[a], window.first[a]);
                r.last[a] = std::min(r.last[a], window_last[a]);
            }
        }
    });
    return std::all_of(ok.begin(), ok.end(), [](char v) { return v != 0; });
}

Decision classify_material_witness(const Placed& solid, const Bounds& wi)
{
    if (!solid.finite) {
        return Decision::indeterminate;
    }
    for (int a = 0; a < 3; ++a) {
        if (!std::isfinite(wi.min[a]) || !std::isfinite(wi.max[a]) || wi.min[a] > wi.max[a] ||
            solid.conservative.min[a] > solid.conservative.max[a]) {
            return Decision::indeterminate;
        }
    }
    for (int a = 0; a < 3; ++a) {
        if (wi.max[a] < solid.conservative.min[a] || wi.min[a] > solid.conservative.max[a]) {
            return Decision::no;
        }
    }
    if (solid.world_exact) {
        Vec3 represented;
        for (int a = 0; a < 3; ++a) {
            represented[a] = midpoint(wi.min[a], wi.max[a]);
        }
        return point_in_material(represented, solid);
    }
    return local_interval_point_in_material(solid, wi);
}

bool analytic_box_axis_inside(double origin, double pitch, std::int64_t index, double dimension, double clearance,
                              const IVec3& cell, int axis)
{
    const Interval& c = cell.v[axis];
    if (c.low < clearance) {
        if (c.high < clearance) {
            return false;
        }
        // compare_grid_expression(origin, pitch, index, {clearance, -1}) (:2102-2142)
        double p, pe;
        exact::two_product(pitch, static_cast<double>(index), p, pe);
        const double terms[4] = { origin, p, pe, -clearance };
        if (exact::sum_sign(terms, 4) == exact::Sign::negative) {
            return false;
        }
    }
    const Interval permitted = subtract_interval(point_interval(dimension), point_interval(clearance));
    if (permitted.valid && c.high <= permitted.low) {
        return true;
    }
    if (permitted.valid && c.low > permitted.high) {
        return false;
    }
    double p, pe;
    exact::two_product(pitch, static_cast<double>(index + 1), p, pe);
    const double terms[5] = { origin, p, pe, -dimension, clearance };
    return exact::sum_sign(terms, 5) != exact::Sign::positive;
}

bool clearance_halo(double clearance, double pitch, std::uint64_t& halo)
{
    if (!std::isfinite(clearance) || clearance < 0.0) {
        return false;
    }
    if (clearance == 0.0) {
        halo = 0;
        return true;
    }
    const long double radius = std::ceil(static_cast<long double>(clearance) / pitch) + 1.0L;
    if (!std::isfinite(radius) || radius > std::numeric_limits<std::uint32_t>::max()) {
        return false;
    }
    halo = static_cast<std::uint64_t>(radius);
    return true;
}

std::vector<std::array<std::int64_t, 3>> make_stencil(std::uint64_t halo, double pitch, double clearance)
{
    std::vector<std::array<std::int64_t, 3>> stencil;
    const auto r = static_cast<std::int64_t>(halo);
    for (std::int64_t z = -r; z <= r; ++z) {
        for (std::int64_t y = -r; y <= r; ++y) {
            for (std::int64_t x = -r; x <= r; ++x) {
                const std::int64_t delta[3] = { x, y, z };
                std::uint64_t squared_sum = 0;
                for (const auto v : delta) {
                    const std::uint64_t magnitude = static_cast<std::uint64_t>(v < 0 ? -v : v);
                    const std::uint64_t gap = magnitude > 1 ? magnitude - 1 : 0;
                    squared_sum += gap * gap;
                }
                bool reaches = true;  // indeterminate counts as reaching
                if (squared_sum <= (std::uint64_t { 1 } << 53)) {
                    const double pitch_squared_low =
                        std::nextafter(pitch * pitch, -std::numeric_limits<double>::infinity());
                    const double distance_squared_low = std::nextafter(pitch_squared_low * static_cast<double>(squared_sum),
                                                                       -std::numeric_limits<double>::infinity());
                    const double clearance_squared_high =
                        std::nextafter(clearance * clearance, std::numeric_limits<double>::infinity());
                    if (std::isfinite(distance_squared_low) && std::isfinite(clearance_squared_high)) {
                        reaches = !(distance_squared_low > clearance_squared_high);
                    }
                }
                if (reaches) {
                    stencil.push_back({ x, y, z });
                }
            }
        }
    }
    return stencil;
}

bool oriented_bounds(const Mesh& mesh, const Quat& q, Bounds& out)
{
    if (!finite_pose_in({ 0, 0, 0 }, q)) {
        return false;
    }
    const auto transform = rotation_transform(q);
    if (!transform) {
        return false;
    }
    if (transform->exact_cardinal) {
        for (int world = 0; world < 3; ++world) {
            const int source = transform->source_axis[world], sign = transform->sign[world];
            const double low = sign * (sign > 0 ? mesh.bounds.min[source] : mesh.bounds.max[source]);
            const double high = sign * (sign > 0 ? mesh.bounds.max[source] : mesh.bounds.min[source]);
            if (!std::isfinite(low) || !std::isfinite(high) || low > high) {
                return false;
            }
            out.min[world] = low;
            out.max[world] = high;
        }
        return true;
    }
    Interval rotation[3][3];
    rotation_intervals(q, rotation);
    bool first = true;
    for (const auto& v : mesh.vertices) {
        for (int world = 0; world < 3; ++world) {
            const Interval iv = transformed_interval(v, { 0, 0, 0 }, rotation, world);
            if (!iv.valid) {
                return false;
            }
            if (first) {
                out.min[world] = iv.low;
                out.max[world] = iv.high;
            }
            else {
                out.min[world] = std::min(out.min[world], iv.low);
                out.max[world] = std::max(out.max[world], iv.high);
            }
        }
        first = false;
    }
    return !first;
}

// validation_kernel::posed_bounds (validation_kernel.cpp:1000-1088) with
// transformed_source_box (:949-997): the conservative bounds the validator's
// pair loop tests.  Cardinal rotations map the source box by the signed axis
// permutation and move each bound one ulp outward; every other rotation
// encloses the eight corners of the source box by their transformed
// intervals.  False where the reference returns no bounds.
bool posed_bounds(const Mesh& mesh, const Vec3& translation, const Quat& q, Bounds& out)
{
    if (!finite_pose_in(translation, q)) {
        return false;
    }
    const auto transform = rotation_transform(q);
    if (!transform) {
        return false;
    }
    const Bounds& local = mesh.bounds;
    constexpr double inf = std::numeric_limits<double>::infinity();
    if (transform->exact_cardinal) {
        for (int axis = 0; axis < 3; ++axis) {
            const int source = transform->source_axis[axis], sign = transform->sign[axis];
            const double low = translation[axis] + sign * (sign > 0 ? local.min[source] : local.max[source]);
            const double high = translation[axis] + sign * (sign > 0 ? local.max[source] : local.min[source]);
            out.min[axis] = std::nextafter(low, -inf);
            out.max[axis] = std::nextafter(high, inf);
        }
    }
    else {
        for (int axis = 0; axis < 3; ++axis) {
            if (!std::isfinite(local.min[axis]) || !std::isfinite(local.max[axis]) || local.min[axis] > local.max[axis]) {
                return false;
            }
        }
        Interval rotation[3][3];
        rotation_intervals(q, rotation);
        for (int axis = 0; axis < 3; ++axis) {
            out.min[axis] = inf;
            out.max[axis] = -inf;
        }
        for (unsigned corner = 0; corner != 8; ++corner) {
            Vec3 point;
            for (unsigned axis = 0; axis != 3; ++axis) {
                point[axis] = corner & (1U << axis) ? local.max[axis] : local.min[axis];
            }
            for (int axis = 0; axis < 3; ++axis) {
                const Interval interval = transformed_interval(point, translation, rotation, axis);
                if (!interval.valid) {
                    return false;
                }
                out.min[axis] = std::min(out.min[axis], interval.low);
                out.max[axis] = std::max(out.max[axis], interval.high);
            }
        }
    }
    for (int axis = 0; axis < 3; ++axis) {
        if (!std::isfinite(out.min[axis]) || !std::isfinite(out.max[axis])) {
            return false;
        }
    }
    return true;
}

std::array<Quat, 24> cube_catalog()
{
    using Matrix = std::array<int, 9>;
    std::array<Matrix, 24> matrices {};
    std::size_t count = 0;
    std::array<int, 3> perm { 0, 1, 2 };
    const auto det = [](const Matrix& m) {
        return m[0] * (m[4] * m[8] - m[5] * m[7]) - m[1] * (m[3] * m[8] - m[5] * m[6]) +
               m[2] * (m[3] * m[7] - m[4] * m[6]);
    };
    do {
        for (const int sx : { -1, 1 }) {
            for (const int sy : { -1, 1 }) {
                for (const int sz : { -1, 1 }) {
                    Matrix m {};
                    m[perm[0]] = sx;
                    m[3 + perm[1]] = sy;
                    m[6 + perm[2]] = sz;
                    if (det(m) == 1) {
                        matrices[count++] = m;
                    }
                }
            }
        }
    } while (std::next_permutation(perm.begin(), perm.end()));
    std::sort(matrices.begin(), matrices.end());
    std::array<Quat, 24> result {};
    for (std::size_t i = 0; i < 24; ++i) {
        const auto& m = matrices[i];
        const int trace = m[0] + m[4] + m[8];
        std::array<int, 4> n {};
        if (trace > 0) {
            n = { m[7] - m[5], m[2] - m[6], m[3] - m[1], trace + 1 };
        }
        else if (m[0] > m[4] && m[0] > m[8]) {
            n = { 1 + m[0] - m[4] - m[8], m[1] + m[3], m[2] + m[6], m[7] - m[5] };
        }
        else if (m[4] > m[8]) {
            n = { m[1] + m[3], 1 + m[4] - m[0] - m[8], m[5] + m[7], m[2] - m[6] };
        }
        else {
            n = { m[2] + m[6], m[5] + m[7], 1 + m[8] - m[0] - m[4], m[3] - m[1] };
        }
        const auto nonzero = std::count_if(n.begin(), n.end(), [](int v) { return v != 0; });
        const double magnitude = nonzero == 1 ? 1.0 : nonzero == 2 ? 0.7071067811865475244 : 0.5;
        Quat q {};
        for (int k = 0; k < 4; ++k) {
            q[k] = n[k] < 0 ? -magnitude : n[k] ? magnitude : 0;
        }
        bool neg = q[3] < 0;
        if (q[3] == 0) {
            for (int k = 0; k < 3; ++k) {
                if (q[k] != 0) {
                    neg = q[k] < 0;
                    break;
                }
            }
        }
        if (neg) {
            for (auto& c : q) {
                c = -c;
            }
        }
        for (auto& c : q) {
            if (c == 0) {
                c = 0;
            }
        }
        result[i] = q;
    }
    return result;
}

Quat canonical(Quat q)
{
    const double n = std::hypot(std::hypot(q[0], q[1]), std::hypot(q[2], q[3]));
    for (auto& v : q) {
        v /= n;
        if (v == 0) {
            v = 0;
        }
    }
    bool neg = q[3] < 0;
    if (q[3] == 0) {
        for (int i = 0; i < 3; ++i) {
            if (q[i] != 0) {
                neg = q[i] < 0;
                break;
            }
        }
    }
    if (neg) {
        for (auto& v : q) {
            v = -v;
        }
    }
    for (auto& v : q) {
        if (v == 0) {
            v = 0;
        }
    }
    return q;
}

bool canonical_unit(const Quat& q)
{
    for (const double v : q) {
        if (!std::isfinite(v)) {
            return false;
        }
    }
    const double norm = std::hypot(std::hypot(q[0], q[1]), std::hypot(q[2], q[3]));
    if (std::fabs(norm - 1.0) > 1e-7) {
        return false;
    }
    if (q[3] != 0.0) {
        return q[3] > 0.0;
    }
    for (int i = 0; i < 3; ++i) {
        if (q[i] != 0.0) {
            return q[i] > 0.0;
        }
    }
    return false;
}

}  // namespace spk::geo
