// Exact geometric predicates on binary64 inputs (host).
//
// Signs of small polynomial expressions are computed exactly with
// floating-point expansions (Shewchuk, "Adaptive Precision Floating-Point
// Arithmetic and Fast Robust Geometric Predicates", 1997): two_sum and an
// FMA-based two_product produce exact non-overlapping expansions, and the
// sign of an expansion is the sign of its largest component.  A float filter
// answers first; the expansion path settles whatever the filter cannot.
#pragma once

#include <array>
#include <cmath>
#include <vector>

namespace spk::exact {

enum class Sign { negative = -1, zero = 0, positive = 1 };

using Expansion = std::vector<double>;  // increasing magnitude, non-overlapping

inline void two_sum(double a, double b, double& s, double& e)
{
    s = a + b;
    const double bv = s - a;
    const double av = s - bv;
    e = (a - av) + (b - bv);
}

inline void two_product(double a, double b, double& p, double& e)
{
    p = a * b;
    e = std::fma(a, b, -p);
}

// h = e + f (Shewchuk's fast-expansion-sum without zero elimination issues:
// implemented as repeated grow-expansion, which is always exact).
inline Expansion expansion_sum(const Expansion& e, const Expansion& f)
{
    Expansion h = e;
    for (double b : f) {
        Expansion next;
        next.reserve(h.size() + 1);
        double q = b;
        for (double a : h) {
            double s, err;
            two_sum(q, a, s, err);
            if (err != 0.0) {
                next.push_back(err);
            }
            q = s;
        }
        if (q != 0.0 || next.empty()) {
            next.push_back(q);
        }
        h.swap(next);
    }
    return h;
}

inline Expansion scale_expansion(const Expansion& e, double b)
{
    Expansion h;
    h.reserve(2 * e.size());
    for (double a : e) {
        double p, pe;
        two_product(a, b, p, pe);
        h = expansion_sum(h, Expansion { pe, p });
    }
    return h;
}

inline Expansion product(const Expansion& a, const Expansion& b)
{
    Expansion r;
    for (double v : b) {
        r = expansion_sum(r, scale_expansion(a, v));
    }
    return r;
}

inline Expansion negate(Expansion e)
{
    for (double& v : e) {
        v = -v;
    }
    return e;
}

inline Sign sign_of(const Expansion& e)
{
    for (auto it = e.rbegin(); it != e.rend(); ++it) {
        if (*it > 0) {
            return Sign::positive;
        }
        if (*it < 0) {
            return Sign::negative;
        }
    }
    return Sign::zero;
}

inline Expansion difference(double a, double b)
{
    double s, e;
    two_sum(a, -b, s, e);
    return e != 0.0 ? Expansion { e, s } : Expansion { s };
}

// Sign of the exact sum of the terms (each term a binary64 value).
inline Sign sum_sign(const double* terms, int n)
{
    Expansion acc;
    for (int i = 0; i < n; ++i) {
        acc = expansion_sum(acc, Expansion { terms[i] });
    }
    return sign_of(acc);
}

using Vec3 = std::array<double, 3>;
using Point2 = std::array<double, 2>;

// sign of det[b-a, c-a] (2D orientation).
inline Sign orient2d(const Point2& a, const Point2& b, const Point2& c)
{
    const double acx = a[0] - c[0], bcx = b[0] - c[0], acy = a[1] - c[1], bcy = b[1] - c[1];
    const double l = acx * bcy, r = acy * bcx;
    const double det = l - r;
    const double bound = 3.3306690738754716e-16 * (std::fabs(l) + std::fabs(r));
    if (det > bound) {
        return Sign::positive;
    }
    if (-det > bound) {
        return Sign::negative;
    }
    const Expansion ax = difference(a[0], c[0]), bx = difference(b[0], c[0]);
    const Expansion ay = difference(a[1], c[1]), by = difference(b[1], c[1]);
    return sign_of(expansion_sum(product(ax, by), negate(product(ay, bx))));
}

// sign of det[a-d, b-d, c-d] (3D orientation of d against plane abc).
inline Sign orient3d(const Vec3& a, const Vec3& b, const Vec3& c, const Vec3& d)
{
    const double adx = a[0] - d[0], bdx = b[0] - d[0], cdx = c[0] - d[0];
    const double ady = a[1] - d[1], bdy = b[1] - d[1], cdy = c[1] - d[1];
    const double adz = a[2] - d[2], bdz = b[2] - d[2], cdz = c[2] - d[2];
    const double bdxcdy = bdx * cdy, cdxbdy = cdx * bdy;
    const double cdxady = cdx * ady, adxcdy = adx * cdy;
    const double adxbdy = adx * bdy, bdxady = bdx * ady;
    const double det = adz * (bdxcdy - cdxbdy) + bdz * (cdxady - adxcdy) + cdz * (adxbdy - bdxady);
    const double permanent = (std::fabs(bdxcdy) + std::fabs(cdxbdy)) * std::fabs(adz) +
                             (std::fabs(cdxady) + std::fabs(adxcdy)) * std::fabs(bdz) +
                             (std::fabs(adxbdy) + std::fabs(bdxady)) * std::fabs(cdz);
    const double bound = 7.771561172376103e-16 * permanent;  // (7 + 56 eps) eps
    if (det > bound) {
        return Sign::positive;
    }
    if (-det > bound) {
        return Sign::negative;
    }
    const Expansion ex[3] = { difference(a[0], d[0]), difference(b[0], d[0]), difference(c[0], d[0]) };
    const Expansion ey[3] = { difference(a[1], d[1]), difference(b[1], d[1]), difference(c[1], d[1]) };
    const Expansion ez[3] = { difference(a[2], d[2]), difference(b[2], d[2]), difference(c[2], d[2]) };
    // det = az (bx cy - cx by) + bz (cx ay - ax cy) + cz (ax by - bx ay)
    const Expansion m0 = expansion_sum(product(ex[1], ey[2]), negate(product(ex[2], ey[1])));
    const Expansion m1 = expansion_sum(product(ex[2], ey[0]), negate(product(ex[0], ey[2])));
    const Expansion m2 = expansion_sum(product(ex[0], ey[1]), negate(product(ex[1], ey[0])));
    const Expansion total =
        expansion_sum(expansion_sum(product(ez[0], m0), product(ez[1], m1)), product(ez[2], m2));
    return sign_of(total);
}

}  // namespace spk::exact
