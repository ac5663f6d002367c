// Host check that face_sat_disjoint(face_sat(tri), box) equals
// triangle_box_disjoint(tri, box) (csrc/interval.cuh) on seeded triangles and
// cells: cells around the triangle at several pitches, degenerate triangles,
// vertex intervals of zero and of a few ulps' width, and magnitudes whose
// products overflow (invalid intervals).  Prints the case counts; exits 1 on
// the first difference.
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <random>

#include "../../cpp-max-packer_b200/csrc/interval.cuh"

using namespace spk;

static Interval around(double v, int ulps)
{
    double lo = v, hi = v;
    for (int i = 0; i < ulps; ++i) {
        lo = std::nextafter(lo, -INFINITY);
        hi = std::nextafter(hi, INFINITY);
    }
    return { lo, hi, std::isfinite(lo) && std::isfinite(hi) };
}

int main()
{
    std::mt19937_64 rng(20261204);
    std::uniform_real_distribution<double> unit(-1.0, 1.0);
    long long cases = 0, disjoint = 0;
    const double scales[] = { 1.0, 37.5, 1e-3, 1e150, 1e200 };
    for (int trial = 0; trial < 60000; ++trial) {
        const double scale = scales[trial % 5];
        double p[3][3];
        for (int k = 0; k < 3; ++k) {
            for (int a = 0; a < 3; ++a) {
                p[k][a] = unit(rng) * scale;
            }
        }
        if (trial % 7 == 0) {  // degenerate: the third vertex on the first edge
            for (int a = 0; a < 3; ++a) {
                p[2][a] = p[0][a] + 0.5 * (p[1][a] - p[0][a]);
            }
        }
        if (trial % 11 == 0) {  // two equal vertices
            for (int a = 0; a < 3; ++a) {
                p[1][a] = p[0][a];
            }
        }
        IVec3 tri[3];
        const int ulps = trial % 3;
        for (int k = 0; k < 3; ++k) {
            for (int a = 0; a < 3; ++a) {
                tri[k].v[a] = around(p[k][a], ulps);
            }
        }
        FaceSat f;
        face_sat(tri, f);
        const double pitch = scale * (trial % 4 == 0 ? 0.05 : trial % 4 == 1 ? 0.2 : trial % 4 == 2 ? 0.7 : 2.0);
        const double origin[3] = { unit(rng) * scale, unit(rng) * scale, unit(rng) * scale };
        for (int c = 0; c < 40; ++c) {
            // A cell near a random point of the triangle.
            const double u = std::fabs(unit(rng)), v = std::fabs(unit(rng)) * (1.0 - std::fabs(unit(rng)));
            std::int64_t index[3];
            for (int a = 0; a < 3; ++a) {
                const double q = p[0][a] + u * (p[1][a] - p[0][a]) + v * (p[2][a] - p[0][a]) + unit(rng) * pitch;
                const double cell = std::floor((q - origin[a]) / pitch);
                index[a] = std::isfinite(cell) && std::fabs(cell) < 1e15 ? static_cast<std::int64_t>(cell) : 0;
            }
            IVec3 box;
            if (!grid_cell_interval(origin, pitch, index, box)) {
                continue;
            }
            const bool want = triangle_box_disjoint(tri, box);
            const bool got = face_sat_disjoint(f, box);
            ++cases;
            disjoint += want;
            if (want != got) {
                std::printf("mismatch at trial %d cell %d: triangle_box_disjoint %d, face_sat_disjoint %d\n", trial, c,
                            want, got);
                return 1;
            }
        }
    }
    std::printf("%lld cases, %lld disjoint, %lld overlapping\n", cases, disjoint, cases - disjoint);
    return 0;
}
