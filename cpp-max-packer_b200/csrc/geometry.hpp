// Host-side geometry of the conservative fields: rigid placement with
// outward intervals, windows, face ranges, component witnesses, the analytic
// box container, clearance stencils, oriented bounds and orientation catalogs.
// Each function restates the reference function named beside it (paths under
// engine/pack_geometry/src unless noted) with the same binary64 arithmetic.
#pragma once

#include <array>
#include <cstdint>
#include <optional>
#include <vector>

#include "interval.cuh"

namespace spk::geo {

using Vec3 = std::array<double, 3>;
using Quat = std::array<double, 4>;
using Tri = std::array<std::uint32_t, 3>;

struct Bounds {
    Vec3 min {};
    Vec3 max {};
};

// An accepted solid's local mesh (AcceptedSolid::mesh(), import.hpp:184-219).
struct Mesh {
    std::vector<Vec3> vertices;
    std::vector<Tri> triangles;
    Bounds bounds;  // mesh_bounds_mm: min/max over the vertices
};

// prepare(): cuboid certificate (validation_kernel.cpp:384-447, 805-827).
// Also keeps each triangle's local vertices and their bounds, which every
// interval witness test reads (local_interval_point_in_material).
struct Prepared {
    const Mesh* mesh {};
    bool is_cuboid {};
    Bounds cuboid {};
    std::vector<std::array<Vec3, 3>> triangles;
    std::vector<Bounds> triangle_bounds;
};
Prepared prepare(const Mesh& mesh);

struct RotationTransform {
    double matrix[3][3] {};
    int source_axis[3] {};
    int sign[3] {};
    bool exact_cardinal {};
};
// rotation_transform (validation_kernel.cpp:572-610) with cardinal_rotation (:454-488).
std::optional<RotationTransform> rotation_transform(Quat q);
// rotation_intervals (:490-508).
void rotation_intervals(const Quat& q, Interval out[3][3]);

struct AxisCoordinate {
    double translation {};
    double local {};
    int sign { 1 };
};

// PlacedSolid (:624-638) built by place() (:829-943).
struct Placed {
    const Prepared* prepared {};
    Vec3 translation {};
    Quat q {};
    bool is_cardinal {};
    int source_axis[3] {};
    int sign[3] {};
    AxisCoordinate cuboid_min[3] {}, cuboid_max[3] {};
    Bounds conservative {};
    bool finite {};
    std::vector<Vec3> world;
    std::vector<IVec3> intervals;
    bool world_exact {};
};
bool place(const Prepared& prepared, const Vec3& translation, const Quat& q, Placed& out);
// finite_pose (validation_kernel.cpp): a finite translation and a finite,
// non-zero quaternion.
bool finite_pose(const Vec3& translation, const Quat& q);

struct Window {
    std::int64_t first[3] {};
    std::uint32_t shape[3] {};
};

// trim_index (conservative_fields.cpp:506-519): floor of the long double ratio, -1/+1.
bool trim_index(double bound, double origin, double pitch, bool lower, std::int64_t& out);
// voxelize_object window (conservative_fields.cpp:946-960).
bool object_window(const Placed& placed, const double* origin, double pitch, Window& out);
// window() (engine/pack_solver/src/spectral_pipeline.cpp:107-140).
bool environment_window(const Bounds& container, const double* origin, double pitch, Window& out);

enum class PlanKind { full_window, cropped_window, certified_empty };
// plan_placed_raw_window (conservative_fields.cpp:530-617).
PlanKind plan_placed_window(const Placed& placed, const Window& whole, const double* origin, double pitch,
                            Window& out);

// Per-face candidate cell ranges of rasterize_boundary (validation_kernel.cpp:3282-3330).
struct FaceRange {
    std::int64_t first[3];
    std::int64_t last[3];
    std::int32_t outside;
    std::int32_t pad;
};
bool face_ranges(const Placed& placed, const Window& window, const double* origin, double pitch,
                 std::vector<FaceRange>& out);

enum class Decision { no, yes, indeterminate };
// outward_grid_cell (validation_kernel.cpp:3444-3455).
bool outward_grid_cell(const double* origin, double pitch, const std::int64_t* index, Bounds& out);
// classify_material_witness (:3401-3438) with point_in_material (:1895-1938),
// local_interval_point_in_material (:3345-3399), local_point_in_material (:2144-2194).
Decision classify_material_witness(const Placed& solid, const Bounds& world_interval);

// classify_analytic_box_cell (:3457-3490), one axis: true when that axis
// certifies the closed cell inside the box after the wall inset.
bool analytic_box_axis_inside(double origin, double pitch, std::int64_t index, double dimension, double clearance,
                              const IVec3& cell, int axis);

// clearance_halo (conservative_fields.cpp:189-204) and make_stencil (:398-434)
// with euclidean_offset_reaches (validation_kernel.cpp:3492-3522).
bool clearance_halo(double clearance, double pitch, std::uint64_t& halo);
std::vector<std::array<std::int64_t, 3>> make_stencil(std::uint64_t halo, double pitch, double clearance);

// physical_bounds (validation_kernel.cpp:1099-1242): oriented bounds of the
// rotated mesh (exact for signed permutations, interval hull otherwise).
bool oriented_bounds(const Mesh& mesh, const Quat& q, Bounds& out);
// validation_kernel::posed_bounds (validation_kernel.cpp:1000-1088).
bool posed_bounds(const Mesh& mesh, const Vec3& translation, const Quat& q, Bounds& out);

// Orientation catalogs (engine/pack_solver/src/orientation_cube.hpp:10-80,
// orientations.cpp:40-66 canonical()).
std::array<Quat, 24> cube_catalog();
Quat canonical(Quat q);
bool canonical_unit(const Quat& q);  // conservative_fields.cpp:82-92

}  // namespace spk::geo
