// Test infrastructure only: a C entry surface over the reference's own
// hot-path C++ (compiled unmodified from its sources by oracle/ref/Makefile)
// so the tests and the CPU baseline can call it through ctypes.  Nothing in
// the product links this library.
//
// Wrapped reference functions:
//   compute::correlate_binary_cpu / correlate_proximity_cpu  correlation.hpp:108-117
//   solver::detail::build_proximity                           field_proximity.hpp:32-132
//   geometry::voxelize_object / _container / _placed          conservative_fields.hpp:106-125
//   geometry::oriented_bounds                                 physical_bounds.cpp:347
//   solver::make_orientation_catalog                          orientations.hpp:41-42
//   solver::detail::build_spectral_pipeline                   spectral_pipeline.hpp:94-99
//   geometry::validate                                        validation.hpp:168
//   validation_kernel::bounds_pair_certificate                validation_kernel.hpp:177-178
//   geometry::RigidTransform::make / apply                    rigid_transform.hpp:15-18
// spkref_export_stl follows the record loop of pack_io's write_stl_stage
// (engine/pack_io/src/result_export.cpp:1034-1123; pack_io itself needs
// nlohmann/json and is not built here) with the reference's RigidTransform
// and the host libm's hypot.
// The greedy driver below follows the non-timed page-merge loop of
// engine/pack_solver/src/spectral.cpp:1460-1591 (run_trial) without the
// physical refinement that starts once every voxel page is exhausted.

#include <algorithm>
#include <chrono>
#include <cstdint>
#include <cstring>
#include <limits>
#include <memory>
#include <optional>
#include <span>
#include <string>
#include <variant>
#include <vector>

#include "field_proximity.hpp"
#include "spectral_pipeline.hpp"
#include "spectrapack/geometry/rigid_transform.hpp"
#include "validation_kernel.hpp"
#include "spectrapack/compute/correlation.hpp"
#include "spectrapack/geometry/conservative_fields.hpp"
#include "spectrapack/geometry/physical_bounds.hpp"
#include "spectrapack/solver/orientations.hpp"

namespace g = spectrapack::geometry;
namespace c = spectrapack::compute;
namespace s = spectrapack::solver;

namespace {

constexpr std::uint64_t kHuge = 1ULL << 60;

void put_error(char* buffer, int capacity, std::string_view code)
{
    if (buffer && capacity > 0) {
        const auto n = std::min<std::size_t>(code.size(), static_cast<std::size_t>(capacity - 1));
        std::memcpy(buffer, code.data(), n);
        buffer[n] = 0;
    }
}

g::RepresentationLimits wide_representation()
{
    g::RepresentationLimits limits;
    limits.max_working_bytes = kHuge;
    limits.max_cells = kHuge;
    limits.max_kernel_work = kHuge;
    limits.max_cell_visits = kHuge;
    limits.max_input_triangles = kHuge;
    return limits;
}

s::SpectralLimits wide_spectral()
{
    s::SpectralLimits limits;
    for (auto* phase : { &limits.baseline, &limits.spectral }) {
        phase->max_candidate_evaluations = kHuge;
        phase->max_search_passes = kHuge;
        phase->max_orientations = kHuge;
        phase->max_copies = kHuge;
        phase->max_axis_cells = kHuge;
        phase->max_working_bytes = kHuge;
        phase->max_geometry_kernel_work = kHuge;
        phase->max_validation_kernel_work = kHuge;
        phase->per_query.max_working_bytes = kHuge;
        phase->per_query.max_kernel_work = kHuge;
        phase->per_query.max_vertex_visits = kHuge;
        phase->per_validation.max_copy_count = kHuge;
        phase->per_validation.max_working_bytes = kHuge;
        phase->per_validation.max_aabb_pair_tests = kHuge;
        phase->per_validation.max_kernel_work = kHuge;
    }
    limits.per_representation = wide_representation();
    limits.per_correlation.max_working_bytes = kHuge;
    limits.per_correlation.max_padded_cells = kHuge;
    limits.per_correlation.max_direct_terms = kHuge;
    limits.max_working_bytes = kHuge;
    limits.max_refinement_evaluations = 0;
    limits.cpu_thread_count = 1;
    limits.timed = false;
    return limits;
}

g::ValidationLimits wide_validation()
{
    g::ValidationLimits limits;
    limits.max_copy_count = kHuge;
    limits.max_working_bytes = kHuge;
    limits.max_aabb_pair_tests = kHuge;
    limits.max_kernel_work = kHuge;
    return limits;
}

struct Asset {
    std::shared_ptr<const g::AcceptedSolid> solid;
};

std::shared_ptr<const g::VoxelGeometry> prepared(const Asset& asset)
{
    auto outcome = g::prepare_voxel_geometry(asset.solid, wide_representation());
    if (!std::holds_alternative<std::shared_ptr<const g::VoxelGeometry>>(outcome)) {
        return {};
    }
    return std::get<std::shared_ptr<const g::VoxelGeometry>>(outcome);
}

int copy_field(const g::RepresentationOutcome<g::CellField>& outcome, std::int64_t* first, std::uint32_t* shape,
               std::uint8_t* cells, std::uint64_t capacity, char* err, int errcap)
{
    if (const auto* failure = std::get_if<g::RepresentationFailure>(&outcome)) {
        put_error(err, errcap, failure->code);
        return 1;
    }
    const auto& field = std::get<std::shared_ptr<const g::CellField>>(outcome);
    const auto& window = field->window();
    for (int a = 0; a != 3; ++a) {
        first[a] = window.first[a];
        shape[a] = window.shape[a];
    }
    const auto data = field->cells();
    if (data.size() > capacity) {
        put_error(err, errcap, "BUFFER_TOO_SMALL");
        return 2;
    }
    std::memcpy(cells, data.data(), data.size());
    return 0;
}

// Captures the arrays the pipeline observes (spectral_pipeline.hpp:53-65).
struct Observation {
    std::vector<std::uint8_t> occupancy;
    std::vector<double> proximity;
    std::vector<std::uint8_t> kernel;
    std::vector<double> binary_values;
    std::vector<double> proximity_values;
    g::GridWindow environment {}, kernel_window {};
    c::Index3 translation_first {};
    c::Shape3 output_shape {};
    bool valid {};
};
thread_local Observation* g_observation {};
thread_local bool g_keep_values {};

void observe(const s::detail::BinaryObservation& value) noexcept
{
    if (!g_observation) {
        return;
    }
    auto& o = *g_observation;
    o.environment = value.environment_window;
    o.kernel_window = value.kernel_window;
    o.occupancy.assign(value.environment.begin(), value.environment.end());
    o.proximity.assign(value.proximity.begin(), value.proximity.end());
    o.kernel.assign(value.kernel.begin(), value.kernel.end());
    if (g_keep_values) {
        o.binary_values.assign(value.values.begin(), value.values.end());
        o.proximity_values.assign(value.proximity_values.begin(), value.proximity_values.end());
    }
    o.translation_first = value.translation_first;
    o.output_shape = value.output_shape;
    o.valid = true;
}

struct Session {
    std::shared_ptr<const g::ValidationContext> context;
    g::GridLattice lattice {};
    s::OrientationCatalog catalog;
    s::SpectralLimits limits = wide_spectral();
    s::detail::SpectralWorkspace workspace;
    std::shared_ptr<const g::ValidatedSolution> working;
    std::uint64_t next_id {};
    Observation last;
};

struct PageEntry {
    std::int64_t t[3];
    double score;
    std::uint64_t orientation;
    double binary_overlap;
    std::int32_t direct_zero;
};

std::string make_id(std::uint64_t n) { return "copy-" + std::to_string(n); }

}  // namespace

extern "C" {

int spkref_correlate(int proximity, const std::uint32_t* env_shape, const std::uint32_t* ker_shape,
                     const std::int64_t* env_first, const std::int64_t* ker_first, const void* environment,
                     const std::uint8_t* kernel, double* out, std::uint64_t out_capacity, std::int64_t* t_first,
                     std::uint32_t* out_shape, double* report, char* err, int errcap)
{
    c::CorrelationSpec spec {};
    std::uint64_t env_cells = 1, ker_cells = 1;
    for (int a = 0; a != 3; ++a) {
        spec.environment_shape[a] = env_shape[a];
        spec.kernel_shape[a] = ker_shape[a];
        spec.environment_first[a] = env_first[a];
        spec.kernel_first[a] = ker_first[a];
        env_cells *= env_shape[a];
        ker_cells *= ker_shape[a];
    }
    c::CorrelationLimits limits;
    limits.max_working_bytes = kHuge;
    limits.max_padded_cells = kHuge;
    limits.max_direct_terms = kHuge;
    const std::span<const std::uint8_t> ker(kernel, ker_cells);
    const auto outcome =
        proximity ? c::correlate_proximity_cpu(spec, { static_cast<const double*>(environment), env_cells }, ker, limits)
                  : c::correlate_binary_cpu(spec, { static_cast<const std::uint8_t*>(environment), env_cells }, ker,
                                            limits);
    if (const auto* failure = std::get_if<c::CorrelationFailure>(&outcome)) {
        put_error(err, errcap, failure->code);
        return 1;
    }
    const auto& result = std::get<c::CorrelationResult>(outcome);
    if (result.values.size() > out_capacity) {
        put_error(err, errcap, "BUFFER_TOO_SMALL");
        return 2;
    }
    std::memcpy(out, result.values.data(), result.values.size() * sizeof(double));
    for (int a = 0; a != 3; ++a) {
        t_first[a] = result.translation_first[a];
        out_shape[a] = result.shape[a];
    }
    report[0] = result.numeric.max_integer_residual;
    report[1] = result.numeric.mass_residual;
    report[2] = result.numeric.max_probe_error;
    return 0;
}

int spkref_build_proximity(const std::uint32_t* shape, const std::uint8_t* occupied, double* values)
{
    const g::CellShape cell_shape { shape[0], shape[1], shape[2] };
    const std::size_t n = std::size_t { shape[0] } * shape[1] * shape[2];
    std::uint64_t work {};
    return s::detail::build_proximity(cell_shape, { occupied, n }, { values, n }, UINT64_MAX, work) ? 0 : 1;
}

void* spkref_asset_from_stl(const std::uint8_t* bytes, std::uint64_t size, int container, char* err, int errcap)
{
    const g::ImportOptions options(container ? g::AssetRole::container : g::AssetRole::object, g::Units::mm);
    auto draft = g::inspect_stl({ reinterpret_cast<const std::byte*>(bytes), size }, options);
    if (const auto* failure = std::get_if<g::ImportFailure>(&draft)) {
        put_error(err, errcap, failure->code);
        return nullptr;
    }
    auto accepted = g::accept_asset(std::get<std::shared_ptr<const g::AssetDraft>>(draft));
    if (const auto* failure = std::get_if<g::ImportFailure>(&accepted)) {
        put_error(err, errcap, failure->code);
        return nullptr;
    }
    return new Asset { std::get<std::shared_ptr<const g::AcceptedSolid>>(accepted) };
}

void spkref_asset_free(void* asset) { delete static_cast<Asset*>(asset); }

// counts[0] vertices, counts[1] triangles; bounds min xyz then max xyz.
int spkref_asset_mesh(void* handle, double* vertices, std::uint64_t vertex_capacity, std::uint32_t* triangles,
                      std::uint64_t triangle_capacity, std::uint64_t* counts, double* bounds)
{
    const auto& solid = *static_cast<Asset*>(handle)->solid;
    const auto mesh = solid.mesh();
    counts[0] = mesh.vertices.size();
    counts[1] = mesh.triangles.size();
    const auto b = solid.bounds_mm();
    for (int a = 0; a != 3; ++a) {
        bounds[a] = b.min[a];
        bounds[3 + a] = b.max[a];
    }
    if (mesh.vertices.size() > vertex_capacity || mesh.triangles.size() > triangle_capacity) {
        return vertices || triangles ? 2 : 0;
    }
    if (vertices) {
        std::memcpy(vertices, mesh.vertices.data(), mesh.vertices.size() * sizeof(g::Vec3));
    }
    if (triangles) {
        std::memcpy(triangles, mesh.triangles.data(), mesh.triangles.size() * sizeof(g::Triangle));
    }
    return 0;
}

int spkref_voxelize_object(void* handle, const double* origin, double pitch, const double* q, std::int64_t* first,
                           std::uint32_t* shape, std::uint8_t* cells, std::uint64_t capacity, char* err, int errcap)
{
    const auto geometry = prepared(*static_cast<Asset*>(handle));
    if (!geometry) {
        put_error(err, errcap, "PREPARE_FAILED");
        return 3;
    }
    const g::GridLattice lattice { { origin[0], origin[1], origin[2] }, pitch };
    return copy_field(g::voxelize_object(geometry, lattice, { q[0], q[1], q[2], q[3] }, wide_representation()), first,
                      shape, cells, capacity, err, errcap);
}

int spkref_voxelize_container(int box, const double* dims, void* handle, const double* origin, double pitch,
                              const std::int64_t* first, const std::uint32_t* shape, double clearance,
                              std::uint8_t* cells, char* err, int errcap)
{
    g::GridWindow window;
    window.lattice = { { origin[0], origin[1], origin[2] }, pitch };
    for (int a = 0; a != 3; ++a) {
        window.first[a] = first[a];
        window.shape[a] = shape[a];
    }
    g::Container container = box ? g::Container { g::BoxDimensions { dims[0], dims[1], dims[2] } }
                                 : g::Container { static_cast<Asset*>(handle)->solid };
    std::int64_t f[3];
    std::uint32_t sh[3];
    const std::uint64_t n = std::uint64_t { shape[0] } * shape[1] * shape[2];
    return copy_field(g::voxelize_container(container, window, clearance, wide_representation()), f, sh, cells, n, err,
                      errcap);
}

int spkref_voxelize_placed(void* handle, const double* origin, double pitch, const std::int64_t* first,
                           const std::uint32_t* shape, const double* translation, const double* q, double clearance,
                           std::uint8_t* cells, char* err, int errcap)
{
    const auto geometry = prepared(*static_cast<Asset*>(handle));
    if (!geometry) {
        put_error(err, errcap, "PREPARE_FAILED");
        return 3;
    }
    g::GridWindow window;
    window.lattice = { { origin[0], origin[1], origin[2] }, pitch };
    for (int a = 0; a != 3; ++a) {
        window.first[a] = first[a];
        window.shape[a] = shape[a];
    }
    const g::CopyPose pose { "placed", { translation[0], translation[1], translation[2] }, { q[0], q[1], q[2], q[3] } };
    std::int64_t f[3];
    std::uint32_t sh[3];
    const std::uint64_t n = std::uint64_t { shape[0] } * shape[1] * shape[2];
    return copy_field(g::voxelize_placed(geometry, window, pose, clearance, wide_representation()), f, sh, cells, n,
                      err, errcap);
}

int spkref_oriented_bounds(void* handle, const double* q, double* out)
{
    g::PhysicalQueryLimits limits;
    limits.max_working_bytes = kHuge;
    limits.max_kernel_work = kHuge;
    limits.max_vertex_visits = kHuge;
    const auto outcome = g::oriented_bounds(static_cast<Asset*>(handle)->solid, { q[0], q[1], q[2], q[3] }, limits);
    if (!std::holds_alternative<g::OrientedBounds>(outcome)) {
        return 1;
    }
    const auto& b = std::get<g::OrientedBounds>(outcome).bounds_mm;
    for (int a = 0; a != 3; ++a) {
        out[a] = b.min[a];
        out[3 + a] = b.max[a];
    }
    return 0;
}

namespace vk = spectrapack::geometry::detail::validation_kernel;

// validation_kernel::bounds_pair_certificate of two poses of the asset:
// 0 no certificate (the validator goes on to its other certificates), 1
// certified by the outward AABBs ("outward-aabb"), 2 certified another way,
// 3 indeterminate, -1 a pose without bounds.
int spkref_bounds_pair(void* handle, const double* t1, const double* q1, const double* t2, const double* q2,
                       double clearance)
{
    vk::Budget budget(kHuge, kHuge);
    const auto& solid = static_cast<Asset*>(handle)->solid;
    const auto a = vk::posed_bounds(solid, { t1[0], t1[1], t1[2] }, { q1[0], q1[1], q1[2], q1[3] }, budget);
    const auto b = vk::posed_bounds(solid, { t2[0], t2[1], t2[2] }, { q2[0], q2[1], q2[2], q2[3] }, budget);
    if (!a || !b) {
        return -1;
    }
    const auto c = vk::bounds_pair_certificate(*a.bounds, *b.bounds, clearance, budget);
    if (!c) {
        return 0;
    }
    if (c->material_overlap == vk::Decision::indeterminate || c->surface_gap == vk::Threshold::indeterminate) {
        return 3;
    }
    return c->method == "outward-aabb" ? 1 : 2;
}

// The binary STL of `copies` posed copies of the asset (see the header
// comment).  1 = a pose without a rigid transform, 2 = a coordinate that is
// not a finite float32, 3 = out too small (*size is the file size).
int spkref_export_stl(void* handle, const double* translations, const double* quaternions, std::uint64_t copies,
                      std::uint8_t* out, std::uint64_t capacity, std::uint64_t* size)
{
    const auto mesh = static_cast<Asset*>(handle)->solid->mesh();
    const std::uint64_t triangles = mesh.triangles.size() * copies;
    *size = 84 + 50 * triangles;
    if (capacity < *size) {
        return 3;
    }
    std::memset(out, 0, 80);
    const auto count32 = static_cast<std::uint32_t>(triangles);
    std::memcpy(out + 80, &count32, 4);
    std::uint8_t* at = out + 84;
    for (std::uint64_t c = 0; c < copies; ++c) {
        const double* t = translations + 3 * c;
        const double* q = quaternions + 4 * c;
        const auto transform = g::RigidTransform::make({ q[0], q[1], q[2], q[3] }, { t[0], t[1], t[2] });
        if (!transform) {
            return 1;
        }
        for (const auto& face : mesh.triangles) {
            std::array<std::array<float, 3>, 3> points {};
            for (std::size_t vertex = 0; vertex != 3; ++vertex) {
                const auto point = transform->apply(mesh.vertices[face[vertex]]);
                for (std::size_t axis = 0; axis != 3; ++axis) {
                    if (!std::isfinite(point[axis]) || point[axis] > std::numeric_limits<float>::max() ||
                        point[axis] < -std::numeric_limits<float>::max()) {
                        return 2;
                    }
                    points[vertex][axis] = static_cast<float>(point[axis]);
                }
            }
            const std::array<double, 3> ea { static_cast<double>(points[1][0]) - points[0][0],
                                             static_cast<double>(points[1][1]) - points[0][1],
                                             static_cast<double>(points[1][2]) - points[0][2] };
            const std::array<double, 3> eb { static_cast<double>(points[2][0]) - points[0][0],
                                             static_cast<double>(points[2][1]) - points[0][1],
                                             static_cast<double>(points[2][2]) - points[0][2] };
            std::array<double, 3> n { ea[1] * eb[2] - ea[2] * eb[1], ea[2] * eb[0] - ea[0] * eb[2],
                                      ea[0] * eb[1] - ea[1] * eb[0] };
            const auto length = std::hypot(std::hypot(n[0], n[1]), n[2]);
            if (length != 0.0 && std::isfinite(length)) {
                for (auto& v : n) {
                    v /= length;
                }
            }
            else {
                n = {};
            }
            const std::array<float, 3> normal { static_cast<float>(n[0]), static_cast<float>(n[1]),
                                                static_cast<float>(n[2]) };
            std::memcpy(at, normal.data(), 12);
            std::memcpy(at + 12, points.data(), 36);
            at[48] = at[49] = 0;
            at += 50;
        }
    }
    return 0;
}

// mode: 0 fixed, 1 cube, 4 catalog (g::OrientationMode values).
int spkref_catalog(int mode, const double* quaternions, std::uint64_t count, double* out, std::uint64_t capacity,
                   std::uint64_t* produced)
{
    g::OrientationPolicy policy;
    policy.mode = static_cast<g::OrientationMode>(mode);
    for (std::uint64_t i = 0; i != count; ++i) {
        policy.catalog_xyzw.push_back({ quaternions[4 * i], quaternions[4 * i + 1], quaternions[4 * i + 2],
                                        quaternions[4 * i + 3] });
    }
    const auto outcome = s::make_orientation_catalog(policy, kHuge);
    if (!std::holds_alternative<s::OrientationCatalog>(outcome)) {
        return 1;
    }
    const auto& catalog = std::get<s::OrientationCatalog>(outcome).quaternions;
    *produced = catalog.size();
    if (catalog.size() > capacity) {
        return 2;
    }
    std::memcpy(out, catalog.data(), catalog.size() * sizeof(g::Quaternion));
    return 0;
}

void* spkref_session_new(void* object, int box, const double* dims, void* container, double pair_clearance,
                         double wall_clearance, const double* origin, double pitch, const double* quaternions,
                         std::uint64_t count, char* err, int errcap)
{
    g::Container shape = box ? g::Container { g::BoxDimensions { dims[0], dims[1], dims[2] } }
                             : g::Container { static_cast<Asset*>(container)->solid };
    g::Constraints constraints;
    constraints.pair_clearance_mm = pair_clearance;
    constraints.wall_clearance_mm = wall_clearance;
    constraints.orientations.mode = g::OrientationMode::catalog;
    for (std::uint64_t i = 0; i != count; ++i) {
        constraints.orientations.catalog_xyzw.push_back(
            { quaternions[4 * i], quaternions[4 * i + 1], quaternions[4 * i + 2], quaternions[4 * i + 3] });
    }
    auto context = g::make_validation_context(static_cast<Asset*>(object)->solid, shape, constraints);
    if (const auto* failure = std::get_if<g::ValidationInputFailure>(&context)) {
        put_error(err, errcap, failure->code);
        return nullptr;
    }
    auto session = std::make_unique<Session>();
    session->context = std::get<std::shared_ptr<const g::ValidationContext>>(context);
    session->lattice = { { origin[0], origin[1], origin[2] }, pitch };
    session->catalog.quaternions = constraints.orientations.catalog_xyzw;
    auto empty = g::make_candidate(session->context, {});
    auto checked = g::validate(session->context, std::get<std::shared_ptr<const g::Candidate>>(empty),
                               wide_validation());
    if (!checked.validated_solution) {
        put_error(err, errcap, "EMPTY_LAYOUT_INVALID");
        return nullptr;
    }
    session->working = checked.validated_solution;
    return session.release();
}

void spkref_session_free(void* session) { delete static_cast<Session*>(session); }

// One page for `orientation` over the current layout (spectral_pipeline.cpp:914-1876).
int spkref_session_page(void* handle, std::uint64_t orientation, int has_cursor, const PageEntry* cursor,
                        int low_overlap, PageEntry* page, std::uint64_t* count, int keep_values, char* err,
                        int errcap)
{
    auto& session = *static_cast<Session*>(handle);
    s::detail::CandidatePageQuery query;
    query.orientation_index = orientation;
    query.mode = low_overlap ? s::detail::CandidatePageMode::low_overlap : s::detail::CandidatePageMode::ordinary;
    if (has_cursor) {
        s::detail::SpectralPipelineResult::RankedCandidate value;
        value.translation = { cursor->t[0], cursor->t[1], cursor->t[2] };
        value.score = cursor->score;
        value.orientation_index = cursor->orientation;
        value.binary_overlap = cursor->binary_overlap;
        value.direct_zero_overlap = cursor->direct_zero != 0;
        query.exclusive_cursor = value;
    }
    session.last = {};
    g_observation = &session.last;
    g_keep_values = keep_values != 0;
    auto result = s::detail::build_spectral_pipeline(session.workspace, session.context, session.lattice,
                                                     session.limits, session.working, session.catalog, query, observe);
    g_observation = nullptr;
    if (!result.complete) {
        put_error(err, errcap, result.diagnostic);
        return 1;
    }
    *count = 0;
    if (!result.ranked_candidates) {
        return 0;
    }
    for (const auto& candidate : *result.ranked_candidates) {
        auto& entry = page[(*count)++];
        for (int a = 0; a != 3; ++a) {
            entry.t[a] = candidate.translation[a];
        }
        entry.score = candidate.score;
        entry.orientation = candidate.orientation_index;
        entry.binary_overlap = candidate.binary_overlap;
        entry.direct_zero = candidate.direct_zero_overlap ? 1 : 0;
    }
    return 0;
}

// Copies the arrays captured by the last page call.  kind: 0 occupancy (u8),
// 1 proximity (f64), 2 kernel (u8), 3 binary values (f64), 4 proximity values
// (f64).  meta: env first[3], env shape[3], kernel first[3], kernel shape[3],
// translation_first[3], output shape[3].
int spkref_session_observed(void* handle, int kind, void* out, std::uint64_t capacity_bytes, std::int64_t* meta)
{
    const auto& o = static_cast<Session*>(handle)->last;
    if (!o.valid) {
        return 1;
    }
    for (int a = 0; a != 3; ++a) {
        meta[a] = o.environment.first[a];
        meta[3 + a] = o.environment.shape[a];
        meta[6 + a] = o.kernel_window.first[a];
        meta[9 + a] = o.kernel_window.shape[a];
        meta[12 + a] = o.translation_first[a];
        meta[15 + a] = o.output_shape[a];
    }
    const void* source {};
    std::uint64_t bytes {};
    switch (kind) {
    case 0: source = o.occupancy.data(); bytes = o.occupancy.size(); break;
    case 1: source = o.proximity.data(); bytes = o.proximity.size() * 8; break;
    case 2: source = o.kernel.data(); bytes = o.kernel.size(); break;
    case 3: source = o.binary_values.data(); bytes = o.binary_values.size() * 8; break;
    case 4: source = o.proximity_values.data(); bytes = o.proximity_values.size() * 8; break;
    default: return 2;
    }
    if (!out) {
        meta[18] = static_cast<std::int64_t>(bytes);
        return 0;
    }
    if (bytes > capacity_bytes) {
        return 3;
    }
    std::memcpy(out, source, bytes);
    return 0;
}

// Validates and appends one lattice pose; returns 0 when accepted.
int spkref_session_place(void* handle, std::uint64_t orientation, const std::int64_t* t)
{
    auto& session = *static_cast<Session*>(handle);
    auto copies = session.working->copies();
    const auto& lattice = session.lattice;
    copies.push_back({ make_id(session.next_id),
                       { lattice.origin_mm[0] + lattice.pitch_mm * t[0], lattice.origin_mm[1] + lattice.pitch_mm * t[1],
                         lattice.origin_mm[2] + lattice.pitch_mm * t[2] },
                       session.catalog.quaternions[orientation] });
    auto candidate = g::make_candidate(session.context, copies);
    if (!std::holds_alternative<std::shared_ptr<const g::Candidate>>(candidate)) {
        return 2;
    }
    auto checked = g::validate_incremental(session.working, std::get<std::shared_ptr<const g::Candidate>>(candidate),
                                           wide_validation());
    if (!checked.validated_solution) {
        return 1;
    }
    session.working = checked.validated_solution;
    ++session.next_id;
    return 0;
}

// Greedy fill from the current layout (spectral.cpp:1460-1591, non-timed, no
// refinement).  Each accepted copy writes orientation, t[3] and score.
int spkref_session_greedy(void* handle, std::uint64_t max_steps, std::uint64_t* orientations, std::int64_t* t,
                          double* scores, std::uint64_t* placed, std::uint64_t* rejected, double* seconds, char* err,
                          int errcap)
{
    auto& session = *static_cast<Session*>(handle);
    const auto start = std::chrono::steady_clock::now();
    const std::size_t n = session.catalog.quaternions.size();
    *placed = 0;
    *rejected = 0;
    const auto rank_less = [](const PageEntry& l, const PageEntry& r) {
        if (l.score != r.score) {
            return l.score < r.score;
        }
        if (l.orientation != r.orientation) {
            return l.orientation < r.orientation;
        }
        return std::tie(l.t[2], l.t[1], l.t[0]) < std::tie(r.t[2], r.t[1], r.t[0]);
    };
    while (*placed < max_steps) {
        std::vector<std::vector<PageEntry>> pages(n);
        std::vector<std::size_t> index(n);
        std::vector<std::optional<PageEntry>> cursors(n);
        std::vector<bool> exhausted(n);
        bool admitted = false;
        for (;;) {
            for (std::size_t o = 0; o != n; ++o) {
                if (exhausted[o] || index[o] != pages[o].size()) {
                    continue;
                }
                PageEntry buffer[32];
                std::uint64_t count {};
                if (spkref_session_page(handle, o, cursors[o].has_value(), cursors[o] ? &*cursors[o] : nullptr, 0,
                                        buffer, &count, 0, err, errcap)) {
                    return 1;
                }
                pages[o].assign(buffer, buffer + count);
                index[o] = 0;
                if (count == 0) {
                    exhausted[o] = true;
                }
            }
            std::optional<std::size_t> chosen;
            for (std::size_t o = 0; o != n; ++o) {
                if (index[o] == pages[o].size()) {
                    continue;
                }
                if (!chosen || rank_less(pages[o][index[o]], pages[*chosen][index[*chosen]])) {
                    chosen = o;
                }
            }
            if (!chosen) {
                break;
            }
            const auto candidate = pages[*chosen][index[*chosen]++];
            cursors[*chosen] = candidate;
            if (!candidate.direct_zero) {
                ++*rejected;
                continue;
            }
            if (spkref_session_place(handle, candidate.orientation, candidate.t) != 0) {
                ++*rejected;
                continue;
            }
            orientations[*placed] = candidate.orientation;
            for (int a = 0; a != 3; ++a) {
                t[3 * *placed + a] = candidate.t[a];
            }
            scores[*placed] = candidate.score;
            ++*placed;
            admitted = true;
            break;
        }
        if (!admitted) {
            break;
        }
    }
    *seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - start).count();
    return 0;
}

}  // extern "C"
