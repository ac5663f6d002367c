// Test infrastructure only: accepted-solid stand-in for the reference's
// engine/pack_geometry/src/import.cpp, which needs fcl/CGAL/manifold that are
// absent here.  It defines inspect_stl/accept_asset and the AssetDraft and
// AcceptedSolid accessors the hot-path TUs link against (import.hpp:184-219),
// for binary STL meshes that are closed and outward-wound by construction (the
// seeded synthetic generators); the solid-analysis checks are not re-run.
//
// The cleanup and frame steps restate import.cpp:509-660: bounds of the
// parsed vertices set the frame, the anchor is the lower corner for a
// container and the box centre (lo/2 + hi/2) for an object, exact duplicate
// vertices merge in first-appearance order, collinear faces (the reference's
// exact::collinear3d) and cyclic duplicates are dropped, unreferenced vertices
// are compacted away and local = scale * v - anchor with -0 normalised to +0.

#include <algorithm>
#include <array>
#include <bit>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <map>
#include <memory>
#include <optional>
#include <span>
#include <unordered_map>
#include <utility>
#include <vector>

#include "exact_predicates.hpp"
#include "spectrapack/geometry/import.hpp"

namespace spectrapack::geometry {

struct AssetDraft::Storage {
    std::vector<Vec3> vertices;
    std::vector<Triangle> triangles;
    Frame frame;
    AssetRole role { AssetRole::object };
    ImportReport report;
};

struct AcceptedSolid::Storage {
    std::shared_ptr<const AssetDraft> accepted;
};

AssetDraft::AssetDraft(std::shared_ptr<const Storage> storage) noexcept : storage_(std::move(storage)) {}
MeshView AssetDraft::mesh() const noexcept { return { storage_->vertices, storage_->triangles }; }
const Frame& AssetDraft::frame() const noexcept { return storage_->frame; }
AssetRole AssetDraft::role() const noexcept { return storage_->role; }
const ImportReport& AssetDraft::report() const noexcept { return storage_->report; }

AcceptedSolid::AcceptedSolid(std::shared_ptr<const Storage> storage) noexcept : storage_(std::move(storage)) {}
MeshView AcceptedSolid::mesh() const noexcept { return storage_->accepted->mesh(); }
bool AcceptedSolid::is_packing_envelope() const noexcept { return false; }
MeshView AcceptedSolid::source_mesh() const noexcept { return mesh(); }
const Frame& AcceptedSolid::frame() const noexcept { return storage_->accepted->frame(); }
AssetRole AcceptedSolid::role() const noexcept { return storage_->accepted->role(); }
const ImportReport& AcceptedSolid::report() const noexcept { return storage_->accepted->report(); }
Bounds AcceptedSolid::bounds_mm() const noexcept
{
    return storage_->accepted->report().mesh_bounds_mm.value_or(Bounds {});
}

namespace {

std::uint64_t payload_bytes(const AssetDraft& draft)
{
    const auto mesh = draft.mesh();
    return static_cast<std::uint64_t>(mesh.vertices.size()) * sizeof(Vec3) +
           static_cast<std::uint64_t>(mesh.triangles.size()) * sizeof(Triangle);
}

double plus_zero(double value) { return value == 0.0 ? 0.0 : value; }

struct Key {
    std::uint64_t x, y, z;
    bool operator==(const Key&) const = default;
};
struct KeyHash {
    std::size_t operator()(const Key& k) const noexcept
    {
        return std::hash<std::uint64_t>()(k.x * 0x9e3779b97f4a7c15ULL ^ k.y * 0xbf58476d1ce4e5b9ULL ^ k.z);
    }
};
Key key_of(const Vec3& v)
{
    return { std::bit_cast<std::uint64_t>(plus_zero(v[0])), std::bit_cast<std::uint64_t>(plus_zero(v[1])),
             std::bit_cast<std::uint64_t>(plus_zero(v[2])) };
}

ImportFailure failure(const char* code, const char* message) { return { code, code, message, std::nullopt }; }

}  // namespace

std::optional<std::uint64_t> AcceptedSolid::resident_buffer_bytes() const noexcept
{
    if (!storage_ || !storage_->accepted) {
        return std::nullopt;
    }
    return payload_bytes(*storage_->accepted);
}

std::optional<RepresentationResidency> AcceptedSolid::representation_residency() const noexcept
{
    if (!storage_ || !storage_->accepted) {
        return std::nullopt;
    }
    RepresentationResidency result;
    result.blocks[result.count++] = { RepresentationResidentKind::accepted_draft_payload, storage_->accepted.get(),
                                      payload_bytes(*storage_->accepted) };
    return result;
}

ImportOutcome<AssetDraft> inspect_stl(std::span<const std::byte> bytes, const ImportOptions& options,
                                      const runtime::OperationControl& control)
{
    if (bytes.size() < 84) {
        return failure("STL_TRUNCATED", "Binary STL header is truncated.");
    }
    std::uint32_t count {};
    std::memcpy(&count, bytes.data() + 80, 4);
    if (bytes.size() != 84 + 50ULL * count || count == 0) {
        return failure("STL_TRUNCATED", "Binary STL size does not match its triangle count.");
    }
    std::vector<Vec3> parsed;
    parsed.reserve(3ULL * count);
    Bounds bounds {};
    for (std::uint32_t t = 0; t != count; ++t) {
        const auto* record = bytes.data() + 84 + 50ULL * t + 12;
        for (int v = 0; v != 3; ++v) {
            Vec3 point {};
            for (int a = 0; a != 3; ++a) {
                float value {};
                std::memcpy(&value, record + 12 * v + 4 * a, 4);
                point[a] = static_cast<double>(value);
            }
            if (parsed.empty()) {
                bounds = { point, point };
            }
            for (int a = 0; a != 3; ++a) {
                bounds.min[a] = std::min(bounds.min[a], point[a]);
                bounds.max[a] = std::max(bounds.max[a], point[a]);
            }
            parsed.push_back(point);
        }
    }
    const double scale = options.units == Units::custom ? options.custom_scale_mm
                         : options.units == Units::inch ? 25.4
                                                        : 1.0;
    auto storage = std::make_shared<AssetDraft::Storage>();
    storage->role = options.role;
    storage->frame.source_bounds = bounds;
    storage->frame.unit_scale_mm = scale;
    for (int a = 0; a != 3; ++a) {
        const double low = scale * bounds.min[a];
        const double high = scale * bounds.max[a];
        const double anchor = options.role == AssetRole::container ? low : low / 2.0 + high / 2.0;
        storage->frame.dimensions_mm[a] = plus_zero(high - low);
        storage->frame.anchor_mm[a] = plus_zero(anchor);
    }
    std::unordered_map<Key, std::uint32_t, KeyHash> index;
    std::vector<Vec3> unique;
    std::vector<std::uint32_t> remap(parsed.size());
    for (std::size_t i = 0; i != parsed.size(); ++i) {
        Vec3 point { plus_zero(parsed[i][0]), plus_zero(parsed[i][1]), plus_zero(parsed[i][2]) };
        const auto [at, inserted] = index.emplace(key_of(point), static_cast<std::uint32_t>(unique.size()));
        if (inserted) {
            unique.push_back(point);
        }
        remap[i] = at->second;
    }
    detail::exact::WorkBudget budget(options.limits.max_predicate_work, control);
    std::vector<Triangle> faces;
    std::map<Triangle, bool> seen;
    std::uint64_t zero_area {}, duplicates {};
    for (std::uint32_t t = 0; t != count; ++t) {
        Triangle face { remap[3 * t], remap[3 * t + 1], remap[3 * t + 2] };
        const auto degenerate = detail::exact::collinear3d(unique[face[0]], unique[face[1]], unique[face[2]], budget);
        if (degenerate == detail::exact::Truth::uncertain) {
            return failure("PREDICATE_WORK_LIMIT", "Collinearity check exhausted its budget.");
        }
        if (degenerate == detail::exact::Truth::yes) {
            ++zero_area;
            continue;
        }
        const Triangle cyclic = std::min({ face, Triangle { face[1], face[2], face[0] },
                                           Triangle { face[2], face[0], face[1] } });
        if (!seen.emplace(cyclic, true).second) {
            ++duplicates;
            continue;
        }
        faces.push_back(face);
    }
    std::vector<bool> referenced(unique.size());
    for (const auto& face : faces) {
        for (const auto v : face) {
            referenced[v] = true;
        }
    }
    std::vector<std::uint32_t> compact(unique.size());
    for (std::uint32_t i = 0; i != unique.size(); ++i) {
        if (!referenced[i]) {
            continue;
        }
        compact[i] = static_cast<std::uint32_t>(storage->vertices.size());
        Vec3 local {};
        for (int a = 0; a != 3; ++a) {
            local[a] = plus_zero(scale * unique[i][a] - storage->frame.anchor_mm[a]);
        }
        storage->vertices.push_back(local);
    }
    for (auto& face : faces) {
        for (auto& v : face) {
            v = compact[v];
        }
    }
    storage->triangles = std::move(faces);
    Bounds local_bounds { storage->vertices.front(), storage->vertices.front() };
    double six {};
    for (const auto& v : storage->vertices) {
        for (int a = 0; a != 3; ++a) {
            local_bounds.min[a] = std::min(local_bounds.min[a], v[a]);
            local_bounds.max[a] = std::max(local_bounds.max[a], v[a]);
        }
    }
    for (const auto& t : storage->triangles) {
        const auto& p = storage->vertices[t[0]];
        const auto& q = storage->vertices[t[1]];
        const auto& r = storage->vertices[t[2]];
        six += p[0] * (q[1] * r[2] - q[2] * r[1]) - p[1] * (q[0] * r[2] - q[2] * r[0]) +
               p[2] * (q[0] * r[1] - q[1] * r[0]);
    }
    auto& report = storage->report;
    report.encoding = StlEncoding::binary;
    report.validity = Validity::valid;
    report.source_byte_size = bytes.size();
    report.source_triangle_count = count;
    report.vertex_count = storage->vertices.size();
    report.triangle_count = storage->triangles.size();
    report.component_count = 1;
    report.zero_area_faces = zero_area;
    report.duplicate_faces = duplicates;
    report.cleanup.zero_area_faces_removed = zero_area;
    report.cleanup.duplicate_faces_removed = duplicates;
    report.cleanup.exact_vertices_merged = parsed.size() - unique.size();
    report.topology_check = CheckState::complete;
    report.intersection_check = CheckState::complete;
    report.containment_check = CheckState::complete;
    report.mesh_bounds_mm = local_bounds;
    report.volume_mm3 = six / 6.0;
    return std::shared_ptr<const AssetDraft>(new AssetDraft(std::move(storage)));
}

ImportOutcome<AcceptedSolid> accept_asset(std::shared_ptr<const AssetDraft> draft)
{
    if (!draft || draft->report().validity != Validity::valid) {
        return failure("ASSET_NOT_VALID", "Only a valid draft can be accepted.");
    }
    auto storage = std::make_shared<AcceptedSolid::Storage>();
    storage->accepted = std::move(draft);
    return std::shared_ptr<const AcceptedSolid>(new AcceptedSolid(std::move(storage)));
}

}  // namespace spectrapack::geometry
