// Placement session and the stateless field entry points.
//
// The session is the device-resident counterpart of the reference's
// SpectralWorkspace (engine/pack_solver/src/spectral_pipeline.cpp:227-252):
// container blocker, BlockedField counts, occupancy, proximity, environment
// spectrum and one kernel per catalog orientation, all kept in HBM.  A layout
// change re-stamps only the new copy (voxelize_placed + add, :1255-1308),
// then rebuilds occupancy (:1323-1334), the exact proximity field (:1343) and
// the environment spectrum once for every orientation's page.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <memory>
#include <optional>
#include <set>
#include <thread>
#include <tuple>
#include <vector>

#include "context.hpp"
#include "edt.cuh"
#include "fields.hpp"
#include "geometry.hpp"
#include "pipeline.hpp"
#include "proposal.hpp"

namespace spk {

namespace {

geo::Mesh to_mesh(const spk_mesh& m)
{
    geo::Mesh mesh;
    mesh.vertices.resize(m.vertex_count);
    mesh.triangles.resize(m.triangle_count);
    std::memcpy(mesh.vertices.data(), m.vertices, m.vertex_count * 24);
    std::memcpy(mesh.triangles.data(), m.triangles, m.triangle_count * 12);
    if (!mesh.vertices.empty()) {
        mesh.bounds = { mesh.vertices.front(), mesh.vertices.front() };
        for (const auto& v : mesh.vertices) {
            for (int a = 0; a < 3; ++a) {
                mesh.bounds.min[a] = std::min(mesh.bounds.min[a], v[a]);
                mesh.bounds.max[a] = std::max(mesh.bounds.max[a], v[a]);
            }
        }
    }
    return mesh;
}

bool valid_mesh(const spk_mesh* m)
{
    if (!m || !m->vertices || !m->triangles || !m->vertex_count || !m->triangle_count) {
        return false;
    }
    for (std::uint64_t i = 0; i < 3 * m->triangle_count; ++i) {
        if (m->triangles[i] >= m->vertex_count) {
            return false;
        }
    }
    return true;
}

bool valid_lattice(const double* origin, double pitch)
{
    return std::isfinite(origin[0]) && std::isfinite(origin[1]) && std::isfinite(origin[2]) && std::isfinite(pitch) &&
           pitch > 0.0;
}

// expanded() (conservative_fields.cpp:169-187).
geo::Window expanded(const geo::Window& w, std::uint64_t halo)
{
    geo::Window r = w;
    for (int a = 0; a < 3; ++a) {
        r.first[a] -= static_cast<std::int64_t>(halo);
        r.shape[a] = static_cast<std::uint32_t>(w.shape[a] + 2 * halo);
    }
    return r;
}

std::uint64_t cells_of(const geo::Window& w)
{
    return static_cast<std::uint64_t>(w.shape[0]) * w.shape[1] * w.shape[2];
}

// voxelize_object into d_cells (device); window returned in `w`.
int object_field(spk_context* ctx, const geo::Prepared& prepared, const double* origin, double pitch,
                 const geo::Quat& q, geo::Window& w, std::vector<std::uint8_t>& host_cells)
{
    if (!geo::canonical_unit(q)) {
        return kFieldInput;
    }
    geo::Placed placed;
    if (!geo::place(prepared, { origin[0], origin[1], origin[2] }, q, placed)) {
        return kFieldInput;
    }
    if (!geo::object_window(placed, origin, pitch, w)) {
        return kFieldIndexOverflow;
    }
    const std::uint64_t n = cells_of(w);
    int status = kOk;
    auto* d = static_cast<std::uint8_t*>(device_buffer(ctx, "obj.cells", n, status));
    if (!d) {
        return status;
    }
    if ((status = raster_fill(ctx, placed, make_window(w, origin, pitch), d, true))) {
        return status;
    }
    host_cells.resize(n);
    cudaMemcpyAsync(host_cells.data(), d, n, cudaMemcpyDeviceToHost, ctx->stream);
    return cudaStreamSynchronize(ctx->stream) == cudaSuccess ? kOk : kCuda;
}

// voxelize_placed into d_out over `requested` (device).  `support`, when
// given, receives a box (cells of `requested`, possibly reaching past its
// edges) outside which every output cell is zero.
int placed_field(spk_context* ctx, const geo::Prepared& prepared, const geo::Window& requested, const double* origin,
                 double pitch, const geo::Vec3& translation, const geo::Quat& q, double clearance,
                 std::uint8_t* d_out, EdtBox* support = nullptr, const std::uint32_t* d_tris = nullptr,
                 const double* d_vertices = nullptr)
{
    if (!geo::canonical_unit(q)) {
        return kFieldInput;
    }
    std::uint64_t halo = 0;
    if (!geo::clearance_halo(clearance, pitch, halo)) {
        return kFieldInput;
    }
    const geo::Window work = expanded(requested, halo);
    geo::Placed placed;
    // With the item's vertices on the device, a non-cardinal pose's vertex
    // intervals are computed there (the host reads back only their bounds).
    bool on_device = false;
    int status = kOk;
    if (d_vertices && d_tris &&
        (status = place_on_device(ctx, prepared, d_vertices, translation, q, placed, on_device))) {
        return status;
    }
    if (!on_device && !geo::place(prepared, translation, q, placed)) {
        return kFieldInput;
    }
    geo::Window plan;
    const auto kind = geo::plan_placed_window(placed, work, origin, pitch, plan);
    const std::uint64_t n = cells_of(requested);
    if (kind == geo::PlanKind::certified_empty) {
        cudaMemsetAsync(d_out, 0, n, ctx->stream);
        if (support) {
            *support = {};
        }
        return kOk;
    }
    // The raster writes only inside `plan`; the clearance dilation reaches
    // `halo` cells further.  Outside that box the field is zero.
    int box_lo[3], box_hi[3];
    for (int a = 0; a < 3; ++a) {
        const long long h = static_cast<long long>(halo);
        const long long lo = plan.first[a] - h - requested.first[a];
        const long long hi = plan.first[a] + static_cast<long long>(plan.shape[a]) + h - requested.first[a];
        const long long top = static_cast<long long>(requested.shape[a]);
        if (support) {
            support->lo[a] = static_cast<int>(std::min(std::max(lo, -1LL), top + 1));
            support->hi[a] = static_cast<int>(std::min(std::max(hi, -1LL), top + 1));
        }
        box_lo[a] = static_cast<int>(std::min(std::max(lo, 0LL), top));
        box_hi[a] = static_cast<int>(std::min(std::max(hi, 0LL), top));
    }
    auto* raw = static_cast<std::uint8_t*>(device_buffer(ctx, "placed.raw", cells_of(plan), status));
    if (!raw) {
        return status;
    }
    if ((status = raster_fill(ctx, placed, make_window(plan, origin, pitch), raw, false, nullptr, d_tris,
                              on_device))) {
        return status;
    }
    return dilate_crop(ctx, raw, make_window(plan, origin, pitch), halo, clearance, false, d_out,
                       make_window(requested, origin, pitch), box_lo, box_hi);
}

// voxelize_container into d_out over `requested` (device).
int container_field(spk_context* ctx, const double* box, const geo::Prepared* prepared, const geo::Window& requested,
                    const double* origin, double pitch, double clearance, std::uint8_t* d_out)
{
    if (!std::isfinite(clearance) || clearance < 0.0) {
        return kFieldInput;
    }
    if (box) {
        for (int a = 0; a < 3; ++a) {
            if (!(box[a] > 0) || !std::isfinite(box[a])) {
                return kFieldInput;
            }
        }
        return box_mask(ctx, box, clearance, make_window(requested, origin, pitch), d_out);
    }
    std::uint64_t halo = 0;
    if (!geo::clearance_halo(clearance, pitch, halo)) {
        return kFieldInput;
    }
    const geo::Window work = expanded(requested, halo);
    geo::Placed placed;
    if (!geo::place(*prepared, { 0, 0, 0 }, { 0, 0, 0, 1 }, placed)) {
        return kFieldInput;
    }
    int status = kOk;
    auto* raw = static_cast<std::uint8_t*>(device_buffer(ctx, "container.raw", cells_of(work), status));
    if (!raw) {
        return status;
    }
    if ((status = raster_fill(ctx, placed, make_window(work, origin, pitch), raw, false))) {
        return status;
    }
    return dilate_crop(ctx, raw, make_window(work, origin, pitch), halo, clearance, true, d_out,
                       make_window(requested, origin, pitch));
}

struct Copy {
    std::uint64_t orientation;
    std::int64_t t[3];
};

struct Session {
    geo::Mesh object_mesh, container_mesh;
    geo::Prepared object, container;
    bool box {};
    double box_mm[3] {};
    double pair {}, wall {};
    double origin[3] {};
    double pitch {};
    geo::Window env {};
    double cmin_z {}, height {};
    std::vector<geo::Quat> catalog;
    std::vector<std::uint64_t> slot_of;  // orientation -> pipeline kernel slot
    std::unique_ptr<Pipeline> pipe;
    std::uint8_t* mask {};
    std::uint32_t* counts {};
    std::uint8_t* occ {};
    std::uint32_t* object_tris {};  // the item's triangle indices on the device (placed-copy rasters)
    double* object_vertices {};     // and its vertices
    std::vector<Copy> copies;
    bool dirty { true };
    __nv_bfloat16* items {};  // every orientation's kernel pooled to 32^3 (proposal input)
    bool items_ready {};
    std::uint64_t items_tag {};  // unique per session: names the pooled items for the network's cache
    spk_validate_fn validator {};  // the caller's native validation of a chosen pose (may be null)
    void* validator_user {};
    std::uint64_t validated {}, rejected {};
    // Set when the only change since the last refresh is one placed copy,
    // whose field is in "session.placed" with its support box: the EDT is
    // then updated in place rather than rebuilt.
    bool one_added {};
    EdtBox added_support {};
};

Session* session_of(spk_context* ctx) { return static_cast<Session*>(ctx->session); }

// The window box of a placed copy's support (its field is zero outside).
void support_box(const Session& s, const EdtBox& support, int (&shape)[3], int (&lo)[3], int (&hi)[3])
{
    for (int a = 0; a < 3; ++a) {
        shape[a] = static_cast<int>(s.env.shape[a]);
        lo[a] = std::min(std::max(support.lo[a], 0), shape[a]);
        hi[a] = std::min(std::max(support.hi[a], 0), shape[a]);
    }
}

// Brings the occupancy up to date on the context's stream and queues the
// pipeline's proximity and spectrum update on the pipeline's own stream
// (refresh_begin), so that work that needs only the occupancy (the
// proposal) runs beside it.
int refresh_async(spk_context* ctx, Session& s)
{
    if (!s.dirty) {
        return kOk;
    }
    s.pipe->refresh_order();
    const long long n = static_cast<long long>(cells_of(s.env));
    int status = kOk;
    if (s.one_added) {
        // One copy added to an up-to-date occupancy: only its support changes.
        int shape[3], lo[3], hi[3];
        support_box(s, s.added_support, shape, lo, hi);
        status = occupancy_box(ctx, s.mask, s.counts, s.occ, shape, lo, hi);
    }
    else {
        status = occupancy(ctx, s.mask, s.counts, s.occ, n);
    }
    if (status) {
        return status;
    }
    if (s.one_added) {
        auto* placed = static_cast<std::uint8_t*>(device_buffer(ctx, "session.placed", cells_of(s.env), status));
        if (!placed || (status = s.pipe->refresh_begin(s.occ, placed, &s.added_support))) {
            return status ? status : kAllocation;
        }
    }
    else if ((status = s.pipe->refresh_begin(s.occ, nullptr, nullptr))) {
        return status;
    }
    s.dirty = false;
    s.one_added = false;
    return kOk;
}

// The same, then the context's stream waits for the update.
int refresh(spk_context* ctx, Session& s)
{
    int status = refresh_async(ctx, s);
    if (!status) {
        s.pipe->refresh_order();
    }
    return status;
}

void to_c(const Candidate& c, spk_candidate& out)
{
    std::memset(&out, 0, sizeof(out));
    std::memcpy(out.translation, c.t, sizeof(out.translation));
    out.score = c.score;
    out.direct_zero_overlap = c.direct_zero ? 1 : 0;
    out.orientation_index = c.orientation;
    out.binary_overlap = c.binary_overlap;
}

Candidate from_c(const spk_candidate& c)
{
    Candidate out {};
    std::memcpy(out.t, c.translation, sizeof(out.t));
    out.score = c.score;
    out.direct_zero = c.direct_zero_overlap != 0;
    out.orientation = c.orientation_index;
    out.binary_overlap = c.binary_overlap;
    return out;
}

bool rank_less(const Candidate& l, const Candidate& r)
{
    if (l.score != r.score) {
        return l.score < r.score;
    }
    if (l.orientation != r.orientation) {
        return l.orientation < r.orientation;
    }
    return std::tie(l.t[2], l.t[1], l.t[0]) < std::tie(r.t[2], r.t[1], r.t[0]);
}

// Copy counts +1 / -1 under a placed copy's field, over its support only.
int stamp_support(spk_context* ctx, Session& s, const std::uint8_t* placed, const EdtBox& support, int direction)
{
    int shape[3], lo[3], hi[3];
    support_box(s, support, shape, lo, hi);
    return stamp_box(ctx, s.counts, placed, shape, lo, hi, direction);
}

int session_place(spk_context* ctx, Session& s, std::uint64_t orientation, const std::int64_t* t)
{
    if (orientation >= s.catalog.size()) {
        return kCatalog;
    }
    s.pipe->refresh_order();  // a queued update may still read the placed-copy buffer
    const geo::Vec3 translation { s.origin[0] + s.pitch * static_cast<double>(t[0]),
                                  s.origin[1] + s.pitch * static_cast<double>(t[1]),
                                  s.origin[2] + s.pitch * static_cast<double>(t[2]) };
    int status = kOk;
    auto* placed = static_cast<std::uint8_t*>(device_buffer(ctx, "session.placed", cells_of(s.env), status));
    if (!placed) {
        return status;
    }
    EdtBox support {};
    if ((status = placed_field(ctx, s.object, s.env, s.origin, s.pitch, translation, s.catalog[orientation], s.pair,
                               placed, &support, s.object_tris, s.object_vertices))) {
        return status;
    }
    if ((status = stamp_support(ctx, s, placed, support, 1))) {
        return status;
    }
    s.copies.push_back({ orientation, { t[0], t[1], t[2] } });
    // One copy added to an up-to-date layout: its EDT can be updated in place.
    s.one_added = !s.dirty;
    s.added_support = support;
    s.dirty = true;
    return kOk;
}

int session_pages_mode(spk_context* ctx, Session& s, const std::vector<PageRequest>& requests,
                       std::vector<PageOutcome>& out, bool full)
{
    int status = refresh(ctx, s);
    if (status) {
        return status;
    }
    return s.pipe->pages(requests, out, full);
}

int session_pages(spk_context* ctx, Session& s, const std::vector<PageRequest>& requests, std::vector<PageOutcome>& out)
{
    return session_pages_mode(ctx, s, requests, out, true);
}

// One greedy placement over the orientations in `subset`: the page merge of
// spectral.cpp:1460-1591.  Pages come from the first pass; an entry is exact
// once its score is <= that page's exact floor.  An orientation whose next
// entry is not yet exact is resolved (certified page) only when its lower
// bound could reach the current best head.  Places the chosen candidate and
// returns it in `chosen` (empty when no orientation of the subset admits one).
//
// Widening (the learned proposal's adaptive policy): `reserve` lists further
// orientations in the order they should join.  After the subset's first
// pages are loaded, while fewer than `min_feasible` of the active
// orientations have a non-empty page, the next `block` orientations of the
// reserve are activated and paged before anything is chosen.  With an empty
// reserve this is the plain merge over `subset`.
int greedy_step(spk_context* ctx, Session& s, const std::vector<std::size_t>& subset, std::optional<Candidate>& chosen,
                const std::vector<std::size_t>& reserve = {}, std::size_t min_feasible = 0, std::size_t block = 0,
                std::size_t* widened = nullptr)
{
    chosen.reset();
    std::size_t next_reserve = 0;
    const std::size_t O = s.catalog.size();
    std::vector<bool> active(O, false);
    for (std::size_t o : subset) {
        if (o < O) {
            active[o] = true;
        }
    }
    std::vector<std::vector<Candidate>> pages(O);
    std::vector<std::size_t> index(O, 0);
    std::vector<double> floor(O, -INFINITY);
    std::vector<std::optional<Candidate>> cursors(O);
    std::vector<bool> exhausted(O, false), loaded(O, false);
    for (std::size_t o = 0; o < O; ++o) {
        exhausted[o] = !active[o];
    }
    for (;;) {
        // (Re)load pages that are consumed: lazily, all at once.
        std::vector<PageRequest> requests;
        std::vector<std::size_t> which;
        for (std::size_t o = 0; o < O; ++o) {
            if (exhausted[o] || (loaded[o] && index[o] != pages[o].size())) {
                continue;
            }
            if (loaded[o] && floor[o] == INFINITY) {
                exhausted[o] = true;  // a complete page was fully consumed
                continue;
            }
            PageRequest r;
            r.slot = s.slot_of[o];
            r.has_cursor = cursors[o].has_value();
            if (r.has_cursor) {
                r.cursor = *cursors[o];
            }
            requests.push_back(r);
            which.push_back(o);
        }
        if (!requests.empty()) {
            std::vector<PageOutcome> out;
            int status = session_pages_mode(ctx, s, requests, out, false);
            if (status) {
                return status;
            }
            for (std::size_t k = 0; k < which.size(); ++k) {
                if (out[k].status) {
                    return out[k].status;
                }
                const auto o = which[k];
                pages[o] = std::move(out[k].page);
                index[o] = 0;
                floor[o] = out[k].exact_floor;
                loaded[o] = true;
                if (pages[o].empty() && floor[o] == INFINITY) {
                    exhausted[o] = true;
                }
            }
            // Widen while too few active orientations admit a copy.
            if (next_reserve < reserve.size() && block > 0) {
                std::size_t feasible = 0;
                for (std::size_t o = 0; o < O; ++o) {
                    feasible += active[o] && !pages[o].empty() ? 1 : 0;
                }
                if (feasible < min_feasible) {
                    for (std::size_t added = 0; added < block && next_reserve < reserve.size(); ++next_reserve) {
                        const std::size_t o = reserve[next_reserve];
                        if (o < O && !active[o]) {
                            active[o] = true;
                            exhausted[o] = false;
                            ++added;
                        }
                    }
                    if (widened) {
                        ++*widened;
                    }
                    continue;
                }
                next_reserve = reserve.size();  // enough feasible orientations: no more widening
            }
        }
        // Best exact head.
        std::optional<std::size_t> best;
        for (std::size_t o = 0; o < O; ++o) {
            if (exhausted[o] || index[o] >= pages[o].size() || pages[o][index[o]].score > floor[o]) {
                continue;
            }
            if (!best || rank_less(pages[o][index[o]], pages[*best][index[*best]])) {
                best = o;
            }
        }
        // Orientations whose next exact candidate could precede it.
        std::vector<PageRequest> resolve;
        std::vector<std::size_t> resolve_which;
        for (std::size_t o = 0; o < O; ++o) {
            if (exhausted[o]) {
                continue;
            }
            const bool exact_next = index[o] < pages[o].size() && pages[o][index[o]].score <= floor[o];
            if (exact_next) {
                continue;
            }
            double lower = floor[o];
            if (index[o] < pages[o].size()) {
                lower = std::min(lower, pages[o][index[o]].score);
            }
            if (best && lower > pages[*best][index[*best]].score) {
                continue;
            }
            PageRequest r;
            r.slot = s.slot_of[o];
            r.has_cursor = cursors[o].has_value();
            if (r.has_cursor) {
                r.cursor = *cursors[o];
            }
            resolve.push_back(r);
            resolve_which.push_back(o);
        }
        if (!resolve.empty()) {
            std::vector<PageOutcome> out;
            int status = session_pages_mode(ctx, s, resolve, out, true);
            if (status) {
                return status;
            }
            for (std::size_t k = 0; k < resolve_which.size(); ++k) {
                if (out[k].status) {
                    return out[k].status;
                }
                const auto o = resolve_which[k];
                pages[o] = std::move(out[k].page);
                index[o] = 0;
                floor[o] = out[k].page.size() == static_cast<std::size_t>(kPageSize) || !out[k].certified
                               ? out[k].exact_floor
                               : INFINITY;
                if (out[k].certified && floor[o] < INFINITY && !pages[o].empty()) {
                    floor[o] = std::max(floor[o], pages[o].back().score);
                }
                loaded[o] = true;
                if (pages[o].empty()) {
                    exhausted[o] = true;
                }
            }
            continue;
        }
        if (!best) {
            break;
        }
        const Candidate c = pages[*best][index[*best]++];
        cursors[*best] = c;
        if (!c.direct_zero) {
            continue;
        }
        // The reference's try_pose: the pose goes to native validation before
        // it joins the layout; a rejected pose leaves the layout unchanged and
        // the merge moves on to the next candidate (spectral.cpp:1289-1430,
        // called at :1571-1591).
        if (s.validator) {
            const double pose[3] = { s.origin[0] + s.pitch * static_cast<double>(c.t[0]),
                                     s.origin[1] + s.pitch * static_cast<double>(c.t[1]),
                                     s.origin[2] + s.pitch * static_cast<double>(c.t[2]) };
            const geo::Quat& q = s.catalog[c.orientation];
            const int verdict = s.validator(s.validator_user, c.orientation, c.t, pose, q.data());
            ++s.validated;
            if (verdict == SPK_POSE_REJECTED) {
                ++s.rejected;
                continue;
            }
            if (verdict != SPK_POSE_ACCEPTED) {
                return kValidationAborted;
            }
        }
        int status = session_place(ctx, s, c.orientation, c.t);
        if (status) {
            return status;
        }
        chosen = c;
        break;
    }
    return kOk;
}

void record(const Candidate& c, std::uint64_t i, std::uint64_t* orientations, std::int64_t* translations,
            double* scores)
{
    if (orientations) {
        orientations[i] = c.orientation;
    }
    if (translations) {
        for (int a = 0; a < 3; ++a) {
            translations[3 * i + a] = c.t[a];
        }
    }
    if (scores) {
        scores[i] = c.score;
    }
}

// Pools every orientation's kernel field to the proposal grid (once per session).
int session_items(spk_context* ctx, Session& s)
{
    if (s.items_ready) {
        return kOk;
    }
    const std::size_t O = s.catalog.size();
    int status = kOk;
    s.items = static_cast<__nv_bfloat16*>(
        device_buffer(ctx, "session.items", O * kProposalVoxels * sizeof(__nv_bfloat16), status));
    if (!s.items) {
        return status;
    }
    std::size_t most = 1;
    for (std::size_t o = 0; o < O; ++o) {
        most = std::max(most, s.pipe->slot(s.slot_of[o]).host_cells.size());
    }
    auto* cells = static_cast<std::uint8_t*>(device_buffer(ctx, "session.item_cells", most * O, status));
    if (!cells) {
        return status;
    }
    for (std::size_t o = 0; o < O; ++o) {
        const KernelSlot& k = s.pipe->slot(s.slot_of[o]);
        cudaMemcpyAsync(cells + o * most, k.host_cells.data(), k.host_cells.size(), cudaMemcpyHostToDevice,
                        ctx->stream);
        if ((status = pool_item(ctx, cells + o * most, k.K, s.items + o * kProposalVoxels))) {
            return status;
        }
    }
    if (cudaStreamSynchronize(ctx->stream) != cudaSuccess) {
        cudaGetLastError();
        return kCuda;
    }
    static std::atomic<std::uint64_t> next_tag { 1 };
    s.items_tag = next_tag++;
    s.items_ready = true;
    return kOk;
}

// Pools the current occupancy to the proposal grid.
int session_crop(spk_context* ctx, Session& s, __nv_bfloat16*& crop)
{
    int status = refresh_async(ctx, s);
    if (status) {
        return status;
    }
    crop = static_cast<__nv_bfloat16*>(
        device_buffer(ctx, "session.crop", kProposalVoxels * sizeof(__nv_bfloat16), status));
    if (!crop) {
        return status;
    }
    const int shape[3] = { static_cast<int>(s.env.shape[0]), static_cast<int>(s.env.shape[1]),
                           static_cast<int>(s.env.shape[2]) };
    return pool_occupancy(ctx, s.occ, shape, crop);
}

// Network score of every orientation for the current layout (host copy).
int session_predict(spk_context* ctx, Session& s, ProposalNet* net, std::vector<float>& pred)
{
    int status = session_items(ctx, s);
    __nv_bfloat16* crop {};
    if (!status) {
        status = session_crop(ctx, s, crop);
    }
    if (status) {
        return status;
    }
    const std::size_t O = s.catalog.size();
    auto* d = static_cast<float*>(device_buffer(ctx, "session.pred", O * sizeof(float), status));
    if (!d) {
        return status;
    }
    if ((status = proposal_predict(ctx, net, static_cast<std::uint32_t>(O), crop, nullptr, s.items, nullptr, s.items_tag,
                                   d))) {
        return status;
    }
    pred.resize(O);
    cudaMemcpyAsync(pred.data(), d, O * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream);
    if (cudaStreamSynchronize(ctx->stream) != cudaSuccess) {
        cudaGetLastError();
        return kCuda;
    }
    return kOk;
}

// The k orientations with the lowest predicted score (ties: lower index).
std::vector<std::size_t> top_k(const std::vector<float>& pred, std::size_t k)
{
    std::vector<std::size_t> order(pred.size());
    for (std::size_t o = 0; o < order.size(); ++o) {
        order[o] = o;
    }
    k = std::min(k, order.size());
    std::partial_sort(order.begin(), order.begin() + static_cast<std::ptrdiff_t>(k), order.end(),
                      [&](std::size_t a, std::size_t b) {
                          const float pa = std::isnan(pred[a]) ? INFINITY : pred[a];
                          const float pb = std::isnan(pred[b]) ? INFINITY : pred[b];
                          return pa != pb ? pa < pb : a < b;
                      });
    order.resize(k);
    return order;
}

}  // namespace

void session_destroy(spk_context* ctx)
{
    delete session_of(ctx);
    ctx->session = nullptr;
}

}  // namespace spk

using namespace spk;

extern "C" {

int spk_voxelize_object(spk_context* ctx, const spk_mesh* object, const double origin[3], double pitch,
                        const double q[4], int64_t first[3], uint32_t shape[3], uint8_t* cells, uint64_t capacity)
{
    try {
        if (!ctx || !valid_mesh(object) || !origin || !q || !first || !shape || !valid_lattice(origin, pitch)) {
            return kFieldInput;
        }
        if (cudaSetDevice(ctx->device) != cudaSuccess) {
            return kCuda;
        }
        const geo::Mesh mesh = to_mesh(*object);
        const geo::Prepared prepared = geo::prepare(mesh);
        geo::Window w;
        std::vector<std::uint8_t> host;
        int status = object_field(ctx, prepared, origin, pitch, { q[0], q[1], q[2], q[3] }, w, host);
        if (status) {
            return status;
        }
        for (int a = 0; a < 3; ++a) {
            first[a] = w.first[a];
            shape[a] = w.shape[a];
        }
        if (!cells || capacity < host.size()) {
            return kInvalidArgument;
        }
        std::memcpy(cells, host.data(), host.size());
        return kOk;
    }
    catch (...) {
        return kAllocation;
    }
}

int spk_voxelize_container(spk_context* ctx, const double box[3], const spk_mesh* container, const double origin[3],
                           double pitch, const int64_t first[3], const uint32_t shape[3], double clearance,
                           uint8_t* cells)
{
    try {
        if (!ctx || !origin || !first || !shape || !cells || !valid_lattice(origin, pitch) ||
            (!box && !valid_mesh(container))) {
            return kFieldInput;
        }
        if (cudaSetDevice(ctx->device) != cudaSuccess) {
            return kCuda;
        }
        geo::Window w;
        for (int a = 0; a < 3; ++a) {
            w.first[a] = first[a];
            w.shape[a] = shape[a];
        }
        geo::Mesh mesh;
        geo::Prepared prepared;
        if (!box) {
            mesh = to_mesh(*container);
            prepared = geo::prepare(mesh);
        }
        int status = kOk;
        auto* d = static_cast<std::uint8_t*>(device_buffer(ctx, "api.container", cells_of(w), status));
        if (!d) {
            return status;
        }
        if ((status = container_field(ctx, box, box ? nullptr : &prepared, w, origin, pitch, clearance, d))) {
            return status;
        }
        cudaMemcpyAsync(cells, d, cells_of(w), cudaMemcpyDeviceToHost, ctx->stream);
        return cudaStreamSynchronize(ctx->stream) == cudaSuccess ? kOk : kCuda;
    }
    catch (...) {
        return kAllocation;
    }
}

int spk_voxelize_placed(spk_context* ctx, const spk_mesh* object, const double origin[3], double pitch,
                        const int64_t first[3], const uint32_t shape[3], const double translation[3],
                        const double q[4], double clearance, uint8_t* cells)
{
    try {
        if (!ctx || !valid_mesh(object) || !origin || !first || !shape || !translation || !q || !cells ||
            !valid_lattice(origin, pitch)) {
            return kFieldInput;
        }
        if (cudaSetDevice(ctx->device) != cudaSuccess) {
            return kCuda;
        }
        geo::Window w;
        for (int a = 0; a < 3; ++a) {
            w.first[a] = first[a];
            w.shape[a] = shape[a];
        }
        const geo::Mesh mesh = to_mesh(*object);
        const geo::Prepared prepared = geo::prepare(mesh);
        int status = kOk;
        auto* d = static_cast<std::uint8_t*>(device_buffer(ctx, "api.placed", cells_of(w), status));
        if (!d) {
            return status;
        }
        if ((status = placed_field(ctx, prepared, w, origin, pitch, { translation[0], translation[1], translation[2] },
                                   { q[0], q[1], q[2], q[3] }, clearance, d))) {
            return status;
        }
        cudaMemcpyAsync(cells, d, cells_of(w), cudaMemcpyDeviceToHost, ctx->stream);
        return cudaStreamSynchronize(ctx->stream) == cudaSuccess ? kOk : kCuda;
    }
    catch (...) {
        return kAllocation;
    }
}

int spk_oriented_bounds(const spk_mesh* object, const double q[4], double bounds[6])
{
    try {
        if (!valid_mesh(object) || !q || !bounds) {
            return kFieldInput;
        }
        const geo::Mesh mesh = to_mesh(*object);
        geo::Bounds b;
        if (!geo::oriented_bounds(mesh, { q[0], q[1], q[2], q[3] }, b)) {
            return kFieldInput;
        }
        for (int a = 0; a < 3; ++a) {
            bounds[a] = b.min[a];
            bounds[3 + a] = b.max[a];
        }
        return kOk;
    }
    catch (...) {
        return kAllocation;
    }
}

int spk_posed_bounds(const spk_mesh* object, const double* translations_mm, const double* q_xyzw, uint64_t count,
                     double* bounds_min, double* bounds_max, uint8_t* finite)
{
    try {
        if (!valid_mesh(object) || (count && (!translations_mm || !q_xyzw || !bounds_min || !bounds_max || !finite))) {
            return kFieldInput;
        }
        const geo::Mesh mesh = to_mesh(*object);
        for (uint64_t i = 0; i < count; ++i) {
            geo::Bounds b;
            const double* t = translations_mm + 3 * i;
            const double* q = q_xyzw + 4 * i;
            const bool ok = geo::posed_bounds(mesh, { t[0], t[1], t[2] }, { q[0], q[1], q[2], q[3] }, b);
            finite[i] = ok ? 1 : 0;
            for (int a = 0; a < 3; ++a) {
                bounds_min[3 * i + a] = ok ? b.min[a] : 0.0;
                bounds_max[3 * i + a] = ok ? b.max[a] : 0.0;
            }
        }
        return kOk;
    }
    catch (...) {
        return kAllocation;
    }
}

int spk_environment_window(const double bounds[6], const double origin[3], double pitch, int64_t first[3],
                           uint32_t shape[3])
{
    if (!bounds || !origin || !first || !shape || !valid_lattice(origin, pitch)) {
        return kFieldInput;
    }
    geo::Bounds b { { bounds[0], bounds[1], bounds[2] }, { bounds[3], bounds[4], bounds[5] } };
    geo::Window w;
    if (!geo::environment_window(b, origin, pitch, w)) {
        return kFieldIndexOverflow;
    }
    for (int a = 0; a < 3; ++a) {
        first[a] = w.first[a];
        shape[a] = w.shape[a];
    }
    return kOk;
}

int spk_cube_catalog(double out[96])
{
    if (!out) {
        return kInvalidArgument;
    }
    try {
        const auto cube = geo::cube_catalog();
        for (int i = 0; i < 24; ++i) {
            for (int k = 0; k < 4; ++k) {
                out[4 * i + k] = cube[i][k];
            }
        }
        return kOk;
    }
    catch (...) {
        return kAllocation;
    }
}

int spk_custom_catalog(const double* in, uint64_t count, double* out, uint64_t* out_count)
{
    if (!in || !out || !out_count || count == 0) {
        return kCatalog;
    }
    try {
        std::vector<geo::Quat> result;
        for (std::uint64_t i = 0; i < count; ++i) {
            const geo::Quat q { in[4 * i], in[4 * i + 1], in[4 * i + 2], in[4 * i + 3] };
            const double n = std::hypot(std::hypot(q[0], q[1]), std::hypot(q[2], q[3]));
            if (!std::isfinite(n) || !(n > 0)) {
                return kCatalog;
            }
            const auto c = geo::canonical(q);
            if (std::find(result.begin(), result.end(), c) == result.end()) {
                result.push_back(c);
            }
        }
        for (std::size_t i = 0; i < result.size(); ++i) {
            for (int k = 0; k < 4; ++k) {
                out[4 * i + k] = result[i][k];
            }
        }
        *out_count = result.size();
        return kOk;
    }
    catch (...) {
        return kAllocation;
    }
}

int spk_session_open(spk_context* ctx, const spk_session_desc* d, spk_session_info* info)
{
    try {
        if (!ctx || !d || !valid_mesh(&d->object) || !valid_lattice(d->lattice_origin_mm, d->lattice_pitch_mm) ||
            !d->orientations_xyzw || !d->orientation_count || (!d->container_is_box && !valid_mesh(&d->container))) {
            return kFieldInput;
        }
        if (cudaSetDevice(ctx->device) != cudaSuccess) {
            return kCuda;
        }
        session_destroy(ctx);
        auto s = std::make_unique<Session>();
        s->object_mesh = to_mesh(d->object);
        s->object = geo::prepare(s->object_mesh);
        s->box = d->container_is_box != 0;
        geo::Bounds cb;
        if (s->box) {
            for (int a = 0; a < 3; ++a) {
                s->box_mm[a] = d->box_mm[a];
            }
            cb = { { 0, 0, 0 }, { d->box_mm[0], d->box_mm[1], d->box_mm[2] } };
        }
        else {
            s->container_mesh = to_mesh(d->container);
            s->container = geo::prepare(s->container_mesh);
            cb = s->container_mesh.bounds;
        }
        s->pair = d->pair_clearance_mm;
        s->wall = d->wall_clearance_mm;
        for (int a = 0; a < 3; ++a) {
            s->origin[a] = d->lattice_origin_mm[a];
        }
        s->pitch = d->lattice_pitch_mm;
        if (!geo::environment_window(cb, s->origin, s->pitch, s->env)) {
            return kFieldIndexOverflow;
        }
        s->cmin_z = cb.min[2];
        s->height = cb.max[2] - cb.min[2];
        if (!std::isfinite(s->height) || s->height <= 0.) {
            return kFieldInput;
        }
        for (std::uint64_t i = 0; i < d->orientation_count; ++i) {
            s->catalog.push_back({ d->orientations_xyzw[4 * i], d->orientations_xyzw[4 * i + 1],
                                   d->orientations_xyzw[4 * i + 2], d->orientations_xyzw[4 * i + 3] });
        }
        const std::uint64_t n = cells_of(s->env);
        int status = kOk;
        s->mask = static_cast<std::uint8_t*>(device_buffer(ctx, "session.mask", n, status));
        s->counts = static_cast<std::uint32_t*>(device_buffer(ctx, "session.counts", n * 4, status));
        s->occ = static_cast<std::uint8_t*>(device_buffer(ctx, "session.occ", n, status));
        const std::size_t tri_bytes = s->object_mesh.triangles.size() * 12;
        const std::size_t vertex_bytes = s->object_mesh.vertices.size() * 24;
        s->object_tris = static_cast<std::uint32_t*>(device_buffer(ctx, "session.object_tris", tri_bytes, status));
        s->object_vertices = static_cast<double*>(device_buffer(ctx, "session.object_vertices", vertex_bytes, status));
        if (!s->mask || !s->counts || !s->occ || !s->object_tris || !s->object_vertices) {
            return status;
        }
        cudaMemcpyAsync(s->object_tris, s->object_mesh.triangles.data(), tri_bytes, cudaMemcpyHostToDevice,
                        ctx->stream);
        cudaMemcpyAsync(s->object_vertices, s->object_mesh.vertices.data(), vertex_bytes, cudaMemcpyHostToDevice,
                        ctx->stream);
        cudaMemsetAsync(s->counts, 0, n * 4, ctx->stream);
        if ((status = container_field(ctx, s->box ? s->box_mm : nullptr, s->box ? nullptr : &s->container, s->env,
                                      s->origin, s->pitch, s->wall, s->mask))) {
            return status;
        }
        s->pipe = std::make_unique<Pipeline>(ctx);
        if ((status = s->pipe->set_geometry(s->env.first, s->env.shape, s->origin, s->pitch, s->cmin_z, s->height))) {
            return status;
        }
        for (std::uint64_t o = 0; o < s->catalog.size(); ++o) {
            geo::Window w;
            std::vector<std::uint8_t> cells;
            if ((status = object_field(ctx, s->object, s->origin, s->pitch, s->catalog[o], w, cells))) {
                return status;
            }
            geo::Bounds ob;
            if (!geo::oriented_bounds(s->object_mesh, s->catalog[o], ob)) {
                return kFieldInput;
            }
            std::uint64_t slot = 0;
            if ((status = s->pipe->add_kernel(o, w.first, w.shape, cells.data(), ob.max[2], slot))) {
                return status;
            }
            s->slot_of.push_back(slot);
        }
        ctx->session = s.release();
        return spk_session_info_get(ctx, info);
    }
    catch (...) {
        return kAllocation;
    }
}

int spk_session_close(spk_context* ctx)
{
    if (!ctx) {
        return kInvalidArgument;
    }
    session_destroy(ctx);
    return kOk;
}

int spk_session_info_get(spk_context* ctx, spk_session_info* info)
{
    if (!ctx || !session_of(ctx)) {
        return kNotReady;
    }
    if (!info) {
        return kOk;
    }
    const auto& s = *session_of(ctx);
    for (int a = 0; a < 3; ++a) {
        info->environment_first[a] = s.env.first[a];
        info->environment_shape[a] = s.env.shape[a];
        info->fft_shape[a] = static_cast<std::uint32_t>(s.pipe->fft_shape()[a]);
    }
    info->copies = s.copies.size();
    info->orientations = s.catalog.size();
    info->container_min_z_mm = s.cmin_z;
    info->container_height_mm = s.height;
    return kOk;
}

int spk_session_place(spk_context* ctx, uint64_t orientation, const int64_t translation[3])
{
    try {
        if (!ctx || !session_of(ctx) || !translation) {
            return kNotReady;
        }
        if (cudaSetDevice(ctx->device) != cudaSuccess) {
            return kCuda;
        }
        return session_place(ctx, *session_of(ctx), orientation, translation);
    }
    catch (...) {
        return kAllocation;
    }
}

int spk_session_remove_last(spk_context* ctx)
{
    try {
        if (!ctx || !session_of(ctx) || session_of(ctx)->copies.empty()) {
            return kNotReady;
        }
        auto& s = *session_of(ctx);
        s.pipe->refresh_order();  // a queued update may still read the placed-copy buffer
        const Copy c = s.copies.back();
        const geo::Vec3 translation { s.origin[0] + s.pitch * static_cast<double>(c.t[0]),
                                      s.origin[1] + s.pitch * static_cast<double>(c.t[1]),
                                      s.origin[2] + s.pitch * static_cast<double>(c.t[2]) };
        int status = kOk;
        auto* placed = static_cast<std::uint8_t*>(device_buffer(ctx, "session.placed", cells_of(s.env), status));
        if (!placed) {
            return status;
        }
        EdtBox support {};
        if ((status = placed_field(ctx, s.object, s.env, s.origin, s.pitch, translation, s.catalog[c.orientation],
                                   s.pair, placed, &support, s.object_tris, s.object_vertices))) {
            return status;
        }
        if ((status = stamp_support(ctx, s, placed, support, -1))) {
            return status;
        }
        s.copies.pop_back();
        s.dirty = true;
        s.one_added = false;  // distances can grow: rebuild
        return kOk;
    }
    catch (...) {
        return kAllocation;
    }
}

int spk_session_pages(spk_context* ctx, uint64_t n, const spk_page_query* queries, spk_candidate* pages,
                      uint32_t* counts, spk_page_report* reports)
{
    try {
        if (!ctx || !session_of(ctx)) {
            return kNotReady;
        }
        if (!queries || !pages || !counts) {
            return kInvalidArgument;
        }
        auto& s = *session_of(ctx);
        std::vector<PageRequest> requests(n);
        for (std::uint64_t i = 0; i < n; ++i) {
            if (queries[i].orientation_index >= s.catalog.size()) {
                return kCatalog;
            }
            if (queries[i].mode > 1) {
                return kInvalidArgument;  // 0 ordinary, 1 low-overlap
            }
            requests[i].slot = s.slot_of[queries[i].orientation_index];
            requests[i].low_overlap = queries[i].mode == 1;
            requests[i].has_cursor = queries[i].has_cursor != 0;
            if (requests[i].has_cursor) {
                requests[i].cursor = from_c(queries[i].exclusive_cursor);
            }
        }
        std::vector<PageOutcome> out;
        int status = session_pages(ctx, s, requests, out);
        if (status) {
            return status;
        }
        for (std::uint64_t i = 0; i < n; ++i) {
            if (out[i].status) {
                return out[i].status;
            }
            counts[i] = static_cast<std::uint32_t>(out[i].page.size());
            for (std::size_t k = 0; k < out[i].page.size(); ++k) {
                to_c(out[i].page[k], pages[i * kPageSize + k]);
            }
            if (reports) {
                reports[i].max_integer_residual = out[i].max_integer_residual;
                reports[i].max_score_error = out[i].max_score_error;
                reports[i].rescored = out[i].rescored;
                reports[i].certified = out[i].certified ? 1 : 0;
                reports[i].threshold_pass = out[i].threshold_pass ? 1 : 0;
            }
        }
        return kOk;
    }
    catch (...) {
        return kAllocation;
    }
}

int spk_session_greedy(spk_context* ctx, uint64_t max_steps, uint64_t* placed, uint64_t* orientations,
                       int64_t* translations, double* scores)
{
    try {
        if (!ctx || !session_of(ctx) || !placed) {
            return kNotReady;
        }
        auto& s = *session_of(ctx);
        *placed = 0;
        std::vector<std::size_t> all(s.catalog.size());
        for (std::size_t o = 0; o < all.size(); ++o) {
            all[o] = o;
        }
        while (*placed < max_steps) {
            std::optional<Candidate> chosen;
            int status = greedy_step(ctx, s, all, chosen);
            if (status) {
                return status;
            }
            if (!chosen) {
                break;
            }
            record(*chosen, *placed, orientations, translations, scores);
            ++*placed;
        }
        return kOk;
    }
    catch (...) {
        return kAllocation;
    }
}

int spk_session_set_validator(spk_context* ctx, spk_validate_fn validator, void* user)
{
    if (!ctx || !session_of(ctx)) {
        return kNotReady;
    }
    auto& s = *session_of(ctx);
    s.validator = validator;
    s.validator_user = user;
    return kOk;
}

int spk_session_validation_counts(spk_context* ctx, uint64_t* validated, uint64_t* rejected)
{
    if (!ctx || !session_of(ctx)) {
        return kNotReady;
    }
    if (!validated || !rejected) {
        return kInvalidArgument;
    }
    *validated = session_of(ctx)->validated;
    *rejected = session_of(ctx)->rejected;
    return kOk;
}

int spk_session_features(spk_context* ctx, float* crop, float* items)
{
    try {
        if (!ctx || !session_of(ctx)) {
            return kNotReady;
        }
        auto& s = *session_of(ctx);
        const std::size_t O = s.catalog.size();
        int status = kOk;
        std::vector<std::uint16_t> host;
        if (crop) {
            __nv_bfloat16* d {};
            if ((status = session_crop(ctx, s, d))) {
                return status;
            }
            host.resize(kProposalVoxels);
            cudaMemcpyAsync(host.data(), d, kProposalVoxels * 2, cudaMemcpyDeviceToHost, ctx->stream);
            if (cudaStreamSynchronize(ctx->stream) != cudaSuccess) {
                return kCuda;
            }
            for (int v = 0; v < kProposalVoxels; ++v) {
                const std::uint32_t bits = static_cast<std::uint32_t>(host[v]) << 16;
                std::memcpy(crop + v, &bits, 4);
            }
        }
        if (items) {
            if ((status = session_items(ctx, s))) {
                return status;
            }
            host.resize(O * kProposalVoxels);
            cudaMemcpyAsync(host.data(), s.items, host.size() * 2, cudaMemcpyDeviceToHost, ctx->stream);
            if (cudaStreamSynchronize(ctx->stream) != cudaSuccess) {
                return kCuda;
            }
            for (std::size_t v = 0; v < host.size(); ++v) {
                const std::uint32_t bits = static_cast<std::uint32_t>(host[v]) << 16;
                std::memcpy(items + v, &bits, 4);
            }
        }
        return kOk;
    }
    catch (...) {
        return kAllocation;
    }
}

int spk_session_propose(spk_context* ctx, spk_proposal* proposal, uint32_t k, uint64_t* orientations,
                        float* predictions)
{
    try {
        if (!ctx || !session_of(ctx)) {
            return kNotReady;
        }
        ProposalNet* net = proposal_net(proposal);
        if (!net || (k && !orientations)) {
            return kInvalidArgument;
        }
        auto& s = *session_of(ctx);
        std::vector<float> pred;
        int status = session_predict(ctx, s, net, pred);
        if (status) {
            return status;
        }
        if (predictions) {
            std::memcpy(predictions, pred.data(), pred.size() * sizeof(float));
        }
        const auto best = top_k(pred, k);
        for (std::size_t i = 0; i < best.size(); ++i) {
            orientations[i] = best[i];
        }
        return kOk;
    }
    catch (...) {
        return kAllocation;
    }
}

int spk_session_greedy_proposed(spk_context* ctx, spk_proposal* proposal, uint32_t k, uint64_t max_steps,
                                uint64_t* placed, uint64_t* orientations, int64_t* translations, double* scores,
                                uint64_t* fallbacks)
{
    try {
        if (!ctx || !session_of(ctx) || !placed) {
            return kNotReady;
        }
        ProposalNet* net = proposal_net(proposal);
        if (!net || k == 0) {
            return kInvalidArgument;
        }
        auto& s = *session_of(ctx);
        *placed = 0;
        if (fallbacks) {
            *fallbacks = 0;
        }
        std::vector<std::size_t> all(s.catalog.size());
        for (std::size_t o = 0; o < all.size(); ++o) {
            all[o] = o;
        }
        std::vector<float> pred;
        while (*placed < max_steps) {
            int status = session_predict(ctx, s, net, pred);
            if (status) {
                return status;
            }
            std::optional<Candidate> chosen;
            if ((status = greedy_step(ctx, s, top_k(pred, k), chosen))) {
                return status;
            }
            if (!chosen) {
                // No proposed orientation admits a copy: the exhaustive step decides.
                if ((status = greedy_step(ctx, s, all, chosen))) {
                    return status;
                }
                if (!chosen) {
                    break;
                }
                if (fallbacks) {
                    ++*fallbacks;
                }
            }
            record(*chosen, *placed, orientations, translations, scores);
            ++*placed;
        }
        return kOk;
    }
    catch (...) {
        return kAllocation;
    }
}

int spk_session_greedy_proposed_margin(spk_context* ctx, spk_proposal* proposal, uint32_t k_min, uint32_t k_max,
                                       float margin, uint64_t max_steps, uint64_t* placed, uint64_t* orientations,
                                       int64_t* translations, double* scores, uint64_t* fallbacks, uint64_t* paged)
{
    try {
        if (!ctx || !session_of(ctx) || !placed) {
            return kNotReady;
        }
        ProposalNet* net = proposal_net(proposal);
        if (!net || k_min == 0 || k_max < k_min || !(margin >= 0.f)) {
            return kInvalidArgument;
        }
        auto& s = *session_of(ctx);
        *placed = 0;
        if (fallbacks) {
            *fallbacks = 0;
        }
        if (paged) {
            *paged = 0;
        }
        const std::size_t O = s.catalog.size();
        std::vector<std::size_t> all(O);
        for (std::size_t o = 0; o < O; ++o) {
            all[o] = o;
        }
        std::vector<float> pred;
        while (*placed < max_steps) {
            int status = session_predict(ctx, s, net, pred);
            if (status) {
                return status;
            }
            const std::vector<std::size_t> ranked = top_k(pred, O);
            // The k_min best, then every further orientation predicted within
            // `margin` of the k_min-th, up to k_max.
            std::size_t n = std::min<std::size_t>(k_min, O);
            const float cut = pred[ranked[n - 1]] + margin;
            while (n < std::min<std::size_t>(k_max, O) && pred[ranked[n]] <= cut) {
                ++n;
            }
            const std::vector<std::size_t> subset(ranked.begin(), ranked.begin() + n);
            if (paged) {
                *paged += n;
            }
            std::optional<Candidate> chosen;
            if ((status = greedy_step(ctx, s, subset, chosen))) {
                return status;
            }
            if (!chosen) {
                if ((status = greedy_step(ctx, s, all, chosen))) {
                    return status;
                }
                if (!chosen) {
                    break;
                }
                if (fallbacks) {
                    ++*fallbacks;
                }
            }
            record(*chosen, *placed, orientations, translations, scores);
            ++*placed;
        }
        return kOk;
    }
    catch (...) {
        return kAllocation;
    }
}

int spk_session_greedy_proposed_adaptive(spk_context* ctx, spk_proposal* proposal, uint32_t k,
                                         uint32_t min_feasible, uint64_t max_steps, uint64_t* placed,
                                         uint64_t* orientations, int64_t* translations, double* scores,
                                         uint64_t* fallbacks, uint64_t* widenings)
{
    try {
        if (!ctx || !session_of(ctx) || !placed) {
            return kNotReady;
        }
        ProposalNet* net = proposal_net(proposal);
        if (!net || k == 0) {
            return kInvalidArgument;
        }
        auto& s = *session_of(ctx);
        *placed = 0;
        if (fallbacks) {
            *fallbacks = 0;
        }
        if (widenings) {
            *widenings = 0;
        }
        const std::size_t O = s.catalog.size();
        std::vector<std::size_t> all(O);
        for (std::size_t o = 0; o < O; ++o) {
            all[o] = o;
        }
        std::vector<float> pred;
        while (*placed < max_steps) {
            int status = session_predict(ctx, s, net, pred);
            if (status) {
                return status;
            }
            const std::vector<std::size_t> ranked = top_k(pred, O);
            const std::vector<std::size_t> subset(ranked.begin(), ranked.begin() + std::min<std::size_t>(k, O));
            const std::vector<std::size_t> reserve(ranked.begin() + subset.size(), ranked.end());
            std::optional<Candidate> chosen;
            std::size_t widened = 0;
            if ((status = greedy_step(ctx, s, subset, chosen, reserve, min_feasible, k, &widened))) {
                return status;
            }
            if (widenings) {
                *widenings += widened;
            }
            if (!chosen) {
                if ((status = greedy_step(ctx, s, all, chosen))) {
                    return status;
                }
                if (!chosen) {
                    break;
                }
                if (fallbacks) {
                    ++*fallbacks;
                }
            }
            record(*chosen, *placed, orientations, translations, scores);
            ++*placed;
        }
        return kOk;
    }
    catch (...) {
        return kAllocation;
    }
}

int spk_jobs_greedy(spk_job* jobs, uint64_t count)
{
    try {
        if (count && !jobs) {
            return kInvalidArgument;
        }
        std::set<const void*> contexts, proposals;
        for (std::uint64_t j = 0; j < count; ++j) {
            if (!jobs[j].context || !contexts.insert(jobs[j].context).second ||
                (jobs[j].proposal && !proposals.insert(jobs[j].proposal).second)) {
                return kInvalidArgument;
            }
        }
        std::vector<std::thread> threads;
        threads.reserve(count);
        for (std::uint64_t j = 0; j < count; ++j) {
            threads.emplace_back([job = &jobs[j]] {
                job->placed = 0;
                job->fallbacks = 0;
                if (cudaSetDevice(job->context->device) != cudaSuccess) {
                    job->status = kCuda;
                    return;
                }
                job->status = job->proposal
                                  ? spk_session_greedy_proposed(job->context, job->proposal, job->k, job->max_steps,
                                                                &job->placed, job->orientations, job->translations,
                                                                job->scores, &job->fallbacks)
                                  : spk_session_greedy(job->context, job->max_steps, &job->placed, job->orientations,
                                                       job->translations, job->scores);
            });
        }
        for (auto& t : threads) {
            t.join();
        }
        return kOk;
    }
    catch (...) {
        return kAllocation;
    }
}

int spk_session_stats(spk_context* ctx, uint64_t out[4], int reset)
{
    if (!ctx || !session_of(ctx) || !out) {
        return kNotReady;
    }
    auto& p = *session_of(ctx)->pipe;
    out[0] = p.stat_pages;
    out[1] = p.stat_threshold_passes;
    out[2] = p.stat_rescored;
    out[3] = p.stat_first_certified;
    if (reset) {
        p.stat_pages = p.stat_threshold_passes = p.stat_rescored = p.stat_first_certified = 0;
    }
    return kOk;
}

int spk_session_field(spk_context* ctx, int kind, uint64_t orientation, int64_t first[3], uint32_t shape[3],
                      void* out, uint64_t capacity)
{
    try {
        if (!ctx || !session_of(ctx) || !first || !shape) {
            return kNotReady;
        }
        auto& s = *session_of(ctx);
        if (kind == 2) {
            if (orientation >= s.catalog.size()) {
                return kCatalog;
            }
            const auto& slot = s.pipe->slot(s.slot_of[orientation]);
            for (int a = 0; a < 3; ++a) {
                first[a] = slot.first[a];
                shape[a] = static_cast<std::uint32_t>(slot.K[a]);
            }
            if (!out) {
                return kOk;
            }
            if (capacity < slot.host_cells.size()) {
                return kInvalidArgument;
            }
            std::memcpy(out, slot.host_cells.data(), slot.host_cells.size());
            return kOk;
        }
        for (int a = 0; a < 3; ++a) {
            first[a] = s.env.first[a];
            shape[a] = s.env.shape[a];
        }
        if (!out) {
            return kOk;
        }
        const std::uint64_t n = cells_of(s.env);
        int status = refresh(ctx, s);
        if (status) {
            return status;
        }
        if (kind == 0 || kind == 1) {
            if (capacity < n) {
                return kInvalidArgument;
            }
            cudaMemcpyAsync(out, kind == 0 ? s.mask : s.occ, n, cudaMemcpyDeviceToHost, ctx->stream);
        }
        else if (kind == 3) {
            if (capacity < n * 8) {
                return kInvalidArgument;
            }
            auto* d = static_cast<double*>(device_buffer(ctx, "session.prox", n * 8, status));
            if (!d) {
                return status;
            }
            if ((status = proximity_from_d2(ctx, s.pipe->d2(), d, s.env.shape, ctx->stream))) {
                return status;
            }
            cudaMemcpyAsync(out, d, n * 8, cudaMemcpyDeviceToHost, ctx->stream);
        }
        else {
            return kInvalidArgument;
        }
        return cudaStreamSynchronize(ctx->stream) == cudaSuccess ? kOk : kCuda;
    }
    catch (...) {
        return kAllocation;
    }
}

}  // extern "C"
