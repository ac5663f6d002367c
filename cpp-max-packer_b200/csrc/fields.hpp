// Device field builders shared by the engine and the stateless entry points.
#pragma once

#include <cstdint>

#include "geometry.hpp"

struct spk_context;

namespace spk {

// A lattice window passed by value to kernels.
struct FieldWindow {
    long long first[3];
    int shape[3];
    double origin[3];
    double pitch;
};

inline FieldWindow make_window(const geo::Window& w, const double* origin, double pitch)
{
    FieldWindow f;
    for (int a = 0; a < 3; ++a) {
        f.first[a] = w.first[a];
        f.shape[a] = static_cast<int>(w.shape[a]);
        f.origin[a] = origin[a];
    }
    f.pitch = pitch;
    return f;
}

// Raster + component fill of `placed` over window `w` into d_cells (u8,
// values 0/1/2/3, or 0/1 when `normalize`).
// d_tris_kept: the mesh's triangle indices already on the device (a
// session keeps its item's), or null to upload them.  device_intervals: the
// vertex intervals are already in the context's "field.vint" buffer
// (place_on_device), so placed.intervals is not read.
int raster_fill(spk_context* ctx, const geo::Placed& placed, const FieldWindow& w, std::uint8_t* d_cells,
                bool normalize, std::uint64_t* uncertain_components = nullptr,
                const std::uint32_t* d_tris_kept = nullptr, bool device_intervals = false);

// place() for a rotation that is not cardinal, with the vertex intervals
// computed on the device (d_vertices: the mesh's vertices there) into the
// context's "field.vint" buffer; on the host `out` receives everything the
// window plan and the witnesses read (conservative bounds, pose), not the
// per-vertex vectors.  done = false: the pose is cardinal, not finite or
// has an invalid interval, and the host's place() must run instead.
int place_on_device(spk_context* ctx, const geo::Prepared& prepared, const double* d_vertices,
                    const geo::Vec3& translation, const geo::Quat& q, geo::Placed& out, bool& done);
// Clearance dilation of a raw field into the requested window.
int dilate_crop(spk_context* ctx, const std::uint8_t* d_raw, const FieldWindow& raw, std::uint64_t halo,
                double clearance, bool invert, std::uint8_t* d_out, const FieldWindow& req,
                const int* box_lo = nullptr, const int* box_hi = nullptr);
// box_lo / box_hi (cell offsets in `req`, hi exclusive): the only cells the
// dilation can set; the rest of d_out is cleared.  Null: the whole window.
// Analytic box container blocker over window w (1 = blocked).
int box_mask(spk_context* ctx, const double* dims, double clearance, const FieldWindow& w, std::uint8_t* d_mask);
int stamp(spk_context* ctx, std::uint32_t* d_counts, const std::uint8_t* d_placed, long long n, int direction);
int occupancy(spk_context* ctx, const std::uint8_t* d_mask, const std::uint32_t* d_counts, std::uint8_t* d_occ,
              long long n);
// stamp / occupancy over the box [lo, hi) of a window of `shape` cells (the
// cells a placed copy's field can set).
int stamp_box(spk_context* ctx, std::uint32_t* d_counts, const std::uint8_t* d_placed, const int* shape,
              const int* lo, const int* hi, int direction);
int occupancy_box(spk_context* ctx, const std::uint8_t* d_mask, const std::uint32_t* d_counts, std::uint8_t* d_occ,
                  const int* shape, const int* lo, const int* hi);

}  // namespace spk
