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
// session keeps its item's), or null to upload them.
int raster_fill(spk_context* ctx, const geo::Placed& placed, const FieldWindow& w, std::uint8_t* d_cells,
                bool normalize, std::uint64_t* uncertain_components = nullptr,
                const std::uint32_t* d_tris_kept = nullptr);
// Clearance dilation of a raw field into the requested window.
int dilate_crop(spk_context* ctx, const std::uint8_t* d_raw, const FieldWindow& raw, std::uint64_t halo,
                double clearance, bool invert, std::uint8_t* d_out, const FieldWindow& req);
// Analytic box container blocker over window w (1 = blocked).
int box_mask(spk_context* ctx, const double* dims, double clearance, const FieldWindow& w, std::uint8_t* d_mask);
int stamp(spk_context* ctx, std::uint32_t* d_counts, const std::uint8_t* d_placed, long long n, int direction);
int occupancy(spk_context* ctx, const std::uint8_t* d_mask, const std::uint32_t* d_counts, std::uint8_t* d_occ,
              long long n);

}  // namespace spk
