// Exact EDT / proximity entry points shared by the pipeline.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

struct spk_context;

namespace spk {

bool proximity_shape_supported(const std::uint32_t* shape);
std::int32_t max_squared_distance(const std::uint32_t* shape);
// Table of exp(-sqrt(v)/2) for v <= max_d2 (host libm), cached on the device.
const double* proximity_table(spk_context* ctx, std::int32_t max_d2, int& status);
// d2 = exact squared distance to the nearest occupied cell, INT32_MAX if none.
int edt_squared(spk_context* ctx, const std::uint8_t* d_occupied, std::int32_t* d_d2, const std::uint32_t* shape,
                cudaStream_t stream);
int proximity_from_d2(spk_context* ctx, const std::int32_t* d_d2, double* d_out, const std::uint32_t* shape,
                      cudaStream_t stream);

// A box of cells, lo inclusive, hi exclusive, per axis.
struct EdtBox {
    int lo[3];
    int hi[3];
};

// Side of the cubic tiles over which the incremental update keeps the largest
// squared distance.
constexpr int kEdtTile = 8;

// tile_max[t] = largest d2 over tile t (INT32_MAX if any cell has no
// occupied cell at all), for every tile.
int edt_tile_max(spk_context* ctx, const std::int32_t* d_d2, const std::uint32_t* shape, std::int32_t* d_tile_max,
                 cudaStream_t stream);

// The exact EDT after new occupied cells (d_sites != 0, all inside `sites`)
// join the occupancy whose EDT d_d2 holds: d2 = min(d2, squared distance to
// the nearest new site).  Only the box spanned by `sites` and by every tile
// whose largest d2 exceeds its squared distance to `sites` is recomputed;
// outside it no d2 can fall.  tile_max is kept current.
int edt_add_sites(spk_context* ctx, const std::uint8_t* d_sites, const EdtBox& sites, std::int32_t* d_d2,
                  std::int32_t* d_tile_max, const std::uint32_t* shape, cudaStream_t stream);

}  // namespace spk
