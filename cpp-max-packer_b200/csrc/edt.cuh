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

}  // namespace spk
