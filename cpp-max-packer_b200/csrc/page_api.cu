// C entry for a single spectral page over a caller-supplied layout.
#include <cuda_runtime.h>

#include <cstring>
#include <vector>

#include "context.hpp"
#include "pipeline.hpp"

using namespace spk;

extern "C" int spk_spectral_page(spk_context* ctx, const spk_page_scene* scene, const uint8_t* occupancy,
                                 const spk_page_kernel* kernel, const uint8_t* kernel_cells,
                                 const spk_page_query* query, spk_candidate* page, uint32_t* count,
                                 spk_page_report* report)
{
    try {
        if (!ctx || !scene || !occupancy || !kernel || !kernel_cells || !query || !page || !count) {
            return kInvalidArgument;
        }
        *count = 0;
        if (query->mode > 1) {
            return kInvalidArgument;  // 0 ordinary, 1 low-overlap
        }
        if (cudaSetDevice(ctx->device) != cudaSuccess) {
            return kCuda;
        }
        Pipeline pipe(ctx);
        int status = pipe.set_geometry(scene->environment_first, scene->environment_shape, scene->lattice_origin_mm,
                                       scene->lattice_pitch_mm, scene->container_min_z_mm,
                                       scene->container_height_mm);
        if (status) {
            return status;
        }
        const std::size_t cells = static_cast<std::size_t>(scene->environment_shape[0]) *
                                  scene->environment_shape[1] * scene->environment_shape[2];
        auto* d_occ = static_cast<std::uint8_t*>(device_buffer(ctx, "page.occ", cells, status));
        if (!d_occ) {
            return status;
        }
        cudaMemcpyAsync(d_occ, occupancy, cells, cudaMemcpyHostToDevice, ctx->stream);
        if ((status = pipe.set_occupancy(d_occ))) {
            return status;
        }
        std::uint64_t slot = 0;
        if ((status = pipe.add_kernel(query->orientation_index, kernel->first, kernel->shape, kernel_cells,
                                      kernel->object_max_z_mm, slot))) {
            return status;
        }
        PageRequest request;
        request.slot = slot;
        request.low_overlap = query->mode == 1;
        request.has_cursor = query->has_cursor != 0;
        if (request.has_cursor) {
            const auto& c = query->exclusive_cursor;
            std::memcpy(request.cursor.t, c.translation, sizeof(request.cursor.t));
            request.cursor.score = c.score;
            request.cursor.orientation = c.orientation_index;
            request.cursor.binary_overlap = c.binary_overlap;
            request.cursor.direct_zero = c.direct_zero_overlap != 0;
        }
        std::vector<PageOutcome> out;
        if ((status = pipe.pages({ request }, out))) {
            return status;
        }
        const auto& o = out[0];
        if (report) {
            report->max_integer_residual = o.max_integer_residual;
            report->max_score_error = o.max_score_error;
            report->rescored = o.rescored;
            report->certified = o.certified ? 1 : 0;
            report->threshold_pass = o.threshold_pass ? 1 : 0;
        }
        if (o.status) {
            return o.status;
        }
        for (std::size_t i = 0; i < o.page.size(); ++i) {
            auto& dst = page[i];
            std::memset(&dst, 0, sizeof(dst));
            std::memcpy(dst.translation, o.page[i].t, sizeof(dst.translation));
            dst.score = o.page[i].score;
            dst.direct_zero_overlap = o.page[i].direct_zero ? 1 : 0;
            dst.orientation_index = o.page[i].orientation;
            dst.binary_overlap = o.page[i].binary_overlap;
        }
        *count = static_cast<std::uint32_t>(o.page.size());
        return kOk;
    }
    catch (...) {
        return kAllocation;
    }
}
