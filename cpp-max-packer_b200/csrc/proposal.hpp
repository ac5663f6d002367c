// Learned orientation proposal: a small 3D CNN that scores every catalog
// orientation of the current layout so that only the best k are paged.
//
// Input  : 2 x 32^3 voxels per sample, channels-last ([z][y][x][c], x fastest
//          before c): channel 0 = the layout's occupancy fraction over the
//          environment window pooled to 32^3, channel 1 = the oriented item's
//          cells pooled to 32^3 (corner aligned).
// Network: conv3d 3^3 pad 1 (ReLU after each):
//            2 -> 16 stride 1 (32^3), 16 -> 32 stride 2 (16^3),
//            32 -> 64 stride 2 (8^3), 64 -> 64 stride 2 (4^3);
//          global mean over the 4^3 voxels, then linear 64 -> 1.
// Output : predicted score gap to the layout's best placement (lower first).
// BF16 operands and activations, FP32 accumulation (tcgen05 MMA in TMEM),
// FP32 master parameters and Adam.
//
// Flat parameter order (FP32): for each conv layer, weights [cout][27][cin]
// (tap = (kz * 3 + ky) * 3 + kx, input voxel = out * stride + k - 1) then
// bias [cout]; then head weights [64] and head bias [1].
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>

struct spk_context;
struct spk_proposal;

namespace spk {

constexpr int kProposalGrid = 32;
constexpr int kProposalVoxels = kProposalGrid * kProposalGrid * kProposalGrid;
constexpr int kProposalLayers = 4;

struct ProposalLayer {
    int cin, cout, stride, s_in;
};
constexpr ProposalLayer kProposalSpec[kProposalLayers] = {
    { 2, 16, 1, 32 }, { 16, 32, 2, 32 }, { 32, 64, 2, 16 }, { 64, 64, 2, 8 } };

struct ProposalNet;
ProposalNet* proposal_net(spk_proposal* handle);

std::uint64_t proposal_parameter_count();

// Scores `batch` samples whose inputs are assembled on the device from pooled
// layouts and pooled items: sample b uses crops[crop_index[b]] (or crops[0]
// when crop_index is null) and items[item_index[b]] (or items[b] when null).
// Predictions land in device memory `pred` (batch floats).  A nonzero
// `items_tag` names an unchanging set of item channels (one layout scored
// against the same items again and again, crop_index and item_index null):
// the first layer's item sums are then cached per (tag, batch, parameters).
int proposal_predict(spk_context* ctx, ProposalNet* net, std::uint32_t batch, const __nv_bfloat16* crops,
                     const std::uint32_t* crop_index, const __nv_bfloat16* items, const std::uint32_t* item_index,
                     std::uint64_t items_tag, float* pred);

// Device pooling helpers (bf16 32^3 outputs, [z][y][x]).
int pool_occupancy(spk_context* ctx, const std::uint8_t* occupancy, const int* shape, __nv_bfloat16* out);
int pool_item(spk_context* ctx, const std::uint8_t* cells, const int* shape, __nv_bfloat16* out);

}  // namespace spk
