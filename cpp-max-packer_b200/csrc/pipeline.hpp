// Spectral page pipeline: legal-translation correlation of one environment
// (occupancy + proximity) against many oriented kernels, fused threshold,
// approximate score and top-k, then exact integer recount and exact FP64
// proximity sums for the selected candidates.
//
// Reference behaviour restated (engine/pack_solver/src/spectral_pipeline.cpp):
//   legal translations  first = env.first - kernel.first, extent E-K+1   :1618-1648
//   score = .65 * (world_z + max_z - c_min_z) / H - .35 * prox / occ      :1794-1800
//   ordinary pages keep round(binary) == 0, rank by (score, o, z, y, x),
//   32 entries after an exclusive cursor                                  :1706-1824
//   direct_zero_overlap = exact u8 recount of each page candidate         :1825-1857
#pragma once

#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <vector>

#include "../../include/spk_b200.h"
#include "common.cuh"
#include "edt.cuh"

struct spk_context;

namespace spk {

constexpr int kPageSize = 32;
constexpr int kExactPerOrientation = 64;
constexpr unsigned kKeyCapacity = 4096;
constexpr unsigned kLargeKeyChunks = 64;  // key range of a 256^3 request: 64 x 4096 = 4096 blocks x 64 keys
constexpr unsigned long long kEmptyKey = ~0ULL;

struct Candidate {
    std::int64_t t[3];
    double score;
    bool direct_zero;
    std::uint64_t orientation;
    double binary_overlap;
};

// One oriented kernel on the device, prepared for a fixed environment shape.
struct KernelSlot {
    std::uint64_t orientation {};
    int K[3] {};
    std::int64_t first[3] {};
    std::uint64_t occupied {};
    double max_z {};
    float2* partial {};           // [z < K2][ky < L1][kx < L0], x and y transformed
    std::int32_t* ones {};        // environment-relative offsets of kernel ones
    double* t65 {};               // .65 * top(z) for each legal z
    int legal[3] {};              // E - K + 1 per axis (0 when the kernel does not fit)
    std::vector<std::uint8_t> host_cells;
};

// One orientation of a batched pass A (256^3 grids).
constexpr int kPassABatch = 16;
struct PassASlot {
    const float2* partial;
    float2* inter;
    int K2;
    int legal_z;
};
struct PassABatch {
    PassASlot slot[kPassABatch];
    int count;
};
// Passes B1 and B2 of a batch of orientations in one launch each: slot g
// owns the blocks from first_block on.
struct PassBSlot {
    float2* inter;
    const double* t65;
    unsigned long long* keys;
    unsigned int* count;
    unsigned long long* tau;
    unsigned long long* resid;
    double inv_occ;
    double cursor_floor;
    float target;
    unsigned int cap;
    int legal_x, legal_y, legal_z;
    int first_block;
};
// Block order: the first `interleaved` blocks go round-robin over the
// slots (block b: slot b % count, the slot's block b / count), covering the
// first `min_blocks` blocks of every slot; the rest follow slot by slot from
// each slot's first_block, as its blocks min_blocks and up.  With
// interleaved = min_blocks = 0 the order is slot by slot.
struct PassBBatch {
    PassBSlot slot[kPassABatch];
    int count;
    int interleaved;
    int min_blocks;
};

struct PageRequest {
    std::uint64_t slot {};
    bool has_cursor {};
    Candidate cursor {};
    // Candidates are the legal translations whose overlap count is this
    // (0: ordinary pages; low-overlap pages use one count at a time).
    std::uint32_t overlap {};
    // A low-overlap page (spectral_pipeline.hpp:45, CandidatePageMode::low_overlap).
    bool low_overlap {};
};

struct PageOutcome {
    int status {};
    std::vector<Candidate> page;
    bool certified {};
    bool threshold_pass {};
    double max_integer_residual {};
    double max_score_error {};
    double excluded_score {};  // lowest approximate score of an unrescored candidate
    // Every candidate left out of the rescored set has an exact score above
    // this bound; page entries scoring <= it are exact and correctly placed.
    double exact_floor { INFINITY };
    std::uint64_t rescored {};
};

class Pipeline {
public:
    explicit Pipeline(spk_context* ctx);
    ~Pipeline();

    // Environment window (global first + shape) and lattice/container terms.
    int set_geometry(const std::int64_t* env_first, const std::uint32_t* env_shape, const double* origin,
                     double pitch, double container_min_z, double container_height);
    // Device occupancy (u8, E^3): runs the exact EDT and the environment spectrum.
    int set_occupancy(const std::uint8_t* d_occupancy);
    // The same after the only change since the last call is that the cells
    // d_sites != 0 (all inside `sites`, window coordinates) became occupied:
    // the EDT is updated in place over the region they can affect.
    int add_occupied(const std::uint8_t* d_occupancy, const std::uint8_t* d_sites, const EdtBox& sites);
    // The same updates queued on the pipeline's own stream, after the work
    // already on the context's stream (d_sites null: set_occupancy), so that
    // the context's stream can run other work (the proposal) meanwhile.
    // refresh_order() makes the context's stream wait for it; pages() does
    // so itself.  Until then nothing the update writes may be read, and
    // nothing it reads (the occupancy, the sites) rewritten.
    int refresh_begin(const std::uint8_t* d_occupancy, const std::uint8_t* d_sites, const EdtBox* sites);
    void refresh_order();
    // Adds an oriented kernel field (host cells, X-fastest); returns the slot.
    int add_kernel(std::uint64_t orientation, const std::int64_t* first, const std::uint32_t* shape,
                   const std::uint8_t* cells, double max_z, std::uint64_t& slot);
    // full = true certifies whole pages (threshold passes where needed);
    // full = false returns first-pass pages with their exact_floor only.
    int pages(const std::vector<PageRequest>& requests, std::vector<PageOutcome>& out, bool full = true);

    const std::uint8_t* occupancy() const { return occ_; }
    const std::int32_t* d2() const { return d2_; }
    const int* env_shape() const { return E_; }
    const int* fft_shape() const { return L_; }
    std::size_t kernels() const { return slots_.size(); }
    const KernelSlot& slot(std::size_t i) const { return slots_[i]; }
    double epsilon_p(const KernelSlot& s) const;

private:
    int ordinary_pages(const std::vector<PageRequest>& requests, std::vector<PageOutcome>& out, bool full);
    int low_overlap_page(const PageRequest& request, PageOutcome& out);
    int run_orientation(const KernelSlot& s, int mode, float target, double threshold, double cursor_floor,
                        unsigned long long* keys, unsigned int* count, unsigned int cap, unsigned long long* tau,
                        unsigned long long* resid);
    int run_b256(const KernelSlot& s, float2* inter, int mode, float target, double threshold, double cursor_floor,
                 unsigned long long* keys, unsigned int* count, unsigned int cap, unsigned long long* tau,
                 unsigned long long* resid);
    double pass_a_bytes(const KernelSlot& s) const;
    int update_spectrum();
    // z_norm_ from the spectrum's partial sums, once the device has them.
    int finish_norm();
    // Transform lengths per axis for the window (the autotuner); sets L_.
    int choose_lengths(const std::uint32_t* env_shape);
    // Pass A for up to kPassABatch orientations in one launch (256^3 grids);
    // orientation i's legal-z intermediate goes to inter[i].
    int run_a256_batch(const KernelSlot* const* slots, int count, float2* const* inter);
    // Passes B1 and B2 (mode 0) of the same batch, one launch each.
    int run_b256_batch(const KernelSlot* const* slots, int count, float2* const* inter, const PassBSlot* outputs);
    // The launch arguments of a batched pass A; returns its algorithmic bytes.
    double fill_a256(const KernelSlot* const* slots, int count, float2* const* inter, PassABatch& batch) const;
    // The launch arguments of batched passes B1 and B2: block counts and
    // algorithmic bytes of each.
    void fill_b256(const KernelSlot* const* slots, int count, float2* const* inter, const PassBSlot* outputs,
                   PassBBatch& b1, PassBBatch& b2, int& blocks1, int& blocks2, double& bytes1, double& bytes2) const;
    // Ordinary pages' passes A, B1 and B2 over `count` batches as a software
    // pipeline: launch k runs pass A of batch k, B1 of batch k - 1 and B2 of
    // batch k - 2 (pass_stage256_kernel).  Batch k uses inter[k % 3].
    struct StageBatch {
        const KernelSlot* slots[kPassABatch];
        PassBSlot outputs[kPassABatch];
        int count;
    };
    int run_stages256(const std::vector<StageBatch>& batches, float2* const* inter, std::size_t stride);
    double score(const KernelSlot& s, const std::int64_t* t, double p) const;
    double approx_epsilon(const KernelSlot& s) const;

    spk_context* ctx_;
    int E_[3] {};
    int L_[3] {};
    std::int64_t env_first_[3] {};
    double origin_[3] {};
    double pitch_ {};
    double cmin_z_ {};
    double height_ {};
    std::uint8_t* occ_ {};
    std::int32_t* d2_ {};
    std::int32_t* tile_max_ {};  // largest d2 per kEdtTile^3 tile (incremental EDT)
    float2* spectrum_ {};
    float2* inter_ {};
    std::size_t inter_bytes_ {};
    bool fused_b_ {};  // 256^3: passes B1 and B2 as one cluster kernel (SPK_PASS_B=fused), else two passes
    bool staged_ {};  // 256^3 ordinary pages: pipelined stage launches (SPK_PAGE_SCHEDULE=staged), else one per pass
    const double* table_ {};
    double z_norm_ {};  // sqrt(sum over cells of b^2 + p^2)
    const double* norm_host_ {};  // pinned partial sums of the last update_spectrum
    int norm_blocks_ {};
    cudaStream_t norm_stream_ {};
    bool norm_pending_ {};
    cudaStream_t side_ {};  // refresh_begin's stream
    cudaEvent_t ev_in_ {}, ev_done_ {};
    bool pending_ {};
    std::vector<KernelSlot> slots_;

public:
    // Work counters since the last reset: first-pass pages, threshold passes,
    // candidates rescored exactly, pages certified by the first pass.
    std::uint64_t stat_pages {}, stat_threshold_passes {}, stat_rescored {}, stat_first_certified {};
};

}  // namespace spk
