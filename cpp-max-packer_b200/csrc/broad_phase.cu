// Validator broad phase on the device: the outward-AABB pair test of
// geometry::validate's pair loop (engine/pack_geometry/src/validation.cpp:
// 404-418, kernel::bounds_pair_certificate -> separated_conservative_bounds,
// validation_kernel.cpp:1245-1261) over every pair of copies at once.
//
// The validator visits pairs (first, second), second < first, first
// ascending then second ascending, skipping pairs whose poses are both
// proven (validate_incremental).  A pair is certified disjoint by its posed
// bounds when, on some axis, nextafter(max + clearance, +inf) of one copy is
// below the other copy's min.  spk_broad_phase returns, in that visiting
// order, the pairs this test does not certify: the pairs for which the
// validator's remaining steps (cardinal proofs, support tables, exact
// classification) still have to run on the host.
//
// Pair p of the full order is (first, second) with p = first (first - 1) / 2
// + second.  One launch counts the uncertified pairs of each block's
// contiguous range of p, one block scans those counts, and a third launch
// writes each block's pairs at its offset in order (a warp-ballot rank
// inside the block), so the output is deterministic and needs no sort.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <vector>

#include "../../include/spk_b200.h"
#include "common.cuh"
#include "context.hpp"
#include "interval.cuh"

namespace spk {
namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kBroadThreads = 256;
constexpr int kPairsPerThread = 8;
constexpr long long kPairsPerBlock = static_cast<long long>(kBroadThreads) * kPairsPerThread;

struct BroadArgs {
    const double* lo;          // [n][3] posed conservative bounds, min corner
    const double* hi;          // [n][3] max corner
    const std::uint8_t* finite;  // [n] ConservativeBounds::finite
    const std::uint8_t* proven;  // [n] or null
    double clearance;
    long long pairs;           // n (n - 1) / 2
};

// (first, second) of pair p in the visiting order.
__device__ __forceinline__ void pair_of(long long p, long long& first, long long& second)
{
    long long f = static_cast<long long>((1.0 + sqrt(1.0 + 8.0 * static_cast<double>(p))) * 0.5);
    while (f * (f - 1) / 2 > p) {
        --f;
    }
    while ((f + 1) * f / 2 <= p) {
        ++f;
    }
    first = f;
    second = p - f * (f - 1) / 2;
}

// separated_conservative_bounds (validation_kernel.cpp:1245-1261) for a
// finite, non-negative clearance: each bound plus the clearance, rounded to
// nearest, moved one ulp up.
__device__ __forceinline__ bool separated(const BroadArgs& a, long long i, long long j)
{
    if (!a.finite[i] || !a.finite[j]) {
        return false;
    }
#pragma unroll
    for (int axis = 0; axis < 3; ++axis) {
        const double x = next_up(f_add(a.hi[3 * i + axis], a.clearance));
        const double y = next_up(f_add(a.hi[3 * j + axis], a.clearance));
        if (x < a.lo[3 * j + axis] || y < a.lo[3 * i + axis]) {
            return true;
        }
    }
    return false;
}

// True when the validator still has work for pair p after the broad phase.
__device__ __forceinline__ bool unresolved(const BroadArgs& a, long long p, long long& first, long long& second)
{
    pair_of(p, first, second);
    if (a.proven && a.proven[first] && a.proven[second]) {
        return false;
    }
    return !separated(a, first, second);
}

__global__ void __launch_bounds__(kBroadThreads) broad_count_kernel(const BroadArgs a,
                                                                   unsigned long long* __restrict__ block_counts)
{
    const long long base = static_cast<long long>(blockIdx.x) * kPairsPerBlock;
    unsigned int mine = 0;
    for (int k = 0; k < kPairsPerThread; ++k) {
        const long long p = base + static_cast<long long>(k) * kBroadThreads + threadIdx.x;
        long long f, s;
        if (p < a.pairs && unresolved(a, p, f, s)) {
            ++mine;
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        mine += __shfl_xor_sync(kFull, mine, o);
    }
    __shared__ unsigned int warp_sums[kBroadThreads / 32];
    if ((threadIdx.x & 31) == 0) {
        warp_sums[threadIdx.x >> 5] = mine;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long total = 0;
        for (int w = 0; w < kBroadThreads / 32; ++w) {
            total += warp_sums[w];
        }
        block_counts[blockIdx.x] = total;
    }
}

// Exclusive scan of the block counts in place; the grand total goes to
// block_counts[blocks].  One block of kBroadThreads threads.
__global__ void __launch_bounds__(kBroadThreads) broad_scan_kernel(unsigned long long* __restrict__ block_counts,
                                                                  long long blocks)
{
    __shared__ unsigned long long carry;
    __shared__ unsigned long long warp_sums[kBroadThreads / 32];
    if (threadIdx.x == 0) {
        carry = 0;
    }
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (long long start = 0; start < blocks; start += kBroadThreads) {
        const long long i = start + threadIdx.x;
        const unsigned long long v = i < blocks ? block_counts[i] : 0ULL;
        unsigned long long inclusive = v;
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned long long other = __shfl_up_sync(kFull, inclusive, o);
            if (lane >= o) {
                inclusive += other;
            }
        }
        if (lane == 31) {
            warp_sums[warp] = inclusive;
        }
        __syncthreads();
        unsigned long long before = carry;
        for (int w = 0; w < warp; ++w) {
            before += warp_sums[w];
        }
        if (i < blocks) {
            block_counts[i] = before + inclusive - v;
        }
        __syncthreads();
        if (threadIdx.x == kBroadThreads - 1) {
            carry = before + inclusive;
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        block_counts[blocks] = carry;
    }
}

// Writes block b's uncertified pairs, in visiting order, from offset
// block_counts[b]; pairs beyond `capacity` are counted but not written.
__global__ void __launch_bounds__(kBroadThreads) broad_write_kernel(const BroadArgs a,
                                                                   const unsigned long long* __restrict__ block_counts,
                                                                   std::uint32_t* __restrict__ out,
                                                                   unsigned long long capacity)
{
    __shared__ unsigned int warp_sums[kBroadThreads / 32];
    __shared__ unsigned long long running;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (threadIdx.x == 0) {
        running = block_counts[blockIdx.x];
    }
    const long long base = static_cast<long long>(blockIdx.x) * kPairsPerBlock;
    for (int k = 0; k < kPairsPerThread; ++k) {
        const long long p = base + static_cast<long long>(k) * kBroadThreads + threadIdx.x;
        long long f = 0, s = 0;
        const bool take = p < a.pairs && unresolved(a, p, f, s);
        const unsigned int mask = __ballot_sync(kFull, take);
        if (lane == 0) {
            warp_sums[warp] = __popc(mask);
        }
        __syncthreads();
        unsigned long long at = running + __popc(mask & ((1u << lane) - 1u));
        for (int w = 0; w < warp; ++w) {
            at += warp_sums[w];
        }
        if (take && at < capacity) {
            out[2 * at] = static_cast<std::uint32_t>(f);
            out[2 * at + 1] = static_cast<std::uint32_t>(s);
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            for (int w = 0; w < kBroadThreads / 32; ++w) {
                running += warp_sums[w];
            }
        }
        __syncthreads();
    }
}

}  // namespace
}  // namespace spk

using namespace spk;

extern "C" int spk_broad_phase(spk_context* ctx, const double* bounds_min, const double* bounds_max,
                               const uint8_t* finite, const uint8_t* proven, uint64_t copies, double clearance_mm,
                               uint32_t* pairs, uint64_t capacity, uint64_t* unresolved_count)
{
    if (!ctx) {
        return kNotReady;
    }
    if (!bounds_min || !bounds_max || !finite || !unresolved_count || (capacity && !pairs)) {
        return fail(ctx, kInvalidArgument, "Broad-phase input is missing.");
    }
    if (copies > (1ULL << 20)) {
        return fail(ctx, kInvalidArgument, "Broad-phase copy count exceeds 2^20.");
    }
    if (!(clearance_mm >= 0.0) || !std::isfinite(clearance_mm)) {
        // validation_kernel.cpp:1248: an invalid clearance certifies nothing.
        return fail(ctx, kInvalidArgument, "Broad-phase clearance must be finite and non-negative.");
    }
    *unresolved_count = 0;
    const long long n = static_cast<long long>(copies);
    const long long total_pairs = n * (n - 1) / 2;
    if (total_pairs == 0) {
        return finish(ctx, kOk);
    }
    const long long blocks = (total_pairs + kPairsPerBlock - 1) / kPairsPerBlock;
    cudaStream_t st = ctx->stream;
    int status = kOk;
    const std::size_t per_copy = 3 * sizeof(double);
    auto* d_lo = static_cast<double*>(device_buffer(ctx, "broad.lo", copies * per_copy, status));
    auto* d_hi = static_cast<double*>(device_buffer(ctx, "broad.hi", copies * per_copy, status));
    auto* d_flags = static_cast<std::uint8_t*>(device_buffer(ctx, "broad.flags", 2 * copies, status));
    auto* d_counts = static_cast<unsigned long long*>(
        device_buffer(ctx, "broad.counts", (static_cast<std::size_t>(blocks) + 1) * 8, status));
    // Output slots on the device: no more than there are pairs.
    const std::uint64_t written =
        capacity < static_cast<std::uint64_t>(total_pairs) ? capacity : static_cast<std::uint64_t>(total_pairs);
    auto* d_out = written ? static_cast<std::uint32_t*>(device_buffer(ctx, "broad.out", written * 8, status)) : nullptr;
    if (!d_lo || !d_hi || !d_flags || !d_counts || (written && !d_out)) {
        return fail(ctx, status ? status : kAllocation, "Broad-phase device buffers could not be allocated.");
    }
    cudaMemcpyAsync(d_lo, bounds_min, copies * per_copy, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(d_hi, bounds_max, copies * per_copy, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(d_flags, finite, copies, cudaMemcpyHostToDevice, st);
    if (proven) {
        cudaMemcpyAsync(d_flags + copies, proven, copies, cudaMemcpyHostToDevice, st);
    }
    BroadArgs a { d_lo, d_hi, d_flags, proven ? d_flags + copies : nullptr, clearance_mm, total_pairs };
    broad_count_kernel<<<static_cast<unsigned>(blocks), kBroadThreads, 0, st>>>(a, d_counts);
    broad_scan_kernel<<<1, kBroadThreads, 0, st>>>(d_counts, blocks);
    broad_write_kernel<<<static_cast<unsigned>(blocks), kBroadThreads, 0, st>>>(a, d_counts, d_out, written);
    ctx->launches += 3;
    unsigned long long total = 0;
    cudaMemcpyAsync(&total, d_counts + blocks, 8, cudaMemcpyDeviceToHost, st);
    if (cudaStreamSynchronize(st) != cudaSuccess) {
        cudaGetLastError();
        return fail(ctx, kCuda, "Broad-phase kernels failed.");
    }
    *unresolved_count = total;
    const std::uint64_t copy_out = total < written ? total : written;
    if (copy_out && cudaMemcpy(pairs, d_out, copy_out * 8, cudaMemcpyDeviceToHost) != cudaSuccess) {
        cudaGetLastError();
        return fail(ctx, kCuda, "Broad-phase pairs could not be copied.");
    }
    if (total > capacity) {
        return fail(ctx, kScratchLimit, "Broad-phase pair capacity is smaller than the unresolved pair count.");
    }
    return finish(ctx, kOk);
}
