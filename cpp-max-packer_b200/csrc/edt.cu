// Exact squared Euclidean distance transform and the proximity field:
// the GPU replacement of solver::detail::build_proximity
// (reference engine/pack_solver/src/field_proximity.hpp:32-132).
//
// d2(c) = min over occupied o of |c - o|^2, computed exactly in integers by
// three separable 1D lower-envelope passes (one thread per line; the minimum
// of parabolas is algorithm-independent, so values equal the reference's).
// proximity(c) = exp(-sqrt(d2)/2), 0 where no cell is occupied.  The exp/sqrt
// values come from a host table built with the host libm for every integer
// d2 that can occur, so the FP64 field is bit-identical to the reference's.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstring>
#include <mutex>
#include <vector>

#include "context.hpp"
#include "edt.cuh"

namespace spk {

namespace {

constexpr std::int32_t kInf = INT32_MAX;

__global__ void edt_init_kernel(const std::uint8_t* __restrict__ occupied, std::int32_t* __restrict__ d2, long long n)
{
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        d2[i] = occupied[i] ? 0 : kInf;
    }
}

// One 1D pass along `axis`.  Line scratch (site positions and the first
// coordinate each site wins from) lives in global memory, one slot per cell.
__global__ void edt_pass_kernel(std::int32_t* __restrict__ d2, std::int32_t* __restrict__ line_f,
                                std::int32_t* __restrict__ site_q, long long* __restrict__ site_start, int sx,
                                int sy, int sz, int axis)
{
    const int length = axis == 0 ? sx : axis == 1 ? sy : sz;
    const long long lines = static_cast<long long>(sx) * sy * sz / length;
    const long long line = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
    if (line >= lines) {
        return;
    }
    long long base, stride;
    if (axis == 0) {
        base = line * sx;
        stride = 1;
    }
    else if (axis == 1) {
        const long long x = line % sx, z = line / sx;
        base = x + z * static_cast<long long>(sx) * sy;
        stride = sx;
    }
    else {
        base = line;
        stride = static_cast<long long>(sx) * sy;
    }
    // Scratch for this line sits at the line's own cells, strided alike.
    int count = 0;
    for (int q = 0; q < length; ++q) {
        const long long at = base + q * stride;
        const std::int32_t f = d2[at];
        line_f[at] = f;
        if (f == kInf) {
            continue;
        }
        long long start = LLONG_MIN;
        while (count > 0) {
            const long long top = base + (count - 1) * stride;
            const long long p = site_q[top];
            const long long numerator =
                static_cast<long long>(f) - static_cast<long long>(line_f[base + p * stride]) + 1LL * q * q - p * p;
            const long long denominator = 2LL * (q - p);
            // The intersection of the two parabolas, rounded down: from one past it on, site q wins.
            long long quotient = numerator / denominator;
            if ((numerator % denominator != 0) && ((numerator < 0) != (denominator < 0))) {
                --quotient;
            }
            start = quotient + 1;
            if (start > site_start[top]) {
                break;
            }
            --count;
        }
        if (count == 0) {
            start = LLONG_MIN;
        }
        const long long slot = base + count * stride;
        site_q[slot] = q;
        site_start[slot] = start;
        ++count;
    }
    int site = 0;
    for (int q = 0; q < length; ++q) {
        const long long at = base + q * stride;
        if (count == 0) {
            d2[at] = kInf;
            continue;
        }
        while (site + 1 < count && site_start[base + (site + 1) * stride] <= q) {
            ++site;
        }
        const long long p = site_q[base + site * stride];
        const long long delta = q - p;
        d2[at] = static_cast<std::int32_t>(line_f[base + p * stride] + delta * delta);
    }
}

// First pass (along x) straight from the occupancy: on a binary line the 1D
// squared distance is the square of the distance to the nearest occupied
// cell, found by a left-to-right and a right-to-left sweep.  One warp per
// line, each lane a run of `per_lane` consecutive cells; warp max/min scans
// carry the nearest occupied position across lanes.  Lines of up to
// 32 * kFirstPassPerLane cells.
constexpr int kFirstPassPerLane = 32;

__global__ void __launch_bounds__(256) edt_first_pass_kernel(const std::uint8_t* __restrict__ occupied,
                                                            std::int32_t* __restrict__ d2, int sx, long long lines)
{
    const int lane = threadIdx.x & 31;
    const long long line = static_cast<long long>(blockIdx.x) * 8 + (threadIdx.x >> 5);
    if (line >= lines) {
        return;  // whole warp: the line index is warp-uniform
    }
    const int per_lane = (sx + 31) / 32;
    const int begin = lane * per_lane;
    const std::uint8_t* row = occupied + line * sx;
    std::int32_t* out = d2 + line * sx;
    constexpr int kNone = 1 << 24;  // beyond any line length
    std::uint32_t bits = 0;  // occupied cells of this lane's run
    for (int i = 0; i < per_lane; ++i) {
        const int x = begin + i;
        if (x < sx && row[x]) {
            bits |= 1u << i;
        }
    }
    // Nearest occupied position at or before the end of each earlier run.
    int last = bits ? begin + 31 - __clz(bits) : -kNone;
    int first = bits ? begin + __ffs(bits) - 1 : kNone;
    int left = last, right = first;
    for (int o = 1; o < 32; o <<= 1) {
        const int l = __shfl_up_sync(0xffffffffu, left, o);
        const int r = __shfl_down_sync(0xffffffffu, right, o);
        if (lane >= o) {
            left = max(left, l);
        }
        if (lane + o < 32) {
            right = min(right, r);
        }
    }
    // Exclusive: occupied positions strictly in earlier / later runs.
    int carry_left = __shfl_up_sync(0xffffffffu, left, 1);
    int carry_right = __shfl_down_sync(0xffffffffu, right, 1);
    if (lane == 0) {
        carry_left = -kNone;
    }
    if (lane == 31) {
        carry_right = kNone;
    }
    for (int i = 0; i < per_lane; ++i) {
        const int x = begin + i;
        if (x >= sx) {
            break;
        }
        const std::uint32_t at_or_after = bits & (~0u << i);
        const std::uint32_t at_or_before = bits & ((2u << i) - 1u);  // i = 31 wraps to every bit
        const int nearest_right = at_or_after ? begin + __ffs(at_or_after) - 1 : carry_right;
        const int nearest_left = at_or_before ? begin + 31 - __clz(at_or_before) : carry_left;
        const int d = min(x - nearest_left, nearest_right - x);
        out[x] = d >= kNone / 2 ? kInf : d * d;
    }
}

// The same 1D pass for lines of at most kSharedLineMax cells, two lanes per
// line.  Lane h of a pair builds the lower envelope of the sites in its half
// of the line, [h * half, min(len, (h + 1) * half)), in shared memory (site q,
// its value f, and the first coordinate it wins from, clamped to
// [-1, length]: a site whose interval lies wholly outside [0, length) wins no
// cell, so the clamp changes no output).  Each lane then writes its half of
// the outputs as the smaller of the two envelopes evaluated there: the lower
// envelope of a union is the minimum of the envelopes.  One warp holds 16
// lines; consecutive line pairs are consecutive lines, so the loads and
// stores of the y and z passes are coalesced.
constexpr int kSharedLineMax = 512;

__device__ __forceinline__ long long envelope_value(const std::int32_t* sf, const std::int16_t* sq,
                                                    const std::int16_t* ss, int count, int owner, int& site, int q)
{
    while (site + 1 < count && ss[(site + 1) * 32 + owner] <= q) {
        ++site;
    }
    const long long delta = q - sq[site * 32 + owner];
    return static_cast<long long>(sf[site * 32 + owner]) + delta * delta;
}

__global__ void __launch_bounds__(32) edt_pass_shared_kernel(std::int32_t* __restrict__ d2, int sx, int sy, int sz,
                                                             int axis)
{
    extern __shared__ __align__(16) unsigned char stack_raw[];
    const int length = axis == 0 ? sx : axis == 1 ? sy : sz;
    const int half = (length + 1) / 2;
    std::int32_t* sf = reinterpret_cast<std::int32_t*>(stack_raw);     // [half][32]
    std::int16_t* sq = reinterpret_cast<std::int16_t*>(sf + half * 32);  // [half][32]
    std::int16_t* ss = sq + half * 32;                                  // [half][32]
    const int lane = threadIdx.x;
    const int h = lane & 1;
    const long long lines = static_cast<long long>(sx) * sy * sz / length;
    const long long line = static_cast<long long>(blockIdx.x) * 16 + (lane >> 1);
    const bool active = line < lines;  // both lanes of a pair agree
    long long base = 0, stride = 1;
    if (active) {
        if (axis == 0) {
            base = line * sx;
        }
        else if (axis == 1) {
            const long long x = line % sx, z = line / sx;
            base = x + z * static_cast<long long>(sx) * sy;
            stride = sx;
        }
        else {
            base = line;
            stride = static_cast<long long>(sx) * sy;
        }
    }
    const int q_begin = h * half, q_end = min(length, q_begin + half);
    int count = 0;
    if (active) {
        for (int q0 = q_begin; q0 < q_end; q0 += 8) {
            // Eight independent loads in flight before the envelope work.
            std::int32_t fv[8];
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                fv[i] = q0 + i < q_end ? d2[base + (q0 + i) * stride] : kInf;
            }
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                const int q = q0 + i;
                const std::int32_t f = fv[i];
                if (f == kInf) {
                    continue;
                }
                int start = -1;
                while (count > 0) {
                    const int top = (count - 1) * 32 + lane;
                    const long long p = sq[top];
                    const long long numerator = static_cast<long long>(f) - sf[top] + 1LL * q * q - p * p;
                    const long long denominator = 2LL * (q - p);  // positive: q > p
                    // The top site keeps cells before floor(n / d) + 1 when that
                    // exceeds its own first cell S, i.e. when n >= S * d.
                    if (numerator >= static_cast<long long>(ss[top]) * denominator) {
                        long long quotient = numerator / denominator;
                        if (numerator % denominator != 0 && numerator < 0) {
                            --quotient;
                        }
                        const long long first = quotient + 1;
                        start = first < -1 ? -1 : first > length ? length : static_cast<int>(first);
                        break;
                    }
                    --count;
                }
                if (count == 0) {
                    start = -1;
                }
                const int slot = count * 32 + lane;
                sf[slot] = f;
                sq[slot] = static_cast<std::int16_t>(q);
                ss[slot] = static_cast<std::int16_t>(start);
                ++count;
            }
        }
    }
    const int partner_count = __shfl_xor_sync(0xffffffffu, count, 1);
    __syncwarp();
    if (!active) {
        return;
    }
    const int partner = lane ^ 1;
    int own_site = 0, partner_site = 0;
    for (int q = q_begin; q < q_end; ++q) {
        long long best = kInf;
        if (count > 0) {
            best = envelope_value(sf, sq, ss, count, lane, own_site, q);
        }
        if (partner_count > 0) {
            const long long other = envelope_value(sf, sq, ss, partner_count, partner, partner_site, q);
            best = other < best ? other : best;
        }
        d2[base + q * stride] = best >= kInf ? kInf : static_cast<std::int32_t>(best);
    }
}

__global__ void proximity_gather_kernel(const std::int32_t* __restrict__ d2, const double* __restrict__ table,
                                        double* __restrict__ out, long long n)
{
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        const std::int32_t v = d2[i];
        out[i] = v == kInf ? 0.0 : table[v];
    }
}

int blocks_for(long long n, int threads)
{
    const long long want = (n + threads - 1) / threads;
    return static_cast<int>(want < 1 ? 1 : (want > 148LL * 32 ? 148LL * 32 : want));
}

// ---- incremental update after new occupied cells ------------------------

// Largest d2 of each kEdtTile^3 tile: one block of 64 threads per tile,
// thread i scanning the tile's x-run at (y, z) = (i % 8, i / 8).  With a
// region, tiles that do not meet it are left as they are.
__global__ void __launch_bounds__(64) edt_tile_max_kernel(const std::int32_t* __restrict__ d2, int sx, int sy,
                                                         int sz, int tx, int ty, std::int32_t* __restrict__ tile_max,
                                                         const EdtBox* __restrict__ region)
{
    const int t = blockIdx.x;
    const int x0 = (t % tx) * kEdtTile, y0 = ((t / tx) % ty) * kEdtTile, z0 = (t / (tx * ty)) * kEdtTile;
    if (region) {
        const EdtBox r = *region;
        if (x0 >= r.hi[0] || x0 + kEdtTile <= r.lo[0] || y0 >= r.hi[1] || y0 + kEdtTile <= r.lo[1] ||
            z0 >= r.hi[2] || z0 + kEdtTile <= r.lo[2]) {
            return;  // the whole block
        }
    }
    const int y = y0 + (threadIdx.x & 7), z = z0 + (threadIdx.x >> 3);
    std::int32_t m = 0;
    if (y < sy && z < sz) {
        const std::int32_t* row = d2 + x0 + static_cast<long long>(sx) * (y + static_cast<long long>(sy) * z);
        for (int i = 0; i < kEdtTile && x0 + i < sx; ++i) {
            m = max(m, row[i]);
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
    }
    __shared__ std::int32_t warp_max[2];
    if ((threadIdx.x & 31) == 0) {
        warp_max[threadIdx.x >> 5] = m;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        tile_max[t] = max(warp_max[0], warp_max[1]);
    }
}

__global__ void edt_region_init_kernel(EdtBox sites, EdtBox* __restrict__ region)
{
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        *region = sites;
    }
}

// Grows `region` (initialised to the sites' box) by every tile that a new
// site could bring nearer: one whose squared distance to the sites' box is
// below its largest d2.  Every cell of any other tile is at least that far
// from each new site, and already that near an old one.
__global__ void edt_region_kernel(const std::int32_t* __restrict__ tile_max, int sx, int sy, int sz, int tx, int ty,
                                  int tz, EdtBox sites, EdtBox* __restrict__ region)
{
    const long long tiles = static_cast<long long>(tx) * ty * tz;
    int lo[3] = { INT32_MAX, INT32_MAX, INT32_MAX }, hi[3] = { INT32_MIN, INT32_MIN, INT32_MIN };
    const int extent[3] = { sx, sy, sz };
    for (long long t = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; t < tiles;
         t += static_cast<long long>(gridDim.x) * blockDim.x) {
        const int c[3] = { static_cast<int>(t % tx), static_cast<int>((t / tx) % ty),
                           static_cast<int>(t / (1LL * tx * ty)) };
        int a0[3], a1[3];
        long long dist = 0;
        for (int a = 0; a < 3; ++a) {
            a0[a] = c[a] * kEdtTile;
            a1[a] = min(a0[a] + kEdtTile, extent[a]);
            const long long gap = max(0, max(sites.lo[a] - (a1[a] - 1), a0[a] - (sites.hi[a] - 1)));
            dist += gap * gap;
        }
        if (dist < static_cast<long long>(tile_max[t])) {
            for (int a = 0; a < 3; ++a) {
                lo[a] = min(lo[a], a0[a]);
                hi[a] = max(hi[a], a1[a]);
            }
        }
    }
    for (int a = 0; a < 3; ++a) {
        for (int o = 16; o > 0; o >>= 1) {
            lo[a] = min(lo[a], __shfl_xor_sync(0xffffffffu, lo[a], o));
            hi[a] = max(hi[a], __shfl_xor_sync(0xffffffffu, hi[a], o));
        }
    }
    if ((threadIdx.x & 31) == 0 && lo[0] != INT32_MAX) {
        for (int a = 0; a < 3; ++a) {
            atomicMin(&region->lo[a], lo[a]);
            atomicMax(&region->hi[a], hi[a]);
        }
    }
}

// First pass of the new sites' EDT: along x, over the region's x range, the
// squared distance to the nearest site on the same line (a left and a right
// sweep).  Only lines through the sites' box hold sites; every other line of
// the region is infinite and is never read.
__global__ void edt_region_x_kernel(const std::uint8_t* __restrict__ sites, std::int32_t* __restrict__ tmp, int sx,
                                    int sy, EdtBox b, const EdtBox* __restrict__ region)
{
    const EdtBox r = *region;
    const int ny = b.hi[1] - b.lo[1], nz = b.hi[2] - b.lo[2];
    const long long line = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
    if (line >= static_cast<long long>(ny) * nz) {
        return;
    }
    const int y = b.lo[1] + static_cast<int>(line % ny), z = b.lo[2] + static_cast<int>(line / ny);
    const long long base = static_cast<long long>(sx) * (y + static_cast<long long>(sy) * z);
    constexpr int kFar = 1 << 24;
    int last = -kFar;
    for (int x = r.lo[0]; x < r.hi[0]; ++x) {
        if (sites[base + x]) {
            last = x;
        }
        tmp[base + x] = x - last;
    }
    int next = kFar;
    for (int x = r.hi[0] - 1; x >= r.lo[0]; --x) {
        if (sites[base + x]) {
            next = x;
        }
        const int d = min(tmp[base + x], next - x);
        tmp[base + x] = d >= kFar / 2 ? kInf : d * d;
    }
}

// Later passes, along `axis` (1: y, 2: z): one thread per line builds the
// lower envelope of the line's parabolas in shared memory (f, site, first
// cell it wins: the integer rule of the full passes above) and evaluates it
// over the region's extent; the last pass takes min with the old d2.  A line
// holds finite values only inside the sites' box along its axis, so only
// those cells are read.  The y pass covers the lines (x in the region,
// z in the sites' box), which are all the z pass reads; the z pass covers
// every (x, y) of the region.
__global__ void __launch_bounds__(32) edt_region_envelope_kernel(std::int32_t* __restrict__ tmp,
                                                                std::int32_t* __restrict__ d2, int sx, int sy,
                                                                int axis, int last, int max_sites, EdtBox b,
                                                                const EdtBox* __restrict__ region)
{
    extern __shared__ __align__(16) unsigned char stack_raw[];
    std::int32_t* sf = reinterpret_cast<std::int32_t*>(stack_raw);           // [max_sites][32]
    std::int16_t* sq = reinterpret_cast<std::int16_t*>(sf + max_sites * 32);  // [max_sites][32]
    std::int16_t* ss = sq + max_sites * 32;                                   // [max_sites][32]
    const EdtBox r = *region;
    const int lane = threadIdx.x;
    const int length = r.hi[axis] - r.lo[axis];
    const int other = axis == 1 ? 2 : 1;  // the second line coordinate; x is the first
    const int w0 = axis == 1 ? b.lo[2] : r.lo[1];
    const int n0 = r.hi[0] - r.lo[0], n1 = axis == 1 ? b.hi[2] - b.lo[2] : r.hi[1] - r.lo[1];
    const long long line = static_cast<long long>(blockIdx.x) * 32 + lane;
    if (line >= static_cast<long long>(n0) * n1) {
        return;
    }
    const int x = r.lo[0] + static_cast<int>(line % n0);
    const int w = w0 + static_cast<int>(line / n0);
    (void)other;
    const long long plane = static_cast<long long>(sx) * sy;
    const long long stride = axis == 1 ? sx : plane;
    const long long base = x + (axis == 1 ? plane * w : static_cast<long long>(sx) * w) + stride * r.lo[axis];
    // Sites along this axis lie in [b.lo, b.hi), as offsets from the region's start.
    const int q_first = b.lo[axis] - r.lo[axis], q_end = b.hi[axis] - r.lo[axis];
    int count = 0;
    for (int q = q_first; q < q_end; ++q) {
        const std::int32_t f = tmp[base + q * stride];
        if (f == kInf) {
            continue;
        }
        int start = -1;
        while (count > 0) {
            const int top = (count - 1) * 32 + lane;
            const long long p = sq[top];
            const long long numerator = static_cast<long long>(f) - sf[top] + 1LL * q * q - p * p;
            const long long denominator = 2LL * (q - p);
            if (numerator >= static_cast<long long>(ss[top]) * denominator) {
                long long quotient = numerator / denominator;
                if (numerator % denominator != 0 && numerator < 0) {
                    --quotient;
                }
                const long long first = quotient + 1;
                start = first < -1 ? -1 : first > length ? length : static_cast<int>(first);
                break;
            }
            --count;
        }
        if (count == 0) {
            start = -1;
        }
        const int slot = count * 32 + lane;
        sf[slot] = f;
        sq[slot] = static_cast<std::int16_t>(q);
        ss[slot] = static_cast<std::int16_t>(start);
        ++count;
    }
    int site = 0;
    for (int q = 0; q < length; ++q) {
        long long value = kInf;
        if (count > 0) {
            while (site + 1 < count && ss[(site + 1) * 32 + lane] <= q) {
                ++site;
            }
            const long long delta = q - sq[site * 32 + lane];
            value = static_cast<long long>(sf[site * 32 + lane]) + delta * delta;
        }
        const long long at = base + q * stride;
        const std::int32_t v = value >= kInf ? kInf : static_cast<std::int32_t>(value);
        if (last) {
            d2[at] = min(d2[at], v);
        }
        else {
            tmp[at] = v;
        }
    }
}

}  // namespace

int edt_tile_max(spk_context* ctx, const std::int32_t* d_d2, const std::uint32_t* shape, std::int32_t* d_tile_max,
                 cudaStream_t stream)
{
    const int tx = (static_cast<int>(shape[0]) + kEdtTile - 1) / kEdtTile;
    const int ty = (static_cast<int>(shape[1]) + kEdtTile - 1) / kEdtTile;
    const int tz = (static_cast<int>(shape[2]) + kEdtTile - 1) / kEdtTile;
    edt_tile_max_kernel<<<tx * ty * tz, 64, 0, stream>>>(d_d2, shape[0], shape[1], shape[2], tx, ty, d_tile_max,
                                                         nullptr);
    ctx->launches++;
    return cudaGetLastError() == cudaSuccess ? kOk : kCuda;
}

int edt_add_sites(spk_context* ctx, const std::uint8_t* d_sites, const EdtBox& sites, std::int32_t* d_d2,
                  std::int32_t* d_tile_max, const std::uint32_t* shape, cudaStream_t stream)
{
    EdtBox box = sites;
    for (int a = 0; a < 3; ++a) {
        box.lo[a] = std::max(box.lo[a], 0);
        box.hi[a] = std::min(box.hi[a], static_cast<int>(shape[a]));
        if (box.lo[a] >= box.hi[a]) {
            return kOk;  // no new site inside the window
        }
    }
    const int sx = static_cast<int>(shape[0]), sy = static_cast<int>(shape[1]), sz = static_cast<int>(shape[2]);
    if (sx > 32767 || sy > 32767 || sz > 32767) {
        return kInvalidArgument;  // sites are held as 16-bit coordinates
    }
    const long long n = static_cast<long long>(sx) * sy * sz;
    int status = kOk;
    auto* region = static_cast<EdtBox*>(device_buffer(ctx, "edt.region", sizeof(EdtBox), status));
    auto* tmp = static_cast<std::int32_t*>(device_buffer(ctx, "edt.tmp", n * sizeof(std::int32_t), status));
    if (!region || !tmp) {
        return status;
    }
    const int tx = (sx + kEdtTile - 1) / kEdtTile, ty = (sy + kEdtTile - 1) / kEdtTile,
              tz = (sz + kEdtTile - 1) / kEdtTile;
    const long long tiles = static_cast<long long>(tx) * ty * tz;
    const int longest = std::max(box.hi[1] - box.lo[1], box.hi[2] - box.lo[2]);
    if (static_cast<long long>(longest) * 32 * 8 > 227LL * 1024) {
        return kInvalidArgument;
    }
    static std::once_flag attribute[64];
    once_per_device(attribute, [] {
        cudaFuncSetAttribute(edt_region_envelope_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
    });
    edt_region_init_kernel<<<1, 32, 0, stream>>>(box, region);
    edt_region_kernel<<<blocks_for(tiles, 256), 256, 0, stream>>>(d_tile_max, sx, sy, sz, tx, ty, tz, box, region);
    const int by = box.hi[1] - box.lo[1], bz = box.hi[2] - box.lo[2];
    edt_region_x_kernel<<<static_cast<unsigned>((static_cast<long long>(by) * bz + 127) / 128), 128, 0, stream>>>(
        d_sites, tmp, sx, sy, box, region);
    edt_region_envelope_kernel<<<static_cast<unsigned>((static_cast<long long>(sx) * bz + 31) / 32), 32,
                                 static_cast<std::size_t>(by) * 32 * 8, stream>>>(tmp, d_d2, sx, sy, 1, 0, by, box,
                                                                                  region);
    edt_region_envelope_kernel<<<static_cast<unsigned>((static_cast<long long>(sx) * sy + 31) / 32), 32,
                                 static_cast<std::size_t>(bz) * 32 * 8, stream>>>(tmp, d_d2, sx, sy, 2, 1, bz, box,
                                                                                  region);
    edt_tile_max_kernel<<<static_cast<unsigned>(tiles), 64, 0, stream>>>(d_d2, sx, sy, sz, tx, ty, d_tile_max,
                                                                          region);
    ctx->launches += 6;
    return cudaGetLastError() == cudaSuccess ? kOk : kCuda;
}

bool proximity_shape_supported(const std::uint32_t* shape)
{
    std::uint64_t sum = 0;
    for (int a = 0; a != 3; ++a) {
        if (shape[a] == 0) {
            return false;
        }
        const std::uint64_t extent = shape[a] - 1;
        if (extent > 94'906'265 || extent * extent > (1ULL << 53) - sum) {
            return false;
        }
        sum += extent * extent;
    }
    return true;
}

std::int32_t max_squared_distance(const std::uint32_t* shape)
{
    std::int64_t sum = 0;
    for (int a = 0; a != 3; ++a) {
        sum += static_cast<std::int64_t>(shape[a] - 1) * (shape[a] - 1);
    }
    return static_cast<std::int32_t>(sum);
}

const double* proximity_table(spk_context* ctx, std::int32_t max_d2, int& status)
{
    const std::size_t want = static_cast<std::size_t>(max_d2) + 1;
    auto& b = ctx->device_buffers["prox.table"];
    if (b.ptr && b.bytes >= want * sizeof(double)) {
        return static_cast<const double*>(b.ptr);
    }
    std::vector<double> host(want);
    for (std::size_t v = 0; v < want; ++v) {
        host[v] = std::exp(-std::sqrt(static_cast<double>(v)) / 2.);
    }
    auto* d = static_cast<double*>(device_buffer(ctx, "prox.table", want * sizeof(double), status));
    if (!d) {
        return nullptr;
    }
    if (!upload_table(ctx, d, host.data(), want * sizeof(double))) {
        status = kCuda;
        return nullptr;
    }
    return d;
}

int edt_squared(spk_context* ctx, const std::uint8_t* d_occupied, std::int32_t* d_d2, const std::uint32_t* shape,
                cudaStream_t stream)
{
    const long long n = static_cast<long long>(shape[0]) * shape[1] * shape[2];
    int status = kOk;
    auto* line_f = static_cast<std::int32_t*>(device_buffer(ctx, "edt.f", n * sizeof(std::int32_t), status));
    auto* site_q = static_cast<std::int32_t*>(device_buffer(ctx, "edt.q", n * sizeof(std::int32_t), status));
    auto* site_s = static_cast<long long*>(device_buffer(ctx, "edt.s", n * sizeof(long long), status));
    if (!line_f || !site_q || !site_s) {
        return status;
    }
    const bool first_fused = shape[0] <= 32u * kFirstPassPerLane;
    if (first_fused) {
        const long long lines = n / shape[0];
        edt_first_pass_kernel<<<static_cast<unsigned>((lines + 7) / 8), 256, 0, stream>>>(d_occupied, d_d2,
                                                                                          shape[0], lines);
    }
    else {
        edt_init_kernel<<<blocks_for(n, 256), 256, 0, stream>>>(d_occupied, d_d2, n);
    }
    ctx->launches++;
    static std::once_flag attribute[64];
    once_per_device(attribute, [] {
        cudaFuncSetAttribute(edt_pass_shared_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (kSharedLineMax + 1) / 2 * 32 * 8);
    });
    for (int axis = first_fused ? 1 : 0; axis != 3; ++axis) {
        const long long lines = n / shape[axis];
        if (shape[axis] <= static_cast<std::uint32_t>(kSharedLineMax)) {
            const unsigned stack_bytes = (shape[axis] + 1) / 2 * 32 * 8;
            edt_pass_shared_kernel<<<static_cast<unsigned>((lines + 15) / 16), 32, stack_bytes, stream>>>(
                d_d2, shape[0], shape[1], shape[2], axis);
        }
        else {
            edt_pass_kernel<<<static_cast<unsigned>((lines + 127) / 128), 128, 0, stream>>>(
                d_d2, line_f, site_q, site_s, shape[0], shape[1], shape[2], axis);
        }
        ctx->launches++;
    }
    return cudaGetLastError() == cudaSuccess ? kOk : kCuda;
}

int proximity_from_d2(spk_context* ctx, const std::int32_t* d_d2, double* d_out, const std::uint32_t* shape,
                      cudaStream_t stream)
{
    int status = kOk;
    const double* table = proximity_table(ctx, max_squared_distance(shape), status);
    if (!table) {
        return status;
    }
    const long long n = static_cast<long long>(shape[0]) * shape[1] * shape[2];
    proximity_gather_kernel<<<blocks_for(n, 256), 256, 0, stream>>>(d_d2, table, d_out, n);
    ctx->launches++;
    return cudaGetLastError() == cudaSuccess ? kOk : kCuda;
}

}  // namespace spk

// ---- allocation-free variant ---------------------------------------------
//
// Scratch for fields of up to kStaticCells cells lives in one file-scope
// device array: squared distances, the three line scratch arrays and the
// exp(-sqrt(v)/2) table.  Host code never uses the array's name as a device
// address; the address comes from cudaGetSymbolAddress, looked up once per
// device with that device current.
namespace spk {
namespace {

constexpr std::uint32_t kStaticCells = SPK_STATIC_PROXIMITY_MAX_CELLS;
constexpr std::int32_t kStaticMaxD2 = 3 * 63 * 63;  // largest d2 of a field whose cells fit (64^3)
constexpr std::size_t kStaticD2 = 0;
constexpr std::size_t kStaticLineF = kStaticD2 + 4ULL * kStaticCells;
constexpr std::size_t kStaticSiteQ = kStaticLineF + 4ULL * kStaticCells;
constexpr std::size_t kStaticSiteS = kStaticSiteQ + 4ULL * kStaticCells;
constexpr std::size_t kStaticTable = kStaticSiteS + 8ULL * kStaticCells;
constexpr std::size_t kStaticBytes = kStaticTable + 8ULL * (kStaticMaxD2 + 1);

__device__ __align__(256) unsigned char g_static_scratch[kStaticBytes];

constexpr int kMaxDevices = 64;
unsigned char* g_scratch_address[kMaxDevices] {};
std::mutex g_scratch_mutex;
double g_table_host[kStaticMaxD2 + 1];
bool g_table_ready = false;

// Largest d2 any shape with at most kStaticCells cells can produce.
std::int32_t static_max_d2(const std::uint32_t* shape) { return max_squared_distance(shape); }

int static_setup(int device, cudaStream_t stream, unsigned char*& base)
{
    std::lock_guard<std::mutex> lock(g_scratch_mutex);
    if (device < 0 || device >= kMaxDevices) {
        return kInvalidArgument;
    }
    if (g_scratch_address[device]) {
        base = g_scratch_address[device];
        return kOk;
    }
    void* address = nullptr;
    if (cudaGetSymbolAddress(&address, g_static_scratch) != cudaSuccess || !address) {
        cudaGetLastError();
        return kCuda;
    }
    if (!g_table_ready) {
        for (std::int32_t v = 0; v <= kStaticMaxD2; ++v) {
            g_table_host[v] = std::exp(-std::sqrt(static_cast<double>(v)) / 2.);
        }
        g_table_ready = true;
    }
    auto* bytes = static_cast<unsigned char*>(address);
    if (cudaMemcpyAsync(bytes + kStaticTable, g_table_host, sizeof(g_table_host), cudaMemcpyHostToDevice, stream) !=
            cudaSuccess ||
        cudaStreamSynchronize(stream) != cudaSuccess) {
        cudaGetLastError();
        return kCuda;
    }
    g_scratch_address[device] = bytes;
    base = bytes;
    return kOk;
}

}  // namespace

}  // namespace spk

using namespace spk;

extern "C" int spk_build_proximity_static(void* stream_handle, const uint32_t shape[3], const uint8_t* occupied,
                                          double* values)
{
    try {
        if (!shape || !occupied || !values) {
            return kInvalidArgument;
        }
        if (!proximity_shape_supported(shape)) {
            return kProximityShape;
        }
        if (shape[0] > 64 || shape[1] > 64 || shape[2] > 64) {
            return kScratchLimit;  // beyond the static scratch: 64 cells per axis
        }
        const unsigned long long n = static_cast<unsigned long long>(shape[0]) * shape[1] * shape[2];
        if (n > kStaticCells || static_max_d2(shape) > kStaticMaxD2) {
            return kScratchLimit;
        }
        int device = 0;
        if (cudaGetDevice(&device) != cudaSuccess) {
            cudaGetLastError();
            return kCuda;
        }
        auto stream = static_cast<cudaStream_t>(stream_handle);
        unsigned char* base = nullptr;
        int status = static_setup(device, stream, base);
        if (status) {
            return status;
        }
        auto* d2 = reinterpret_cast<std::int32_t*>(base + kStaticD2);
        auto* line_f = reinterpret_cast<std::int32_t*>(base + kStaticLineF);
        auto* site_q = reinterpret_cast<std::int32_t*>(base + kStaticSiteQ);
        auto* site_s = reinterpret_cast<long long*>(base + kStaticSiteS);
        const auto* table = reinterpret_cast<const double*>(base + kStaticTable);
        const long long cells = static_cast<long long>(n);
        // Every scratch cell that is read is written first in this call.
        edt_init_kernel<<<blocks_for(cells, 256), 256, 0, stream>>>(occupied, d2, cells);
        for (int axis = 0; axis != 3; ++axis) {
            const long long lines = cells / shape[axis];
            edt_pass_kernel<<<static_cast<unsigned>((lines + 127) / 128), 128, 0, stream>>>(
                d2, line_f, site_q, site_s, shape[0], shape[1], shape[2], axis);
        }
        proximity_gather_kernel<<<blocks_for(cells, 256), 256, 0, stream>>>(d2, table, values, cells);
        return cudaGetLastError() == cudaSuccess ? kOk : kCuda;
    }
    catch (...) {
        return kCuda;
    }
}

extern "C" int spk_build_proximity(spk_context* ctx, const uint32_t shape[3], const uint8_t* occupied, double* values)
{
    try {
        if (!ctx || !shape || !occupied || !values) {
            return kInvalidArgument;
        }
        if (!proximity_shape_supported(shape)) {
            return kProximityShape;
        }
        if (cudaSetDevice(ctx->device) != cudaSuccess) {
            return kCuda;
        }
        const long long n = static_cast<long long>(shape[0]) * shape[1] * shape[2];
        int status = kOk;
        auto* d_occ = static_cast<std::uint8_t*>(device_buffer(ctx, "prox.occ", n, status));
        auto* d_d2 = static_cast<std::int32_t*>(device_buffer(ctx, "prox.d2", n * sizeof(std::int32_t), status));
        auto* d_out = static_cast<double*>(device_buffer(ctx, "prox.out", n * sizeof(double), status));
        if (!d_occ || !d_d2 || !d_out) {
            return status;
        }
        cudaMemcpyAsync(d_occ, occupied, n, cudaMemcpyHostToDevice, ctx->stream);
        if ((status = edt_squared(ctx, d_occ, d_d2, shape, ctx->stream))) {
            return status;
        }
        if ((status = proximity_from_d2(ctx, d_d2, d_out, shape, ctx->stream))) {
            return status;
        }
        cudaMemcpyAsync(values, d_out, n * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream);
        return cudaStreamSynchronize(ctx->stream) == cudaSuccess ? kOk : kCuda;
    }
    catch (...) {
        return kAllocation;
    }
}
