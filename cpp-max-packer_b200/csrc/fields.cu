// Conservative fields on the GPU: boundary rasterisation, component labelling,
// witness fill, clearance dilation, the analytic box container, and the
// blocked-field stamp/unstamp with occupancy extraction.
//
// Reference (engine/pack_geometry/src): rasterize_boundary + run_raster_cursor
// (validation_kernel.cpp:3248-3340, 3668-3762) tag a cell 2 when the closed
// cell's interval box and a triangle's vertex intervals are not SAT-disjoint;
// fill_components (conservative_fields.cpp:257-360) gives every 6-connected
// component of non-2 cells the decision of its first cell in scan order
// (0 void, 1 material, 3 uncertain); dilate_and_crop (:436-504) marks every
// requested cell reached by a seed through the clearance stencil;
// BlockedField::add/remove/blocked (:1666-1886) keep per-cell copy counts and
// report mask || count.  The rasterised tags are an OR over faces, so one warp
// per face with benign same-value writes reproduces them exactly; component
// roots are the minimum linear index (= first in scan order) by union-find.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <vector>

#include "context.hpp"
#include "fields.hpp"
#include "interval.cuh"

namespace spk {

namespace {

int blocks_for(long long n, int threads)
{
    const long long want = (n + threads - 1) / threads;
    return static_cast<int>(std::min<long long>(std::max<long long>(want, 1), 148LL * 32));
}

// The placed copy's vertex intervals (place(), validation_kernel.cpp:
// 805-943) on the device, for a rotation that is not cardinal: each
// coordinate is transformed_interval_at, the code the host runs.  Each block
// also reduces its vertices' bounds (lowest low, highest high per axis) into
// partial[block]; error[0] is set when an interval is not valid.
struct PoseIntervals {
    Interval rotation[3][3];
    double translation[3];
};

__global__ void __launch_bounds__(256) vertex_intervals_kernel(const double* __restrict__ vertices, int count,
                                                              const PoseIntervals pose, IVec3* __restrict__ vint,
                                                              double* __restrict__ partial, int* __restrict__ error)
{
    __shared__ double lows[3][256], highs[3][256];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double lo[3], hi[3];
    for (int a = 0; a < 3; ++a) {
        lo[a] = INFINITY;
        hi[a] = -INFINITY;
    }
    if (i < count) {
        const double point[3] = { vertices[3 * i], vertices[3 * i + 1], vertices[3 * i + 2] };
        IVec3 out;
        bool valid = true;
        for (int a = 0; a < 3; ++a) {
            out.v[a] = transformed_interval_at(point, pose.translation, pose.rotation, a);
            valid = valid && out.v[a].valid;
            lo[a] = out.v[a].low;
            hi[a] = out.v[a].high;
        }
        vint[i] = out;
        if (!valid) {
            atomicOr(error, 1);
        }
    }
    for (int a = 0; a < 3; ++a) {
        lows[a][threadIdx.x] = lo[a];
        highs[a][threadIdx.x] = hi[a];
    }
    __syncthreads();
    for (int h = 128; h > 0; h >>= 1) {
        if (threadIdx.x < h) {
            for (int a = 0; a < 3; ++a) {
                lows[a][threadIdx.x] = f_min(lows[a][threadIdx.x], lows[a][threadIdx.x + h]);
                highs[a][threadIdx.x] = f_max(highs[a][threadIdx.x], highs[a][threadIdx.x + h]);
            }
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        for (int a = 0; a < 3; ++a) {
            partial[6 * blockIdx.x + a] = lows[a][0];
            partial[6 * blockIdx.x + 3 + a] = highs[a][0];
        }
    }
}

// The blocks' partial bounds reduced to out[0..5] (one thread).
__global__ void vertex_bounds_kernel(const double* __restrict__ partial, int blocks, double* __restrict__ out)
{
    double b[6] = { INFINITY, INFINITY, INFINITY, -INFINITY, -INFINITY, -INFINITY };
    for (int k = 0; k < blocks; ++k) {
        for (int a = 0; a < 3; ++a) {
            b[a] = f_min(b[a], partial[6 * k + a]);
            b[3 + a] = f_max(b[3 + a], partial[6 * k + 3 + a]);
        }
    }
    for (int a = 0; a < 6; ++a) {
        out[a] = b[a];
    }
}

// Per-face candidate cell ranges on the device: face_ranges
// (validation_kernel.cpp:3248-3340 cursor bounds) with the host's binary64
// path, floor((v - origin) / pitch) when the quotient lies farther than
// |q| 2^-48 + 2^-60 from every integer.  Nearer to an integer n the host
// takes the floor of a long double quotient, which is n - 1 or n; here the
// range takes n - 1 for its low end and n for its high end instead.  The
// range is then at most one cell wider than the host's, and a cell it adds
// lies outside the face's padded interval bounds, where the SAT's first
// three axes separate it: the raster is the same.  Quotients of magnitude
// 2^50 or more, or not finite, set bit 4 of error[0] (the host path then
// runs).  counts[f] = the clipped range's cell count (0 when outside).
__global__ void face_ranges_kernel(const std::uint32_t* __restrict__ tris, const IVec3* __restrict__ vint, int faces,
                                   FieldWindow w, geo::FaceRange* __restrict__ ranges,
                                   long long* __restrict__ counts, int* __restrict__ error)
{
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= faces) {
        return;
    }
    geo::FaceRange r;
    r.outside = 0;
    r.pad = 0;
    bool host_needed = false;
    for (int a = 0; a < 3; ++a) {
        const IVec3& v0 = vint[tris[3 * f]];
        double low = v0.v[a].low, high = v0.v[a].high;
        for (int k = 1; k < 3; ++k) {
            const IVec3& vk = vint[tris[3 * f + k]];
            low = f_min(low, vk.v[a].low);
            high = f_max(high, vk.v[a].high);
        }
        long long ends[2];
        for (int e = 0; e < 2; ++e) {
            const double q = f_div(f_sub(e == 0 ? low : high, w.origin[a]), w.pitch);
            if (!(fabs(q) < 0x1p50)) {
                host_needed = true;
                ends[e] = 0;
                continue;
            }
            const double fl = floor(q);
            const double margin = f_add(f_mul(fabs(q), 0x1p-48), 0x1p-60);
            if (f_sub(q, fl) > margin && f_sub(f_add(fl, 1.0), q) > margin) {
                ends[e] = static_cast<long long>(fl);
            }
            else {
                const long long n = static_cast<long long>(rint(q));
                ends[e] = e == 0 ? n - 1 : n;
            }
        }
        r.first[a] = ends[0] - 1;
        r.last[a] = ends[1] + 1;
        const long long wlast = w.first[a] + static_cast<long long>(w.shape[a] - 1);
        if (r.last[a] < w.first[a] || r.first[a] > wlast) {
            r.outside = 1;
        }
        r.first[a] = r.first[a] > w.first[a] ? r.first[a] : w.first[a];
        r.last[a] = r.last[a] < wlast ? r.last[a] : wlast;
    }
    if (host_needed) {
        atomicOr(error, 4);
    }
    ranges[f] = r;
    long long cells = 0;
    if (!r.outside && r.last[0] >= r.first[0] && r.last[1] >= r.first[1] && r.last[2] >= r.first[2]) {
        cells = (r.last[0] - r.first[0] + 1) * (r.last[1] - r.first[1] + 1) * (r.last[2] - r.first[2] + 1);
    }
    counts[f] = cells;
}

// offsets[0] = 0, offsets[f + 1] = counts[0] + ... + counts[f], in place
// over offsets[1..faces] (the counts); one block of 1024 threads.
__global__ void __launch_bounds__(1024) face_offsets_kernel(long long* __restrict__ offsets, int faces)
{
    __shared__ long long warp_sums[32];
    __shared__ long long carry;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (threadIdx.x == 0) {
        carry = 0;
        offsets[0] = 0;
    }
    __syncthreads();
    for (int start = 0; start < faces; start += 1024) {
        const int i = start + threadIdx.x;
        const long long v = i < faces ? offsets[1 + i] : 0;
        long long inclusive = v;
        for (int o = 1; o < 32; o <<= 1) {
            const long long other = __shfl_up_sync(0xffffffffu, inclusive, o);
            if (lane >= o) {
                inclusive += other;
            }
        }
        if (lane == 31) {
            warp_sums[warp] = inclusive;
        }
        __syncthreads();
        long long before = carry;
        for (int k = 0; k < warp; ++k) {
            before += warp_sums[k];
        }
        if (i < faces) {
            offsets[1 + i] = before + inclusive;
        }
        __syncthreads();
        if (threadIdx.x == 1023) {
            carry = before + inclusive;
        }
        __syncthreads();
    }
}

// One thread per (face, cell) pair.  `offsets` is the exclusive prefix sum of
// the faces' clipped cell-range sizes (outside faces count 0), so small faces
// pack densely into warps instead of leaving most lanes of a per-face warp idle.
// The pair count is offsets[faces], read on the device.
// The triangle-only part of each face's separating-axis test (face_sat),
// once per face before the raster: 16 threads per face, thread i < 10
// computing axis i and thread 10 the box-axis bounds.
__global__ void face_sat_kernel(const std::uint32_t* __restrict__ tris, const IVec3* __restrict__ vint, int faces,
                                FaceSat* __restrict__ sats)
{
    const long long thread = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    const long long face = thread >> 4;
    const int i = static_cast<int>(thread & 15);
    if (face >= faces || i > 10) {
        return;
    }
    IVec3 tri[3];
    for (int k = 0; k < 3; ++k) {
        tri[k] = vint[tris[3 * face + k]];
    }
    if (i == 10) {
        face_sat_bounds(tri, sats[face]);
    }
    else {
        face_sat_axis(tri, i, sats[face]);
    }
}

__global__ void __launch_bounds__(128, 6) raster_kernel(const FaceSat* __restrict__ sats,
                              const geo::FaceRange* __restrict__ ranges, const long long* __restrict__ offsets,
                              int faces, FieldWindow w, std::uint8_t* __restrict__ cells,
                              int* __restrict__ error)
{
    const long long total = offsets[faces];
    for (long long item = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; item < total;
         item += static_cast<long long>(gridDim.x) * blockDim.x) {
        int lo = 0, hi = faces - 1;  // last face whose offset is <= item: the face that owns it
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (offsets[mid] <= item) {
                lo = mid;
            } else {
                hi = mid - 1;
            }
        }
        const int face = lo;
        const geo::FaceRange r = ranges[face];
        const long long nx = r.last[0] - r.first[0] + 1, ny = r.last[1] - r.first[1] + 1;
        const long long c = item - offsets[face];
        std::int64_t index[3];
        index[0] = r.first[0] + c % nx;
        index[1] = r.first[1] + (c / nx) % ny;
        index[2] = r.first[2] + c / (nx * ny);
        const long long flat = (index[0] - w.first[0]) +
                               static_cast<long long>(w.shape[0]) *
                                   ((index[1] - w.first[1]) + static_cast<long long>(w.shape[1]) * (index[2] - w.first[2]));
        if (cells[flat] == 2) {
            continue;
        }
        IVec3 box;
        if (!grid_cell_interval(w.origin, w.pitch, index, box)) {
            atomicOr(error, 1);
            continue;
        }
        if (!face_sat_disjoint(sats[face], box)) {
            cells[flat] = 2;
        }
    }
}

__device__ int find_root(const int* __restrict__ parent, int i)
{
    for (int guard = 0; guard < (1 << 26); ++guard) {
        const int p = parent[i];
        if (p == i) {
            return i;
        }
        i = p;
    }
    return i;
}

__global__ void ccl_init_kernel(const std::uint8_t* __restrict__ cells, int* __restrict__ parent, long long n)
{
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        parent[i] = cells[i] == 2 ? -1 : static_cast<int>(i);
    }
}

__device__ void unite(int* parent, int a, int b, int* error)
{
    for (int guard = 0; guard < (1 << 24); ++guard) {
        a = find_root(parent, a);
        b = find_root(parent, b);
        if (a == b) {
            return;
        }
        if (a < b) {
            const int t = a;
            a = b;
            b = t;
        }
        const int old = atomicMin(&parent[a], b);
        if (old == a) {
            return;
        }
        a = old;
    }
    atomicOr(error, 2);  // bounded retries exhausted: reported, never spun forever
}

__global__ void ccl_union_kernel(const std::uint8_t* __restrict__ cells, int* __restrict__ parent, int sx, int sy,
                                 int sz, int* __restrict__ error)
{
    const long long n = static_cast<long long>(sx) * sy * sz;
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        if (cells[i] == 2) {
            continue;
        }
        const int x = static_cast<int>(i % sx);
        const long long r = i / sx;
        const int y = static_cast<int>(r % sy);
        const int z = static_cast<int>(r / sy);
        if (x > 0 && cells[i - 1] != 2) {
            unite(parent, static_cast<int>(i), static_cast<int>(i - 1), error);
        }
        if (y > 0 && cells[i - sx] != 2) {
            unite(parent, static_cast<int>(i), static_cast<int>(i - sx), error);
        }
        if (z > 0 && cells[i - static_cast<long long>(sx) * sy] != 2) {
            unite(parent, static_cast<int>(i), static_cast<int>(i - static_cast<long long>(sx) * sy), error);
        }
    }
}

__global__ void ccl_compress_kernel(int* __restrict__ parent, long long n, int* __restrict__ roots,
                                    unsigned int* __restrict__ root_count, unsigned int root_capacity)
{
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        if (parent[i] < 0) {
            continue;
        }
        const int root = find_root(parent, static_cast<int>(i));
        parent[i] = root;
        if (root == static_cast<int>(i)) {
            const unsigned int slot = atomicAdd(root_count, 1u);
            if (slot < root_capacity) {
                roots[slot] = root;
            }
        }
    }
}

__global__ void scatter_decisions_kernel(const int* __restrict__ roots, const std::uint8_t* __restrict__ values,
                                         int count, std::uint8_t* __restrict__ root_value)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < count) {
        root_value[roots[i]] = values[i];
    }
}

__global__ void fill_kernel(std::uint8_t* __restrict__ cells, const int* __restrict__ parent,
                            const std::uint8_t* __restrict__ root_value, long long n, int normalize)
{
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        std::uint8_t v = cells[i];
        if (v != 2) {
            v = root_value[parent[i]];
        }
        cells[i] = normalize ? (v != 0 ? 1 : 0) : v;
    }
}

// out[t] over `req` = OR over stencil deltas d of seed(raw[t - d]) inside `raw`.
// A sub-box [lo, lo + extent) of a window (cell offsets from its first
// cell); the box kernels visit its cells only.
struct CellBox {
    int lo[3];
    int extent[3];
};

__device__ __forceinline__ long long box_cells(const CellBox& b)
{
    return static_cast<long long>(b.extent[0]) * b.extent[1] * b.extent[2];
}

// Offset (x, y, z) from the window's first cell of the box's cell i.
__device__ __forceinline__ void box_cell(const CellBox& b, long long i, int (&c)[3])
{
    c[0] = b.lo[0] + static_cast<int>(i % b.extent[0]);
    c[1] = b.lo[1] + static_cast<int>((i / b.extent[0]) % b.extent[1]);
    c[2] = b.lo[2] + static_cast<int>(i / (static_cast<long long>(b.extent[0]) * b.extent[1]));
}

__global__ void dilate_kernel(const std::uint8_t* __restrict__ raw, FieldWindow rw,
                              const int* __restrict__ stencil, int stencil_count, int invert,
                              std::uint8_t* __restrict__ out, FieldWindow req, CellBox box)
{
    const long long n = box_cells(box);
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        int c[3];
        box_cell(box, i, c);
        const long long t[3] = { req.first[0] + c[0], req.first[1] + c[1], req.first[2] + c[2] };
        const long long at = c[0] + static_cast<long long>(req.shape[0]) * (c[1] + static_cast<long long>(req.shape[1]) * c[2]);
        std::uint8_t value = 0;
        for (int s = 0; s < stencil_count && !value; ++s) {
            const long long sx = t[0] - stencil[3 * s] - rw.first[0];
            const long long sy = t[1] - stencil[3 * s + 1] - rw.first[1];
            const long long sz = t[2] - stencil[3 * s + 2] - rw.first[2];
            if (sx < 0 || sy < 0 || sz < 0 || sx >= rw.shape[0] || sy >= rw.shape[1] || sz >= rw.shape[2]) {
                continue;
            }
            const std::uint8_t v = raw[sx + rw.shape[0] * (sy + static_cast<long long>(rw.shape[1]) * sz)];
            value = invert ? (v != 1) : (v != 0);
        }
        out[at] = value;
    }
}

__global__ void box_mask_kernel(const std::uint8_t* __restrict__ ax, const std::uint8_t* __restrict__ ay,
                                const std::uint8_t* __restrict__ az, int sx, int sy, int sz,
                                std::uint8_t* __restrict__ mask)
{
    const long long n = static_cast<long long>(sx) * sy * sz;
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        const int x = static_cast<int>(i % sx);
        const long long r = i / sx;
        const int y = static_cast<int>(r % sy);
        const int z = static_cast<int>(r / sy);
        mask[i] = (ax[x] && ay[y] && az[z]) ? 0 : 1;
    }
}

__global__ void stamp_box_kernel(std::uint32_t* __restrict__ counts, const std::uint8_t* __restrict__ placed,
                                 int sx, int sy, CellBox box, int direction)
{
    const long long n = box_cells(box);
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        int c[3];
        box_cell(box, i, c);
        const long long at = c[0] + static_cast<long long>(sx) * (c[1] + static_cast<long long>(sy) * c[2]);
        if (placed[at]) {
            counts[at] += direction > 0 ? 1u : static_cast<std::uint32_t>(-1);
        }
    }
}

__global__ void occupancy_box_kernel(const std::uint8_t* __restrict__ mask, const std::uint32_t* __restrict__ counts,
                                     std::uint8_t* __restrict__ occ, int sx, int sy, CellBox box)
{
    const long long n = box_cells(box);
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        int c[3];
        box_cell(box, i, c);
        const long long at = c[0] + static_cast<long long>(sx) * (c[1] + static_cast<long long>(sy) * c[2]);
        occ[at] = (mask[at] != 0 || counts[at] != 0) ? 1 : 0;
    }
}

__global__ void stamp_kernel(std::uint32_t* __restrict__ counts, const std::uint8_t* __restrict__ placed, long long n,
                             int direction)
{
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        if (placed[i]) {
            counts[i] += direction > 0 ? 1u : static_cast<std::uint32_t>(-1);
        }
    }
}

__global__ void occupancy_kernel(const std::uint8_t* __restrict__ mask, const std::uint32_t* __restrict__ counts,
                                 std::uint8_t* __restrict__ occ, long long n)
{
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        occ[i] = (mask[i] != 0 || counts[i] != 0) ? 1 : 0;
    }
}

}  // namespace

namespace {

int raster_fill_impl(spk_context* ctx, const geo::Placed& placed, const FieldWindow& w, std::uint8_t* d_cells,
                     bool normalize, std::uint64_t* uncertain_components, const std::uint32_t* d_tris_kept,
                     bool device_intervals, bool host_ranges)
{
    cudaStream_t st = ctx->stream;
    const auto& mesh = *placed.prepared->mesh;
    const long long n = static_cast<long long>(w.shape[0]) * w.shape[1] * w.shape[2];
    if (n >= (1LL << 31)) {
        return kCellLimit;
    }
    const std::size_t F = mesh.triangles.size(), V = mesh.vertices.size();
    int status = kOk;
    auto* d_tris = d_tris_kept ? const_cast<std::uint32_t*>(d_tris_kept)
                               : static_cast<std::uint32_t*>(device_buffer(ctx, "field.tris", F * 12, status));
    auto* d_vint = static_cast<IVec3*>(device_buffer(ctx, "field.vint", V * sizeof(IVec3), status));
    auto* h_vint = static_cast<IVec3*>(host_buffer(ctx, "field.vint", V * sizeof(IVec3), status));
    auto* d_ranges = static_cast<geo::FaceRange*>(device_buffer(ctx, "field.ranges", F * sizeof(geo::FaceRange), status));
    auto* d_offsets = static_cast<long long*>(device_buffer(ctx, "field.offsets", (F + 1) * sizeof(long long), status));
    auto* d_sats = static_cast<FaceSat*>(device_buffer(ctx, "field.sats", F * sizeof(FaceSat), status));
    auto* d_parent = static_cast<int*>(device_buffer(ctx, "field.parent", n * sizeof(int), status));
    auto* d_rootv = static_cast<std::uint8_t*>(device_buffer(ctx, "field.rootv", n, status));
    auto* d_misc = static_cast<int*>(device_buffer(ctx, "field.misc", 64, status));
    const unsigned int root_capacity = 1u << 20;
    auto* d_roots = static_cast<int*>(device_buffer(ctx, "field.roots", root_capacity * 4ULL, status));
    if (!d_tris || !d_vint || !h_vint || !d_ranges || !d_offsets || !d_sats || !d_parent || !d_rootv || !d_misc ||
        !d_roots) {
        return status;
    }
    if (!d_tris_kept) {
        cudaMemcpyAsync(d_tris, mesh.triangles.data(), F * 12, cudaMemcpyHostToDevice, st);
    }
    if (!device_intervals) {
        // The vertex intervals go through pinned memory (the previous call's
        // copy finished at its synchronisation below).
        std::memcpy(h_vint, placed.intervals.data(), V * sizeof(IVec3));
        cudaMemcpyAsync(d_vint, h_vint, V * sizeof(IVec3), cudaMemcpyHostToDevice, st);
    }
    cudaMemsetAsync(d_cells, 0, n, st);
    cudaMemsetAsync(d_misc, 0, 64, st);
    const int threads = 256;
    if (F > 0) {
        if (host_ranges) {
            geo::Window gw;
            for (int a = 0; a < 3; ++a) {
                gw.first[a] = w.first[a];
                gw.shape[a] = w.shape[a];
            }
            // The host reads the vertex intervals; those made on the device
            // come back first.
            const geo::Placed* source = &placed;
            geo::Placed with_intervals;
            if (device_intervals) {
                with_intervals = placed;
                with_intervals.intervals.resize(V);
                if (cudaMemcpyAsync(with_intervals.intervals.data(), d_vint, V * sizeof(IVec3), cudaMemcpyDeviceToHost,
                                    st) != cudaSuccess ||
                    cudaStreamSynchronize(st) != cudaSuccess) {
                    cudaGetLastError();
                    return kCuda;
                }
                source = &with_intervals;
            }
            std::vector<geo::FaceRange> ranges;
            if (!geo::face_ranges(*source, gw, w.origin, w.pitch, ranges)) {
                return kFieldIndexOverflow;
            }
            std::vector<long long> offsets(F + 1, 0);
            for (std::size_t f = 0; f < F; ++f) {
                const auto& r = ranges[f];
                long long cells = 0;
                if (!r.outside && r.last[0] >= r.first[0] && r.last[1] >= r.first[1] && r.last[2] >= r.first[2]) {
                    cells = (r.last[0] - r.first[0] + 1) * (r.last[1] - r.first[1] + 1) * (r.last[2] - r.first[2] + 1);
                }
                offsets[f + 1] = offsets[f] + cells;
            }
            cudaMemcpyAsync(d_ranges, ranges.data(), F * sizeof(geo::FaceRange), cudaMemcpyHostToDevice, st);
            cudaMemcpyAsync(d_offsets, offsets.data(), (F + 1) * sizeof(long long), cudaMemcpyHostToDevice, st);
            if (cudaStreamSynchronize(st) != cudaSuccess) {  // the host vectors end with this scope
                cudaGetLastError();
                return kCuda;
            }
        }
        else {
            face_ranges_kernel<<<static_cast<unsigned>((F + 255) / 256), 256, 0, st>>>(
                d_tris, d_vint, static_cast<int>(F), w, d_ranges, d_offsets + 1, d_misc);
            face_offsets_kernel<<<1, 1024, 0, st>>>(d_offsets, static_cast<int>(F));
        }
        // 128-thread blocks, six to an SM: the SAT's dependent FP64 chains need
        // the resident warps more than the registers that spill (measured).
        // The pair count is on the device; a grid of four waves loops over it.
        face_sat_kernel<<<static_cast<unsigned>((16 * F + 127) / 128), 128, 0, st>>>(d_tris, d_vint,
                                                                                  static_cast<int>(F), d_sats);
        raster_kernel<<<148 * 6 * 4, 128, 0, st>>>(d_sats, d_ranges, d_offsets, static_cast<int>(F), w, d_cells,
                                                  d_misc);
        ctx->launches += 4;
    }
    ccl_init_kernel<<<blocks_for(n, threads), threads, 0, st>>>(d_cells, d_parent, n);
    ccl_union_kernel<<<blocks_for(n, threads), threads, 0, st>>>(d_cells, d_parent, w.shape[0], w.shape[1],
                                                                   w.shape[2], d_misc);
    auto* d_root_count = reinterpret_cast<unsigned int*>(d_misc + 4);
    ccl_compress_kernel<<<blocks_for(n, threads), threads, 0, st>>>(d_parent, n, d_roots, d_root_count, root_capacity);
    ctx->launches += 3;
    int h_misc[8];
    cudaMemcpyAsync(h_misc, d_misc, 32, cudaMemcpyDeviceToHost, st);
    if (cudaStreamSynchronize(st) != cudaSuccess) {
        cudaGetLastError();
        return kCuda;
    }
    if (h_misc[0] & 4) {
        // A quotient the device's binary64 path does not cover: the host's
        // face ranges (with their long double floors) decide, and the raster
        // and labels run again from them.
        return raster_fill_impl(ctx, placed, w, d_cells, normalize, uncertain_components, d_tris_kept,
                                device_intervals, true);
    }
    if (h_misc[0] & 1) {
        return kFieldIndexOverflow;
    }
    if (h_misc[0] & 2) {
        return kKernelWait;
    }
    const unsigned int roots = static_cast<unsigned int>(h_misc[4]);
    if (roots > root_capacity) {
        return kCellLimit;
    }
    std::vector<int> h_roots(roots);
    cudaMemcpy(h_roots.data(), d_roots, roots * 4ULL, cudaMemcpyDeviceToHost);
    std::vector<std::uint8_t> values(roots);
    std::uint64_t uncertain = 0;
    for (unsigned int k = 0; k < roots; ++k) {
        const long long i = h_roots[k];
        const std::int64_t index[3] = { w.first[0] + i % w.shape[0], w.first[1] + (i / w.shape[0]) % w.shape[1],
                                         w.first[2] + i / (static_cast<long long>(w.shape[0]) * w.shape[1]) };
        geo::Bounds witness;
        if (!geo::outward_grid_cell(w.origin, w.pitch, index, witness)) {
            return kFieldIndexOverflow;
        }
        const auto decision = geo::classify_material_witness(placed, witness);
        values[k] = decision == geo::Decision::indeterminate ? 3 : decision == geo::Decision::yes ? 1 : 0;
        uncertain += decision == geo::Decision::indeterminate;
    }
    if (uncertain_components) {
        *uncertain_components = uncertain;
    }
    if (roots) {
        auto* d_values = static_cast<std::uint8_t*>(device_buffer(ctx, "field.values", roots, status));
        if (!d_values) {
            return status;
        }
        cudaMemcpyAsync(d_values, values.data(), roots, cudaMemcpyHostToDevice, st);
        scatter_decisions_kernel<<<(roots + 255) / 256, 256, 0, st>>>(d_roots, d_values, static_cast<int>(roots),
                                                                      d_rootv);
        ctx->launches++;
    }
    fill_kernel<<<blocks_for(n, threads), threads, 0, st>>>(d_cells, d_parent, d_rootv, n, normalize ? 1 : 0);
    ctx->launches++;
    return cudaGetLastError() == cudaSuccess ? kOk : kCuda;
}

}  // namespace

int raster_fill(spk_context* ctx, const geo::Placed& placed, const FieldWindow& w, std::uint8_t* d_cells, bool normalize,
                std::uint64_t* uncertain_components, const std::uint32_t* d_tris_kept, bool device_intervals)
{
    return raster_fill_impl(ctx, placed, w, d_cells, normalize, uncertain_components, d_tris_kept, device_intervals,
                            false);
}

int place_on_device(spk_context* ctx, const geo::Prepared& prepared, const double* d_vertices,
                    const geo::Vec3& translation, const geo::Quat& q, geo::Placed& out, bool& done)
{
    done = false;
    if (!geo::finite_pose(translation, q)) {
        return kOk;  // the host's place() decides
    }
    const auto transform = geo::rotation_transform(q);
    if (!transform || transform->exact_cardinal) {
        return kOk;
    }
    const auto& mesh = *prepared.mesh;
    const int V = static_cast<int>(mesh.vertices.size());
    if (V == 0) {
        return kOk;
    }
    cudaStream_t st = ctx->stream;
    int status = kOk;
    const int blocks = (V + 255) / 256;
    auto* d_vint = static_cast<IVec3*>(device_buffer(ctx, "field.vint", V * sizeof(IVec3), status));
    auto* d_partial = static_cast<double*>(device_buffer(ctx, "field.vpartial", (6 * blocks + 6) * 8, status));
    auto* d_err = static_cast<int*>(device_buffer(ctx, "field.verr", 4, status));
    auto* h_out = static_cast<double*>(host_buffer(ctx, "field.vbounds", 8 * 8, status));
    if (!d_vint || !d_partial || !d_err || !h_out) {
        return status;
    }
    PoseIntervals pose {};
    geo::rotation_intervals(q, pose.rotation);
    for (int a = 0; a < 3; ++a) {
        pose.translation[a] = translation[a];
    }
    cudaMemsetAsync(d_err, 0, 4, st);
    vertex_intervals_kernel<<<blocks, 256, 0, st>>>(d_vertices, V, pose, d_vint, d_partial, d_err);
    vertex_bounds_kernel<<<1, 1, 0, st>>>(d_partial, blocks, d_partial + 6 * blocks);
    ctx->launches += 2;
    cudaMemcpyAsync(h_out, d_partial + 6 * blocks, 48, cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(h_out + 6, d_err, 4, cudaMemcpyDeviceToHost, st);
    if (cudaStreamSynchronize(st) != cudaSuccess) {
        cudaGetLastError();
        return kCuda;
    }
    int invalid = 0;
    std::memcpy(&invalid, h_out + 6, 4);
    if (invalid) {
        return kOk;  // the host's place() decides (it returns false)
    }
    out = geo::Placed {};
    out.prepared = &prepared;
    out.translation = translation;
    out.q = q;
    out.is_cardinal = false;
    for (int a = 0; a < 3; ++a) {
        out.source_axis[a] = transform->source_axis[a];
        out.sign[a] = transform->sign[a];
        out.conservative.min[a] = h_out[a];
        out.conservative.max[a] = h_out[3 + a];
    }
    out.finite = true;
    out.world_exact = false;
    done = true;
    return kOk;
}

int dilate_crop(spk_context* ctx, const std::uint8_t* d_raw, const FieldWindow& raw, std::uint64_t halo,
                double clearance, bool invert, std::uint8_t* d_out, const FieldWindow& req, const int* box_lo,
                const int* box_hi)
{
    const auto stencil = geo::make_stencil(halo, req.pitch, clearance);
    std::vector<int> flat(3 * stencil.size());
    for (std::size_t i = 0; i < stencil.size(); ++i) {
        for (int a = 0; a < 3; ++a) {
            flat[3 * i + a] = static_cast<int>(stencil[i][a]);
        }
    }
    int status = kOk;
    auto* d_stencil = static_cast<int*>(device_buffer(ctx, "field.stencil", std::max<std::size_t>(flat.size(), 3) * 4,
                                                      status));
    if (!d_stencil) {
        return status;
    }
    cudaMemcpyAsync(d_stencil, flat.data(), flat.size() * 4, cudaMemcpyHostToDevice, ctx->stream);
    const long long n = static_cast<long long>(req.shape[0]) * req.shape[1] * req.shape[2];
    CellBox box {};
    for (int a = 0; a < 3; ++a) {
        box.lo[a] = box_lo ? box_lo[a] : 0;
        box.extent[a] = (box_hi ? box_hi[a] : req.shape[a]) - box.lo[a];
        if (box.extent[a] <= 0) {
            box.extent[a] = 0;
        }
    }
    const long long m = static_cast<long long>(box.extent[0]) * box.extent[1] * box.extent[2];
    if (m < n) {
        cudaMemsetAsync(d_out, 0, n, ctx->stream);  // no stencil offset reaches the raw window from outside the box
    }
    if (m > 0) {
        dilate_kernel<<<blocks_for(m, 256), 256, 0, ctx->stream>>>(d_raw, raw, d_stencil,
                                                                   static_cast<int>(stencil.size()), invert ? 1 : 0,
                                                                   d_out, req, box);
        ctx->launches++;
    }
    return cudaGetLastError() == cudaSuccess ? kOk : kCuda;
}

int box_mask(spk_context* ctx, const double* dims, double clearance, const FieldWindow& w, std::uint8_t* d_mask)
{
    std::vector<std::uint8_t> axes[3];
    for (int a = 0; a < 3; ++a) {
        axes[a].resize(w.shape[a]);
        for (std::uint32_t k = 0; k < w.shape[a]; ++k) {
            std::int64_t index[3] = { w.first[0], w.first[1], w.first[2] };
            index[a] = w.first[a] + k;
            IVec3 cell;
            if (!grid_cell_interval(w.origin, w.pitch, index, cell)) {
                return kFieldIndexOverflow;
            }
            axes[a][k] = geo::analytic_box_axis_inside(w.origin[a], w.pitch, index[a], dims[a], clearance, cell, a) ? 1
                                                                                                                   : 0;
        }
    }
    int status = kOk;
    auto* d_axes = static_cast<std::uint8_t*>(
        device_buffer(ctx, "field.axes", static_cast<std::size_t>(w.shape[0]) + w.shape[1] + w.shape[2], status));
    if (!d_axes) {
        return status;
    }
    cudaMemcpyAsync(d_axes, axes[0].data(), w.shape[0], cudaMemcpyHostToDevice, ctx->stream);
    cudaMemcpyAsync(d_axes + w.shape[0], axes[1].data(), w.shape[1], cudaMemcpyHostToDevice, ctx->stream);
    cudaMemcpyAsync(d_axes + w.shape[0] + w.shape[1], axes[2].data(), w.shape[2], cudaMemcpyHostToDevice, ctx->stream);
    const long long n = static_cast<long long>(w.shape[0]) * w.shape[1] * w.shape[2];
    box_mask_kernel<<<blocks_for(n, 256), 256, 0, ctx->stream>>>(d_axes, d_axes + w.shape[0],
                                                                 d_axes + w.shape[0] + w.shape[1], w.shape[0],
                                                                 w.shape[1], w.shape[2], d_mask);
    ctx->launches++;
    return cudaGetLastError() == cudaSuccess ? kOk : kCuda;
}

int stamp(spk_context* ctx, std::uint32_t* d_counts, const std::uint8_t* d_placed, long long n, int direction)
{
    stamp_kernel<<<blocks_for(n, 256), 256, 0, ctx->stream>>>(d_counts, d_placed, n, direction);
    ctx->launches++;
    return cudaGetLastError() == cudaSuccess ? kOk : kCuda;
}

int stamp_box(spk_context* ctx, std::uint32_t* d_counts, const std::uint8_t* d_placed, const int* shape,
              const int* lo, const int* hi, int direction)
{
    CellBox box {};
    for (int a = 0; a < 3; ++a) {
        box.lo[a] = lo[a];
        box.extent[a] = hi[a] > lo[a] ? hi[a] - lo[a] : 0;
    }
    const long long m = static_cast<long long>(box.extent[0]) * box.extent[1] * box.extent[2];
    if (m > 0) {
        stamp_box_kernel<<<blocks_for(m, 256), 256, 0, ctx->stream>>>(d_counts, d_placed, shape[0], shape[1], box,
                                                                      direction);
        ctx->launches++;
    }
    return cudaGetLastError() == cudaSuccess ? kOk : kCuda;
}

int occupancy_box(spk_context* ctx, const std::uint8_t* d_mask, const std::uint32_t* d_counts, std::uint8_t* d_occ,
                  const int* shape, const int* lo, const int* hi)
{
    CellBox box {};
    for (int a = 0; a < 3; ++a) {
        box.lo[a] = lo[a];
        box.extent[a] = hi[a] > lo[a] ? hi[a] - lo[a] : 0;
    }
    const long long m = static_cast<long long>(box.extent[0]) * box.extent[1] * box.extent[2];
    if (m > 0) {
        occupancy_box_kernel<<<blocks_for(m, 256), 256, 0, ctx->stream>>>(d_mask, d_counts, d_occ, shape[0], shape[1],
                                                                          box);
        ctx->launches++;
    }
    return cudaGetLastError() == cudaSuccess ? kOk : kCuda;
}

int occupancy(spk_context* ctx, const std::uint8_t* d_mask, const std::uint32_t* d_counts, std::uint8_t* d_occ,
              long long n)
{
    occupancy_kernel<<<blocks_for(n, 256), 256, 0, ctx->stream>>>(d_mask, d_counts, d_occ, n);
    ctx->launches++;
    return cudaGetLastError() == cudaSuccess ? kOk : kCuda;
}

}  // namespace spk
