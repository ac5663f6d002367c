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
            // Floor division, then the first integer where q is strictly nearer.
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

}  // namespace

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
    cudaMemcpy(d, host.data(), want * sizeof(double), cudaMemcpyHostToDevice);
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
    edt_init_kernel<<<blocks_for(n, 256), 256, 0, stream>>>(d_occupied, d_d2, n);
    ctx->launches++;
    for (int axis = 0; axis != 3; ++axis) {
        const long long lines = n / shape[axis];
        edt_pass_kernel<<<static_cast<unsigned>((lines + 127) / 128), 128, 0, stream>>>(
            d_d2, line_f, site_q, site_s, shape[0], shape[1], shape[2], axis);
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

using namespace spk;

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
