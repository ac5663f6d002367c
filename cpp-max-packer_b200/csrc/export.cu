// STL export of a placement sequence on the device: every copy of the
// item's mesh transformed by its pose, as the float32 binary STL that
// pack_io's write_stl_stage writes (engine/pack_io/src/result_export.cpp:
// 1034-1123).
//
// Per triangle, as the reference does it:
//   - each vertex through RigidTransform::apply (rigid_transform.cpp:37-42):
//     m[r][0] x + m[r][1] y + m[r][2] z + t[r], left to right, binary64
//     round-to-nearest with no fused multiply-add, then rounded to float32;
//     a coordinate that is not a finite float32 fails the export;
//   - the normal from the float32 points, in binary64: edges, cross product,
//     length = hypot(hypot(n0, n1), n2), each component divided by the length
//     (zero when the length is zero or not finite), rounded to float32;
//   - a zero 16-bit attribute.
// The rotation matrices are the host's rotation_transform (bit-exact with
// validation_kernel::rotation_transform).  hypot is the one step whose
// rounding the device library does not share with the host's libm; each
// normal component is therefore checked on the device: when its float32
// rounding would change for a length 8 binary64 ulps larger or smaller (far
// beyond both libraries' hypot error), the triangle is listed and the host
// recomputes its normal with its own hypot.  Everything else is computed
// once, on the device.
//
// Records are 50 bytes; 128 triangles (6,400 bytes, a multiple of 16) are
// staged per block in shared memory and stored as 16-byte words.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <vector>

#include "../../include/spk_b200.h"
#include "common.cuh"
#include "context.hpp"
#include "geometry.hpp"
#include "interval.cuh"

namespace spk {
namespace {

constexpr int kExportThreads = 128;
constexpr int kRecordBytes = 50;
constexpr std::uint64_t kChunkRecords = 1ULL << 22;  // 200 MB of records per chunk
static_assert(kExportThreads * kRecordBytes % 16 == 0, "a block's records are stored as 16-byte words");
static_assert(kChunkRecords % kExportThreads == 0, "chunks hold whole blocks");

struct ExportArgs {
    const double* vertices;    // [V][3]
    const std::uint32_t* tris;  // [F][3]
    const double* transforms;  // [copies][12]: row-major 3 x 4 (rotation | translation)
    long long faces;
    long long records;         // triangles of this chunk
    long long first_record;    // of this chunk in the whole sequence
    std::uint8_t* out;         // this chunk's records
    unsigned int* flags;       // [0]: a coordinate is not a finite float32; [1]: unstable normals
    unsigned long long* unstable;  // indices (whole sequence) of triangles whose normal the host recomputes
    unsigned int unstable_capacity;
};

// float32 rounding of q that holds for every value within 2^-49 |q| of it.
__device__ __forceinline__ bool stable_float(double q)
{
    const double m = fabs(q) * 0x1p-49;
    return __double2float_rn(q - m) == __double2float_rn(q + m);
}

__global__ void __launch_bounds__(kExportThreads) stl_records_kernel(const ExportArgs a)
{
    __shared__ __align__(16) std::uint8_t stage[kExportThreads * kRecordBytes];
    const long long item = static_cast<long long>(blockIdx.x) * kExportThreads + threadIdx.x;
    if (item < a.records) {
        const long long global = a.first_record + item;
        const long long copy = global / a.faces - a.first_record / a.faces;
        const long long face = global % a.faces;
        const double* m = a.transforms + 12 * copy;
        float p[3][3];
        bool finite = true;
        for (int k = 0; k < 3; ++k) {
            const double* v = a.vertices + 3 * static_cast<long long>(a.tris[3 * face + k]);
            for (int r = 0; r < 3; ++r) {
                const double w = f_add(f_add(f_add(f_mul(m[4 * r], v[0]), f_mul(m[4 * r + 1], v[1])),
                                             f_mul(m[4 * r + 2], v[2])),
                                       m[4 * r + 3]);
                finite = finite && isfinite(w) && w <= 3.4028234663852886e38 && w >= -3.4028234663852886e38;
                p[k][r] = __double2float_rn(w);
            }
        }
        if (!finite) {
            atomicOr(a.flags, 1u);
        }
        double ea[3], eb[3];
        for (int r = 0; r < 3; ++r) {
            ea[r] = f_sub(static_cast<double>(p[1][r]), static_cast<double>(p[0][r]));
            eb[r] = f_sub(static_cast<double>(p[2][r]), static_cast<double>(p[0][r]));
        }
        double n[3] = { f_sub(f_mul(ea[1], eb[2]), f_mul(ea[2], eb[1])),
                        f_sub(f_mul(ea[2], eb[0]), f_mul(ea[0], eb[2])),
                        f_sub(f_mul(ea[0], eb[1]), f_mul(ea[1], eb[0])) };
        const double length = hypot(hypot(n[0], n[1]), n[2]);
        float nf[3] = { 0.f, 0.f, 0.f };
        if (length != 0.0 && isfinite(length)) {
            bool stable = true;
            for (int r = 0; r < 3; ++r) {
                const double q = f_div(n[r], length);
                stable = stable && stable_float(q);
                nf[r] = __double2float_rn(q);
            }
            if (!stable) {
                const unsigned int slot = atomicAdd(a.flags + 1, 1u);
                if (slot < a.unstable_capacity) {
                    a.unstable[slot] = static_cast<unsigned long long>(global);
                }
            }
        }
        std::uint8_t* rec = stage + threadIdx.x * kRecordBytes;
        std::memcpy(rec, nf, 12);
        std::memcpy(rec + 12, p, 36);
        rec[48] = 0;
        rec[49] = 0;
    }
    __syncthreads();
    const long long first = static_cast<long long>(blockIdx.x) * kExportThreads;
    const long long count = a.records - first < kExportThreads ? a.records - first : kExportThreads;
    const int bytes = static_cast<int>(count) * kRecordBytes;
    std::uint8_t* dst = a.out + first * kRecordBytes;
    const int words = bytes / 16;
    for (int i = threadIdx.x; i < words; i += kExportThreads) {
        reinterpret_cast<uint4*>(dst)[i] = reinterpret_cast<const uint4*>(stage)[i];
    }
    for (int i = words * 16 + threadIdx.x; i < bytes; i += kExportThreads) {
        dst[i] = stage[i];
    }
}

}  // namespace
}  // namespace spk

using namespace spk;

extern "C" int spk_export_stl(spk_context* ctx, const spk_mesh* object, const double* translations_mm,
                              const double* q_xyzw, uint64_t copies, uint8_t* out, uint64_t capacity,
                              uint64_t* size)
{
    if (!ctx) {
        return kNotReady;
    }
    try {
        if (!object || !object->vertices || !object->triangles || !object->vertex_count || !size ||
            (copies && (!translations_mm || !q_xyzw))) {
            return fail(ctx, kInvalidArgument, "STL export input is missing.");
        }
        for (std::uint64_t i = 0; i < 3 * object->triangle_count; ++i) {
            if (object->triangles[i] >= object->vertex_count) {
                return fail(ctx, kInvalidArgument, "STL export triangle refers to a missing vertex.");
            }
        }
        const std::uint64_t faces = object->triangle_count;
        const std::uint64_t triangles = faces * copies;
        if (faces && triangles / faces != copies) {
            return fail(ctx, kInvalidArgument, "STL triangle count exceeds uint32 range.");
        }
        if (triangles > std::numeric_limits<std::uint32_t>::max()) {
            // result_export.cpp:1423-1426 (EXPORT_SIZE_LIMIT)
            return fail(ctx, kInvalidArgument, "STL triangle count exceeds uint32 range.");
        }
        *size = 84 + kRecordBytes * triangles;
        if (capacity < *size || !out) {
            return fail(ctx, kScratchLimit, "STL output buffer is smaller than the file.");
        }
        // RigidTransform::make (rigid_transform.cpp:11-33) for every pose.
        std::vector<double> transforms(12 * copies);
        for (std::uint64_t c = 0; c < copies; ++c) {
            const double* t = translations_mm + 3 * c;
            const double* q = q_xyzw + 4 * c;
            bool finite = true;
            for (int i = 0; i < 4; ++i) {
                finite = finite && std::isfinite(q[i]);
            }
            for (int i = 0; i < 3; ++i) {
                finite = finite && std::isfinite(t[i]);
            }
            const auto rotation = finite ? geo::rotation_transform({ q[0], q[1], q[2], q[3] })
                                         : std::optional<geo::RotationTransform> {};
            if (!rotation) {
                return fail(ctx, kInvalidArgument, "A source pose has no rigid transform.");
            }
            for (int r = 0; r < 3; ++r) {
                for (int k = 0; k < 3; ++k) {
                    transforms[12 * c + 4 * r + k] = rotation->matrix[r][k];
                }
                transforms[12 * c + 4 * r + 3] = t[r];
            }
        }
        std::memset(out, 0, 80);
        const auto count32 = static_cast<std::uint32_t>(triangles);
        std::memcpy(out + 80, &count32, 4);
        if (triangles == 0) {
            return finish(ctx, kOk);
        }
        cudaStream_t st = ctx->stream;
        int status = kOk;
        const std::size_t V = object->vertex_count;
        auto* d_vertices = static_cast<double*>(device_buffer(ctx, "stl.vertices", 24 * V, status));
        auto* d_tris = static_cast<std::uint32_t*>(device_buffer(ctx, "stl.tris", 12 * faces, status));
        const std::uint64_t chunk = std::min<std::uint64_t>(triangles, kChunkRecords);
        auto* d_out = static_cast<std::uint8_t*>(device_buffer(ctx, "stl.records", kRecordBytes * chunk, status));
        auto* d_transforms = static_cast<double*>(device_buffer(ctx, "stl.transforms", 96 * copies, status));
        constexpr unsigned int kUnstableCapacity = 1u << 16;
        auto* d_flags = static_cast<unsigned int*>(device_buffer(ctx, "stl.flags", 8, status));
        auto* d_unstable = static_cast<unsigned long long*>(
            device_buffer(ctx, "stl.unstable", 8ULL * kUnstableCapacity, status));
        if (!d_vertices || !d_tris || !d_out || !d_transforms || !d_flags || !d_unstable) {
            return fail(ctx, status ? status : kAllocation, "STL export device buffers could not be allocated.");
        }
        cudaMemcpyAsync(d_vertices, object->vertices, 24 * V, cudaMemcpyHostToDevice, st);
        cudaMemcpyAsync(d_tris, object->triangles, 12 * faces, cudaMemcpyHostToDevice, st);
        cudaMemcpyAsync(d_transforms, transforms.data(), 96 * copies, cudaMemcpyHostToDevice, st);
        std::vector<unsigned long long> unstable;
        for (std::uint64_t first = 0; first < triangles; first += chunk) {
            const std::uint64_t records = std::min(chunk, triangles - first);
            const std::uint64_t first_copy = first / faces;
            cudaMemsetAsync(d_flags, 0, 8, st);
            ExportArgs a { d_vertices, d_tris, d_transforms + 12 * first_copy, static_cast<long long>(faces),
                           static_cast<long long>(records), static_cast<long long>(first), d_out, d_flags,
                           d_unstable, kUnstableCapacity };
            stl_records_kernel<<<static_cast<unsigned>((records + kExportThreads - 1) / kExportThreads),
                                 kExportThreads, 0, st>>>(a);
            ctx->launches++;
            unsigned int flags[2] {};
            cudaMemcpyAsync(flags, d_flags, 8, cudaMemcpyDeviceToHost, st);
            if (cudaMemcpyAsync(out + 84 + kRecordBytes * first, d_out, kRecordBytes * records,
                                cudaMemcpyDeviceToHost, st) != cudaSuccess ||
                cudaStreamSynchronize(st) != cudaSuccess) {
                cudaGetLastError();
                return fail(ctx, kCuda, "STL export kernels failed.");
            }
            if (flags[0]) {
                return fail(ctx, kInvalidArgument, "A transformed STL coordinate is not finite float32.");
            }
            if (flags[1] > kUnstableCapacity) {
                return fail(ctx, kScratchLimit, "Too many STL normals need the host's hypot.");
            }
            if (flags[1]) {
                const std::size_t base = unstable.size();
                unstable.resize(base + flags[1]);
                if (cudaMemcpy(unstable.data() + base, d_unstable, 8ULL * flags[1], cudaMemcpyDeviceToHost) !=
                    cudaSuccess) {
                    cudaGetLastError();
                    return fail(ctx, kCuda, "STL export kernels failed.");
                }
            }
        }
        // Normals whose float32 rounding the device's hypot could not settle:
        // recomputed from the record's own float32 points with the host's.
        for (const unsigned long long index : unstable) {
            std::uint8_t* rec = out + 84 + kRecordBytes * index;
            float p[3][3];
            std::memcpy(p, rec + 12, 36);
            const double ea[3] = { static_cast<double>(p[1][0]) - p[0][0], static_cast<double>(p[1][1]) - p[0][1],
                                   static_cast<double>(p[1][2]) - p[0][2] };
            const double eb[3] = { static_cast<double>(p[2][0]) - p[0][0], static_cast<double>(p[2][1]) - p[0][1],
                                   static_cast<double>(p[2][2]) - p[0][2] };
            double n[3] = { ea[1] * eb[2] - ea[2] * eb[1], ea[2] * eb[0] - ea[0] * eb[2],
                            ea[0] * eb[1] - ea[1] * eb[0] };
            const double length = std::hypot(std::hypot(n[0], n[1]), n[2]);
            float nf[3] = { 0.f, 0.f, 0.f };
            if (length != 0.0 && std::isfinite(length)) {
                for (int r = 0; r < 3; ++r) {
                    nf[r] = static_cast<float>(n[r] / length);
                }
            }
            std::memcpy(rec, nf, 12);
        }
        return finish(ctx, kOk);
    }
    catch (const std::bad_alloc&) {
        return fail(ctx, kAllocation, "STL export host allocation failed.");
    }
}
