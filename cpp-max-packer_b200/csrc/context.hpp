// Context: device, stream, device-memory arena, twiddle tables and the
// host-side stop/deadline poll shared by every entry point.
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <utility>
#include <vector>

#include "../../include/spk_b200.h"
#include "common.cuh"

struct spk_context {
    int device {};
    std::uint64_t cap_bytes {};
    cudaStream_t stream {};
    std::atomic<std::uint64_t> launches { 0 };
    std::uint64_t bytes_in_use {};
    struct Buffer {
        void* ptr {};
        std::size_t bytes {};
    };
    std::map<std::string, Buffer> device_buffers;
    std::map<std::string, Buffer> host_buffers;  // pinned staging
    std::map<std::pair<int, int>, void*> twiddles;  // (sizeof scalar, L) -> table
    void* session {};                              // placement session (engine.cpp)
    bool profiling {};
    static constexpr int kPasses = 5;  // A, B1, B2, merge + exact, the pipelined A/B1/B2 stage
    std::uint64_t pass_launches[kPasses] {};
    double pass_ms[kPasses] {};
    double pass_bytes[kPasses] {};  // algorithmic bytes of the profiled launches
    std::vector<std::pair<int, std::pair<cudaEvent_t, cudaEvent_t>>> pending;  // (pass, events)
    const char* message { "" };  // static text of the last correlation failure on this context
};

namespace spk {

// Grows (never shrinks) a named device buffer; returns nullptr on failure.
inline void* device_buffer(spk_context* ctx, const std::string& name, std::size_t bytes, int& status)
{
    auto& b = ctx->device_buffers[name];
    if (b.bytes >= bytes && b.ptr) {
        return b.ptr;
    }
    const std::uint64_t next = ctx->bytes_in_use - b.bytes + bytes;
    if (ctx->cap_bytes && next > ctx->cap_bytes) {
        status = kMemoryLimit;
        return nullptr;
    }
    if (b.ptr) {
        cudaFree(b.ptr);
        ctx->bytes_in_use -= b.bytes;
        b = {};
    }
    void* p {};
    if (cudaMalloc(&p, bytes ? bytes : 1) != cudaSuccess) {
        cudaGetLastError();
        status = kAllocation;
        return nullptr;
    }
    b.ptr = p;
    b.bytes = bytes;
    ctx->bytes_in_use += bytes;
    return p;
}

inline void* host_buffer(spk_context* ctx, const std::string& name, std::size_t bytes, int& status)
{
    auto& b = ctx->host_buffers[name];
    if (b.bytes >= bytes && b.ptr) {
        return b.ptr;
    }
    if (b.ptr) {
        cudaFreeHost(b.ptr);
        b = {};
    }
    void* p {};
    if (cudaMallocHost(&p, bytes ? bytes : 1) != cudaSuccess) {
        cudaGetLastError();
        status = kAllocation;
        return nullptr;
    }
    b.ptr = p;
    b.bytes = bytes;
    return p;
}

// Copies a host table into device memory and returns once the copy has
// landed.  A plain cudaMemcpy from pageable memory may return before its DMA
// reaches the device, and it runs on the legacy stream, which the context's
// non-blocking streams do not wait for: a kernel launched right after it
// could read the table half written.  Here the copy is ordered on the
// context's stream and that stream is drained before returning.
inline bool upload_table(spk_context* ctx, void* dst, const void* src, std::size_t bytes)
{
    if (cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, ctx->stream) != cudaSuccess ||
        cudaStreamSynchronize(ctx->stream) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return true;
}

// exp(-2 pi i m / L) for m < L, FP64-computed, stored as T.
template <typename T>
const cplx_t<T>* twiddle_table(spk_context* ctx, int L, int& status)
{
    const auto key = std::make_pair(static_cast<int>(sizeof(T)), L);
    auto it = ctx->twiddles.find(key);
    if (it != ctx->twiddles.end()) {
        return static_cast<const cplx_t<T>*>(it->second);
    }
    std::vector<cplx_t<T>> host(L);
    const double pi = 3.14159265358979323846264338327950288;
    for (int m = 0; m < L; ++m) {
        // Exact values at the quarter points keep the table symmetric.
        double c, s;
        if (4 * m % L == 0) {
            const int quadrant = 4 * m / L;
            c = quadrant == 0 ? 1.0 : quadrant == 2 ? -1.0 : 0.0;
            s = quadrant == 1 ? -1.0 : quadrant == 3 ? 1.0 : 0.0;
        }
        else {
            const double angle = -2.0 * pi * static_cast<double>(m) / static_cast<double>(L);
            c = std::cos(angle);
            s = std::sin(angle);
        }
        host[m].x = static_cast<T>(c);
        host[m].y = static_cast<T>(s);
    }
    void* p {};
    if (cudaMalloc(&p, sizeof(cplx_t<T>) * L) != cudaSuccess) {
        cudaGetLastError();
        status = kAllocation;
        return nullptr;
    }
    if (!upload_table(ctx, p, host.data(), sizeof(cplx_t<T>) * L)) {
        cudaFree(p);
        status = kCuda;
        return nullptr;
    }
    ctx->twiddles[key] = p;
    return static_cast<const cplx_t<T>*>(p);
}

std::int64_t monotonic_ns();

// Records the reference's message for a failure site and returns its status.
inline int fail(spk_context* ctx, int status, const char* message)
{
    ctx->message = message;
    return status;
}

// A failing status whose site left no message gets the reference's wording
// for its code (correlation.cpp:268-270,587) or the library's own.
inline int finish(spk_context* ctx, int status)
{
    if (status && ctx && !*ctx->message) {
        switch (status) {
        case kCancelled:
        case kDeadline: ctx->message = "Correlation interrupted."; break;
        case kAllocation: ctx->message = "Correlation allocation failed."; break;
        case kMemoryLimit: ctx->message = "Correlation buffers and FFT workspace exceed their memory limit."; break;
        case kCuda: ctx->message = "CUDA runtime call failed."; break;
        case kInvalidArgument: ctx->message = "Invalid argument."; break;
        default: break;
        }
    }
    return status;
}

// The reference polls stop first, then the deadline (operation_control.hpp:33-42).
inline int poll(const spk_control* control)
{
    if (!control) {
        return kOk;
    }
    if (control->stop_word && *control->stop_word) {
        return kCancelled;
    }
    if (control->deadline_ns && monotonic_ns() >= control->deadline_ns) {
        return kDeadline;
    }
    return kOk;
}

// Brackets one pass launch with events when profiling is on.
inline std::pair<cudaEvent_t, cudaEvent_t> pass_begin(spk_context* ctx)
{
    std::pair<cudaEvent_t, cudaEvent_t> ev {};
    if (ctx->profiling) {
        cudaEventCreate(&ev.first);
        cudaEventCreate(&ev.second);
        cudaEventRecord(ev.first, ctx->stream);
    }
    return ev;
}
inline void pass_end(spk_context* ctx, int pass, std::pair<cudaEvent_t, cudaEvent_t> ev, double bytes = 0.0)
{
    if (ctx->profiling && ev.first) {
        cudaEventRecord(ev.second, ctx->stream);
        ctx->pending.push_back({ pass, ev });
        ctx->pass_bytes[pass] += bytes;
    }
}
inline void pass_collect(spk_context* ctx)
{
    for (auto& [pass, ev] : ctx->pending) {
        float ms = 0.f;
        if (cudaEventSynchronize(ev.second) == cudaSuccess && cudaEventElapsedTime(&ms, ev.first, ev.second) ==
                                                                 cudaSuccess) {
            ctx->pass_ms[pass] += ms;
            ctx->pass_launches[pass] += 1;
        }
        cudaEventDestroy(ev.first);
        cudaEventDestroy(ev.second);
    }
    ctx->pending.clear();
}

inline std::uint32_t next_pow2(std::uint64_t v)
{
    std::uint32_t p = 1;
    while (p < v) {
        p <<= 1;
    }
    return p;
}

}  // namespace spk
