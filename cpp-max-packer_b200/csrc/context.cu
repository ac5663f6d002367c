// Context lifetime, status strings and launch accounting.
#include <cuda_runtime.h>

#include <new>

#include "context.hpp"

namespace spk {
void session_destroy(spk_context* ctx);
}

extern "C" {

int spk_context_create(int device, uint64_t max_device_bytes, spk_context** out)
{
    if (!out) {
        return spk::kInvalidArgument;
    }
    *out = nullptr;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || device < 0 || device >= count) {
        cudaGetLastError();
        return spk::kCuda;
    }
    if (cudaSetDevice(device) != cudaSuccess) {
        return spk::kCuda;
    }
    auto* ctx = new (std::nothrow) spk_context();
    if (!ctx) {
        return spk::kAllocation;
    }
    ctx->device = device;
    ctx->cap_bytes = max_device_bytes;
    if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete ctx;
        return spk::kCuda;
    }
    *out = ctx;
    return spk::kOk;
}

void spk_context_destroy(spk_context* ctx)
{
    if (!ctx) {
        return;
    }
    cudaSetDevice(ctx->device);
    spk::session_destroy(ctx);
    cudaStreamSynchronize(ctx->stream);
    for (auto& [name, b] : ctx->device_buffers) {
        cudaFree(b.ptr);
    }
    for (auto& [name, b] : ctx->host_buffers) {
        cudaFreeHost(b.ptr);
    }
    for (auto& [key, p] : ctx->twiddles) {
        cudaFree(p);
    }
    cudaStreamDestroy(ctx->stream);
    delete ctx;
}

uint64_t spk_context_launches(const spk_context* ctx) { return ctx ? ctx->launches.load() : 0; }

void* spk_context_stream(const spk_context* ctx) { return ctx ? static_cast<void*>(ctx->stream) : nullptr; }

int spk_context_set_profiling(spk_context* ctx, int enabled)
{
    if (!ctx) {
        return spk::kInvalidArgument;
    }
    spk::pass_collect(ctx);
    ctx->profiling = enabled != 0;
    for (int i = 0; i < spk_context::kPasses; ++i) {
        ctx->pass_launches[i] = 0;
        ctx->pass_ms[i] = 0;
        ctx->pass_bytes[i] = 0;
    }
    return spk::kOk;
}

int spk_context_pass_bytes(const spk_context* ctx, double* bytes, uint32_t capacity)
{
    if (!ctx || !bytes) {
        return spk::kInvalidArgument;
    }
    for (uint32_t i = 0; i < capacity && i < static_cast<uint32_t>(spk_context::kPasses); ++i) {
        bytes[i] = ctx->pass_bytes[i];
    }
    return spk::kOk;
}

int spk_context_pass_times(const spk_context* ctx, uint64_t* launches, double* total_ms, uint32_t capacity)
{
    if (!ctx || !launches || !total_ms) {
        return spk::kInvalidArgument;
    }
    spk::pass_collect(const_cast<spk_context*>(ctx));
    for (uint32_t i = 0; i < capacity && i < static_cast<uint32_t>(spk_context::kPasses); ++i) {
        launches[i] = ctx->pass_launches[i];
        total_ms[i] = ctx->pass_ms[i];
    }
    return spk::kOk;
}

const char* spk_context_message(const spk_context* ctx)
{
    return ctx && ctx->message ? ctx->message : "";
}

const char* spk_status_code(int status)
{
    switch (status) {
    case spk::kOk: return "OK";
    case spk::kShapeOverflow: return "CORRELATION_SHAPE_OVERFLOW";
    case spk::kIndexOverflow: return "CORRELATION_INDEX_OVERFLOW";
    case spk::kInvalidField: return "CORRELATION_INVALID_FIELD";
    case spk::kInvalidEnvironment: return "CORRELATION_INVALID_ENVIRONMENT";
    case spk::kInvalidKernel: return "CORRELATION_INVALID_KERNEL";
    case spk::kNumericRange: return "CORRELATION_NUMERIC_RANGE";
    case spk::kPaddedCellLimit: return "CORRELATION_PADDED_CELL_LIMIT";
    case spk::kMemoryLimit: return "CORRELATION_MEMORY_LIMIT";
    case spk::kNumeric: return "CORRELATION_NUMERIC";
    case spk::kDirectTermLimit: return "CORRELATION_DIRECT_TERM_LIMIT";
    case spk::kAllocation: return "CORRELATION_ALLOCATION";
    case spk::kCancelled: return "OPERATION_CANCELLED";
    case spk::kDeadline: return "DEADLINE_EXCEEDED";
    case spk::kCuda: return "CUDA_RUNTIME_ERROR";
    case spk::kInvalidArgument: return "SPK_INVALID_ARGUMENT";
    case spk::kUnsupportedLength: return "SPK_UNSUPPORTED_FFT_LENGTH";
    case spk::kFieldInput: return "FIELD_INPUT";
    case spk::kFieldIndexOverflow: return "FIELD_INDEX_OVERFLOW";
    case spk::kCellLimit: return "FIELD_CELL_LIMIT";
    case spk::kEmptyKernel: return "SPECTRAL_PIPELINE_EMPTY_KERNEL";
    case spk::kProximityShape: return "SPECTRAL_PIPELINE_PROXIMITY_SHAPE";
    case spk::kCatalog: return "SPECTRAL_PIPELINE_CATALOG";
    case spk::kNoCandidate: return "SPECTRAL_PIPELINE_COMPLETE";
    case spk::kKernelWait: return "SPK_DEVICE_WAIT_LIMIT";
    case spk::kScratchLimit: return "SPK_SCRATCH_LIMIT";
    case spk::kNotReady: return "SPK_CONTEXT_STATE";
    case spk::kValidationAborted: return "SPECTRAL_VALIDATION_ABORTED";
    default: return "SPK_UNKNOWN_STATUS";
    }
}

}  // extern "C"
