// Shared device/host helpers for the spectral placement kernels.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>

#define SPK_HD __host__ __device__ __forceinline__

namespace spk {

// Status codes mirror the reference's string codes (correlation.hpp:52-56,
// spectral_pipeline.cpp diagnostics); spk_status_code() maps them back.
enum Status : int {
    kOk = 0,
    kShapeOverflow = 1,        // CORRELATION_SHAPE_OVERFLOW
    kIndexOverflow = 2,        // CORRELATION_INDEX_OVERFLOW
    kInvalidField = 3,         // CORRELATION_INVALID_FIELD
    kInvalidEnvironment = 4,   // CORRELATION_INVALID_ENVIRONMENT
    kInvalidKernel = 5,        // CORRELATION_INVALID_KERNEL
    kNumericRange = 6,         // CORRELATION_NUMERIC_RANGE
    kPaddedCellLimit = 7,      // CORRELATION_PADDED_CELL_LIMIT
    kMemoryLimit = 8,          // CORRELATION_MEMORY_LIMIT
    kNumeric = 9,              // CORRELATION_NUMERIC
    kDirectTermLimit = 10,     // CORRELATION_DIRECT_TERM_LIMIT
    kAllocation = 11,          // CORRELATION_ALLOCATION
    kCancelled = 12,           // OPERATION_CANCELLED
    kDeadline = 13,            // DEADLINE_EXCEEDED
    kCuda = 14,                // CUDA_RUNTIME_ERROR
    kInvalidArgument = 15,     // SPK_INVALID_ARGUMENT
    kUnsupportedLength = 16,   // SPK_UNSUPPORTED_FFT_LENGTH
    kFieldInput = 17,          // FIELD_INPUT
    kFieldIndexOverflow = 18,  // FIELD_INDEX_OVERFLOW
    kCellLimit = 19,           // FIELD_CELL_LIMIT
    kEmptyKernel = 20,         // SPECTRAL_PIPELINE_EMPTY_KERNEL
    kProximityShape = 21,      // SPECTRAL_PIPELINE_PROXIMITY_SHAPE
    kCatalog = 22,             // SPECTRAL_PIPELINE_CATALOG
    kNoCandidate = 23,         // SPECTRAL_PIPELINE_COMPLETE with an empty page
    kKernelWait = 24,          // SPK_DEVICE_WAIT_LIMIT (bounded device wait expired)
    kScratchLimit = 25,        // SPK_SCRATCH_LIMIT
    kNotReady = 26,            // SPK_CONTEXT_STATE
    kValidationAborted = 27,   // SPECTRAL_VALIDATION_ABORTED
};

template <typename T>
struct Cplx;
template <>
struct Cplx<float> {
    using type = float2;
};
template <>
struct Cplx<double> {
    using type = double2;
};
template <typename T>
using cplx_t = typename Cplx<T>::type;

template <typename C>
SPK_HD C cmake(decltype(C::x) re, decltype(C::x) im)
{
    C c;
    c.x = re;
    c.y = im;
    return c;
}
template <typename C>
SPK_HD C cadd(C a, C b)
{
    return cmake<C>(a.x + b.x, a.y + b.y);
}
template <typename C>
SPK_HD C csub(C a, C b)
{
    return cmake<C>(a.x - b.x, a.y - b.y);
}
template <typename C>
SPK_HD C cmul(C a, C b)
{
    return cmake<C>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// a * conj(b)
template <typename C>
SPK_HD C cmulconj(C a, C b)
{
    return cmake<C>(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}
template <typename C>
SPK_HD C cconj(C a)
{
    return cmake<C>(a.x, -a.y);
}
template <typename C>
SPK_HD C cscale(C a, decltype(C::x) s)
{
    return cmake<C>(a.x * s, a.y * s);
}

SPK_HD int ilog2(unsigned v)
{
    int r = 0;
    while (v > 1) {
        v >>= 1;
        ++r;
    }
    return r;
}

SPK_HD bool is_pow2(std::uint64_t v) { return v && !(v & (v - 1)); }

// Runs `set_up` once per device (kernel attributes are per device), safely
// from any number of host threads.
template <typename F>
inline void once_per_device(std::once_flag (&flags)[64], F set_up)
{
    int device = 0;
    cudaGetDevice(&device);
    std::call_once(flags[device & 63], set_up);
}

}  // namespace spk
