// Full-range FFT cross-correlation: the GPU replacement of
// compute::correlate_binary_cpu / correlate_proximity_cpu
// (reference engine/pack_compute/src/correlation.cpp:238-655).
//
// Math: out(t) = sum_i E[i + t] * K[i] for every t in the (E+K-1)^3 range,
// t_first = env_first - kernel_first - (K-1)  (correlation.cpp:281-304).
// The environment and kernel are packed as one complex field Z = E + iK on a
// power-of-two grid L >= E+K-1 per axis (no wrap for any output), one forward
// 3D FFT gives both spectra through Hermitian symmetry, W = E^ conj(K^) is
// formed, and one inverse 3D FFT (scaled 1/N) yields the correlation in the
// real part; the imaginary part must stay below the reference's tolerance.
// The extraction kernel applies the reference's per-cell checks
// (correlation.cpp:494-540); mass and the 8 direct probes
// (correlation.cpp:542-577) run on the host over the same input buffers.

#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <vector>

#include "context.hpp"
#include "fft.cuh"

namespace spk {

std::int64_t monotonic_ns()
{
    return std::chrono::duration_cast<std::chrono::nanoseconds>(std::chrono::steady_clock::now().time_since_epoch())
        .count();
}

namespace {

constexpr std::uint64_t kExactInteger = 1ULL << 53;

struct Grid {
    int L[3];
    SPK_HD long long n() const { return static_cast<long long>(L[0]) * L[1] * L[2]; }
};

template <typename T, typename E>
__global__ void pack_kernel(cplx_t<T>* __restrict__ z, Grid g, const E* __restrict__ env, int ex, int ey, int ez,
                            const std::uint8_t* __restrict__ ker, int kx, int ky, int kz)
{
    const long long n = g.n();
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        const int x = static_cast<int>(i % g.L[0]);
        const long long r = i / g.L[0];
        const int y = static_cast<int>(r % g.L[1]);
        const int zz = static_cast<int>(r / g.L[1]);
        T re = 0, im = 0;
        if (x < ex && y < ey && zz < ez) {
            re = static_cast<T>(env[x + static_cast<long long>(ex) * (y + static_cast<long long>(ey) * zz)]);
        }
        if (x < kx && y < ky && zz < kz) {
            im = static_cast<T>(ker[x + static_cast<long long>(kx) * (y + static_cast<long long>(ky) * zz)]);
        }
        z[i] = cmake<cplx_t<T>>(re, im);
    }
}

// W(k) = E^(k) conj(K^(k)) with E^ = (Z(k) + conj Z(-k))/2, K^ = (Z(k) - conj Z(-k))/(2i).
template <typename T>
__global__ void spectrum_product_kernel(const cplx_t<T>* __restrict__ z, cplx_t<T>* __restrict__ w, Grid g)
{
    using C = cplx_t<T>;
    const long long n = g.n();
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        const int x = static_cast<int>(i % g.L[0]);
        const long long r = i / g.L[0];
        const int y = static_cast<int>(r % g.L[1]);
        const int zz = static_cast<int>(r / g.L[1]);
        const int mx = x == 0 ? 0 : g.L[0] - x;
        const int my = y == 0 ? 0 : g.L[1] - y;
        const int mz = zz == 0 ? 0 : g.L[2] - zz;
        const C a = z[i];
        const C b = cconj(z[mx + static_cast<long long>(g.L[0]) * (my + static_cast<long long>(g.L[1]) * mz)]);
        const C e = cscale(cadd(a, b), static_cast<T>(0.5));
        const C d = csub(a, b);  // = 2i K^
        const C k = cmake<C>(d.y * static_cast<T>(0.5), -d.x * static_cast<T>(0.5));
        w[i] = cmulconj(e, k);
    }
}

// FP16 storage of the joint spectrum: z * scale rounded to half precision.
__global__ void spectrum_to_half_kernel(const float2* __restrict__ z, __half2* __restrict__ zh, long long n, float scale)
{
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        zh[i] = __floats2half2_rn(z[i].x * scale, z[i].y * scale);
    }
}

// The spectrum product of spectrum_product_kernel reading the FP16 spectrum.
__global__ void spectrum_product_half_kernel(const __half2* __restrict__ zh, float2* __restrict__ w, Grid g,
                                             float unscale)
{
    const long long n = g.n();
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        const int x = static_cast<int>(i % g.L[0]);
        const long long r = i / g.L[0];
        const int y = static_cast<int>(r % g.L[1]);
        const int zz = static_cast<int>(r / g.L[1]);
        const int mx = x == 0 ? 0 : g.L[0] - x;
        const int my = y == 0 ? 0 : g.L[1] - y;
        const int mz = zz == 0 ? 0 : g.L[2] - zz;
        const float2 a0 = __half22float2(zh[i]);
        const float2 b0 = __half22float2(zh[mx + static_cast<long long>(g.L[0]) * (my + static_cast<long long>(g.L[1]) * mz)]);
        const float2 a = make_float2(a0.x * unscale, a0.y * unscale);
        const float2 b = make_float2(b0.x * unscale, -b0.y * unscale);
        const float2 e = cscale(cadd(a, b), 0.5f);
        const float2 d = csub(a, b);
        const float2 k = make_float2(d.y * 0.5f, -d.x * 0.5f);
        w[i] = cmulconj(e, k);
    }
}

// v mod L for v in (-L, 2L).
__device__ __forceinline__ int wrap(int v, int L)
{
    return v < 0 ? v + L : v >= L ? v - L : v;
}

struct ExtractStats {
    double mass;          // sum of unrounded real parts (per block)
    double max_abs;       // largest |value| in the block
    long long max_index;  // first index holding it
};

template <typename T>
__global__ void extract_kernel(const cplx_t<T>* __restrict__ w, Grid g, int ox, int oy, int oz, int kx, int ky,
                               int kz, int binary, double maximum_output, double imag_tolerance,
                               double range_tolerance, double* __restrict__ out, ExtractStats* __restrict__ stats,
                               unsigned long long* __restrict__ max_residual_bits,
                               unsigned long long* __restrict__ first_failure)
{
    __shared__ double s_mass[256];
    __shared__ double s_abs[256];
    __shared__ long long s_idx[256];
    const long long n = static_cast<long long>(ox) * oy * oz;
    double mass = 0.0, best = -1.0, residual_max = 0.0;
    long long best_i = 0;
    // Lowest failing output index per kind: [0] non-finite or non-real,
    // [1] integer or range.  The reference scans outputs in index order and
    // reports the first cell that fails, checking non-real before range.
    unsigned long long bad_real = ~0ULL, bad_range = ~0ULL;
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        const int x = static_cast<int>(i % ox);
        const long long r = i / ox;
        const int y = static_cast<int>(r % oy);
        const int z = static_cast<int>(r / oy);
        // The output's cell on the transform grid, wrapped into [0, L).
        const int sx = wrap(x - (kx - 1), g.L[0]);
        const int sy = wrap(y - (ky - 1), g.L[1]);
        const int sz = wrap(z - (kz - 1), g.L[2]);
        const cplx_t<T> v = w[sx + static_cast<long long>(g.L[0]) * (sy + static_cast<long long>(g.L[1]) * sz)];
        const double value = static_cast<double>(v.x);
        const double imag = static_cast<double>(v.y);
        if (!isfinite(value) || !isfinite(imag) || fabs(imag) >= imag_tolerance) {
            bad_real = min(bad_real, static_cast<unsigned long long>(i));
        }
        mass += value;
        if (fabs(value) > best) {
            best = fabs(value);
            best_i = i;
        }
        if (binary) {
            const double rounded = round(value);
            const double residual = fabs(value - rounded);
            residual_max = fmax(residual_max, residual);
            if (residual >= 0.25 || rounded < 0.0 || rounded > maximum_output) {
                bad_range = min(bad_range, static_cast<unsigned long long>(i));
            }
            out[i] = rounded;
        }
        else {
            if (value < -range_tolerance || value > maximum_output + range_tolerance) {
                bad_range = min(bad_range, static_cast<unsigned long long>(i));
            }
            out[i] = value;
        }
    }
    if (bad_real != ~0ULL) {
        atomicMin(&first_failure[0], bad_real);
    }
    if (bad_range != ~0ULL) {
        atomicMin(&first_failure[1], bad_range);
    }
    if (binary) {
        atomicMax(max_residual_bits, static_cast<unsigned long long>(__double_as_longlong(residual_max)));
    }
    s_mass[threadIdx.x] = mass;
    s_abs[threadIdx.x] = best;
    s_idx[threadIdx.x] = best_i;
    __syncthreads();
    for (int half = blockDim.x / 2; half > 0; half >>= 1) {
        if (threadIdx.x < half) {
            s_mass[threadIdx.x] += s_mass[threadIdx.x + half];
            const double a = s_abs[threadIdx.x + half];
            const long long ai = s_idx[threadIdx.x + half];
            if (a > s_abs[threadIdx.x] || (a == s_abs[threadIdx.x] && ai < s_idx[threadIdx.x])) {
                s_abs[threadIdx.x] = a;
                s_idx[threadIdx.x] = ai;
            }
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        stats[blockIdx.x] = { s_mass[0], s_abs[0], s_idx[0] };
    }
}

// Translation mask over a caller's box of absolute translations, from the
// rounded full-range counts: inside the range, 1 where the count is zero
// (want_zero) or non-zero (otherwise); outside the range, 0.  These are the
// free and blocked rules of gap_fill.cpp:404-420 and :443-446.  dx..dz are the
// box's first translation minus the range's first, clamped on the host so
// that dx + x cannot overflow.
__global__ void mask_kernel(const double* __restrict__ counts, long long ox, long long oy, long long oz, long long dx,
                            long long dy, long long dz, long long bx, long long by, long long bz, int want_zero,
                            std::uint8_t* __restrict__ mask)
{
    const long long n = bx * by * bz;
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        const long long x = dx + i % bx;
        const long long r = i / bx;
        const long long y = dy + r % by;
        const long long z = dz + r / by;
        std::uint8_t m = 0;
        if (x >= 0 && y >= 0 && z >= 0 && x < ox && y < oy && z < oz) {
            const bool zero = counts[x + ox * (y + oy * z)] == 0.0;
            m = (zero == (want_zero != 0)) ? 1 : 0;
        }
        mask[i] = m;
    }
}

// A request to threshold on the device: the mask is written to host memory
// and the FP64 counts stay on the device.
struct MaskRequest {
    std::int64_t first[3];
    std::uint32_t shape[3];
    bool want_zero;
    std::uint8_t* mask;
    std::uint64_t capacity;
};

struct Compensated {
    double value {}, correction {};
    void add(double v)
    {
        const double adjusted = v - correction;
        const double next = value + adjusted;
        correction = (next - value) - adjusted;
        value = next;
    }
};

bool checked_mul(std::uint64_t a, std::uint64_t b, std::uint64_t& r)
{
    if (a && b > UINT64_MAX / a) {
        return false;
    }
    r = a * b;
    return true;
}

// Output-index probe, the reference's direct_probe (correlation.cpp:153-218).
template <typename E>
bool direct_probe(const spk_correlation_spec& spec, const E* env, const std::uint8_t* ker, const std::uint32_t* oshape,
                  std::uint64_t index, std::uint64_t max_terms, std::uint64_t& terms, double& expected)
{
    const std::uint64_t x = index % oshape[0];
    const std::uint64_t yz = index / oshape[0];
    const std::uint64_t y = yz % oshape[1];
    const std::uint64_t z = yz / oshape[1];
    const std::int64_t shift[3] = { static_cast<std::int64_t>(x) - (static_cast<std::int64_t>(spec.kernel_shape[0]) - 1),
                                    static_cast<std::int64_t>(y) - (static_cast<std::int64_t>(spec.kernel_shape[1]) - 1),
                                    static_cast<std::int64_t>(z) - (static_cast<std::int64_t>(spec.kernel_shape[2]) - 1) };
    std::uint64_t integer_sum = 0;
    Compensated real_sum;
    const auto* es = spec.environment_shape;
    const auto* ks = spec.kernel_shape;
    for (std::uint32_t kz = 0; kz != ks[2]; ++kz) {
        for (std::uint32_t ky = 0; ky != ks[1]; ++ky) {
            for (std::uint32_t kx = 0; kx != ks[0]; ++kx) {
                const std::int64_t cx = kx + shift[0], cy = ky + shift[1], cz = kz + shift[2];
                if (cx < 0 || cy < 0 || cz < 0 || cx >= es[0] || cy >= es[1] || cz >= es[2]) {
                    continue;
                }
                if (terms == max_terms) {
                    return false;
                }
                ++terms;
                const std::uint64_t eo = cx + std::uint64_t { es[0] } * (cy + std::uint64_t { es[1] } * cz);
                const std::uint64_t ko = kx + std::uint64_t { ks[0] } * (ky + std::uint64_t { ks[1] } * kz);
                if constexpr (std::is_same_v<E, std::uint8_t>) {
                    integer_sum += static_cast<std::uint64_t>(env[eo]) * ker[ko];
                }
                else {
                    real_sum.add(env[eo] * ker[ko]);
                }
            }
        }
    }
    if constexpr (std::is_same_v<E, std::uint8_t>) {
        if (integer_sum > kExactInteger) {
            return false;
        }
        expected = static_cast<double>(integer_sum);
    }
    else {
        expected = real_sum.value;
    }
    return true;
}

template <typename T>
int run_fft3(spk_context* ctx, cplx_t<T>* data, const Grid& g, bool inverse, T final_scale)
{
    int status = kOk;
    for (int axis = 0; axis != 3; ++axis) {
        const auto* tw = twiddle_table<T>(ctx, g.L[axis], status);
        if (!tw) {
            return status;
        }
        const T scale = (inverse && axis == 2) ? final_scale : static_cast<T>(1);
        if (fft_axis<T>(data, g.L[0], g.L[1], g.L[2], axis, inverse, scale, tw, ctx->stream) != cudaSuccess) {
            return kCuda;
        }
        ctx->launches++;
    }
    return kOk;
}

int grid_blocks(long long n, int threads)
{
    const long long want = (n + threads - 1) / threads;
    return static_cast<int>(std::min<long long>(std::max<long long>(want, 1), 148LL * 16));
}

template <typename T, typename E>
int correlate(spk_context* ctx, const spk_correlation_spec* spec_ptr, const E* environment, const std::uint8_t* kernel,
              const spk_correlation_limits* limits_ptr, const spk_control* control, double* out_values,
              std::uint64_t out_capacity, spk_correlation_result* result, bool half_spectra = false,
              const MaskRequest* mask_request = nullptr)
{
    constexpr bool binary = std::is_same_v<E, std::uint8_t>;
    if (!ctx || !spec_ptr || !environment || !kernel || !result) {
        return kInvalidArgument;
    }
    const auto& spec = *spec_ptr;
    spk_correlation_limits limits { 512ULL << 20, 0, 16'777'216, 200'000'000 };
    if (limits_ptr) {
        limits = *limits_ptr;
    }
    std::memset(result, 0, sizeof(*result));
    ctx->message = "";
    // The reference admits its own call metadata before anything else
    // (correlation.cpp:255-259); here that is the result record.
    if (limits.reserved_bytes > limits.max_working_bytes ||
        limits.max_working_bytes - limits.reserved_bytes < sizeof(spk_correlation_result)) {
        return fail(ctx, kMemoryLimit, "Correlation metadata exceeds its memory limit.");
    }
    if (int s = poll(control)) {
        return fail(ctx, s, "Correlation interrupted.");
    }
    std::uint64_t env_count = 1, ker_count = 1, padded_count = 1;
    std::uint32_t padded[3];
    for (int a = 0; a != 3; ++a) {
        if (spec.environment_shape[a] == 0 || spec.kernel_shape[a] == 0 ||
            !checked_mul(env_count, spec.environment_shape[a], env_count) ||
            !checked_mul(ker_count, spec.kernel_shape[a], ker_count)) {
            return fail(ctx, kShapeOverflow, "Correlation extents must be positive and representable.");
        }
        const std::uint64_t length = std::uint64_t { spec.environment_shape[a] } + spec.kernel_shape[a] - 1;
        if (length > UINT32_MAX || !checked_mul(padded_count, length, padded_count)) {
            return fail(ctx, kShapeOverflow, "Padded correlation shape overflowed.");
        }
        padded[a] = static_cast<std::uint32_t>(length);
        const std::int64_t ef = spec.environment_first[a], kf = spec.kernel_first[a];
        if ((kf > 0 && ef < INT64_MIN + kf) || (kf < 0 && ef > INT64_MAX + kf)) {
            return fail(ctx, kIndexOverflow, "The first output translation is not representable.");
        }
        const std::int64_t diff = ef - kf;
        const std::int64_t k1 = static_cast<std::int64_t>(spec.kernel_shape[a]) - 1;
        if (diff < INT64_MIN + k1) {
            return fail(ctx, kIndexOverflow, "The first output translation is not representable.");
        }
        result->translation_first[a] = diff - k1;
        if (result->translation_first[a] > INT64_MAX - static_cast<std::int64_t>(length - 1)) {
            return fail(ctx, kIndexOverflow, "The last output translation is not representable.");
        }
        result->shape[a] = padded[a];
    }
    // Input validation and masses (correlation.cpp:316-365).
    std::uint64_t env_ones = 0, ker_ones = 0;
    Compensated env_mass_sum;
    for (std::uint64_t i = 0; i != env_count; ++i) {
        const double value = static_cast<double>(environment[i]);
        if (!std::isfinite(value) || value < 0.0 || value > 1.0) {
            return fail(ctx, kInvalidEnvironment, "Environment cells must be finite values in [0,1].");
        }
        if constexpr (binary) {
            env_ones += environment[i];
        }
        else {
            env_mass_sum.add(value);
        }
    }
    for (std::uint64_t i = 0; i != ker_count; ++i) {
        if (kernel[i] > 1) {
            return fail(ctx, kInvalidKernel, "Kernel cells must be binary.");
        }
        ker_ones += kernel[i];
    }
    double expected_mass, environment_mass;
    if constexpr (binary) {
        std::uint64_t product;
        if (!checked_mul(env_ones, ker_ones, product) || product > kExactInteger) {
            return fail(ctx, kNumericRange, "Binary correlation mass is not exactly representable.");
        }
        environment_mass = static_cast<double>(env_ones);
        expected_mass = static_cast<double>(product);
    }
    else {
        environment_mass = env_mass_sum.value;
        expected_mass = environment_mass * static_cast<double>(ker_ones);
        if (!std::isfinite(environment_mass) || !std::isfinite(expected_mass)) {
            return fail(ctx, kNumericRange, "Proximity correlation mass is not representable.");
        }
    }
    result->padded_cells = padded_count;
    if (padded_count > limits.max_padded_cells) {
        return fail(ctx, kPaddedCellLimit, "Padded field exceeds its cell limit.");
    }
    Grid g;
    for (int a = 0; a != 3; ++a) {
        const std::uint32_t L = transform_length(padded[a]);
        if (L == 0) {
            return fail(ctx, kUnsupportedLength, "Padded extent exceeds the device FFT's longest axis.");
        }
        g.L[a] = static_cast<int>(L);
        result->padded_shape[a] = L;
    }
    using C = cplx_t<T>;
    const std::uint64_t grid_bytes = static_cast<std::uint64_t>(g.n()) * sizeof(C);
    const std::uint64_t out_bytes = padded_count * sizeof(double);
    const int extract_threads = 256;
    const int extract_blocks = grid_blocks(static_cast<long long>(padded_count), extract_threads);
    const std::uint64_t half_bytes = half_spectra ? static_cast<std::uint64_t>(g.n()) * 4 : 0;
    std::uint64_t mask_count = 0;
    if (mask_request) {
        mask_count = 1;
        for (int a = 0; a != 3; ++a) {
            if (!checked_mul(mask_count, mask_request->shape[a], mask_count)) {
                return fail(ctx, kShapeOverflow, "Mask box size is not representable.");
            }
        }
    }
    const std::uint64_t working = limits.reserved_bytes + 2 * grid_bytes + half_bytes + out_bytes +
                                  env_count * sizeof(E) + ker_count + extract_blocks * sizeof(ExtractStats) + 64 +
                                  mask_count;
    if (working > limits.max_working_bytes) {
        return fail(ctx, kMemoryLimit, "Correlation buffers and FFT workspace exceed their memory limit.");
    }
    result->working_bytes_peak = working;
    if (mask_request ? (mask_request->capacity < mask_count || (mask_count && !mask_request->mask))
                     : (out_capacity < padded_count || !out_values)) {
        return kInvalidArgument;
    }
    int status = kOk;
    auto* z = static_cast<C*>(device_buffer(ctx, "corr.z", grid_bytes, status));
    auto* w = static_cast<C*>(device_buffer(ctx, "corr.w", grid_bytes, status));
    auto* d_env = static_cast<E*>(device_buffer(ctx, "corr.env", env_count * sizeof(E), status));
    auto* d_ker = static_cast<std::uint8_t*>(device_buffer(ctx, "corr.ker", ker_count, status));
    auto* d_out = static_cast<double*>(device_buffer(ctx, "corr.out", out_bytes, status));
    auto* d_stats = static_cast<ExtractStats*>(
        device_buffer(ctx, "corr.stats", extract_blocks * sizeof(ExtractStats) + 32, status));
    if (!z || !w || !d_env || !d_ker || !d_out || !d_stats) {
        return status;
    }
    auto* d_flags = reinterpret_cast<unsigned long long*>(reinterpret_cast<char*>(d_stats) +
                                                          extract_blocks * sizeof(ExtractStats));
    cudaStream_t st = ctx->stream;
    cudaMemcpyAsync(d_env, environment, env_count * sizeof(E), cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(d_ker, kernel, ker_count, cudaMemcpyHostToDevice, st);
    cudaMemsetAsync(d_flags, 0, 16, st);
    cudaMemsetAsync(d_flags + 2, 0xff, 16, st);
    const int threads = 256;
    pack_kernel<T, E><<<grid_blocks(g.n(), threads), threads, 0, st>>>(
        z, g, d_env, spec.environment_shape[0], spec.environment_shape[1], spec.environment_shape[2], d_ker,
        spec.kernel_shape[0], spec.kernel_shape[1], spec.kernel_shape[2]);
    ctx->launches++;
    if ((status = run_fft3<T>(ctx, z, g, false, 1))) {
        return status;
    }
    if (int s = poll(control)) {
        return s;
    }
    if constexpr (std::is_same_v<T, float>) {
        if (half_spectra) {
            // |Z(k)| <= sum |e| + sum |k|: a power-of-two scale puts that bound at 2^15 or below.
            const double bound = environment_mass + static_cast<double>(ker_ones);
            const int shift = bound > 0 ? 15 - static_cast<int>(std::ceil(std::log2(bound))) : 0;
            auto* zh = static_cast<__half2*>(device_buffer(ctx, "corr.zh", half_bytes, status));
            if (!zh) {
                return status;
            }
            spectrum_to_half_kernel<<<grid_blocks(g.n(), threads), threads, 0, st>>>(
                z, zh, g.n(), std::ldexp(1.0f, shift));
            spectrum_product_half_kernel<<<grid_blocks(g.n(), threads), threads, 0, st>>>(zh, w, g,
                                                                                         std::ldexp(1.0f, -shift));
            ctx->launches += 2;
        }
    }
    if (!half_spectra) {
        spectrum_product_kernel<T><<<grid_blocks(g.n(), threads), threads, 0, st>>>(z, w, g);
        ctx->launches++;
    }
    if ((status = run_fft3<T>(ctx, w, g, true, static_cast<T>(1.0 / static_cast<double>(g.n()))))) {
        return status;
    }
    if (int s = poll(control)) {
        return s;
    }
    const double maximum_output = binary ? static_cast<double>(std::min(env_ones, ker_ones))
                                         : std::min(environment_mass, static_cast<double>(ker_ones));
    // FP64 keeps the reference's 1e-10 proximity tolerance; FP32 states its
    // own bound, 2^-13 relative to the output scale (2^-8 with FP16 spectra).
    const double rel = sizeof(T) == 8 ? 1e-10 : half_spectra ? 1.0 / 256.0 : 1.0 / 8192.0;
    const double proximity_tolerance = rel * std::max(1.0, maximum_output);
    const double imag_tolerance = binary ? 0.25 : proximity_tolerance;
    extract_kernel<T><<<extract_blocks, extract_threads, 0, st>>>(
        w, g, padded[0], padded[1], padded[2], spec.kernel_shape[0], spec.kernel_shape[1], spec.kernel_shape[2],
        binary ? 1 : 0, maximum_output, imag_tolerance, proximity_tolerance, d_out, d_stats, d_flags, d_flags + 2);
    ctx->launches++;
    if (mask_request && mask_count) {
        // Box offset from the range's first translation, per axis.  A box
        // more than 2^33 away lies wholly outside the < 2^32-wide range, so
        // the offset is clamped there and dx + x stays far from overflow.
        long long delta[3];
        for (int a = 0; a != 3; ++a) {
            long long d;
            if (__builtin_sub_overflow(mask_request->first[a], result->translation_first[a], &d)) {
                d = mask_request->first[a] < 0 ? -(1LL << 33) : (1LL << 33);
            }
            delta[a] = std::max(-(1LL << 33), std::min(1LL << 33, d));
        }
        auto* d_mask = static_cast<std::uint8_t*>(device_buffer(ctx, "corr.mask", mask_count, status));
        if (!d_mask) {
            return status;
        }
        mask_kernel<<<grid_blocks(static_cast<long long>(mask_count), threads), threads, 0, st>>>(
            d_out, padded[0], padded[1], padded[2], delta[0], delta[1], delta[2], mask_request->shape[0],
            mask_request->shape[1], mask_request->shape[2], mask_request->want_zero ? 1 : 0, d_mask);
        ctx->launches++;
        cudaMemcpyAsync(mask_request->mask, d_mask, mask_count, cudaMemcpyDeviceToHost, st);
    }
    std::vector<ExtractStats> stats(extract_blocks);
    unsigned long long flags[4] {};
    if (!mask_request) {
        cudaMemcpyAsync(out_values, d_out, out_bytes, cudaMemcpyDeviceToHost, st);
    }
    cudaMemcpyAsync(stats.data(), d_stats, extract_blocks * sizeof(ExtractStats), cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(flags, d_flags, 32, cudaMemcpyDeviceToHost, st);
    if (cudaStreamSynchronize(st) != cudaSuccess) {
        cudaGetLastError();
        return kCuda;
    }
    if (flags[2] != ~0ULL || flags[3] != ~0ULL) {
        if (flags[2] <= flags[3]) {
            return fail(ctx, kNumeric, "FFT produced a nonfinite or non-real value.");
        }
        return fail(ctx, kNumeric, binary ? "Binary FFT output failed its integer or range check."
                                          : "Proximity FFT output failed its range check.");
    }
    double max_residual = 0;
    std::memcpy(&max_residual, &flags[0], 8);
    Compensated output_mass;
    double best = -1.0;
    std::uint64_t best_index = 0;
    for (const auto& s : stats) {
        output_mass.add(s.mass);
        if (s.max_abs > best) {
            best = s.max_abs;
            best_index = static_cast<std::uint64_t>(s.max_index);
        }
    }
    const double mass_residual = std::fabs(output_mass.value - expected_mass);
    const double mass_tolerance = binary ? 0.25 : rel * std::max(1.0, std::fabs(expected_mass));
    if (!std::isfinite(mass_residual) || (binary ? mass_residual >= mass_tolerance : mass_residual > mass_tolerance)) {
        return fail(ctx, kNumeric, "FFT output failed its total-mass check.");
    }
    // Deterministic direct checks (correlation.cpp:549-577).
    std::uint64_t probes[8];
    std::size_t probe_count = 0;
    const auto add_probe = [&](std::uint64_t candidate) {
        for (std::size_t i = 0; i != probe_count; ++i) {
            if (probes[i] == candidate) {
                return;
            }
        }
        if (probe_count < 8) {
            probes[probe_count++] = candidate;
        }
    };
    const std::uint64_t count = padded_count;
    add_probe(0);
    add_probe(count - 1);
    add_probe(count / 2);
    add_probe(best_index);
    add_probe(count / 4);
    add_probe(count / 3);
    add_probe((count / 3) * 2);
    add_probe((count / 4) * 3);
    // With a mask request the counts stay on the device: fetch the probed ones.
    double probe_values[8] {};
    if (mask_request) {
        for (std::size_t p = 0; p != probe_count; ++p) {
            cudaMemcpyAsync(&probe_values[p], d_out + probes[p], sizeof(double), cudaMemcpyDeviceToHost, st);
        }
        if (cudaStreamSynchronize(st) != cudaSuccess) {
            cudaGetLastError();
            return kCuda;
        }
    }
    double max_probe_error = 0;
    std::uint64_t terms = 0;
    for (std::size_t p = 0; p != probe_count; ++p) {
        double expected = 0;
        if (!direct_probe(spec, environment, kernel, padded, probes[p], limits.max_direct_terms, terms, expected)) {
            result->direct_terms = terms;
            if (int s = poll(control)) {
                return fail(ctx, s, "Correlation interrupted.");
            }
            return fail(ctx, kDirectTermLimit, "Deterministic direct checks exhausted their work limit.");
        }
        const double error = std::fabs((mask_request ? probe_values[p] : out_values[probes[p]]) - expected);
        max_probe_error = std::max(max_probe_error, error);
        // FP64 keeps the reference's per-probe relative tolerance; FP32 and
        // FP16 state their bounds relative to the output scale.
        const double tolerance =
            binary ? 0.25 : rel * std::max(1.0, sizeof(T) == 8 ? std::fabs(expected) : maximum_output);
        if (!std::isfinite(error) || (binary ? error >= tolerance : error > tolerance)) {
            result->direct_terms = terms;
            return fail(ctx, kNumeric, "FFT output failed a deterministic direct check.");
        }
    }
    result->direct_terms = terms;
    result->max_integer_residual = max_residual;
    result->mass_residual = mass_residual;
    result->max_probe_error = max_probe_error;
    if (int s = poll(control)) {
        return fail(ctx, s, "Correlation interrupted.");
    }
    return kOk;
}

}  // namespace
}  // namespace spk

using namespace spk;

extern "C" {

int spk_estimate_correlation(const spk_correlation_spec* spec, uint32_t precision, spk_correlation_estimate* out)
{
    if (!spec || !out) {
        return kInvalidArgument;
    }
    std::memset(out, 0, sizeof(*out));
    std::uint64_t padded_cells = 1, grid = 1;
    for (int a = 0; a != 3; ++a) {
        const std::uint64_t length = std::uint64_t { spec->environment_shape[a] } + spec->kernel_shape[a] - 1;
        if (!spec->environment_shape[a] || !spec->kernel_shape[a] || length > UINT32_MAX ||
            !checked_mul(padded_cells, length, padded_cells)) {
            return kShapeOverflow;
        }
        const std::uint32_t L = transform_length(length);
        if (L == 0) {
            return kUnsupportedLength;
        }
        out->padded_shape[a] = L;
        grid *= L;
    }
    out->padded_cells = padded_cells;
    out->working_bytes = 2 * grid * (precision == SPK_FP64 ? 16 : 8) + (precision == SPK_FP16 ? 4 * grid : 0) +
                         padded_cells * 8;
    return kOk;
}

int spk_correlate_binary(spk_context* ctx, const spk_correlation_spec* spec, const uint8_t* environment,
                         const uint8_t* kernel, const spk_correlation_limits* limits, const spk_control* control,
                         uint32_t precision, double* out_values, uint64_t out_capacity, spk_correlation_result* result)
{
    try {
        if (ctx) {
            ctx->message = "";
        }
        if (ctx && cudaSetDevice(ctx->device) != cudaSuccess) {
            return finish(ctx, kCuda);
        }
        if (precision > SPK_FP16) {
            return finish(ctx, kInvalidArgument);
        }
        return finish(ctx, precision == SPK_FP64
                               ? correlate<double, std::uint8_t>(ctx, spec, environment, kernel, limits, control,
                                                                 out_values, out_capacity, result)
                               : correlate<float, std::uint8_t>(ctx, spec, environment, kernel, limits, control,
                                                                out_values, out_capacity, result,
                                                                precision == SPK_FP16));
    }
    catch (...) {
        return ctx ? fail(ctx, kAllocation, "Correlation allocation failed.") : kAllocation;
    }
}

int spk_correlate_binary_mask(spk_context* ctx, const spk_correlation_spec* spec, const uint8_t* environment,
                              const uint8_t* kernel, const spk_correlation_limits* limits, const spk_control* control,
                              uint32_t precision, const int64_t box_first[3], const uint32_t box_shape[3],
                              uint32_t select, uint8_t* mask, uint64_t mask_capacity, spk_correlation_result* result)
{
    try {
        if (ctx) {
            ctx->message = "";
        }
        if (ctx && cudaSetDevice(ctx->device) != cudaSuccess) {
            return finish(ctx, kCuda);
        }
        if (precision > SPK_FP16 || select > SPK_MASK_NONZERO || !box_first || !box_shape) {
            return finish(ctx, kInvalidArgument);
        }
        MaskRequest request {};
        for (int a = 0; a != 3; ++a) {
            request.first[a] = box_first[a];
            request.shape[a] = box_shape[a];
        }
        request.want_zero = select == SPK_MASK_ZERO;
        request.mask = mask;
        request.capacity = mask_capacity;
        return finish(ctx, precision == SPK_FP64
                               ? correlate<double, std::uint8_t>(ctx, spec, environment, kernel, limits, control,
                                                                 nullptr, 0, result, false, &request)
                               : correlate<float, std::uint8_t>(ctx, spec, environment, kernel, limits, control,
                                                                nullptr, 0, result, precision == SPK_FP16,
                                                                &request));
    }
    catch (...) {
        return ctx ? fail(ctx, kAllocation, "Correlation allocation failed.") : kAllocation;
    }
}

int spk_correlate_proximity(spk_context* ctx, const spk_correlation_spec* spec, const double* environment,
                            const uint8_t* kernel, const spk_correlation_limits* limits, const spk_control* control,
                            uint32_t precision, double* out_values, uint64_t out_capacity,
                            spk_correlation_result* result)
{
    try {
        if (ctx) {
            ctx->message = "";
        }
        if (ctx && cudaSetDevice(ctx->device) != cudaSuccess) {
            return finish(ctx, kCuda);
        }
        if (precision > SPK_FP16) {
            return finish(ctx, kInvalidArgument);
        }
        return finish(ctx, precision == SPK_FP64
                               ? correlate<double, double>(ctx, spec, environment, kernel, limits, control,
                                                           out_values, out_capacity, result)
                               : correlate<float, double>(ctx, spec, environment, kernel, limits, control, out_values,
                                                          out_capacity, result, precision == SPK_FP16));
    }
    catch (...) {
        return ctx ? fail(ctx, kAllocation, "Correlation allocation failed.") : kAllocation;
    }
}

}  // extern "C"
