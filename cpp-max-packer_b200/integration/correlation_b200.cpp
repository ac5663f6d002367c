// Maintainer-side binding of libspk_b200 into SpectraPack's pack_compute:
// the reference's correlation types (engine/pack_compute/include/spectrapack/
// compute/correlation.hpp:22-117) mapped onto the C ABI of spk_b200.h.
//
// The reference's contract is kept.  Nothing throws.  Failures are
// CorrelationFailure values with the reference's static code strings and
// messages.  `values` is owned by the returned result.  The
// OperationControl's stop token and deadline reach the library as a stop
// word and a CLOCK_MONOTONIC deadline, which it polls between device phases.
// A stop or an expired deadline seen before the call returns the reference's
// interruption failure (correlation.cpp:263-275) without touching the device.
#include "correlation_b200.hpp"

#include <time.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <limits>
#include <new>
#include <stop_token>
#include <string_view>
#include <vector>

#include "spk_b200.h"

namespace spectrapack::compute {
namespace {

// The reference's metadata admission (correlation.cpp:67-72,255-259): the
// call's own outcome, values vector and control, before anything else.
constexpr std::uint64_t kMetadataBytes =
    2 * sizeof(CorrelationOutcome) + sizeof(std::vector<double>) + sizeof(runtime::OperationControl);

CorrelationFailure failure(std::string_view code, std::string_view message, CorrelationStats stats = {}) noexcept
{
    return CorrelationFailure { code, message, stats };
}

std::optional<CorrelationFailure> metadata_limit(const CorrelationLimits& limits) noexcept
{
    std::uint64_t metadata {};
    if (__builtin_add_overflow(limits.reserved_bytes, kMetadataBytes, &metadata) ||
        metadata > limits.max_working_bytes) {
        return failure("CORRELATION_MEMORY_LIMIT", "Correlation metadata exceeds its memory limit.");
    }
    return std::nullopt;
}

// One context per process on device 0, created on first use.  Calls are
// serialised by the caller's coordinator (correlation.hpp:78-79).
spk_context* device_context() noexcept
{
    static spk_context* const context = [] {
        spk_context* c {};
        return spk_context_create(0, 0, &c) == 0 ? c : nullptr;
    }();
    return context;
}

std::int64_t monotonic_ns() noexcept
{
    timespec ts {};
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return static_cast<std::int64_t>(ts.tv_sec) * 1'000'000'000 + ts.tv_nsec;
}

// The OperationControl as the library's spk_control: a stop word raised by a
// stop_callback, and the time left before the deadline (measured on the
// control's own clock, which tests may replace) added to CLOCK_MONOTONIC.
class ControlBridge {
public:
    explicit ControlBridge(const runtime::OperationControl& control) :
        word_(control.stop.stop_requested() ? 1u : 0u), on_stop_(control.stop, Raise { &word_ })
    {
        c_.stop_word = reinterpret_cast<const volatile std::uint32_t*>(&word_);
        if (control.deadline) {
            const auto left = std::chrono::duration_cast<std::chrono::nanoseconds>(*control.deadline - control.now())
                                  .count();
            const std::int64_t now = monotonic_ns();
            const std::int64_t room = std::numeric_limits<std::int64_t>::max() - now;
            c_.deadline_ns = now + std::clamp<std::int64_t>(left, 1, room);
        }
    }
    ControlBridge(const ControlBridge&) = delete;
    ControlBridge& operator=(const ControlBridge&) = delete;
    const spk_control* get() const noexcept { return &c_; }

private:
    struct Raise {
        std::atomic<std::uint32_t>* word;
        void operator()() const noexcept { word->store(1); }
    };
    static_assert(sizeof(std::atomic<std::uint32_t>) == sizeof(std::uint32_t) &&
                  std::atomic<std::uint32_t>::is_always_lock_free);
    std::atomic<std::uint32_t> word_;
    std::stop_callback<Raise> on_stop_;
    spk_control c_ {};
};

std::optional<CorrelationFailure> interrupted(const runtime::OperationControl& control) noexcept
{
    switch (control.poll()) {
    case runtime::StopCause::user_stopped:
        return failure("OPERATION_CANCELLED", "Correlation interrupted.");
    case runtime::StopCause::deadline:
        return failure("DEADLINE_EXCEEDED", "Correlation interrupted.");
    default:
        return std::nullopt;
    }
}

// The reference's spec and field checks, in its order and with its message
// per site (correlation.cpp:276-314): per axis the extents, the padded
// length, the first and the last translation; then the storage size and the
// supplied cell counts.  The library repeats the axis checks; the cell counts
// only the caller's spans hold.
std::optional<CorrelationFailure> check_fields(const CorrelationSpec& spec, std::size_t environment_size,
                                               std::size_t kernel_size, std::uint64_t& output_count) noexcept
{
    std::uint64_t env_cells = 1, ker_cells = 1, count = 1;
    for (int a = 0; a < 3; ++a) {
        const std::uint64_t e = spec.environment_shape[a], k = spec.kernel_shape[a];
        if (!e || !k || __builtin_mul_overflow(env_cells, e, &env_cells) ||
            __builtin_mul_overflow(ker_cells, k, &ker_cells)) {
            return failure("CORRELATION_SHAPE_OVERFLOW", "Correlation extents must be positive and representable.");
        }
        const std::uint64_t length = e + k - 1;
        if (length > std::numeric_limits<std::uint32_t>::max() || __builtin_mul_overflow(count, length, &count)) {
            return failure("CORRELATION_SHAPE_OVERFLOW", "Padded correlation shape overflowed.");
        }
        std::int64_t difference {}, first {}, last {};
        if (__builtin_sub_overflow(spec.environment_first[a], spec.kernel_first[a], &difference) ||
            __builtin_sub_overflow(difference, static_cast<std::int64_t>(k) - 1, &first)) {
            return failure("CORRELATION_INDEX_OVERFLOW", "The first output translation is not representable.");
        }
        if (__builtin_add_overflow(first, static_cast<std::int64_t>(length) - 1, &last)) {
            return failure("CORRELATION_INDEX_OVERFLOW", "The last output translation is not representable.");
        }
    }
    if (env_cells > std::numeric_limits<std::size_t>::max() || ker_cells > std::numeric_limits<std::size_t>::max() ||
        count > std::numeric_limits<std::size_t>::max()) {
        return failure("CORRELATION_SHAPE_OVERFLOW", "Correlation storage size is not representable.");
    }
    if (environment_size != env_cells || kernel_size != ker_cells) {
        return failure("CORRELATION_INVALID_FIELD", "Shape does not match supplied cells.");
    }
    output_count = count;
    return std::nullopt;
}

// A library failure as the reference's value: its code, and the message the
// library recorded for the failing site.
CorrelationFailure library_failure(spk_context* context, int status, CorrelationStats stats) noexcept
{
    return failure(spk_status_code(status), spk_context_message(context), stats);
}

spk_correlation_spec to_spk(const CorrelationSpec& s) noexcept
{
    spk_correlation_spec out {};
    for (int a = 0; a < 3; ++a) {
        out.environment_shape[a] = s.environment_shape[a];
        out.kernel_shape[a] = s.kernel_shape[a];
        out.environment_first[a] = s.environment_first[a];
        out.kernel_first[a] = s.kernel_first[a];
    }
    return out;
}

spk_correlation_limits to_spk(const CorrelationLimits& l) noexcept
{
    return { l.max_working_bytes, l.reserved_bytes, l.max_padded_cells, l.max_direct_terms };
}

CorrelationStats stats_of(const spk_correlation_result& r) noexcept
{
    return { r.padded_cells, r.working_bytes_peak, r.direct_terms };
}

template <class Env, class Call>
CorrelationOutcome run(const CorrelationSpec& spec, std::span<const Env> environment,
                       std::span<const std::uint8_t> kernel, const CorrelationLimits& limits,
                       const runtime::OperationControl& control, Call call) noexcept
{
    try {
        if (auto limit = metadata_limit(limits)) {
            return *limit;
        }
        if (auto stop = interrupted(control)) {
            return *stop;
        }
        std::uint64_t count = 0;
        if (auto bad = check_fields(spec, environment.size(), kernel.size(), count)) {
            return *bad;
        }
        spk_context* context = device_context();
        if (!context) {
            return failure("CORRELATION_ALLOCATION", "Correlation allocation failed.");
        }
        std::vector<double> values(count);
        const spk_correlation_spec s = to_spk(spec);
        const spk_correlation_limits l = to_spk(limits);
        const ControlBridge bridge(control);
        spk_correlation_result r {};
        const int status = call(context, &s, environment.data(), kernel.data(), &l, bridge.get(), SPK_FP64,
                                values.data(), count, &r);
        if (status != 0) {
            return library_failure(context, status, stats_of(r));
        }
        return CorrelationResult { { r.translation_first[0], r.translation_first[1], r.translation_first[2] },
                                   { r.shape[0], r.shape[1], r.shape[2] },
                                   values,
                                   { r.max_integer_residual, r.mass_residual, r.max_probe_error },
                                   stats_of(r) };
    }
    catch (const std::bad_alloc&) {
        return failure("CORRELATION_ALLOCATION", "Correlation allocation failed.");
    }
    catch (...) {
        return failure("CORRELATION_OPERATION", "Correlation operation failed.");
    }
}

}  // namespace

CorrelationOutcome correlate_binary_b200(const CorrelationSpec& spec, std::span<const std::uint8_t> environment,
                                         std::span<const std::uint8_t> kernel, const CorrelationLimits& limits,
                                         const runtime::OperationControl& control) noexcept
{
    return run(spec, environment, kernel, limits, control, spk_correlate_binary);
}

CorrelationOutcome correlate_proximity_b200(const CorrelationSpec& spec, std::span<const double> environment,
                                            std::span<const std::uint8_t> kernel, const CorrelationLimits& limits,
                                            const runtime::OperationControl& control) noexcept
{
    return run(spec, environment, kernel, limits, control, spk_correlate_proximity);
}

std::optional<CorrelationFailure> correlate_binary_mask_b200(const CorrelationSpec& spec,
                                                             std::span<const std::uint8_t> environment,
                                                             std::span<const std::uint8_t> kernel,
                                                             const TranslationBox& box, MaskRule rule,
                                                             std::span<std::uint8_t> mask,
                                                             const CorrelationLimits& limits,
                                                             const runtime::OperationControl& control) noexcept
{
    try {
        if (auto limit = metadata_limit(limits)) {
            return limit;
        }
        if (auto stop = interrupted(control)) {
            return stop;
        }
        std::uint64_t count = 0;
        if (auto bad = check_fields(spec, environment.size(), kernel.size(), count)) {
            return bad;
        }
        spk_context* context = device_context();
        if (!context) {
            return failure("CORRELATION_ALLOCATION", "Correlation allocation failed.");
        }
        const spk_correlation_spec s = to_spk(spec);
        const spk_correlation_limits l = to_spk(limits);
        const ControlBridge bridge(control);
        spk_correlation_result r {};
        const int status = spk_correlate_binary_mask(
            context, &s, environment.data(), kernel.data(), &l, bridge.get(), SPK_FP64, box.first.data(),
            box.shape.data(), rule == MaskRule::zero_count ? SPK_MASK_ZERO : SPK_MASK_NONZERO, mask.data(),
            mask.size(), &r);
        if (status != 0) {
            return library_failure(context, status, stats_of(r));
        }
        return std::nullopt;
    }
    catch (const std::bad_alloc&) {
        return failure("CORRELATION_ALLOCATION", "Correlation allocation failed.");
    }
    catch (...) {
        return failure("CORRELATION_OPERATION", "Correlation operation failed.");
    }
}

}  // namespace spectrapack::compute
