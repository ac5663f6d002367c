// Maintainer-side binding of libspk_b200 into SpectraPack's pack_compute.
//
// These declarations sit beside compute::correlate_binary_cpu and
// compute::correlate_proximity_cpu (engine/pack_compute/include/spectrapack/
// compute/correlation.hpp:108-117) and take the same arguments, minus the
// FftExecution*: the library's context owns its stream and device memory.
// A caller switches a call site by name under #if SPECTRAPACK_B200.
#pragma once

#include <cstdint>
#include <optional>
#include <span>

#include "spectrapack/compute/correlation.hpp"

namespace spectrapack::compute {

// correlate_binary_cpu on the B200: the same full-range rounded counts, the
// same checks and the same failure codes (correlation.cpp:238-592,643-648).
[[nodiscard]] CorrelationOutcome correlate_binary_b200(const CorrelationSpec& spec,
                                                       std::span<const std::uint8_t> environment,
                                                       std::span<const std::uint8_t> kernel,
                                                       const CorrelationLimits& limits = {},
                                                       const runtime::OperationControl& control = {}) noexcept;

// correlate_proximity_cpu on the B200 (correlation.cpp:650-655).
[[nodiscard]] CorrelationOutcome correlate_proximity_b200(const CorrelationSpec& spec,
                                                          std::span<const double> environment,
                                                          std::span<const std::uint8_t> kernel,
                                                          const CorrelationLimits& limits = {},
                                                          const runtime::OperationControl& control = {}) noexcept;

// The solver's mask callers (gap_fill.cpp:392-420 free translations,
// gap_fill.cpp:432-446 blocked offsets, slab_lattice.cpp:675-691 no-fit
// maps) round the full-range counts into one byte per translation.  This does
// the rounding on the device: `mask` receives, X fastest over `box`, 1 where
// the translation lies in the correlation range and its count is zero
// (zero_count) or non-zero (nonzero_count), else 0.  The checks and failure
// codes are those of correlate_binary_b200; on failure `mask` is unspecified.
struct TranslationBox {
    Index3 first;
    Shape3 shape;
};
enum class MaskRule { zero_count, nonzero_count };
[[nodiscard]] std::optional<CorrelationFailure> correlate_binary_mask_b200(
    const CorrelationSpec& spec, std::span<const std::uint8_t> environment, std::span<const std::uint8_t> kernel,
    const TranslationBox& box, MaskRule rule, std::span<std::uint8_t> mask, const CorrelationLimits& limits = {},
    const runtime::OperationControl& control = {}) noexcept;

}  // namespace spectrapack::compute
