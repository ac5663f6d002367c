// Test infrastructure only: FP64 per-axis FFT stand-in for the reference's
// pocketfft-backed engine/pack_compute/src/fft_execution.cpp.
//
// The reference pins pocketfft 2023-09-25 (vcpkg.json:22-25), which is not
// present in this environment.  This file defines the symbols that
// engine/pack_compute/src/correlation.cpp links against
// (fft_execution_internal.hpp:16-20, correlation.hpp:80-98) with a
// project-written complex FFT: iterative radix-2 for power-of-two lengths and
// Bluestein's chirp-z algorithm (a published method) for every other length.
// Conventions follow the reference's use: forward = exp(-2*pi*i*j*k/n),
// backward = exp(+2*pi*i*j*k/n), both unscaled, then every value times
// `factor` (correlation.cpp:466-478 passes 1/P on axis 0 of the inverse).
// The correlation's own integer, mass and probe checks still guard it.

#include <cmath>
#include <complex>
#include <cstdint>
#include <memory>
#include <optional>
#include <variant>
#include <vector>

#include "fft_execution_internal.hpp"

namespace spectrapack::compute {

struct FftExecution::Storage {
    std::uint32_t threads { 1 };
};

FftExecution::FftExecution(std::uint32_t count) : storage_(std::make_unique<Storage>())
{
    storage_->threads = count;
}
FftExecution::~FftExecution() = default;
std::uint32_t FftExecution::thread_count() const noexcept { return storage_ ? storage_->threads : 1; }
std::uint64_t FftExecution::reserved_bytes() const noexcept { return 0; }

std::optional<std::uint64_t> estimate_fft_execution_bytes(std::uint32_t count) noexcept
{
    if (count == 0 || count > 8) {
        return std::nullopt;
    }
    return std::uint64_t {};
}

std::variant<std::unique_ptr<FftExecution>, CorrelationFailure> make_fft_execution(std::uint32_t count,
                                                                                  std::uint64_t)
{
    if (count == 0 || count > 8) {
        return CorrelationFailure { "CPU_THREAD_COUNT_UNSUPPORTED", "Unsupported FFT thread count.", {} };
    }
    return std::unique_ptr<FftExecution>(new FftExecution(count));
}

namespace detail {

void set_fft_test_options(FftTestOptions) noexcept {}

namespace {

using Complex = std::complex<double>;
constexpr double kPi = 3.14159265358979323846264338327950288;

bool power_of_two(std::size_t n) { return n && !(n & (n - 1)); }

// In-place iterative radix-2 transform; sign -1 forward, +1 backward.
void radix2(std::vector<Complex>& a, int sign, const std::vector<Complex>& roots)
{
    const std::size_t n = a.size();
    for (std::size_t i = 1, j = 0; i < n; ++i) {
        std::size_t bit = n >> 1;
        for (; j & bit; bit >>= 1) {
            j ^= bit;
        }
        j ^= bit;
        if (i < j) {
            std::swap(a[i], a[j]);
        }
    }
    for (std::size_t len = 2; len <= n; len <<= 1) {
        const std::size_t step = n / len;
        for (std::size_t i = 0; i < n; i += len) {
            for (std::size_t k = 0; k < len / 2; ++k) {
                Complex w = roots[k * step];
                if (sign > 0) {
                    w = std::conj(w);
                }
                const Complex u = a[i + k];
                const Complex v = a[i + k + len / 2] * w;
                a[i + k] = u + v;
                a[i + k + len / 2] = u - v;
            }
        }
    }
}

// Plan for one length: forward roots exp(-2 pi i k / m) for the radix-2 core
// and, for non-power-of-two n, the Bluestein chirp and its transformed filter.
struct Plan {
    std::size_t n {}, m {};
    std::vector<Complex> roots;
    std::vector<Complex> chirp;        // exp(-i pi k^2 / n), k < n
    std::vector<Complex> filter_fwd;   // FFT of conj(chirp) wrapped, forward transform
    std::vector<Complex> filter_bwd;   // FFT of chirp wrapped, backward transform
    std::vector<Complex> work;
};

Plan make_plan(std::size_t n)
{
    Plan plan;
    plan.n = n;
    plan.m = n;
    if (!power_of_two(n)) {
        plan.m = 1;
        while (plan.m < 2 * n - 1) {
            plan.m <<= 1;
        }
    }
    plan.roots.resize(plan.m / 2 + 1);
    for (std::size_t k = 0; k <= plan.m / 2; ++k) {
        const double angle = -2.0 * kPi * static_cast<double>(k) / static_cast<double>(plan.m);
        plan.roots[k] = { std::cos(angle), std::sin(angle) };
    }
    if (plan.m != n) {
        plan.chirp.resize(n);
        for (std::size_t k = 0; k < n; ++k) {
            // k^2 mod 2n keeps the angle argument small and exact.
            const auto square = static_cast<std::uint64_t>(k) * k % (2 * static_cast<std::uint64_t>(n));
            const double angle = -kPi * static_cast<double>(square) / static_cast<double>(n);
            plan.chirp[k] = { std::cos(angle), std::sin(angle) };
        }
        for (int pass = 0; pass != 2; ++pass) {
            std::vector<Complex> b(plan.m);
            for (std::size_t k = 0; k < n; ++k) {
                const Complex value = pass == 0 ? std::conj(plan.chirp[k]) : plan.chirp[k];
                b[k] = value;
                if (k) {
                    b[plan.m - k] = value;
                }
            }
            radix2(b, -1, plan.roots);
            (pass == 0 ? plan.filter_fwd : plan.filter_bwd) = std::move(b);
        }
        plan.work.resize(plan.m);
    }
    return plan;
}

// Transform one gathered line of length n in place.
void transform_line(Plan& plan, std::vector<Complex>& line, bool forward)
{
    const int sign = forward ? -1 : 1;
    if (plan.m == plan.n) {
        radix2(line, sign, plan.roots);
        return;
    }
    const std::size_t n = plan.n, m = plan.m;
    auto& a = plan.work;
    for (std::size_t k = 0; k < n; ++k) {
        a[k] = line[k] * (forward ? plan.chirp[k] : std::conj(plan.chirp[k]));
    }
    for (std::size_t k = n; k < m; ++k) {
        a[k] = 0.0;
    }
    radix2(a, -1, plan.roots);
    const auto& filter = forward ? plan.filter_fwd : plan.filter_bwd;
    for (std::size_t k = 0; k < m; ++k) {
        a[k] *= filter[k];
    }
    radix2(a, 1, plan.roots);
    const double scale = 1.0 / static_cast<double>(m);
    for (std::size_t k = 0; k < n; ++k) {
        line[k] = a[k] * scale * (forward ? plan.chirp[k] : std::conj(plan.chirp[k]));
    }
}

}  // namespace

void FftAccess::join(FftExecution*) noexcept {}

std::optional<CorrelationFailure> FftAccess::run(FftExecution*, Shape3 shape, std::size_t axis, bool forward,
                                                 std::complex<double>* data, double factor,
                                                 const runtime::OperationControl& control)
{
    try {
        const std::size_t n = shape[axis];
        const std::size_t stride = axis == 0 ? 1 : axis == 1 ? shape[0] : std::size_t { shape[0] } * shape[1];
        const std::size_t total = std::size_t { shape[0] } * shape[1] * shape[2];
        Plan plan = make_plan(n);
        std::vector<Complex> line(plan.m == n ? n : n);
        std::uint32_t polls {};
        for (std::size_t base = 0; base != total; ++base) {
            if ((base / stride) % n != 0) {
                continue;
            }
            if ((++polls & 255U) == 0 && control.poll() != runtime::StopCause::none) {
                return CorrelationFailure { control.poll() == runtime::StopCause::user_stopped ? "OPERATION_CANCELLED"
                                                                                               : "DEADLINE_EXCEEDED",
                                            "Correlation interrupted.",
                                            {} };
            }
            line.resize(n);
            for (std::size_t q = 0; q != n; ++q) {
                line[q] = data[base + q * stride];
            }
            transform_line(plan, line, forward);
            for (std::size_t q = 0; q != n; ++q) {
                data[base + q * stride] = line[q] * factor;
            }
        }
        return std::nullopt;
    }
    catch (const std::bad_alloc&) {
        return CorrelationFailure { "CORRELATION_ALLOCATION", "Correlation allocation failed.", {} };
    }
}

}  // namespace detail
}  // namespace spectrapack::compute
