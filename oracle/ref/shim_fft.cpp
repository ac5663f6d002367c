// Test infrastructure only: FP64 per-axis FFT stand-in for the reference's
// pocketfft-backed engine/pack_compute/src/fft_execution.cpp.
//
// The reference pins pocketfft 2023-09-25 (vcpkg.json:22-25), which is not
// present in this environment.  This file defines the symbols that
// engine/pack_compute/src/correlation.cpp links against
// (fft_execution_internal.hpp:16-20, correlation.hpp:80-98) with a
// project-written complex FFT of the same algorithm class as pocketfft's:
// mixed-radix Cooley-Tukey (radices 4, 2, 3, 5 with dedicated butterflies,
// every other prime factor up to 31 by a direct small DFT), in Stockham
// autosort order, and Bluestein's chirp-z algorithm (a published method) for
// lengths with a larger prime factor, whose inner convolution length is the
// smallest 2^a 3^b 5^c at or above 2n - 1.  Lines are transformed in blocks
// of kBlock lines interleaved innermost, so every butterfly runs over
// contiguous values and strided axes are gathered a cache line at a time.
// Conventions follow the reference's use: forward = exp(-2*pi*i*j*k/n),
// backward = exp(+2*pi*i*j*k/n), both unscaled, then every value times
// `factor` (correlation.cpp:466-478 passes 1/P on axis 0 of the inverse).
// The correlation's own integer, mass and probe checks still guard it.

#include <algorithm>
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
constexpr std::size_t kBlock = 16;       // lines per block (interleaved innermost)
constexpr std::size_t kLargestRadix = 31;  // larger prime factors go through Bluestein

// exp(sign * 2 pi i * k / n) with k reduced mod n first.
Complex root(std::size_t k, std::size_t n, int sign)
{
    k %= n;
    const double angle = 2.0 * kPi * static_cast<double>(k) / static_cast<double>(n);
    return { std::cos(angle), sign * std::sin(angle) };
}

std::vector<std::size_t> factorise(std::size_t n)
{
    std::vector<std::size_t> radices;
    while (n % 4 == 0) {
        radices.push_back(4);
        n /= 4;
    }
    if (n % 2 == 0) {
        radices.push_back(2);
        n /= 2;
    }
    for (std::size_t p = 3; p * p <= n; p += 2) {
        while (n % p == 0) {
            radices.push_back(p);
            n /= p;
        }
    }
    if (n > 1) {
        radices.push_back(n);
    }
    return radices;
}

std::size_t smooth_at_least(std::size_t n)
{
    for (std::size_t m = n;; ++m) {
        std::size_t r = m;
        for (std::size_t p : { 2, 3, 5 }) {
            while (r % p == 0) {
                r /= p;
            }
        }
        if (r == 1) {
            return m;
        }
    }
}

// Mixed-radix Stockham transform of `lines` interleaved sequences of length n
// (value i of line b at a[b + lines * i]).  Each stage splits the current
// length len = p * m: y[r + s (p q + k)] = W_len^(q k) * sum_j x[r + s (q + m j)] W_p^(j k),
// with s the running stride (lines at the first stage); outputs land in
// natural order.
struct Radix {
    std::size_t n {};
    std::vector<std::size_t> radices;
    std::vector<std::vector<Complex>> twiddles[2];  // [direction][stage]: W_len^(q k), q < m, k < p
    std::vector<std::vector<Complex>> small[2];     // [direction][stage]: W_p^(j k mod p)

    void prepare(std::size_t length)
    {
        n = length;
        radices = factorise(n);
        for (int d = 0; d != 2; ++d) {
            const int sign = d == 0 ? -1 : 1;
            twiddles[d].clear();
            small[d].clear();
            std::size_t len = n;
            for (std::size_t p : radices) {
                const std::size_t m = len / p;
                std::vector<Complex> tw(m * p);
                for (std::size_t q = 0; q != m; ++q) {
                    for (std::size_t k = 0; k != p; ++k) {
                        tw[q * p + k] = root(q * k, len, sign);
                    }
                }
                std::vector<Complex> w(p);
                for (std::size_t k = 0; k != p; ++k) {
                    w[k] = root(k, p, sign);
                }
                twiddles[d].push_back(std::move(tw));
                small[d].push_back(std::move(w));
                len = m;
            }
        }
    }

    // Transforms in place; `scratch` holds as many values as `a`.
    void run(Complex* a, Complex* scratch, std::size_t lines, bool forward) const
    {
        const int d = forward ? 0 : 1;
        const double sign = forward ? -1.0 : 1.0;
        Complex* x = a;
        Complex* y = scratch;
        std::size_t len = n, s = lines;
        for (std::size_t stage = 0; stage != radices.size(); ++stage) {
            const std::size_t p = radices[stage], m = len / p;
            const Complex* tw = twiddles[d][stage].data();
            const Complex* w = small[d][stage].data();
            for (std::size_t q = 0; q != m; ++q) {
                const Complex* t = tw + q * p;
                for (std::size_t r = 0; r != s; ++r) {
                    const Complex* in = x + r + s * q;
                    Complex* out = y + r + s * p * q;
                    const std::size_t step = s * m;
                    if (p == 4) {
                        const Complex a0 = in[0], a1 = in[step], a2 = in[2 * step], a3 = in[3 * step];
                        const Complex s02 = a0 + a2, d02 = a0 - a2, s13 = a1 + a3, d13 = a1 - a3;
                        // multiplication by sign * i
                        const Complex rot { -sign * d13.imag(), sign * d13.real() };
                        out[0] = s02 + s13;
                        out[s] = (d02 + rot) * t[1];
                        out[2 * s] = (s02 - s13) * t[2];
                        out[3 * s] = (d02 - rot) * t[3];
                    }
                    else if (p == 2) {
                        const Complex a0 = in[0], a1 = in[step];
                        out[0] = a0 + a1;
                        out[s] = (a0 - a1) * t[1];
                    }
                    else if (p == 3) {
                        const Complex a0 = in[0], a1 = in[step], a2 = in[2 * step];
                        const Complex sum = a1 + a2, diff = a1 - a2;
                        const Complex mid = a0 - 0.5 * sum;
                        const double h = sign * 0.86602540378443864676372317075293618;
                        const Complex rot { -h * diff.imag(), h * diff.real() };
                        out[0] = a0 + sum;
                        out[s] = (mid + rot) * t[1];
                        out[2 * s] = (mid - rot) * t[2];
                    }
                    else {
                        Complex v[kLargestRadix];
                        for (std::size_t j = 0; j != p; ++j) {
                            v[j] = in[j * step];
                        }
                        for (std::size_t k = 0; k != p; ++k) {
                            Complex acc = v[0];
                            std::size_t e = 0;
                            for (std::size_t j = 1; j != p; ++j) {
                                e += k;
                                if (e >= p) {
                                    e -= p;
                                }
                                acc += v[j] * w[e];
                            }
                            out[k * s] = k ? acc * t[k] : acc;
                        }
                    }
                }
            }
            std::swap(x, y);
            s *= p;
            len = m;
        }
        if (x != a) {
            std::copy(x, x + n * lines, a);
        }
    }
};

// One length: direct mixed radix, or Bluestein over a smooth inner length.
struct Plan {
    std::size_t n {}, m {};
    bool bluestein {};
    Radix inner;
    std::vector<Complex> chirp;     // exp(-i pi k^2 / n), k < n
    std::vector<Complex> filter[2];  // inner forward transform of the wrapped conj(chirp) / chirp
    std::vector<Complex> work, scratch;

    explicit Plan(std::size_t length) : n(length)
    {
        const auto radices = factorise(n);
        bluestein = !radices.empty() && radices.back() > kLargestRadix;
        m = bluestein ? smooth_at_least(2 * n - 1) : n;
        inner.prepare(m);
        if (bluestein) {
            chirp.resize(n);
            for (std::size_t k = 0; k < n; ++k) {
                // k^2 mod 2n keeps the angle argument small and exact.
                const auto square = static_cast<std::uint64_t>(k) * k % (2 * static_cast<std::uint64_t>(n));
                const double angle = -kPi * static_cast<double>(square) / static_cast<double>(n);
                chirp[k] = { std::cos(angle), std::sin(angle) };
            }
            std::vector<Complex> tmp(m);
            for (int d = 0; d != 2; ++d) {
                std::vector<Complex> b(m);
                for (std::size_t k = 0; k < n; ++k) {
                    const Complex value = d == 0 ? std::conj(chirp[k]) : chirp[k];
                    b[k] = value;
                    if (k) {
                        b[m - k] = value;
                    }
                }
                inner.run(b.data(), tmp.data(), 1, true);
                filter[d] = std::move(b);
            }
        }
    }

    // Transforms `lines` interleaved lines of length n held in `a`.
    void run(Complex* a, std::size_t lines, bool forward)
    {
        if (!bluestein) {
            scratch.resize(n * lines);
            inner.run(a, scratch.data(), lines, forward);
            return;
        }
        work.resize(m * lines);
        scratch.resize(m * lines);
        const auto& filt = filter[forward ? 0 : 1];
        for (std::size_t k = 0; k < n; ++k) {
            const Complex c = forward ? chirp[k] : std::conj(chirp[k]);
            for (std::size_t b = 0; b != lines; ++b) {
                work[b + lines * k] = a[b + lines * k] * c;
            }
        }
        std::fill(work.begin() + static_cast<std::ptrdiff_t>(n * lines), work.end(), Complex {});
        inner.run(work.data(), scratch.data(), lines, true);
        for (std::size_t k = 0; k < m; ++k) {
            for (std::size_t b = 0; b != lines; ++b) {
                work[b + lines * k] *= filt[k];
            }
        }
        inner.run(work.data(), scratch.data(), lines, false);
        const double scale = 1.0 / static_cast<double>(m);
        for (std::size_t k = 0; k < n; ++k) {
            const Complex c = (forward ? chirp[k] : std::conj(chirp[k])) * scale;
            for (std::size_t b = 0; b != lines; ++b) {
                a[b + lines * k] = work[b + lines * k] * c;
            }
        }
    }
};

}  // namespace

void FftAccess::join(FftExecution*) noexcept {}

std::optional<CorrelationFailure> FftAccess::run(FftExecution*, Shape3 shape, std::size_t axis, bool forward,
                                                 std::complex<double>* data, double factor,
                                                 const runtime::OperationControl& control)
{
    try {
        const std::size_t n = shape[axis];
        const std::size_t sx = shape[0], sy = shape[1], sz = shape[2];
        const std::size_t stride = axis == 0 ? 1 : axis == 1 ? sx : sx * sy;
        Plan plan(n);
        std::vector<Complex> block(n * kBlock);
        // Lines are enumerated so that kBlock consecutive ones are adjacent in
        // memory (x for axes 1 and 2, whole rows for axis 0).
        const std::size_t inner_count = axis == 0 ? sy * sz : sx;               // lines per outer group
        const std::size_t outer_count = axis == 0 ? 1 : axis == 1 ? sz : sy;    // groups
        const std::size_t inner_step = axis == 0 ? sx : 1;                      // base step between lines
        const std::size_t outer_step = axis == 1 ? sx * sy : axis == 2 ? sx : 0;
        std::uint32_t polls {};
        for (std::size_t outer = 0; outer != outer_count; ++outer) {
            for (std::size_t first = 0; first < inner_count; first += kBlock) {
                if ((++polls & 15U) == 0 && control.poll() != runtime::StopCause::none) {
                    return CorrelationFailure { control.poll() == runtime::StopCause::user_stopped
                                                    ? "OPERATION_CANCELLED"
                                                    : "DEADLINE_EXCEEDED",
                                                "Correlation interrupted.",
                                                {} };
                }
                const std::size_t lines = std::min(kBlock, inner_count - first);
                const std::size_t base0 = outer * outer_step + first * inner_step;
                for (std::size_t q = 0; q != n; ++q) {
                    const Complex* src = data + base0 + q * stride;
                    Complex* dst = block.data() + lines * q;
                    for (std::size_t b = 0; b != lines; ++b) {
                        dst[b] = src[b * inner_step];
                    }
                }
                plan.run(block.data(), lines, forward);
                for (std::size_t q = 0; q != n; ++q) {
                    Complex* dst = data + base0 + q * stride;
                    const Complex* src = block.data() + lines * q;
                    for (std::size_t b = 0; b != lines; ++b) {
                        dst[b * inner_step] = src[b] * factor;
                    }
                }
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
