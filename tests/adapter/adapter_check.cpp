// Check of the maintainer-side adapter (cpp-max-packer_b200/integration/
// correlation_b200.cpp) against the reference's own correlate_binary_cpu and
// correlate_proximity_cpu, linked from the reference build.  Test
// infrastructure only.
//
// Every case runs through both functions on the same inputs and compares the
// outcome kind and code, and with a device also the values (binary exactly,
// proximity within the reference's 1e-10).  Without a device the adapter must
// fail closed with CORRELATION_ALLOCATION on the cases that reach the library.  Prints
// one line per case and "PASS" at the end; exits non-zero on a mismatch.
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdint>
#include <stop_token>
#include <string>
#include <variant>
#include <vector>

#include "correlation_b200.hpp"

namespace compute = spectrapack::compute;
namespace runtime = spectrapack::runtime;

namespace {

int failures = 0;

std::string code_of(const compute::CorrelationOutcome& o)
{
    if (const auto* f = std::get_if<compute::CorrelationFailure>(&o)) {
        return std::string(f->code);
    }
    return "OK";
}

void report(const char* name, bool ok, const std::string& detail)
{
    std::printf("%s %s %s\n", ok ? "ok" : "MISMATCH", name, detail.c_str());
    failures += ok ? 0 : 1;
}

// The adapter's answer must be the reference's.  Without a device, a case
// that gets past the adapter's own checks (stop, deadline, extents,
// translation range, cell counts) fails closed with CORRELATION_ALLOCATION,
// whatever the library would have answered.
void compare(const char* name, const compute::CorrelationOutcome& ours, const compute::CorrelationOutcome& ref,
             bool proximity)
{
    const std::string a = code_of(ours), b = code_of(ref);
    const bool adapter_side = b == "OPERATION_CANCELLED" || b == "DEADLINE_EXCEEDED" ||
                              b == "CORRELATION_SHAPE_OVERFLOW" || b == "CORRELATION_INDEX_OVERFLOW" ||
                              b == "CORRELATION_INVALID_FIELD";
    if (a == "CORRELATION_ALLOCATION" && b != a && !adapter_side) {
        report(name, true, "no device: fails closed (reference: " + b + ")");
        return;
    }
    if (a != b) {
        report(name, false, a + " vs " + b);
        return;
    }
    if (a != "OK") {
        // Same code: the message must be the reference's for the same site.
        const auto& fa = std::get<compute::CorrelationFailure>(ours);
        const auto& fb = std::get<compute::CorrelationFailure>(ref);
        report(name, fa.message == fb.message,
               a + " '" + std::string(fa.message) + "' vs '" + std::string(fb.message) + "'");
        return;
    }
    const auto& x = std::get<compute::CorrelationResult>(ours);
    const auto& y = std::get<compute::CorrelationResult>(ref);
    bool same = x.translation_first == y.translation_first && x.shape == y.shape && x.values.size() == y.values.size();
    for (std::size_t i = 0; same && i != x.values.size(); ++i) {
        same = proximity ? std::fabs(x.values[i] - y.values[i]) <= 1e-10 * std::max(1.0, std::fabs(y.values[i]))
                         : x.values[i] == y.values[i];
    }
    report(name, same, "values");
}

std::vector<std::uint8_t> pattern(std::size_t n, std::uint32_t salt)
{
    std::vector<std::uint8_t> cells(n);
    for (std::size_t i = 0; i != n; ++i) {
        cells[i] = static_cast<std::uint8_t>(((i * 7 + salt * 3) % 11) < 4);
    }
    cells.front() = 1;
    return cells;
}

runtime::Clock::time_point fake_now(void* ticks) noexcept
{
    auto& count = *static_cast<std::uint64_t*>(ticks);
    return runtime::Clock::time_point {} + std::chrono::milliseconds(++count);
}

}  // namespace

int main()
{
    const compute::CorrelationSpec spec { { 7, 5, 4 }, { 3, 2, 2 }, { 4, -3, 9 }, { -1, 2, -5 } };
    const auto env = pattern(7 * 5 * 4, 2);
    const auto ker = pattern(3 * 2 * 2, 5);
    std::vector<double> prox(env.size());
    for (std::size_t i = 0; i != prox.size(); ++i) {
        prox[i] = static_cast<double>((i * 5) % 9) / 8.0;
    }

    compare("binary", compute::correlate_binary_b200(spec, env, ker),
            compute::correlate_binary_cpu(spec, env, ker), false);
    compare("proximity", compute::correlate_proximity_b200(spec, prox, ker),
            compute::correlate_proximity_cpu(spec, prox, ker), true);

    std::stop_source stop;
    stop.request_stop();
    runtime::OperationControl stopped;
    stopped.stop = stop.get_token();
    compare("stopped", compute::correlate_binary_b200(spec, env, ker, {}, stopped),
            compute::correlate_binary_cpu(spec, env, ker, {}, stopped), false);

    // A deadline that the control's own clock has already passed.
    std::uint64_t ticks_a = 100, ticks_b = 100;
    runtime::OperationControl late_a, late_b;
    late_a.deadline = late_b.deadline = runtime::Clock::time_point {} + std::chrono::milliseconds(5);
    late_a.now_fn = late_b.now_fn = fake_now;
    late_a.now_context = &ticks_a;
    late_b.now_context = &ticks_b;
    compare("deadline", compute::correlate_binary_b200(spec, env, ker, {}, late_a),
            compute::correlate_binary_cpu(spec, env, ker, {}, late_b), false);

    const std::vector<std::uint8_t> short_env(env.begin(), env.end() - 1);
    compare("invalid_field", compute::correlate_binary_b200(spec, short_env, ker),
            compute::correlate_binary_cpu(spec, short_env, ker), false);

    const compute::CorrelationSpec empty { { 7, 0, 4 }, { 3, 2, 2 }, {}, {} };
    compare("zero_extent", compute::correlate_binary_b200(empty, env, ker),
            compute::correlate_binary_cpu(empty, env, ker), false);

    const compute::CorrelationSpec far { { 7, 5, 4 }, { 3, 2, 2 }, { INT64_MIN + 1, 0, 0 }, { 5, 0, 0 } };
    compare("index_overflow", compute::correlate_binary_b200(far, env, ker),
            compute::correlate_binary_cpu(far, env, ker), false);

    // A stopped control with no working bytes at all: the metadata limit is
    // checked before the stop (correlation.cpp:255-275).
    compute::CorrelationLimits none;
    none.max_working_bytes = 0;
    compare("stopped_no_memory", compute::correlate_binary_b200(spec, env, ker, none, stopped),
            compute::correlate_binary_cpu(spec, env, ker, none, stopped), false);

    // The first translation fits, the last does not.
    const compute::CorrelationSpec edge { { 7, 5, 4 }, { 3, 2, 2 }, { INT64_MAX - 4, 0, 0 }, { 0, 0, 0 } };
    compare("last_translation", compute::correlate_binary_b200(edge, env, ker),
            compute::correlate_binary_cpu(edge, env, ker), false);

    std::vector<double> bad_prox = prox;
    bad_prox[3] = 1.5;
    compare("invalid_environment", compute::correlate_proximity_b200(spec, bad_prox, ker),
            compute::correlate_proximity_cpu(spec, bad_prox, ker), true);

    // Padded cells over the caller's limit, reached in the library.
    compute::CorrelationLimits few;
    few.max_padded_cells = 10;
    compare("padded_limit", compute::correlate_binary_b200(spec, env, ker, few),
            compute::correlate_binary_cpu(spec, env, ker, few), false);

    std::vector<std::uint8_t> bad_kernel = ker;
    bad_kernel[1] = 2;
    compare("invalid_kernel", compute::correlate_binary_b200(spec, env, bad_kernel),
            compute::correlate_binary_cpu(spec, env, bad_kernel), false);

    // The mask variant: the free mask over the legal box, from the reference's
    // counts by gap_fill.cpp:404-420's rule.
    const compute::TranslationBox box { { 5, -5, 14 }, { 5, 4, 3 } };
    std::vector<std::uint8_t> mask(5 * 4 * 3, 9);
    const auto masked = compute::correlate_binary_mask_b200(spec, env, ker, box, compute::MaskRule::zero_count, mask);
    const auto counts = compute::correlate_binary_cpu(spec, env, ker);
    const auto& r = std::get<compute::CorrelationResult>(counts);
    if (masked && masked->code == "CORRELATION_ALLOCATION") {
        report("mask", true, "no device: fails closed");
    }
    else if (masked) {
        report("mask", false, std::string(masked->code));
    }
    else {
        bool same = true;
        for (std::uint32_t z = 0; z != box.shape[2]; ++z) {
            for (std::uint32_t y = 0; y != box.shape[1]; ++y) {
                for (std::uint32_t x = 0; x != box.shape[0]; ++x) {
                    const std::int64_t o[3] = { box.first[0] + x - r.translation_first[0],
                                                box.first[1] + y - r.translation_first[1],
                                                box.first[2] + z - r.translation_first[2] };
                    bool inside = true;
                    for (int a = 0; a != 3; ++a) {
                        inside = inside && o[a] >= 0 && o[a] < static_cast<std::int64_t>(r.shape[a]);
                    }
                    const std::uint8_t want =
                        inside && std::round(r.values[o[0] + r.shape[0] * (o[1] + r.shape[1] * o[2])]) == 0;
                    same = same && mask[x + box.shape[0] * (y + box.shape[1] * z)] == want;
                }
            }
        }
        report("mask", same, "values");
    }
    std::printf("%s\n", failures ? "FAIL" : "PASS");
    return failures ? 1 : 0;
}
