// Exact fixed-point accumulator for sums of non-negative binary64 values.
//
// The sum is held as limbs of 32 bits (each in an int64 for carry-free adds)
// covering bit positions [kLowBit, kLowBit + 32 * kLimbs).  Every binary64
// value >= 2^-652 is placed exactly; the final conversion rounds to nearest,
// ties to even, so the result is the correctly rounded exact sum - the same
// double the oracle's Shewchuk/fsum summation returns, independent of order.
#pragma once

#include <cstdint>
#include <cstring>

#include "common.cuh"

namespace spk {

constexpr int kSuperLimbs = 23;
constexpr int kSuperLowBit = -704;  // multiple of 32

struct SuperAcc {
    long long limb[kSuperLimbs];
};

SPK_HD void super_clear(SuperAcc& a)
{
    for (int i = 0; i < kSuperLimbs; ++i) {
        a.limb[i] = 0;
    }
}

// Adds v >= 0.  Returns false if v is below the represented range (not
// reachable for proximity values on grids up to 512 cells per axis).
SPK_HD bool super_add(SuperAcc& a, double v)
{
    if (!(v > 0.0)) {
        return v == 0.0;
    }
    unsigned long long bits;
#ifdef __CUDA_ARCH__
    bits = static_cast<unsigned long long>(__double_as_longlong(v));
#else
    std::memcpy(&bits, &v, 8);
#endif
    const int field = static_cast<int>(bits >> 52);
    unsigned long long mant = bits & ((1ULL << 52) - 1);
    int e;
    if (field == 0) {
        e = -1074;
    }
    else {
        mant |= 1ULL << 52;
        e = field - 1075;
    }
    const int shift = e - kSuperLowBit;
    if (shift < 0) {
        return false;
    }
    const int li = shift >> 5;
    const int off = shift & 31;
    const unsigned long long lo = mant << off;              // low 64 bits of mant << off
    const unsigned long long hi = off ? mant >> (64 - off) : 0ULL;
    a.limb[li] += static_cast<long long>(lo & 0xffffffffULL);
    if (li + 1 < kSuperLimbs) {
        a.limb[li + 1] += static_cast<long long>(lo >> 32);
    }
    if (li + 2 < kSuperLimbs) {
        a.limb[li + 2] += static_cast<long long>(hi);
    }
    return true;
}

SPK_HD void super_merge(SuperAcc& a, const SuperAcc& b)
{
    for (int i = 0; i < kSuperLimbs; ++i) {
        a.limb[i] += b.limb[i];
    }
}

// Correctly rounded (nearest, ties to even) binary64 value of the sum.
SPK_HD double super_round(const SuperAcc& in)
{
    unsigned int w[kSuperLimbs];
    long long carry = 0;
    for (int i = 0; i < kSuperLimbs; ++i) {
        const long long v = in.limb[i] + carry;
        w[i] = static_cast<unsigned int>(v & 0xffffffffLL);
        carry = v >> 32;  // limbs are non-negative: arithmetic shift is exact
    }
    int h = kSuperLimbs - 1;
    while (h >= 0 && w[h] == 0) {
        --h;
    }
    if (h < 0) {
        return 0.0;
    }
    int lead = 31;
    while (!((w[h] >> lead) & 1U)) {
        --lead;
    }
    const int msb = 32 * h + lead;  // bit index relative to kSuperLowBit
    const auto bit = [&](int pos) -> unsigned int {
        if (pos < 0) {
            return 0U;
        }
        return (w[pos >> 5] >> (pos & 31)) & 1U;
    };
    unsigned long long m = 0;
    for (int k = 0; k < 53; ++k) {
        m = (m << 1) | bit(msb - k);
    }
    const unsigned int round = bit(msb - 53);
    bool sticky = false;
    const int top_sticky = msb - 54;  // highest position folded into the sticky bit
    if (top_sticky >= 0) {
        const int li = top_sticky >> 5;
        const int off = top_sticky & 31;
        const unsigned int mask = off == 31 ? 0xffffffffU : ((1U << (off + 1)) - 1U);
        sticky = (w[li] & mask) != 0;
        for (int i = li - 1; i >= 0 && !sticky; --i) {
            sticky = w[i] != 0;
        }
    }
    int exponent = msb + kSuperLowBit;  // value = 1.m * 2^exponent
    if (round && (sticky || (m & 1ULL))) {
        ++m;
        if (m == (1ULL << 53)) {
            m >>= 1;
            ++exponent;
        }
    }
    // exponent stays within the normal range for every sum this path forms.
    const unsigned long long out =
        (static_cast<unsigned long long>(exponent + 1023) << 52) | (m & ((1ULL << 52) - 1));
#ifdef __CUDA_ARCH__
    return __longlong_as_double(static_cast<long long>(out));
#else
    double d;
    std::memcpy(&d, &out, 8);
    return d;
#endif
}

}  // namespace spk
