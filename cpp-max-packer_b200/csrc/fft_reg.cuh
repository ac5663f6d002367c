// Register-resident 256-point complex FFT (four-step, 256 = 16 x 16).
//
// A line is held by 16 threads, 16 values each.  With n = 16 n1 + n2 and
// k = k1 + 16 k2:
//   X[k1 + 16 k2] = sum_n2 w16^(n2 k2) * [ w256^(n2 k1) * sum_n1 x[16 n1 + n2] w16^(n1 k1) ]
// Thread n2 holds x[16 n1 + n2] (n1 = 0..15), does a 16-point DFT in
// registers, applies w256^(n2 k1), and exchanges through shared memory so
// thread k1 holds the 16 values over n2; a second 16-point DFT leaves thread
// t holding X[t + 16 k2] (k2 = 0..15).  That output distribution is exactly the
// input distribution of the next transform (n2 = t, n1 = k2), so a forward
// transform, a pointwise product and an inverse transform chain with one
// shared-memory exchange each and no other synchronisation.
// Forward uses w = exp(-2 pi i / N); the inverse conjugates every twiddle.
#pragma once

#include "common.cuh"

namespace spk {

constexpr int kRegLine = 273;  // shared complex slots per line (16 x 17 + 1: bank spread)
constexpr int kTwRow = 18;     // complex slots per twiddle row (16 + 2: bank spread of 16-byte reads)

// Shared twiddles of the register FFT: for each lane-in-line t, the row
// w256^(t k) for k < 16 (the 16-point DFTs' own roots are immediates).  A
// thread reads its row two roots at a time (16-byte loads); with rows 144
// bytes apart, the eight threads of a quarter warp that hold different t
// read distinct banks.
struct RegTwiddles {
    __align__(16) float2 row[16 * kTwRow];
};

// Fills `tw` from the 256 roots in global memory; a block of 256 threads
// calls it, then synchronises before the first transform.
__device__ __forceinline__ void load_twiddles(RegTwiddles& tw, const float2* __restrict__ twiddles)
{
    const int i = threadIdx.x, t = i >> 4, k = i & 15;
    tw.row[t * kTwRow + k] = twiddles[(t * k) & 255];
}

template <bool INV>
__device__ __forceinline__ void dft4(float2& a, float2& b, float2& c, float2& d)
{
    const float2 t0 = make_float2(a.x + c.x, a.y + c.y);
    const float2 t1 = make_float2(a.x - c.x, a.y - c.y);
    const float2 t2 = make_float2(b.x + d.x, b.y + d.y);
    const float2 u = make_float2(b.x - d.x, b.y - d.y);
    // forward: -i * u ; inverse: +i * u
    const float2 t3 = INV ? make_float2(-u.y, u.x) : make_float2(u.y, -u.x);
    a = make_float2(t0.x + t2.x, t0.y + t2.y);
    c = make_float2(t0.x - t2.x, t0.y - t2.y);
    b = make_float2(t1.x + t3.x, t1.y + t3.y);
    d = make_float2(t1.x - t3.x, t1.y - t3.y);
}

__device__ __forceinline__ float2 cmulf(float2 a, float2 b)
{
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// 16-point DFT in registers: x[n] natural in, X[k] natural out.
template <bool INV>
__device__ __forceinline__ void dft16(float2 (&x)[16])
{
    // w16^m for m = 0..9 (only b*c <= 9 occurs), forward sign.
    constexpr float c1 = 0.92387953251128675613f, s1 = 0.38268343236508977173f;
    constexpr float r2 = 0.70710678118654752440f;
#pragma unroll
    for (int b = 0; b < 4; ++b) {
        dft4<INV>(x[b], x[4 + b], x[8 + b], x[12 + b]);  // Y[b][c] now at x[4c + b]
    }
    // twiddle Y[b][c] *= w16^(b c)
    const float2 w[10] = { make_float2(1.f, 0.f),  make_float2(c1, -s1),   make_float2(r2, -r2),
                           make_float2(s1, -c1),   make_float2(0.f, -1.f), make_float2(-s1, -c1),
                           make_float2(-r2, -r2),  make_float2(-c1, -s1),  make_float2(-1.f, 0.f),
                           make_float2(-c1, s1) };
#pragma unroll
    for (int c = 1; c < 4; ++c) {
#pragma unroll
        for (int b = 1; b < 4; ++b) {
            if (b * c == 4) {
                // w16^4 = -i (forward) or +i (inverse): a swap and a sign.
                const float2 u = x[4 * c + b];
                x[4 * c + b] = INV ? make_float2(-u.y, u.x) : make_float2(u.y, -u.x);
                continue;
            }
            float2 tw = w[b * c];
            if (INV) {
                tw.y = -tw.y;
            }
            x[4 * c + b] = cmulf(x[4 * c + b], tw);
        }
    }
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        dft4<INV>(x[4 * c], x[4 * c + 1], x[4 * c + 2], x[4 * c + 3]);  // X[c + 4d] at x[4c + d]
    }
    // back to natural order: X[k] -> slot k
    float2 y[16];
#pragma unroll
    for (int k = 0; k < 16; ++k) {
        y[k] = x[4 * (k & 3) + (k >> 2)];
    }
#pragma unroll
    for (int k = 0; k < 16; ++k) {
        x[k] = y[k];
    }
}

// How fft256 orders its shared-memory exchange:
//   kBlockSync - the line's threads may lie in different warps; the block
//                synchronises before the exchange (earlier readers of `line`
//                are done) and between its writes and reads;
//   kFirstUse  - as kBlockSync, for the first use of `line` in the kernel
//                after a block barrier: only the second synchronisation;
//   kHalfWarp  - the line's 16 threads are one half of a warp (thread t of
//                line j is threadIdx 16 j + t): __syncwarp orders the
//                exchange, and only the calling warps need take part.
enum FftSync { kBlockSync = 0, kFirstUse = 1, kHalfWarp = 2 };

// v[k1] *= w256^(t k1) (conjugated for the inverse), k1 = 1..15, from the
// thread's twiddle row.
template <bool INV>
__device__ __forceinline__ void twiddle_row(float2 (&v)[16], const RegTwiddles& tw, int t)
{
    const float4* row = reinterpret_cast<const float4*>(tw.row + t * kTwRow);
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const float4 q = row[i];
        if (i > 0) {
            v[2 * i] = cmulf(v[2 * i], make_float2(q.x, INV ? -q.y : q.y));
        }
        v[2 * i + 1] = cmulf(v[2 * i + 1], make_float2(q.z, INV ? -q.w : q.w));
    }
}

// Four-step 256-point transform of the line held by the 16 threads with
// lane-in-line index t.  `line` points at this line's kRegLine shared slots.
// With kBlockSync or kFirstUse every thread of the block must call it; with
// kHalfWarp every thread of the warp.
template <bool INV, int SYNC = kBlockSync>
__device__ __forceinline__ void fft256(float2 (&v)[16], float2* line, int t, const RegTwiddles& tw)
{
    dft16<INV>(v);  // thread t: Y[t][k1] = v[k1]
    twiddle_row<INV>(v, tw, t);
    if (SYNC == kBlockSync) {
        __syncthreads();  // the previous reader of `line` is done
    }
    else if (SYNC == kHalfWarp) {
        __syncwarp();
    }
#pragma unroll
    for (int k1 = 0; k1 < 16; ++k1) {
        line[t * 17 + k1] = v[k1];
    }
    if (SYNC == kHalfWarp) {
        __syncwarp();
    }
    else {
        __syncthreads();
    }
#pragma unroll
    for (int n2 = 0; n2 < 16; ++n2) {
        v[n2] = line[n2 * 17 + t];
    }
    dft16<INV>(v);  // thread t: X[t + 16 k2] = v[k2]
}

// The forward transform of a line whose inputs are zero beyond index 31:
// thread t holds x[t] in a and x[16 + t] in b.  The first 16-point DFT over
// n1 then has two non-zero terms, Y[k1] = a + b w16^k1; the rest is the
// four-step transform above.  Output distribution as fft256.
__device__ __forceinline__ void fft256_first32(float2 a, float2 b, float2 (&v)[16], float2* line, int t,
                                               const RegTwiddles& tw)
{
    // w16^k1 = w256^(16 k1) as immediates (the table's values: FP32 roundings
    // of cos and sin at multiples of pi/8, exact at the quarter points).
    constexpr float c1 = 0.92387953251128675613f, s1 = 0.38268343236508977173f;
    constexpr float r2 = 0.70710678118654752440f;
    const float2 w16[16] = { make_float2(1.f, 0.f),  make_float2(c1, -s1),  make_float2(r2, -r2),
                             make_float2(s1, -c1),   make_float2(0.f, -1.f), make_float2(-s1, -c1),
                             make_float2(-r2, -r2),  make_float2(-c1, -s1), make_float2(-1.f, 0.f),
                             make_float2(-c1, s1),   make_float2(-r2, r2),  make_float2(-s1, c1),
                             make_float2(0.f, 1.f),  make_float2(s1, c1),   make_float2(r2, r2),
                             make_float2(c1, s1) };
#pragma unroll
    for (int k1 = 0; k1 < 16; ++k1) {
        const float2 w = w16[k1];
        v[k1] = make_float2(a.x + b.x * w.x - b.y * w.y, a.y + b.x * w.y + b.y * w.x);
    }
    twiddle_row<false>(v, tw, t);
    __syncthreads();  // the previous reader of `line` is done
#pragma unroll
    for (int k1 = 0; k1 < 16; ++k1) {
        line[t * 17 + k1] = v[k1];
    }
    __syncthreads();
#pragma unroll
    for (int n2 = 0; n2 < 16; ++n2) {
        v[n2] = line[n2 * 17 + t];
    }
    dft16<false>(v);  // thread t: X[t + 16 k2] = v[k2]
}

}  // namespace spk
