// Batched complex FFT building blocks for sm_100a.
//
// Lines of a length L (16..512) are staged in shared memory and transformed
// by a Stockham autosort sequence, ping-ponging between two shared buffers:
// radix-4 stages (plus one radix-2 stage when log2 L is odd) for powers of
// two, stages of radix 4, 2, 3 and 5 for other 2^a 3^b 5^c lengths.
// Forward uses exp(-2 pi i jk / L), inverse exp(+2 pi i jk / L), both unscaled
// unless a scale is applied on store.  Twiddles come from a table of
// exp(-2 pi i m / L), m < L, computed on the host in FP64.
#pragma once

#include <algorithm>

#include "common.cuh"

namespace spk {

constexpr int kMaxFftLength = 512;

// Lengths the shared-memory transform takes: 2^a 3^b 5^c, at most
// kMaxFftLength.
SPK_HD bool fft_length_supported(std::uint64_t v)
{
    if (v == 0 || v > static_cast<std::uint64_t>(kMaxFftLength)) {
        return false;
    }
    while (v % 2 == 0) {
        v /= 2;
    }
    while (v % 3 == 0) {
        v /= 3;
    }
    while (v % 5 == 0) {
        v /= 5;
    }
    return v == 1;
}

// The smallest supported transform length >= n (0 if none).
SPK_HD std::uint32_t transform_length(std::uint64_t n)
{
    for (std::uint64_t L = n < 2 ? 2 : n; L <= static_cast<std::uint64_t>(kMaxFftLength); ++L) {
        if (fft_length_supported(L)) {
            return static_cast<std::uint32_t>(L);
        }
    }
    return 0;
}

// Mixed-radix Stockham transform of `lines` lines of a 2^a 3^b 5^c length
// L: stages of radix 4, then 2, 3 and 5.  A stage of radix p on the current
// length len = p m with running stride s computes, for q < m, r < s, k < p,
//   out[r + s (p q + k)] = W_len^(q k) * sum_j in[r + s (q + m j)] W_p^(j k),
// which leaves the result in natural order after the last stage.  Twiddles
// come from the length-L table: W_len^e = tw[e L / len].
template <typename C>
__device__ C* fft_lines_smem_mixed(C* a, C* b, const C* __restrict__ tw, int L, int lines, int pitch, bool inverse)
{
    using T = decltype(C::x);
    const int tid = threadIdx.x;
    const int nthreads = blockDim.x;
    const T sign = inverse ? T(1) : T(-1);
    const T h3 = sign * T(0.86602540378443864676372317075293618);
    const T c1 = T(0.30901699437494742410229341718281906), c2 = T(-0.80901699437494742410229341718281906);
    const T s1 = sign * T(0.95105651629515357211643933337938214), s2 = sign * T(0.58778525229247312916870595463907277);
    C* in = a;
    C* out = b;
    int len = L, s = 1;
    while (len > 1) {
        const int p = len % 4 == 0 ? 4 : len % 2 == 0 ? 2 : len % 3 == 0 ? 3 : 5;
        const int m = len / p;
        const int step = L / len;
        const int per_line = m * s;
        for (int e = tid; e < lines * per_line; e += nthreads) {
            const int jl = e / per_line;
            const int i = e - jl * per_line;
            const int r = i % s;
            const int q = i / s;
            const C* x = in + jl * pitch + r + s * q;
            C* y = out + jl * pitch + r + s * p * q;
            const int gap = s * m;
            // Output k, times W_len^(q k).
            const auto put = [&](int k, C value) {
                if (q && k) {
                    C w = tw[q * k * step];
                    if (inverse) {
                        w = cconj(w);
                    }
                    value = cmul(value, w);
                }
                y[k * s] = value;
            };
            if (p == 4) {
                const C v0 = x[0], v1 = x[gap], v2 = x[2 * gap], v3 = x[3 * gap];
                const C s02 = cadd(v0, v2), d02 = csub(v0, v2);
                const C s13 = cadd(v1, v3), d13 = csub(v1, v3);
                const C rot = cmake<C>(-sign * d13.y, sign * d13.x);  // sign * i * d13
                put(0, cadd(s02, s13));
                put(1, cadd(d02, rot));
                put(2, csub(s02, s13));
                put(3, csub(d02, rot));
            }
            else if (p == 2) {
                const C v0 = x[0], v1 = x[gap];
                put(0, cadd(v0, v1));
                put(1, csub(v0, v1));
            }
            else if (p == 3) {
                const C v0 = x[0], v1 = x[gap], v2 = x[2 * gap];
                const C sum = cadd(v1, v2), diff = csub(v1, v2);
                const C mid = cmake<C>(v0.x - T(0.5) * sum.x, v0.y - T(0.5) * sum.y);
                const C rot = cmake<C>(-h3 * diff.y, h3 * diff.x);  // i * h3 * diff
                put(0, cadd(v0, sum));
                put(1, cadd(mid, rot));
                put(2, csub(mid, rot));
            }
            else {
                const C v0 = x[0], v1 = x[gap], v2 = x[2 * gap], v3 = x[3 * gap], v4 = x[4 * gap];
                const C a1 = cadd(v1, v4), a2 = cadd(v2, v3);
                const C b1 = csub(v1, v4), b2 = csub(v2, v3);
                const C t1 = cmake<C>(v0.x + c1 * a1.x + c2 * a2.x, v0.y + c1 * a1.y + c2 * a2.y);
                const C t2 = cmake<C>(v0.x + c2 * a1.x + c1 * a2.x, v0.y + c2 * a1.y + c1 * a2.y);
                // With the sign folded into the sines: u1 = i (s1 b1 + s2 b2), u2 = i (s2 b1 - s1 b2).
                const C w1 = cmake<C>(s1 * b1.x + s2 * b2.x, s1 * b1.y + s2 * b2.y);
                const C w2 = cmake<C>(s2 * b1.x - s1 * b2.x, s2 * b1.y - s1 * b2.y);
                const C u1 = cmake<C>(-w1.y, w1.x), u2 = cmake<C>(-w2.y, w2.x);
                put(0, cadd(v0, cadd(a1, a2)));
                put(1, cadd(t1, u1));
                put(2, cadd(t2, u2));
                put(3, csub(t2, u2));
                put(4, csub(t1, u1));
            }
        }
        __syncthreads();
        C* t = in;
        in = out;
        out = t;
        s *= p;
        len = m;
    }
    return in;
}

// Runs the whole transform on `lines` lines held at `a + j * pitch`.
// Returns the buffer (a or b) that holds the result.  All threads of the
// block must call it; it synchronises internally.  Power-of-two lengths take
// the radix-4 path below, other 2^a 3^b 5^c lengths the mixed-radix one.
template <typename C>
__device__ C* fft_lines_smem(C* a, C* b, const C* __restrict__ tw, int L, int lines, int pitch, bool inverse)
{
    if (!is_pow2(static_cast<std::uint64_t>(L))) {
        return fft_lines_smem_mixed(a, b, tw, L, lines, pitch, inverse);
    }
    const int tid = threadIdx.x;
    const int nthreads = blockDim.x;
    const int log2L = ilog2(static_cast<unsigned>(L));
    C* in = a;
    C* out = b;
    int ns = 1;
    if (log2L & 1) {
        // Radix-2 first stage (ns = 1, no twiddles).
        const int half = L >> 1;
        for (int e = tid; e < lines * half; e += nthreads) {
            const int j = e / half;
            const int i = e - j * half;
            const C a0 = in[j * pitch + i];
            const C a1 = in[j * pitch + i + half];
            out[j * pitch + 2 * i] = cadd(a0, a1);
            out[j * pitch + 2 * i + 1] = csub(a0, a1);
        }
        __syncthreads();
        C* t = in;
        in = out;
        out = t;
        ns = 2;
    }
    const int quarter = L >> 2;
    while (ns < L) {
        const int step = L / (4 * ns);  // table index per unit of r*k
        for (int e = tid; e < lines * quarter; e += nthreads) {
            const int j = e / quarter;
            const int i = e - j * quarter;
            const int k = i & (ns - 1);
            C v0 = in[j * pitch + i];
            C v1 = in[j * pitch + i + quarter];
            C v2 = in[j * pitch + i + 2 * quarter];
            C v3 = in[j * pitch + i + 3 * quarter];
            if (ns > 1) {
                C w1 = tw[k * step];
                C w2 = tw[2 * k * step];
                C w3 = tw[3 * k * step];
                if (inverse) {
                    w1 = cconj(w1);
                    w2 = cconj(w2);
                    w3 = cconj(w3);
                }
                v1 = cmul(v1, w1);
                v2 = cmul(v2, w2);
                v3 = cmul(v3, w3);
            }
            const C t0 = cadd(v0, v2);
            const C t1 = csub(v0, v2);
            const C t2 = cadd(v1, v3);
            const C d = csub(v1, v3);
            // forward: -i * d ; inverse: +i * d
            const C t3 = inverse ? cmake<C>(-d.y, d.x) : cmake<C>(d.y, -d.x);
            const int base = j * pitch + (i - k) * 4 + k;
            out[base] = cadd(t0, t2);
            out[base + ns] = cadd(t1, t3);
            out[base + 2 * ns] = csub(t0, t2);
            out[base + 3 * ns] = csub(t1, t3);
        }
        __syncthreads();
        C* t = in;
        in = out;
        out = t;
        ns *= 4;
    }
    return in;
}

// One pass of 1D transforms along `axis` of a dense [z][y][x] complex array.
// Each block stages `group` lines (consecutive in the contiguous direction for
// axes 1 and 2, consecutive lines for axis 0) so global accesses coalesce.
template <typename T>
__global__ void fft_axis_kernel(cplx_t<T>* __restrict__ data, int Lx, int Ly, int Lz, int axis, int inverse,
                                T scale, const cplx_t<T>* __restrict__ twiddles, int group, int store_limit)
{
    using C = cplx_t<T>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int L = axis == 0 ? Lx : axis == 1 ? Ly : Lz;
    const int pitch = L + 1;
    C* tw = reinterpret_cast<C*>(smem_raw);
    C* buf_a = tw + L;
    C* buf_b = buf_a + group * pitch;
    for (int m = threadIdx.x; m < L; m += blockDim.x) {
        tw[m] = twiddles[m];
    }
    const long long plane = static_cast<long long>(Lx) * Ly;
    const long long line0 = static_cast<long long>(blockIdx.x) * group;
    long long base;
    long long stride;
    if (axis == 0) {
        base = line0 * Lx;
        stride = 1;
    }
    else if (axis == 1) {
        const long long x0 = line0 % Lx;
        const long long z = line0 / Lx;
        base = x0 + z * plane;
        stride = Lx;
    }
    else {
        base = line0;
        stride = plane;
    }
    if (axis == 0) {
        for (int e = threadIdx.x; e < group * L; e += blockDim.x) {
            const int j = e / L;
            const int q = e - j * L;
            buf_a[j * pitch + q] = data[base + e];
        }
    }
    else {
        for (int e = threadIdx.x; e < group * L; e += blockDim.x) {
            const int j = e % group;
            const int q = e / group;
            buf_a[j * pitch + q] = data[base + j + q * stride];
        }
    }
    __syncthreads();
    C* result = fft_lines_smem(buf_a, buf_b, tw, L, group, pitch, inverse != 0);
    if (axis == 0) {
        for (int e = threadIdx.x; e < group * L; e += blockDim.x) {
            const int j = e / L;
            const int q = e - j * L;
            data[base + e] = cscale(result[j * pitch + q], scale);
        }
    }
    else {
        for (int e = threadIdx.x; e < group * store_limit; e += blockDim.x) {
            const int j = e % group;
            const int q = e / group;
            data[base + j + q * stride] = cscale(result[j * pitch + q], scale);
        }
    }
}

// Host-side launcher for one axis pass; returns the CUDA launch status.
// store_limit (axes 1 and 2 only): positions q >= store_limit are not written back.
template <typename T>
cudaError_t fft_axis(cplx_t<T>* data, int Lx, int Ly, int Lz, int axis, bool inverse, T scale,
                     const cplx_t<T>* twiddles, cudaStream_t stream, int store_limit = -1)
{
    using C = cplx_t<T>;
    const int L = axis == 0 ? Lx : axis == 1 ? Ly : Lz;
    const long long lines = static_cast<long long>(Lx) * Ly * Lz / L;
    int group = sizeof(T) == 4 ? 16 : 8;
    if (axis == 1) {
        // A block's lines are consecutive x at one z: the group divides Lx.
        group = std::min(group, Lx);
        while (Lx % group) {
            --group;
        }
    }
    else {
        while (group > 1 && lines % group) {
            group >>= 1;
        }
    }
    const size_t smem = sizeof(C) * (L + 2 * static_cast<size_t>(group) * (L + 1));
    static std::once_flag attribute[64];
    once_per_device(attribute, [] {
        cudaFuncSetAttribute(fft_axis_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    });
    const int threads = 256;
    const long long blocks = lines / group;
    fft_axis_kernel<T><<<static_cast<unsigned>(blocks), threads, smem, stream>>>(data, Lx, Ly, Lz, axis,
                                                                                  inverse ? 1 : 0, scale, twiddles,
                                                                                  group, store_limit < 0 ? L : store_limit);
    return cudaGetLastError();
}

}  // namespace spk
