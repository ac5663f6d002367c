// Batched complex FFT building blocks for sm_100a.
//
// Lines of a power-of-two length L (64..512) are staged in shared memory and
// transformed by a Stockham autosort sequence of radix-4 stages (plus one
// radix-2 stage when log2 L is odd), ping-ponging between two shared buffers.
// Forward uses exp(-2 pi i jk / L), inverse exp(+2 pi i jk / L), both unscaled
// unless a scale is applied on store.  Twiddles come from a table of
// exp(-2 pi i m / L), m < L, computed on the host in FP64.
#pragma once

#include "common.cuh"

namespace spk {

constexpr int kMaxFftLength = 512;

// Runs the whole transform on `lines` lines held at `a + j * pitch`.
// Returns the buffer (a or b) that holds the result.  All threads of the
// block must call it; it synchronises internally.
template <typename C>
__device__ C* fft_lines_smem(C* a, C* b, const C* __restrict__ tw, int L, int lines, int pitch, bool inverse)
{
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
    if (axis == 1 && group > Lx) {
        group = Lx;
    }
    while (group > 1 && lines % group) {
        group >>= 1;
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
