// Spectral page pipeline kernels and host orchestration (see pipeline.hpp).
//
// Per environment (once per layout): Z = B + iP on an L^3 grid (B the u8
// occupancy, P the FP32 proximity) and its forward FFT, scaled by 1/N.
// Per oriented kernel (once per run): the kernel transformed along x and y,
// kept for its K2 nonzero z-planes ("partial spectrum").
// Per page request:
//   pass A  - per (kx, ky) column: finish the kernel FFT along z, multiply by
//             the conjugate into the environment spectrum, inverse FFT along
//             z, keep the legal z outputs;
//   pass B1 - inverse FFT along y, keep the legal y rows;
//   pass B2 - inverse FFT along x, then the fused epilogue: real part = overlap
//             count, imaginary part = proximity sum; threshold |b| < 0.5,
//             approximate score, per-warp sorted top-32 of 64-bit keys
//             (orderable score, legal linear index z-major) and a per-request
//             pruning bound;
//   merge   - per request, sort the surviving keys;
//   exact   - per selected key, exact u8 overlap recount and the exact,
//             correctly rounded FP64 proximity sum (superaccumulator).
// The host then scores exactly, orders by (score, z, y, x), applies the
// cursor and certifies that no excluded candidate could enter the page; an
// uncertified page is recomputed in threshold mode (every candidate whose
// approximate score is within the error bound of the page's last entry).
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <tuple>
#include <vector>

#include "context.hpp"
#include "edt.cuh"
#include "fft.cuh"
#include "fft_reg.cuh"
#include "pipeline.hpp"
#include "superacc.cuh"

namespace spk {

namespace cg = cooperative_groups;

namespace {

constexpr std::int32_t kInf = INT32_MAX;
constexpr unsigned kFull = 0xffffffffu;
constexpr int kB2Rows = 8;
constexpr int kColumnGroup = 16;

int launch_blocks(long long n, int threads)
{
    const long long want = (n + threads - 1) / threads;
    return static_cast<int>(std::min<long long>(std::max<long long>(want, 1), 148LL * 32));
}

__global__ void env_pack_kernel(float2* __restrict__ z, int L0, int L1, int L2, int E0, int E1, int E2,
                                const std::uint8_t* __restrict__ occ, const std::int32_t* __restrict__ d2,
                                const double* __restrict__ table, double* __restrict__ norm_partial)
{
    __shared__ double s[256];
    const long long n = static_cast<long long>(L0) * L1 * L2;
    double acc = 0;
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        const int x = static_cast<int>(i % L0);
        const long long r = i / L0;
        const int y = static_cast<int>(r % L1);
        const int w = static_cast<int>(r / L1);
        float b = 0.f, p = 0.f;
        if (x < E0 && y < E1 && w < E2) {
            const long long e = x + static_cast<long long>(E0) * (y + static_cast<long long>(E1) * w);
            b = occ[e] ? 1.f : 0.f;
            const std::int32_t v = d2[e];
            p = v == kInf ? 0.f : static_cast<float>(table[v]);
        }
        acc += static_cast<double>(b) * b + static_cast<double>(p) * p;
        z[i] = make_float2(b, p);
    }
    s[threadIdx.x] = acc;
    __syncthreads();
    for (int h = blockDim.x / 2; h > 0; h >>= 1) {
        if (threadIdx.x < h) {
            s[threadIdx.x] += s[threadIdx.x + h];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        norm_partial[blockIdx.x] = s[0];
    }
}

__global__ void kernel_pack_kernel(float2* __restrict__ kp, int L0, int L1, int K0, int K1, int K2,
                                   const std::uint8_t* __restrict__ cells)
{
    const long long n = static_cast<long long>(L0) * L1 * K2;
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        const int x = static_cast<int>(i % L0);
        const long long r = i / L0;
        const int y = static_cast<int>(r % L1);
        const int w = static_cast<int>(r / L1);
        float v = 0.f;
        if (x < K0 && y < K1) {
            v = cells[x + static_cast<long long>(K0) * (y + static_cast<long long>(K1) * w)] ? 1.f : 0.f;
        }
        kp[i] = make_float2(v, 0.f);
    }
}

// Pass A: one block per group of 16 consecutive kx at one ky.
__global__ void pass_a_kernel(const float2* __restrict__ spectrum, const float2* __restrict__ partial,
                              float2* __restrict__ inter, int L0, int L1, int L2, int K2, int legal_z,
                              const float2* __restrict__ twiddles)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int pitch = L2 + 1;
    float2* tw = reinterpret_cast<float2*>(smem_raw);
    float2* a = tw + L2;
    float2* b = a + kColumnGroup * pitch;
    float2* s = b + kColumnGroup * pitch;
    for (int m = threadIdx.x; m < L2; m += blockDim.x) {
        tw[m] = twiddles[m];
    }
    const int groups_x = L0 / kColumnGroup;
    const int ky = blockIdx.x / groups_x;
    const int kx0 = (blockIdx.x % groups_x) * kColumnGroup;
    const long long plane = static_cast<long long>(L0) * L1;
    const long long column = kx0 + static_cast<long long>(L0) * ky;
    for (int e = threadIdx.x; e < kColumnGroup * L2; e += blockDim.x) {
        const int j = e % kColumnGroup;
        const int q = e / kColumnGroup;
        const long long at = column + j + plane * q;
        s[j * L2 + q] = spectrum[at];
        a[j * pitch + q] = q < K2 ? partial[at] : make_float2(0.f, 0.f);
    }
    __syncthreads();
    float2* k = fft_lines_smem(a, b, tw, L2, kColumnGroup, pitch, false);
    float2* o = k == a ? b : a;
    for (int e = threadIdx.x; e < kColumnGroup * L2; e += blockDim.x) {
        const int j = e / L2;
        const int q = e - j * L2;
        o[j * pitch + q] = cmulconj(s[j * L2 + q], k[j * pitch + q]);
    }
    __syncthreads();
    float2* w = fft_lines_smem(o, k, tw, L2, kColumnGroup, pitch, true);
    for (int e = threadIdx.x; e < kColumnGroup * legal_z; e += blockDim.x) {
        const int j = e % kColumnGroup;
        const int q = e / kColumnGroup;
        inter[column + j + plane * q] = w[j * pitch + q];
    }
}

__device__ __forceinline__ unsigned long long make_key(double score, unsigned int index)
{
    const float f = __double2float_rd(score);
    const unsigned int u = __float_as_uint(f);
    const unsigned int k = (u & 0x80000000u) ? ~u : (u | 0x80000000u);
    return (static_cast<unsigned long long>(k) << 32) | index;
}

// The FP32 score in a key's high half (the inverse of make_key's mapping).
__device__ __forceinline__ float key_score_f32(unsigned long long key)
{
    const unsigned int k = static_cast<unsigned int>(key >> 32);
    return __uint_as_float((k & 0x80000000u) ? (k & 0x7fffffffu) : ~k);
}

// Prefilter of the epilogue, per legal z: the proximity sum below which a
// cell's key is certainly above `bound`, so the cell needs no FP64 score.
// The score t65z - 0.35 p / occ falls as p grows; a key exceeds the bound
// when its score, rounded down to FP32, exceeds the bound's FP32 score S,
// which holds once the score reaches the next float above S.  The returned
// value lies below the exact crossing by a margin far wider than the FP64
// rounding of the score, and is itself rounded down to FP32, so every p
// below it gives a key above the bound.  No bound yet: -inf (no cell skips).
__device__ __forceinline__ float skip_below(unsigned long long bound, double t65z, double inv_occ)
{
    if (bound == kEmptyKey) {
        return -INFINITY;
    }
    const float s = key_score_f32(bound);
    if (!isfinite(s)) {
        return -INFINITY;
    }
    const double next = static_cast<double>(nextafterf(s, INFINITY));
    const double scale = 0.35 * inv_occ;
    const double crossing = (t65z - next) / scale;
    const double margin = 1e-9 * (fabs(t65z) + fabs(next)) / scale;
    return __double2float_rd(crossing - margin);
}

__device__ __forceinline__ unsigned long long warp_sort32(unsigned long long v, int lane)
{
    for (int k = 2; k <= 32; k <<= 1) {
        for (int j = k >> 1; j > 0; j >>= 1) {
            const unsigned long long o = __shfl_xor_sync(kFull, v, j);
            const bool up = (lane & k) == 0;
            const bool lower = (lane & j) == 0;
            v = (lower == up) ? (v < o ? v : o) : (v > o ? v : o);
        }
    }
    return v;
}

// Sorts a bitonic 32-sequence held one key per lane (ascending).
__device__ __forceinline__ unsigned long long warp_bitonic_finish(unsigned long long m, int lane)
{
    for (int j = 16; j > 0; j >>= 1) {
        const unsigned long long o = __shfl_xor_sync(kFull, m, j);
        m = ((lane & j) == 0) ? (m < o ? m : o) : (m > o ? m : o);
    }
    return m;
}

// Keeps the 64 smallest keys seen by the warp: lo holds ranks 0..31 and hi
// ranks 32..63, each sorted ascending across lanes.
__device__ __forceinline__ void warp_insert(unsigned long long& lo, unsigned long long& hi, unsigned long long key,
                                            int lane)
{
    const unsigned long long worst = __shfl_sync(kFull, hi, 31);
    if (!__any_sync(kFull, key < worst)) {
        return;
    }
    key = warp_sort32(key, lane);
    // split lo | key into the 32 smallest (new lo) and the 32 largest (spill)
    unsigned long long rev = __shfl_sync(kFull, key, 31 - lane);
    const unsigned long long small = lo < rev ? lo : rev;
    const unsigned long long large = lo < rev ? rev : lo;
    lo = warp_bitonic_finish(small, lane);
    const unsigned long long spill = warp_bitonic_finish(large, lane);
    // keep the 32 smallest of hi | spill
    rev = __shfl_sync(kFull, spill, 31 - lane);
    hi = warp_bitonic_finish(hi < rev ? hi : rev, lane);
}

// Pass B2: inverse FFT along x for 8 legal rows, then the fused epilogue.
// A candidate is a legal translation whose rounded overlap count is `target`
// (0 for ordinary pages).  mode 0: warp top-32 lists + pruning bound in *tau;
// mode 1: append every candidate whose approximate score is <= threshold and
// count every candidate past the cursor floor in *tau; mode 2: histogram of
// the rounded overlap counts of every legal translation into `keys` read as
// `cap` u32 bins (the last bin holds every larger count).
__global__ void pass_b2_kernel(const float2* __restrict__ inter, int L0, int L1, int legal_x, int legal_y,
                               int legal_z, const float2* __restrict__ twiddles, const double* __restrict__ t65,
                               double inv_occ, int mode, float target, double threshold, double cursor_floor,
                               unsigned long long* __restrict__ keys, unsigned int* __restrict__ count,
                               unsigned int cap, unsigned long long* __restrict__ tau,
                               unsigned long long* __restrict__ resid)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int pitch = L0 + 1;
    float2* tw = reinterpret_cast<float2*>(smem_raw);
    float2* a = tw + L0;
    float2* b = a + kB2Rows * pitch;
    for (int m = threadIdx.x; m < L0; m += blockDim.x) {
        tw[m] = twiddles[m];
    }
    const long long rows = static_cast<long long>(legal_y) * legal_z;
    const long long row0 = static_cast<long long>(blockIdx.x) * kB2Rows;
    for (int e = threadIdx.x; e < kB2Rows * L0; e += blockDim.x) {
        const int j = e / L0;
        const int q = e - j * L0;
        const long long row = row0 + j;
        float2 v = make_float2(0.f, 0.f);
        if (row < rows) {
            const long long y = row % legal_y;
            const long long zz = row / legal_y;
            v = inter[q + static_cast<long long>(L0) * (y + static_cast<long long>(L1) * zz)];
        }
        a[j * pitch + q] = v;
    }
    __syncthreads();
    const float2* res = fft_lines_smem(a, b, tw, L0, kB2Rows, pitch, true);
    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    const long long row = row0 + warp;
    if (warp >= kB2Rows || row >= rows) {
        return;
    }
    const int y = static_cast<int>(row % legal_y);
    const int zz = static_cast<int>(row / legal_y);
    const double t65z = t65[zz];
    const float skip = mode == 0 ? skip_below(*reinterpret_cast<volatile unsigned long long*>(tau), t65z, inv_occ)
                                 : -INFINITY;
    unsigned long long list_lo = kEmptyKey, list_hi = kEmptyKey;
    float residual = 0.f;
    const unsigned int row_index = static_cast<unsigned int>(legal_x) * (y + static_cast<unsigned int>(legal_y) * zz);
    for (int c = 0; c < legal_x; c += 32) {
        const int x = c + lane;
        unsigned long long key = kEmptyKey;
        bool take = false;
        if (x < legal_x) {
            const float2 v = res[warp * pitch + x];
            residual = fmaxf(residual, fabsf(v.x - rintf(v.x)));
            if (mode == 2) {
                const float c = rintf(v.x);
                const unsigned int bin = c <= 0.f ? 0u : c >= static_cast<float>(cap - 1) ? cap - 1
                                                                                           : static_cast<unsigned int>(c);
                atomicAdd(reinterpret_cast<unsigned int*>(keys) + bin, 1u);
            }
            else if (fabsf(v.x - target) < 0.5f && !(v.y < skip)) {
                const double score = t65z - 0.35 * (static_cast<double>(v.y) * inv_occ);
                if (score >= cursor_floor) {
                    key = make_key(score, row_index + x);
                    take = mode == 1 && score <= threshold;
                    if (mode == 1) {
                        atomicAdd(tau, 1ULL);
                    }
                }
            }
        }
        if (mode == 0) {
            warp_insert(list_lo, list_hi, key, lane);
        }
        else {
            const unsigned mask = __ballot_sync(kFull, take);
            if (mask) {
                unsigned int base = 0;
                if (lane == 0) {
                    base = atomicAdd(count, static_cast<unsigned int>(__popc(mask)));
                }
                base = __shfl_sync(kFull, base, 0);
                const unsigned int rank = __popc(mask & ((1u << lane) - 1u));
                if (take && base + rank < cap) {
                    keys[base + rank] = key;
                }
            }
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        residual = fmaxf(residual, __shfl_xor_sync(kFull, residual, o));
    }
    if (lane == 0 && residual > 0.f) {
        atomicMax(resid, static_cast<unsigned long long>(__float_as_uint(residual)));
    }
    if (mode == 0) {
        const unsigned long long bound = *reinterpret_cast<volatile unsigned long long*>(tau);
        for (int half = 0; half < 2; ++half) {
            const unsigned long long v = half ? list_hi : list_lo;
            const bool take = v != kEmptyKey && v <= bound;
            const unsigned mask = __ballot_sync(kFull, take);
            if (mask) {
                unsigned int base = 0;
                if (lane == 0) {
                    base = atomicAdd(count, static_cast<unsigned int>(__popc(mask)));
                }
                base = __shfl_sync(kFull, base, 0);
                const unsigned int rank = __popc(mask & ((1u << lane) - 1u));
                if (take && base + rank < cap) {
                    keys[base + rank] = v;
                }
            }
        }
        const unsigned long long worst = __shfl_sync(kFull, list_hi, 31);
        if (lane == 0 && worst != kEmptyKey) {
            atomicMin(tau, worst);
        }
    }
}

// ---- 256^3 grids: register four-step FFT kernels ---------------------------
// Block = 16 lines x 16 threads per line (see fft_reg.cuh).

__global__ void __launch_bounds__(256) pass_a256_kernel(const float2* __restrict__ spectrum,
                                                       const float2* __restrict__ partial,
                                                       float2* __restrict__ inter, int K2, int legal_z,
                                                       const float2* __restrict__ twiddles)
{
    __shared__ RegTwiddles tw;
    __shared__ float2 lines[16 * kRegLine];
    load_twiddles(tw, twiddles);
    __syncthreads();
    const int j = threadIdx.x & 15;  // column within the group (coalesced direction)
    const int t = threadIdx.x >> 4;  // lane within the line
    const int ky = blockIdx.x >> 4;
    const long long col = ((blockIdx.x & 15) << 4) + j + 256LL * ky;
    const long long plane = 65536;
    float2 v[16], sp[16];
    // The environment spectrum column is fetched first so its latency
    // overlaps the forward transform of the kernel column.
#pragma unroll
    for (int k2 = 0; k2 < 16; ++k2) {
        sp[k2] = __ldcs(spectrum + col + plane * (t + 16 * k2));
    }
#pragma unroll
    for (int n1 = 0; n1 < 16; ++n1) {
        const int z = 16 * n1 + t;
        v[n1] = z < K2 ? partial[col + plane * z] : make_float2(0.f, 0.f);
    }
    float2* line = lines + j * kRegLine;
    fft256<false, kFirstUse>(v, line, t, tw);  // v[k2] = K^(t + 16 k2)
#pragma unroll
    for (int k2 = 0; k2 < 16; ++k2) {
        const float2 sv = sp[k2];
        v[k2] = make_float2(sv.x * v[k2].x + sv.y * v[k2].y, sv.y * v[k2].x - sv.x * v[k2].y);
    }
    fft256<true>(v, line, t, tw);  // v[m2] = w(z = t + 16 m2)
#pragma unroll
    for (int m2 = 0; m2 < 16; ++m2) {
        const int z = t + 16 * m2;
        if (z < legal_z) {
            inter[col + plane * z] = v[m2];
        }
    }
}

// Pass A over a batch of orientations on 256^3 grids: the environment
// spectrum column is read once per block and kept in shared memory (32 KB,
// [k2][thread]) while each orientation of the batch finishes its kernel
// column, multiplies and inverts along z.  The spectrum (134 MB at 256^3)
// then crosses HBM once per batch instead of once per orientation.  Held in
// shared memory rather than registers, it leaves the kernel at 80
// registers: three blocks per SM instead of two.  The next orientation's
// kernel planes are fetched before the current one's transforms.
constexpr std::size_t kPassASmem = sizeof(float2) * 16 * 256;

// Block `block` of a batched pass A; `sp_s` is kPassASmem bytes of shared
// memory.  The caller has loaded `tw` (no barrier needed after it: the
// spectrum staging below ends with one).
__device__ __forceinline__ void a_block256(const float2* __restrict__ spectrum, const PassABatch& batch,
                                           const RegTwiddles& tw, float2* lines, float2* sp_s, unsigned int block)
{
    const int j = threadIdx.x & 15;  // column within the group (coalesced direction)
    const int t = threadIdx.x >> 4;  // lane within the line
    const int ky = static_cast<int>(block >> 4);
    const long long col = ((block & 15) << 4) + j + 256LL * ky;
    const long long plane = 65536;
#pragma unroll
    for (int k2 = 0; k2 < 16; ++k2) {
        sp_s[k2 * 256 + threadIdx.x] = __ldcs(spectrum + col + plane * (t + 16 * k2));
    }
    __syncthreads();
    float2* line = lines + j * kRegLine;
    // Kernel planes z = t and z = 16 + t of the next orientation (almost
    // every kernel has K2 <= 32; deeper planes are read in the loop).
    float2 next0 = make_float2(0.f, 0.f), next1 = make_float2(0.f, 0.f);
    if (batch.count > 0) {
        const PassASlot& s0 = batch.slot[0];
        next0 = t < s0.K2 ? s0.partial[col + plane * t] : next0;
        next1 = 16 + t < s0.K2 ? s0.partial[col + plane * (16 + t)] : next1;
    }
#pragma unroll 1
    for (int g = 0; g < batch.count; ++g) {
        const PassASlot s = batch.slot[g];
        float2 v[16];
        const float2 first = next0, second = next1;
        if (g + 1 < batch.count) {
            const PassASlot& sn = batch.slot[g + 1];
            next0 = t < sn.K2 ? sn.partial[col + plane * t] : make_float2(0.f, 0.f);
            next1 = 16 + t < sn.K2 ? sn.partial[col + plane * (16 + t)] : make_float2(0.f, 0.f);
        }
        if (s.K2 <= 32) {
            fft256_first32(first, second, v, line, t, tw);  // v[k2] = K^(t + 16 k2)
        }
        else {
            v[0] = first;
            v[1] = second;
#pragma unroll
            for (int n1 = 2; n1 < 16; ++n1) {
                const int z = 16 * n1 + t;
                v[n1] = z < s.K2 ? s.partial[col + plane * z] : make_float2(0.f, 0.f);
            }
            fft256<false>(v, line, t, tw);  // v[k2] = K^(t + 16 k2)
        }
#pragma unroll
        for (int k2 = 0; k2 < 16; ++k2) {
            const float2 sv = sp_s[k2 * 256 + threadIdx.x];
            v[k2] = make_float2(sv.x * v[k2].x + sv.y * v[k2].y, sv.y * v[k2].x - sv.x * v[k2].y);
        }
        fft256<true>(v, line, t, tw);  // v[m2] = w(z = t + 16 m2)
#pragma unroll
        for (int m2 = 0; m2 < 16; ++m2) {
            const int z = t + 16 * m2;
            if (z < s.legal_z) {
                s.inter[col + plane * z] = v[m2];
            }
        }
    }
}

__global__ void __launch_bounds__(256, 3) pass_a256_batch_kernel(const float2* __restrict__ spectrum,
                                                                const PassABatch batch,
                                                                const float2* __restrict__ twiddles)
{
    __shared__ RegTwiddles tw;
    __shared__ float2 lines[16 * kRegLine];
    extern __shared__ float2 sp_s[];  // [k2][threadIdx.x]
    load_twiddles(tw, twiddles);
    a_block256(spectrum, batch, tw, lines, sp_s, blockIdx.x);
}

// Environment spectrum on 256^3 grids, register four-step FFTs (see
// fft_reg.cuh).  The row kernel packs Z = B + iP straight from the occupancy,
// squared distances and the proximity table, accumulates sum(b^2 + p^2) for
// the error bound, and transforms along x; the column kernel transforms y or
// z in place (16 adjacent columns per block, coalesced along x).
__global__ void __launch_bounds__(256) env_row256_kernel(float2* __restrict__ spectrum, int E0, int E1, int E2,
                                                        const std::uint8_t* __restrict__ occ,
                                                        const std::int32_t* __restrict__ d2,
                                                        const double* __restrict__ table,
                                                        const float2* __restrict__ twiddles,
                                                        double* __restrict__ norm_partial)
{
    __shared__ RegTwiddles tw;
    __shared__ float2 lines[16 * kRegLine];
    __shared__ double red[256];
    load_twiddles(tw, twiddles);
    __syncthreads();
    const int t = threadIdx.x & 15, j = threadIdx.x >> 4;
    const int row = blockIdx.x * 16 + j;  // y + 256 z
    const int y = row & 255, z = row >> 8;
    float2 v[16];
    double acc = 0;
#pragma unroll
    for (int n1 = 0; n1 < 16; ++n1) {
        const int x = 16 * n1 + t;
        float b = 0.f, p = 0.f;
        if (x < E0 && y < E1 && z < E2) {
            const long long e = x + static_cast<long long>(E0) * (y + static_cast<long long>(E1) * z);
            b = occ[e] ? 1.f : 0.f;
            const std::int32_t dv = d2[e];
            p = dv == kInf ? 0.f : static_cast<float>(table[dv]);
        }
        acc += static_cast<double>(b) * b + static_cast<double>(p) * p;
        v[n1] = make_float2(b, p);
    }
    fft256<false, kHalfWarp>(v, lines + j * kRegLine, t, tw);
    float2* out = spectrum + 256LL * row;
#pragma unroll
    for (int k2 = 0; k2 < 16; ++k2) {
        out[t + 16 * k2] = v[k2];
    }
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int h = 128; h > 0; h >>= 1) {
        if (threadIdx.x < h) {
            red[threadIdx.x] += red[threadIdx.x + h];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        norm_partial[blockIdx.x] = red[0];
    }
}

__global__ void __launch_bounds__(256) env_column256_kernel(float2* __restrict__ spectrum, long long line_stride,
                                                           long long other_stride, float scale,
                                                           const float2* __restrict__ twiddles)
{
    __shared__ RegTwiddles tw;
    __shared__ float2 lines[16 * kRegLine];
    load_twiddles(tw, twiddles);
    __syncthreads();
    const int j = threadIdx.x & 15, t = threadIdx.x >> 4;
    const long long col = 16 * (blockIdx.x & 15) + j + other_stride * (blockIdx.x >> 4);
    float2 v[16];
#pragma unroll
    for (int n1 = 0; n1 < 16; ++n1) {
        v[n1] = spectrum[col + line_stride * (16 * n1 + t)];
    }
    fft256<false, kFirstUse>(v, lines + j * kRegLine, t, tw);
#pragma unroll
    for (int k2 = 0; k2 < 16; ++k2) {
        spectrum[col + line_stride * (t + 16 * k2)] = make_float2(v[k2].x * scale, v[k2].y * scale);
    }
}

// Inverse y of 16 columns kx of one legal z plane: block b of an
// orientation covers plane b / 16, columns 16 (b % 16) ...
__device__ __forceinline__ void b1_block256(float2* __restrict__ inter, int legal_y, const RegTwiddles& tw,
                                            float2* lines, unsigned int block)
{
    const int j = threadIdx.x & 15;
    const int t = threadIdx.x >> 4;
    const long long zz = block >> 4;
    const long long col = ((block & 15) << 4) + j + 65536LL * zz;
    float2 v[16];
#pragma unroll
    for (int n1 = 0; n1 < 16; ++n1) {
        v[n1] = inter[col + 256LL * (16 * n1 + t)];
    }
    fft256<true, kFirstUse>(v, lines + j * kRegLine, t, tw);
#pragma unroll
    for (int m2 = 0; m2 < 16; ++m2) {
        const int y = t + 16 * m2;
        if (y < legal_y) {
            inter[col + 256LL * y] = v[m2];
        }
    }
}

__global__ void __launch_bounds__(256) pass_b1_256_kernel(float2* __restrict__ inter, int legal_y,
                                                         const float2* __restrict__ twiddles)
{
    __shared__ RegTwiddles tw;
    __shared__ float2 lines[16 * kRegLine];
    load_twiddles(tw, twiddles);
    __syncthreads();
    b1_block256(inter, legal_y, tw, lines, blockIdx.x);
}

// Slot of a batched launch that owns this block.
__device__ __forceinline__ int batch_slot(const PassBBatch& b, unsigned int block)
{
    int g = 0;
    while (g + 1 < b.count && b.slot[g + 1].first_block <= static_cast<int>(block)) {
        ++g;
    }
    return g;
}

// The slot of block `block` of a batch and the block's index within it
// (PassBBatch's block order).
__device__ __forceinline__ int batch_block(const PassBBatch& b, unsigned int block, unsigned int& local)
{
    if (block < static_cast<unsigned int>(b.interleaved)) {
        local = block / static_cast<unsigned int>(b.count);
        return static_cast<int>(block % static_cast<unsigned int>(b.count));
    }
    const int g = batch_slot(b, block);
    local = static_cast<unsigned int>(b.min_blocks) + block - static_cast<unsigned int>(b.slot[g].first_block);
    return g;
}

__global__ void __launch_bounds__(256) pass_b1_256_batch_kernel(const __grid_constant__ PassBBatch b,
                                                               const float2* __restrict__ twiddles)
{
    __shared__ RegTwiddles tw;
    __shared__ float2 lines[16 * kRegLine];
    load_twiddles(tw, twiddles);
    __syncthreads();
    const int g = batch_slot(b, blockIdx.x);
    b1_block256(b.slot[g].inter, b.slot[g].legal_y, tw, lines, blockIdx.x - b.slot[g].first_block);
}

// Pass B2 on 256^3 grids: 16 rows per block, 16 threads per row.
//   mode 0: every key whose block cannot hold 64 smaller keys is emitted.
//     The block's keys overwrite its staged rows in shared memory, a
//     1024-bin histogram of their high 32 bits between the block's smallest
//     and largest finds the first bin T by which 64 keys have accumulated,
//     and keys in bins <= T that are also <= the request's pruning bound are
//     appended; T's upper edge then lowers the bound.  A key in a bin above T
//     has 64 smaller keys in its own block, so no key of the request's top 64
//     is ever left out.
//   mode 1: every candidate with approximate score <= threshold is appended
//     and every candidate past the cursor floor is counted in *tau.
struct B2Shared {
    unsigned int hist[1024];
    unsigned int block_lo, block_hi, warp_sums[8];
    int cut_bin;
    unsigned long long emit_bound;
};

// The inverse x transform of 16 legal rows and the fused epilogue above.
// Thread (row j = threadIdx / 16, lane t = threadIdx % 16) holds in v[n1]
// its row's value at kx = 16 n1 + t; `valid` rows are (y, zz).  Every thread
// of the block calls it; it may be called again for the next 16 rows.
__device__ __forceinline__ void b2_rows256_generic(float2 (&v)[16], float2* lines, const RegTwiddles& tw, B2Shared& sh,
                                           bool valid, int y, int zz, int legal_x, int legal_y,
                                           const double* __restrict__ t65, double inv_occ, int mode, float target,
                                           double threshold, double cursor_floor,
                                           unsigned long long* __restrict__ keys, unsigned int* __restrict__ count,
                                           unsigned int cap, unsigned long long* __restrict__ tau,
                                           unsigned long long* __restrict__ resid)
{
    constexpr int kBins = 1024;
    const int t = threadIdx.x & 15;  // lane within the row (coalesced direction)
    const int j = threadIdx.x >> 4;  // row within the block
    const int lane = threadIdx.x & 31;
    __syncthreads();  // the previous rows' readers of `sh` are done
    if (threadIdx.x == 0) {
        sh.block_lo = 0xffffffffu;
        sh.block_hi = 0u;
        sh.cut_bin = kBins - 1;
    }
    float2* line = lines + j * kRegLine;
    fft256<true, kHalfWarp>(v, line, t, tw);  // v[m2] = value at x = t + 16 m2
    // Stage the row in shared memory (each thread reads back only its own
    // outputs) so the epilogue loop indexes it without a local-memory array.
    __syncthreads();
#pragma unroll
    for (int m2 = 0; m2 < 16; ++m2) {
        line[t + 16 * m2] = v[m2];
    }
    // Keys replace the staged values slot for slot (mode 0).
    auto* row_keys = reinterpret_cast<unsigned long long*>(line);
    const double t65z = valid ? t65[zz] : 0.0;
    const unsigned int row_index = static_cast<unsigned int>(legal_x) * (y + static_cast<unsigned int>(legal_y) * zz);
    float residual = 0.f;
    // Keys above the request's pruning bound cannot enter its top 64.
    const unsigned long long bound = mode == 0 ? *reinterpret_cast<volatile unsigned long long*>(tau) : ~0ULL;
    const float skip = mode == 0 && valid ? skip_below(bound, t65z, inv_occ) : -INFINITY;
    unsigned int lo = 0xffffffffu, hi = 0u;
#pragma unroll 1
    for (int m2 = 0; m2 < 16; ++m2) {
        const int x = t + 16 * m2;
        unsigned long long key = kEmptyKey;
        bool take = false;
        if (valid && x < legal_x) {
            const float2 w = line[x];
            // Under the residual guard (< 0.25) the rounded value is the
            // overlap count, so the rounding doubles as the feasibility test.
            const float rounded = rintf(w.x);
            residual = fmaxf(residual, fabsf(w.x - rounded));
            if (rounded == target && !(w.y < skip)) {
                const double score = t65z - 0.35 * (static_cast<double>(w.y) * inv_occ);
                if (score >= cursor_floor) {
                    key = make_key(score, row_index + x);
                    if (mode == 0 && key > bound) {
                        key = kEmptyKey;
                    }
                    take = mode == 1 && score <= threshold;
                    if (mode == 1) {
                        atomicAdd(tau, 1ULL);
                    }
                }
            }
        }
        if (mode == 0) {
            row_keys[x] = key;
            if (key != kEmptyKey) {
                const unsigned int h = static_cast<unsigned int>(key >> 32);
                lo = min(lo, h);
                hi = max(hi, h);
            }
        }
        else {
            const unsigned mask = __ballot_sync(kFull, take);
            if (mask) {
                unsigned int slot = 0;
                if (lane == 0) {
                    slot = atomicAdd(count, static_cast<unsigned int>(__popc(mask)));
                }
                slot = __shfl_sync(kFull, slot, 0);
                const unsigned int rank = __popc(mask & ((1u << lane) - 1u));
                if (take && slot + rank < cap) {
                    keys[slot + rank] = key;
                }
            }
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        residual = fmaxf(residual, __shfl_xor_sync(kFull, residual, o));
    }
    if (lane == 0 && residual > 0.f) {
        atomicMax(resid, static_cast<unsigned long long>(__float_as_uint(residual)));
    }
    if (mode != 0) {
        return;
    }
    // Block range of the keys' high words, then the histogram over it.
    for (int o = 16; o > 0; o >>= 1) {
        lo = min(lo, __shfl_xor_sync(kFull, lo, o));
        hi = max(hi, __shfl_xor_sync(kFull, hi, o));
    }
    for (int b = threadIdx.x; b < kBins; b += 256) {
        sh.hist[b] = 0;
    }
    if (lane == 0 && lo <= hi) {
        atomicMin(&sh.block_lo, lo);
        atomicMax(&sh.block_hi, hi);
    }
    __syncthreads();
    const unsigned int range_lo = sh.block_lo;
    if (range_lo > sh.block_hi) {
        return;  // no key in these rows (uniform: every thread sees the same shared values)
    }
    int shift = 0;
    while (shift < 32 && ((sh.block_hi - range_lo) >> shift) >= static_cast<unsigned int>(kBins)) {
        ++shift;
    }
#pragma unroll 1
    for (int m2 = 0; m2 < 16; ++m2) {
        const int x = t + 16 * m2;
        if (valid && x < legal_x) {
            const unsigned long long key = row_keys[x];
            if (key != kEmptyKey) {
                atomicAdd(&sh.hist[(static_cast<unsigned int>(key >> 32) - range_lo) >> shift], 1u);
            }
        }
    }
    __syncthreads();
    // First bin at which 64 keys have accumulated: each thread sums four
    // consecutive bins, a block scan of those sums locates the crossing.
    unsigned int mine = 0;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        mine += sh.hist[4 * threadIdx.x + q];
    }
    unsigned int inclusive = mine;
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned int other = __shfl_up_sync(kFull, inclusive, o);
        if (lane >= o) {
            inclusive += other;
        }
    }
    const int warp = threadIdx.x >> 5;
    if (lane == 31) {
        sh.warp_sums[warp] = inclusive;
    }
    __syncthreads();
    unsigned int before = 0, total = 0;
    for (int w = 0; w < 8; ++w) {
        before += w < warp ? sh.warp_sums[w] : 0u;
        total += sh.warp_sums[w];
    }
    const unsigned int start = before + inclusive - mine;
    constexpr unsigned int kNeed = kExactPerOrientation;
    if (total >= kNeed && start < kNeed && start + mine >= kNeed) {
        unsigned int running = start;
        for (int q = 0; q < 4; ++q) {
            running += sh.hist[4 * threadIdx.x + q];
            if (running >= kNeed) {
                sh.cut_bin = 4 * threadIdx.x + q;
                break;
            }
        }
    }
    __syncthreads();
    const int cut = sh.cut_bin;
    if (threadIdx.x == 0) {
        unsigned long long b = *reinterpret_cast<volatile unsigned long long*>(tau);
        const unsigned long long edge = static_cast<unsigned long long>(range_lo) +
                                        (static_cast<unsigned long long>(cut + 1) << shift);
        if (total >= kNeed && edge <= 0xffffffffULL) {
            // Every key of bins <= cut is below (edge << 32): an upper bound of
            // this block's 64th smallest key, hence of the request's.
            const unsigned long long upper = (edge << 32) - 1;
            const unsigned long long old = atomicMin(tau, upper);
            b = old < upper ? old : upper;
        }
        sh.emit_bound = b;
    }
    __syncthreads();
    const unsigned long long limit = sh.emit_bound;
#pragma unroll 1
    for (int m2 = 0; m2 < 16; ++m2) {
        const int x = t + 16 * m2;
        bool take = false;
        unsigned long long key = kEmptyKey;
        if (valid && x < legal_x) {
            key = row_keys[x];
            take = key != kEmptyKey && key <= limit &&
                   static_cast<int>((static_cast<unsigned int>(key >> 32) - range_lo) >> shift) <= cut;
        }
        const unsigned mask = __ballot_sync(kFull, take);
        if (mask) {
            unsigned int slot = 0;
            if (lane == 0) {
                slot = atomicAdd(count, static_cast<unsigned int>(__popc(mask)));
            }
            slot = __shfl_sync(kFull, slot, 0);
            const unsigned int rank = __popc(mask & ((1u << lane) - 1u));
            if (take && slot + rank < cap) {
                keys[slot + rank] = key;
            }
        }
    }
}

// Mode 0 of the epilogue above with the values kept in registers: every
// cell gets the residual check and two FP32 compares, and only cells that
// pass them (below the prefilter's bound) get an FP64 score and a key slot
// in shared memory; `present` marks those slots, so the histogram and the
// emission visit only them.  Same keys, same emission rule as the generic
// path.
__device__ __forceinline__ void b2_rows256_select(float2 (&v)[16], float2* lines, const RegTwiddles& tw, B2Shared& sh,
                                                  bool valid, int y, int zz, int legal_x, int legal_y,
                                                  const double* __restrict__ t65, double inv_occ, float target,
                                                  double cursor_floor, unsigned long long* __restrict__ keys,
                                                  unsigned int* __restrict__ count, unsigned int cap,
                                                  unsigned long long* __restrict__ tau,
                                                  unsigned long long* __restrict__ resid)
{
    constexpr int kBins = 1024;
    const int t = threadIdx.x & 15;  // lane within the row (coalesced direction)
    const int j = threadIdx.x >> 4;  // row within the block
    const int lane = threadIdx.x & 31;
    __syncthreads();  // the previous rows' readers of `sh` are done
    if (threadIdx.x == 0) {
        sh.block_lo = 0xffffffffu;
        sh.block_hi = 0u;
        sh.cut_bin = kBins - 1;
    }
    float2* line = lines + j * kRegLine;
    fft256<true, kHalfWarp>(v, line, t, tw);  // v[m2] = value at x = t + 16 m2
    auto* row_keys = reinterpret_cast<unsigned long long*>(line);
    const double t65z = valid ? t65[zz] : 0.0;
    const unsigned int row_index = static_cast<unsigned int>(legal_x) * (y + static_cast<unsigned int>(legal_y) * zz);
    // Keys above the request's pruning bound cannot enter its top 64.
    const unsigned long long bound = *reinterpret_cast<volatile unsigned long long*>(tau);
    const float skip = valid ? skip_below(bound, t65z, inv_occ) : -INFINITY;
    float residual = 0.f;
    unsigned int lo = 0xffffffffu, hi = 0u, present = 0u;
    __syncthreads();  // the transform's reads of `line` are done before keys overwrite it
#pragma unroll
    for (int m2 = 0; m2 < 16; ++m2) {
        const int x = t + 16 * m2;
        const float2 w = v[m2];
        if (valid && x < legal_x) {
            // Under the residual guard (< 0.25) the rounded value is the
            // overlap count, so the rounding doubles as the feasibility test.
            const float rounded = rintf(w.x);
            residual = fmaxf(residual, fabsf(w.x - rounded));
            if (rounded == target && !(w.y < skip)) {
                const double score = t65z - 0.35 * (static_cast<double>(w.y) * inv_occ);
                if (score >= cursor_floor) {
                    const unsigned long long key = make_key(score, row_index + x);
                    if (key <= bound) {
                        row_keys[x] = key;
                        present |= 1u << m2;
                        const unsigned int h = static_cast<unsigned int>(key >> 32);
                        lo = min(lo, h);
                        hi = max(hi, h);
                    }
                }
            }
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        residual = fmaxf(residual, __shfl_xor_sync(kFull, residual, o));
    }
    if (lane == 0 && residual > 0.f) {
        atomicMax(resid, static_cast<unsigned long long>(__float_as_uint(residual)));
    }
    // Block range of the keys' high words, then the histogram over it.
    for (int o = 16; o > 0; o >>= 1) {
        lo = min(lo, __shfl_xor_sync(kFull, lo, o));
        hi = max(hi, __shfl_xor_sync(kFull, hi, o));
    }
    for (int b = threadIdx.x; b < kBins; b += 256) {
        sh.hist[b] = 0;
    }
    if (lane == 0 && lo <= hi) {
        atomicMin(&sh.block_lo, lo);
        atomicMax(&sh.block_hi, hi);
    }
    __syncthreads();
    const unsigned int range_lo = sh.block_lo;
    if (range_lo > sh.block_hi) {
        return;  // no key in these rows (uniform: every thread sees the same shared values)
    }
    int shift = 0;
    while (shift < 32 && ((sh.block_hi - range_lo) >> shift) >= static_cast<unsigned int>(kBins)) {
        ++shift;
    }
    for (unsigned int bits = present; bits; bits &= bits - 1) {
        const int m2 = __ffs(bits) - 1;
        const unsigned long long key = row_keys[t + 16 * m2];
        atomicAdd(&sh.hist[(static_cast<unsigned int>(key >> 32) - range_lo) >> shift], 1u);
    }
    __syncthreads();
    // First bin at which 64 keys have accumulated: each thread sums four
    // consecutive bins, a block scan of those sums locates the crossing.
    unsigned int mine = 0;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        mine += sh.hist[4 * threadIdx.x + q];
    }
    unsigned int inclusive = mine;
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned int other = __shfl_up_sync(kFull, inclusive, o);
        if (lane >= o) {
            inclusive += other;
        }
    }
    const int warp = threadIdx.x >> 5;
    if (lane == 31) {
        sh.warp_sums[warp] = inclusive;
    }
    __syncthreads();
    unsigned int before = 0, total = 0;
    for (int w = 0; w < 8; ++w) {
        before += w < warp ? sh.warp_sums[w] : 0u;
        total += sh.warp_sums[w];
    }
    const unsigned int start = before + inclusive - mine;
    constexpr unsigned int kNeed = kExactPerOrientation;
    if (total >= kNeed && start < kNeed && start + mine >= kNeed) {
        unsigned int running = start;
        for (int q = 0; q < 4; ++q) {
            running += sh.hist[4 * threadIdx.x + q];
            if (running >= kNeed) {
                sh.cut_bin = 4 * threadIdx.x + q;
                break;
            }
        }
    }
    __syncthreads();
    const int cut = sh.cut_bin;
    if (threadIdx.x == 0) {
        unsigned long long b = *reinterpret_cast<volatile unsigned long long*>(tau);
        const unsigned long long edge = static_cast<unsigned long long>(range_lo) +
                                        (static_cast<unsigned long long>(cut + 1) << shift);
        if (total >= kNeed && edge <= 0xffffffffULL) {
            // Every key of bins <= cut is below (edge << 32): an upper bound of
            // this block's 64th smallest key, hence of the request's.
            const unsigned long long upper = (edge << 32) - 1;
            const unsigned long long old = atomicMin(tau, upper);
            b = old < upper ? old : upper;
        }
        sh.emit_bound = b;
    }
    __syncthreads();
    const unsigned long long limit = sh.emit_bound;
    // Slots any lane of the warp holds, visited together by the whole warp.
    const unsigned int warp_present = __reduce_or_sync(kFull, present);
    for (unsigned int bits = warp_present; bits; bits &= bits - 1) {
        const int m2 = __ffs(bits) - 1;
        bool take = false;
        unsigned long long key = kEmptyKey;
        if ((present >> m2) & 1u) {
            key = row_keys[t + 16 * m2];
            take = key <= limit &&
                   static_cast<int>((static_cast<unsigned int>(key >> 32) - range_lo) >> shift) <= cut;
        }
        const unsigned mask = __ballot_sync(kFull, take);
        if (mask) {
            unsigned int slot = 0;
            if (lane == 0) {
                slot = atomicAdd(count, static_cast<unsigned int>(__popc(mask)));
            }
            slot = __shfl_sync(kFull, slot, 0);
            const unsigned int rank = __popc(mask & ((1u << lane) - 1u));
            if (take && slot + rank < cap) {
                keys[slot + rank] = key;
            }
        }
    }
}

// Mode 2 of the epilogue: the histogram of the 16 rows' rounded overlap
// counts, gathered in shared memory and added to the request's `bins` u32
// bins in `hist` (the last bin holds every larger count).
__device__ __forceinline__ void b2_rows256_hist(float2 (&v)[16], float2* lines, const RegTwiddles& tw, B2Shared& sh,
                                                bool valid, int legal_x, unsigned int* __restrict__ hist,
                                                unsigned int bins, unsigned long long* __restrict__ resid)
{
    const int t = threadIdx.x & 15;
    const int j = threadIdx.x >> 4;
    const int lane = threadIdx.x & 31;
    const unsigned int local_bins = bins < 1024u ? bins : 1024u;
    __syncthreads();  // the previous rows' readers of `sh` are done
    for (unsigned int b = threadIdx.x; b < local_bins; b += blockDim.x) {
        sh.hist[b] = 0;
    }
    fft256<true, kHalfWarp>(v, lines + j * kRegLine, t, tw);  // v[m2] = value at x = t + 16 m2
    float residual = 0.f;
#pragma unroll
    for (int m2 = 0; m2 < 16; ++m2) {
        const int x = t + 16 * m2;
        if (valid && x < legal_x) {
            const float w = v[m2].x;
            residual = fmaxf(residual, fabsf(w - rintf(w)));
            const float c = rintf(w);
            const unsigned int bin = c <= 0.f ? 0u : c >= static_cast<float>(bins - 1) ? bins - 1
                                                                                       : static_cast<unsigned int>(c);
            if (bin < local_bins) {
                atomicAdd(&sh.hist[bin], 1u);
            }
            else {
                atomicAdd(hist + bin, 1u);
            }
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        residual = fmaxf(residual, __shfl_xor_sync(kFull, residual, o));
    }
    if (lane == 0 && residual > 0.f) {
        atomicMax(resid, static_cast<unsigned long long>(__float_as_uint(residual)));
    }
    __syncthreads();
    for (unsigned int b = threadIdx.x; b < local_bins; b += blockDim.x) {
        if (sh.hist[b]) {
            atomicAdd(hist + b, sh.hist[b]);
        }
    }
}

// Mode 0 (first pass) takes the register path, mode 1 (threshold pass) the
// generic one, mode 2 the count histogram.
__device__ __forceinline__ void b2_rows256(float2 (&v)[16], float2* lines, const RegTwiddles& tw, B2Shared& sh,
                                           bool valid, int y, int zz, int legal_x, int legal_y,
                                           const double* __restrict__ t65, double inv_occ, int mode, float target,
                                           double threshold, double cursor_floor,
                                           unsigned long long* __restrict__ keys, unsigned int* __restrict__ count,
                                           unsigned int cap, unsigned long long* __restrict__ tau,
                                           unsigned long long* __restrict__ resid)
{
    if (mode == 0) {
        b2_rows256_select(v, lines, tw, sh, valid, y, zz, legal_x, legal_y, t65, inv_occ, target, cursor_floor, keys,
                          count, cap, tau, resid);
    }
    else if (mode == 2) {
        b2_rows256_hist(v, lines, tw, sh, valid, legal_x, reinterpret_cast<unsigned int*>(keys), cap, resid);
    }
    else {
        b2_rows256_generic(v, lines, tw, sh, valid, y, zz, legal_x, legal_y, t65, inv_occ, mode, target, threshold,
                           cursor_floor, keys, count, cap, tau, resid);
    }
}

// Inverse x of 16 legal rows of one orientation and the epilogue: block b
// covers rows 16 b ... (row = y + legal_y zz).
__device__ __forceinline__ void b2_block256(const float2* __restrict__ inter, int legal_x, int legal_y, int legal_z,
                                            const RegTwiddles& tw, float2* lines, B2Shared& sh,
                                            const double* __restrict__ t65, double inv_occ, int mode, float target,
                                            double threshold, double cursor_floor,
                                            unsigned long long* __restrict__ keys, unsigned int* __restrict__ count,
                                            unsigned int cap, unsigned long long* __restrict__ tau,
                                            unsigned long long* __restrict__ resid, unsigned int block)
{
    const int t = threadIdx.x & 15;
    const int j = threadIdx.x >> 4;
    const long long rows = static_cast<long long>(legal_y) * legal_z;
    const long long row = static_cast<long long>(block) * 16 + j;
    const bool valid = row < rows;
    const int y = valid ? static_cast<int>(row % legal_y) : 0;
    const int zz = valid ? static_cast<int>(row / legal_y) : 0;
    const long long base = 256LL * (y + 256LL * zz);
    float2 v[16];
#pragma unroll
    for (int n1 = 0; n1 < 16; ++n1) {
        v[n1] = valid ? inter[base + 16 * n1 + t] : make_float2(0.f, 0.f);
    }
    b2_rows256(v, lines, tw, sh, valid, y, zz, legal_x, legal_y, t65, inv_occ, mode, target, threshold, cursor_floor,
               keys, count, cap, tau, resid);
}

__global__ void __launch_bounds__(256) pass_b2_256_kernel(const float2* __restrict__ inter, int legal_x,
                                                         int legal_y, int legal_z,
                                                         const float2* __restrict__ twiddles,
                                                         const double* __restrict__ t65, double inv_occ, int mode,
                                                         float target, double threshold, double cursor_floor,
                                                         unsigned long long* __restrict__ keys,
                                                         unsigned int* __restrict__ count, unsigned int cap,
                                                         unsigned long long* __restrict__ tau,
                                                         unsigned long long* __restrict__ resid)
{
    __shared__ RegTwiddles tw;
    __shared__ float2 lines[16 * kRegLine];
    __shared__ B2Shared sh;
    load_twiddles(tw, twiddles);
    __syncthreads();
    b2_block256(inter, legal_x, legal_y, legal_z, tw, lines, sh, t65, inv_occ, mode, target, threshold, cursor_floor,
                keys, count, cap, tau, resid, blockIdx.x);
}

__global__ void __launch_bounds__(256) pass_b2_256_batch_kernel(const __grid_constant__ PassBBatch b,
                                                               const float2* __restrict__ twiddles)
{
    __shared__ RegTwiddles tw;
    __shared__ float2 lines[16 * kRegLine];
    __shared__ B2Shared sh;
    load_twiddles(tw, twiddles);
    __syncthreads();
    unsigned int local = 0;
    const PassBSlot& s = b.slot[batch_block(b, blockIdx.x, local)];
    b2_block256(s.inter, s.legal_x, s.legal_y, s.legal_z, tw, lines, sh, s.t65, s.inv_occ, 0, s.target, 0.0,
                s.cursor_floor, s.keys, s.count, s.cap, s.tau, s.resid, local);
}

// One stage of the software-pipelined page passes on 256^3 grids: pass A of
// batch k, pass B1 of batch k - 1 and pass B2 of batch k - 2 in one launch,
// each batch on its own intermediate (three in rotation).  Pass B1 streams
// HBM at the copy peak while passes A and B2 are bound by instruction issue;
// run as separate launches, each leaves the other resource idle.  Here the
// three roles' blocks are interleaved through the grid in proportion to
// their counts (block b takes role A when floor((b + 1) nA / n) passes an
// integer, and the rest split the same way between B1 and B2), so every SM
// holds a mix of them throughout the launch.  Each block runs the same code
// as the corresponding block of the separate kernels.
//
// Measured slower than the separate launches (1.16 ms per stage launch; a
// 32-orientation step's passes took 4.6 ms against 3.7 ms), so it runs only
// under SPK_PAGE_SCHEDULE=staged: with three blocks per SM for every role,
// the B1 blocks on an SM keep too few loads in flight to stream HBM, and
// the long pass A blocks dispatched last leave a tail.
struct PassStage {
    const float2* spectrum;
    PassABatch a;
    PassBBatch b1, b2;
    unsigned int blocks_a, blocks_b1;
};

__global__ void __launch_bounds__(256, 3) pass_stage256_kernel(const __grid_constant__ PassStage p,
                                                              const float2* __restrict__ twiddles)
{
    __shared__ RegTwiddles tw;
    __shared__ float2 lines[16 * kRegLine];
    // Pass A: the spectrum column (kPassASmem bytes); pass B2: its B2Shared.
    extern __shared__ __align__(16) unsigned char stage_smem[];
    load_twiddles(tw, twiddles);
    const unsigned long long b = blockIdx.x, n = gridDim.x;
    const unsigned long long a_before = b * p.blocks_a / n, a_upto = (b + 1) * p.blocks_a / n;
    if (a_upto > a_before) {
        a_block256(p.spectrum, p.a, tw, lines, reinterpret_cast<float2*>(stage_smem),
                   static_cast<unsigned int>(a_before));
        return;
    }
    __syncthreads();
    const unsigned long long q = b - a_before, m = n - p.blocks_a;
    const unsigned long long b1_before = q * p.blocks_b1 / m, b1_upto = (q + 1) * p.blocks_b1 / m;
    if (b1_upto > b1_before) {
        const unsigned int block = static_cast<unsigned int>(b1_before);
        const PassBSlot& s = p.b1.slot[batch_slot(p.b1, block)];
        b1_block256(s.inter, s.legal_y, tw, lines, block - static_cast<unsigned int>(s.first_block));
        return;
    }
    unsigned int local = 0;
    const PassBSlot& s = p.b2.slot[batch_block(p.b2, static_cast<unsigned int>(q - b1_before), local)];
    b2_block256(s.inter, s.legal_x, s.legal_y, s.legal_z, tw, lines, *reinterpret_cast<B2Shared*>(stage_smem), s.t65,
                s.inv_occ, 0, s.target, 0.0, s.cursor_floor, s.keys, s.count, s.cap, s.tau, s.resid, local);
}
static_assert(sizeof(B2Shared) <= kPassASmem, "pass B2's shared state must fit the stage kernel's dynamic buffer");

// Passes B1 and B2 fused on 256^3 grids: one cluster of 8 CTAs per legal z
// plane.  CTA c inverts along y the 32 columns kx = 32c..32c+31 of the plane
// (read from HBM once) and keeps them in its shared memory; after a cluster
// barrier each CTA gathers whole rows y = c, c + 8, ... from the 8 CTAs'
// shared memory (distributed shared memory) and runs the inverse x
// transform and the epilogue of pass B2 on them.  The legal-row
// intermediate that B1 wrote and B2 read back never reaches HBM.
constexpr int kFusedCluster = 8;
constexpr std::size_t kFusedSmem = sizeof(float2) * (256 * 32 + 16 * kRegLine) + sizeof(RegTwiddles) + sizeof(B2Shared);
static_assert(sizeof(float2) * (256 * 32 + 16 * kRegLine) % 16 == 0, "the twiddle rows need 16-byte alignment");

__global__ void __cluster_dims__(kFusedCluster, 1, 1) __launch_bounds__(256)
    pass_b_fused_256_kernel(const float2* __restrict__ inter, int legal_x, int legal_y,
                            const float2* __restrict__ twiddles, const double* __restrict__ t65, double inv_occ,
                            int mode, float target, double threshold, double cursor_floor,
                            unsigned long long* __restrict__ keys,
                            unsigned int* __restrict__ count, unsigned int cap, unsigned long long* __restrict__ tau,
                            unsigned long long* __restrict__ resid)
{
    extern __shared__ __align__(16) unsigned char fused_smem[];
    float2* cols = reinterpret_cast<float2*>(fused_smem);  // [y < 256][kx_local < 32]
    float2* lines = cols + 256 * 32;
    RegTwiddles& tw = *reinterpret_cast<RegTwiddles*>(lines + 16 * kRegLine);
    B2Shared& sh = *reinterpret_cast<B2Shared*>(&tw + 1);
    cg::cluster_group cluster = cg::this_cluster();
    const unsigned int rank = cluster.block_rank();
    const int zz = static_cast<int>(blockIdx.x / kFusedCluster);
    load_twiddles(tw, twiddles);
    __syncthreads();
    const long long plane = 65536LL * zz;
    // Inverse y of this CTA's 32 columns, 16 at a time (coalesced along kx).
#pragma unroll 1
    for (int r = 0; r < 2; ++r) {
        const int j = threadIdx.x & 15, t = threadIdx.x >> 4;
        const int kx_local = 16 * r + j;
        const int kx = 32 * static_cast<int>(rank) + kx_local;
        float2 v[16];
#pragma unroll
        for (int n1 = 0; n1 < 16; ++n1) {
            v[n1] = inter[plane + 256LL * (16 * n1 + t) + kx];
        }
        fft256<true>(v, lines + j * kRegLine, t, tw);  // v[m2] = value at y = t + 16 m2
#pragma unroll
        for (int m2 = 0; m2 < 16; ++m2) {
            cols[(t + 16 * m2) * 32 + kx_local] = v[m2];
        }
    }
    cluster.sync();
    // Rows y = rank + 8 i, gathered across the cluster: kx = 16 n1 + t lives
    // in CTA n1 / 2 at local column 16 (n1 % 2) + t.
#pragma unroll 1
    for (int r = 0; r < 2; ++r) {
        const int t = threadIdx.x & 15, j = threadIdx.x >> 4;
        const int y = static_cast<int>(rank) + kFusedCluster * (16 * r + j);
        const bool valid = y < legal_y;
        float2 v[16];
#pragma unroll
        for (int n1 = 0; n1 < 16; ++n1) {
            const float2* src = cluster.map_shared_rank(cols, n1 >> 1);
            v[n1] = valid ? src[y * 32 + 16 * (n1 & 1) + t] : make_float2(0.f, 0.f);
        }
        b2_rows256(v, lines, tw, sh, valid, valid ? y : 0, zz, legal_x, legal_y, t65, inv_occ, mode, target,
                   threshold, cursor_floor, keys, count, cap, tau, resid);
    }
    cluster.sync();  // no CTA leaves while another may still read its columns
}

// Bitonic sort of n <= capacity keys in shared memory (padded with kEmptyKey
// to a power of two); the block then holds them in ascending order in s[].
__device__ unsigned int block_sort(const unsigned long long* __restrict__ src, unsigned int n,
                                   unsigned long long* s)
{
    unsigned int size = 1;
    while (size < n) {
        size <<= 1;
    }
    for (unsigned int i = threadIdx.x; i < size; i += blockDim.x) {
        s[i] = i < n ? src[i] : kEmptyKey;
    }
    __syncthreads();
    for (unsigned int k = 2; k <= size; k <<= 1) {
        for (unsigned int j = k >> 1; j > 0; j >>= 1) {
            for (unsigned int i = threadIdx.x; i < size; i += blockDim.x) {
                const unsigned int p = i ^ j;
                if (p > i) {
                    const bool up = (i & k) == 0;
                    const unsigned long long x = s[i], y = s[p];
                    if ((x > y) == up) {
                        s[i] = y;
                        s[p] = x;
                    }
                }
            }
            __syncthreads();
        }
    }
    return size;
}

// Keeps the smallest kExactPerOrientation + 1 keys of each request: request
// r's keys start at keys + r * stride and number min(counts[r], limit) (or
// `limit` when counts is null).  Dynamic shared memory holds `limit` keys.
__global__ void merge_kernel(const unsigned long long* __restrict__ keys, long long stride,
                             const unsigned int* __restrict__ counts, unsigned int limit,
                             unsigned long long* __restrict__ selected)
{
    extern __shared__ unsigned long long sorted[];
    const int r = blockIdx.x;
    const unsigned int n = counts ? min(counts[r], limit) : limit;
    const unsigned int size = block_sort(keys + static_cast<long long>(r) * stride, n, sorted);
    for (int i = threadIdx.x; i <= kExactPerOrientation; i += blockDim.x) {
        selected[static_cast<long long>(r) * (kExactPerOrientation + 1) + i] =
            static_cast<unsigned int>(i) < size ? sorted[i] : kEmptyKey;
    }
}

// Second stage for large key ranges: request r's `lists` sorted lists of
// `per` keys each (the first stage's chunk winners) merged into their `per`
// smallest, ascending, by one warp-pair per request: thread c holds the head
// of list c, and each round the smallest head (keys are distinct, empty
// slots are kEmptyKey) is written out and its list advances.  The result is
// the first `per` keys of the sorted union, as a full sort would give.
__global__ void __launch_bounds__(64) merge_lists_kernel(const unsigned long long* __restrict__ partial, int lists,
                                                        int per, unsigned long long* __restrict__ selected)
{
    __shared__ unsigned long long warp_min[2];
    const int r = blockIdx.x, c = threadIdx.x, lane = c & 31, warp = c >> 5;
    const unsigned long long* list = partial + (static_cast<long long>(r) * lists + c) * per;
    int head = 0;
    unsigned long long value = c < lists ? list[0] : kEmptyKey;
    for (int i = 0; i < per; ++i) {
        unsigned long long m = value;
        for (int o = 16; o > 0; o >>= 1) {
            const unsigned long long other = __shfl_xor_sync(kFull, m, o);
            m = other < m ? other : m;
        }
        if (lane == 0) {
            warp_min[warp] = m;
        }
        __syncthreads();
        const unsigned long long best = warp_min[0] < warp_min[1] ? warp_min[0] : warp_min[1];
        __syncthreads();
        if (c == 0) {
            selected[static_cast<long long>(r) * per + i] = best;
        }
        if (value == best && best != kEmptyKey) {
            ++head;
            value = head < per ? list[head] : kEmptyKey;
        }
    }
}

// First stage for large key ranges: chunk c (kKeyCapacity keys) of request r
// keeps its smallest kExactPerOrientation + 1 keys in
// partial[(r * chunks + c) * (kExactPerOrientation + 1) ...].
__global__ void merge_chunk_kernel(const unsigned long long* __restrict__ keys, unsigned int cap,
                                   const unsigned int* __restrict__ counts, unsigned long long* __restrict__ partial)
{
    __shared__ unsigned long long sorted[kKeyCapacity];
    const int c = blockIdx.x, r = blockIdx.y, chunks = gridDim.x;
    const unsigned int n_r = min(counts[r], cap);
    const unsigned int begin = static_cast<unsigned int>(c) * kKeyCapacity;
    const unsigned int n = begin < n_r ? min(kKeyCapacity, n_r - begin) : 0u;
    unsigned long long* out = partial + (static_cast<long long>(r) * chunks + c) * (kExactPerOrientation + 1);
    if (n == 0) {
        for (int i = threadIdx.x; i <= kExactPerOrientation; i += blockDim.x) {
            out[i] = kEmptyKey;
        }
        return;
    }
    const unsigned int size = block_sort(keys + static_cast<long long>(r) * cap + begin, n, sorted);
    for (int i = threadIdx.x; i <= kExactPerOrientation; i += blockDim.x) {
        out[i] = static_cast<unsigned int>(i) < size ? sorted[i] : kEmptyKey;
    }
}

struct ExactJob {
    const std::int32_t* ones;
    int ones_count;
    int legal_x, legal_y;
};

// One block per selected key: exact overlap recount and exact proximity sum.
__global__ void exact_kernel(const unsigned long long* __restrict__ selected, const ExactJob* __restrict__ jobs,
                             int per_request, const std::uint8_t* __restrict__ occ,
                             const std::int32_t* __restrict__ d2, const double* __restrict__ table, int E0, int E1,
                             long long* __restrict__ out_count, double* __restrict__ out_p,
                             int* __restrict__ range_error)
{
    const int request = static_cast<int>(blockIdx.x / per_request);
    const unsigned long long key = selected[blockIdx.x];
    if (key == kEmptyKey) {
        if (threadIdx.x == 0) {
            out_count[blockIdx.x] = -1;
            out_p[blockIdx.x] = 0.0;
        }
        return;
    }
    const ExactJob job = jobs[request];
    const unsigned int index = static_cast<unsigned int>(key & 0xffffffffULL);
    const long long sx = index % job.legal_x;
    const long long rest = index / job.legal_x;
    const long long sy = rest % job.legal_y;
    const long long sz = rest / job.legal_y;
    const long long base = sx + E0 * (sy + static_cast<long long>(E1) * sz);
    SuperAcc acc;
    super_clear(acc);
    long long overlap = 0;
    bool ok = true;
    for (int i = threadIdx.x; i < job.ones_count; i += blockDim.x) {
        const long long cell = base + job.ones[i];
        overlap += occ[cell];
        const std::int32_t v = d2[cell];
        ok &= super_add(acc, v == kInf ? 0.0 : table[v]);
    }
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    for (int o = 16; o > 0; o >>= 1) {
        overlap += __shfl_xor_sync(kFull, overlap, o);
        for (int l = 0; l < kSuperLimbs; ++l) {
            acc.limb[l] += __shfl_xor_sync(kFull, acc.limb[l], o);
        }
    }
    __shared__ long long s_limbs[8][kSuperLimbs];
    __shared__ long long s_overlap[8];
    if (lane == 0) {
        s_overlap[warp] = overlap;
        for (int l = 0; l < kSuperLimbs; ++l) {
            s_limbs[warp][l] = acc.limb[l];
        }
    }
    if (!ok) {
        atomicOr(range_error, 1);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        SuperAcc total;
        super_clear(total);
        long long count = 0;
        for (int w = 0; w < static_cast<int>(blockDim.x >> 5); ++w) {
            count += s_overlap[w];
            for (int l = 0; l < kSuperLimbs; ++l) {
                total.limb[l] += s_limbs[w][l];
            }
        }
        out_count[blockIdx.x] = count;
        out_p[blockIdx.x] = super_round(total);
    }
}

double decode_key_score(unsigned long long key)
{
    const unsigned int k = static_cast<unsigned int>(key >> 32);
    const unsigned int u = (k & 0x80000000u) ? (k & 0x7fffffffu) : ~k;
    float f;
    std::memcpy(&f, &u, 4);
    return static_cast<double>(f);
}

bool rank_less(const Candidate& l, const Candidate& r)
{
    if (l.score != r.score) {
        return l.score < r.score;
    }
    if (l.orientation != r.orientation) {
        return l.orientation < r.orientation;
    }
    return std::tie(l.t[2], l.t[1], l.t[0]) < std::tie(r.t[2], r.t[1], r.t[0]);
}

template <typename Kernel>
void allow_large_smem(Kernel k)
{
    cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
}

}  // namespace

Pipeline::Pipeline(spk_context* ctx) : ctx_(ctx)
{
    const char* mode = std::getenv("SPK_PASS_B");
    fused_b_ = mode && std::strcmp(mode, "fused") == 0;
    const char* schedule = std::getenv("SPK_PAGE_SCHEDULE");
    staged_ = schedule && std::strcmp(schedule, "staged") == 0;
}

Pipeline::~Pipeline()
{
    if (side_) {
        cudaStreamSynchronize(side_);
        cudaEventDestroy(ev_in_);
        cudaEventDestroy(ev_done_);
        cudaStreamDestroy(side_);
    }
    for (auto& s : slots_) {
        cudaFree(s.partial);
        cudaFree(s.ones);
        cudaFree(s.t65);
    }
}

// ---- transform-length autotuner --------------------------------------------
//
// A window of E cells per axis needs a circular transform of any length
// L >= E (legal translations never wrap).  The candidates are the supported
// 2^a 3^b 5^c lengths from max(E, 16) to the next power of two; the x axis
// also needs a multiple of 16 (pass A's column groups).  Each candidate's cost
// per transformed point is measured once per device and axis (fft_axis on a
// scratch grid, the fastest of three timed runs after a warm-up); the register
// four-step path, used when every axis is 256, is measured the same way on
// its own column kernel.  The chosen lengths minimise the modelled page cost,
// points x the sum of the three axes' per-point costs.
namespace {

std::mutex g_tune_mutex;
std::map<std::tuple<int, int, int>, double> g_tune_cost;  // (device, axis or -1 for the 256 path, L) -> ns/point

std::vector<int> length_candidates(int E, int axis)
{
    const int lo = std::max(E, 16);
    const int hi = static_cast<int>(next_pow2(static_cast<std::uint32_t>(lo)));
    std::vector<int> out;
    for (int L = lo; L <= hi && L <= kMaxFftLength; ++L) {
        if (fft_length_supported(static_cast<std::uint64_t>(L)) && (axis != 0 || L % 16 == 0)) {
            out.push_back(L);
        }
    }
    return out;
}

// Nanoseconds per point of one transform pass, measured on `scratch`
// (512 x 64 x 64 complex values).
double measure_pass(spk_context* ctx, int axis, int L, float2* scratch, int& status)
{
    cudaStream_t st = ctx->stream;
    const auto* tw = twiddle_table<float>(ctx, L, status);
    if (!tw) {
        return -1.0;
    }
    int shape[3] = { 64, 64, 64 };
    long long points = 0;
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    float best = 1e30f;
    for (int rep = 0; rep < 4; ++rep) {
        cudaEventRecord(a, st);
        if (axis < 0) {
            // The register four-step path: the y pass of env_column256_kernel
            // over 256 x 256 x 16 values.
            env_column256_kernel<<<16 * 16, 256, 0, st>>>(scratch, 256, 65536, 1.f, tw);
            points = 256LL * 256 * 16;
        }
        else {
            shape[axis] = L;
            fft_axis<float>(scratch, shape[0], shape[1], shape[2], axis, false, 1.f, tw, st);
            points = static_cast<long long>(shape[0]) * shape[1] * shape[2];
        }
        cudaEventRecord(b, st);
        cudaEventSynchronize(b);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, a, b);
        if (rep > 0) {
            best = std::min(best, ms);
        }
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    ctx->launches += 4;
    if (cudaGetLastError() != cudaSuccess) {
        status = kCuda;
        return -1.0;
    }
    return 1e6 * static_cast<double>(best) / static_cast<double>(points);
}

double pass_cost(spk_context* ctx, int axis, int L, float2*& scratch, int& status)
{
    int device = 0;
    cudaGetDevice(&device);
    const auto key = std::make_tuple(device, axis, L);
    {
        std::lock_guard<std::mutex> lock(g_tune_mutex);
        const auto it = g_tune_cost.find(key);
        if (it != g_tune_cost.end()) {
            return it->second;
        }
    }
    if (!scratch) {
        // Large enough for 512 x 64 x 64 (any axis) and 256 x 256 x 16 values.
        const std::size_t bytes = sizeof(float2) * 512ULL * 64 * 64;
        scratch = static_cast<float2*>(device_buffer(ctx, "tune.scratch", bytes, status));
        if (!scratch) {
            return -1.0;
        }
        cudaMemsetAsync(scratch, 0, bytes, ctx->stream);
    }
    const double cost = measure_pass(ctx, axis, L, scratch, status);
    if (cost >= 0) {
        std::lock_guard<std::mutex> lock(g_tune_mutex);
        g_tune_cost[key] = cost;
    }
    return cost;
}

}  // namespace

int Pipeline::choose_lengths(const std::uint32_t* env_shape)
{
    std::vector<int> cand[3];
    for (int a = 0; a < 3; ++a) {
        cand[a] = length_candidates(static_cast<int>(env_shape[a]), a);
        if (cand[a].empty()) {
            return kUnsupportedLength;
        }
    }
    if (cand[0].size() == 1 && cand[1].size() == 1 && cand[2].size() == 1) {
        for (int a = 0; a < 3; ++a) {
            L_[a] = cand[a][0];
        }
        return kOk;
    }
    int status = kOk;
    float2* scratch = nullptr;
    double best = INFINITY;
    std::vector<double> cost[3];
    for (int a = 0; a < 3; ++a) {
        for (int L : cand[a]) {
            const double c = pass_cost(ctx_, a, L, scratch, status);
            if (c < 0) {
                return status ? status : kCuda;
            }
            cost[a].push_back(c);
        }
    }
    for (std::size_t i = 0; i < cand[0].size(); ++i) {
        for (std::size_t j = 0; j < cand[1].size(); ++j) {
            for (std::size_t k = 0; k < cand[2].size(); ++k) {
                const double points = static_cast<double>(cand[0][i]) * cand[1][j] * cand[2][k];
                double model = points * (cost[0][i] + cost[1][j] + cost[2][k]);
                if (cand[0][i] == 256 && cand[1][j] == 256 && cand[2][k] == 256) {
                    const double reg = pass_cost(ctx_, -1, 256, scratch, status);
                    if (reg < 0) {
                        return status ? status : kCuda;
                    }
                    model = points * 3 * reg;
                }
                if (model < best) {
                    best = model;
                    L_[0] = cand[0][i];
                    L_[1] = cand[1][j];
                    L_[2] = cand[2][k];
                }
            }
        }
    }
    return kOk;
}

int Pipeline::set_geometry(const std::int64_t* env_first, const std::uint32_t* env_shape, const double* origin,
                           double pitch, double container_min_z, double container_height)
{
    for (int a = 0; a != 3; ++a) {
        if (env_shape[a] == 0) {
            return kInvalidArgument;
        }
        E_[a] = static_cast<int>(env_shape[a]);
        env_first_[a] = env_first[a];
        origin_[a] = origin[a];
    }
    if (const char* fixed = std::getenv("SPK_FFT_LENGTHS"); fixed && std::strcmp(fixed, "pow2") == 0) {
        for (int a = 0; a != 3; ++a) {
            const std::uint32_t L = next_pow2(std::max<std::uint32_t>(env_shape[a], 16));
            if (L > static_cast<std::uint32_t>(kMaxFftLength)) {
                return kUnsupportedLength;
            }
            L_[a] = static_cast<int>(L);
        }
    }
    else if (int status = choose_lengths(env_shape)) {
        return status;
    }
    pitch_ = pitch;
    cmin_z_ = container_min_z;
    height_ = container_height;
    const long long cells = static_cast<long long>(E_[0]) * E_[1] * E_[2];
    const long long grid = static_cast<long long>(L_[0]) * L_[1] * L_[2];
    int status = kOk;
    occ_ = static_cast<std::uint8_t*>(device_buffer(ctx_, "pipe.occ", cells, status));
    d2_ = static_cast<std::int32_t*>(device_buffer(ctx_, "pipe.d2", cells * sizeof(std::int32_t), status));
    spectrum_ = static_cast<float2*>(device_buffer(ctx_, "pipe.spectrum", grid * sizeof(float2), status));
    const long long tiles = static_cast<long long>((E_[0] + kEdtTile - 1) / kEdtTile) *
                            ((E_[1] + kEdtTile - 1) / kEdtTile) * ((E_[2] + kEdtTile - 1) / kEdtTile);
    tile_max_ = static_cast<std::int32_t*>(device_buffer(ctx_, "pipe.tile_max", tiles * sizeof(std::int32_t), status));
    if (!occ_ || !d2_ || !spectrum_ || !tile_max_) {
        return status;
    }
    const std::uint32_t shape[3] = { env_shape[0], env_shape[1], env_shape[2] };
    if (!proximity_shape_supported(shape)) {
        return kProximityShape;
    }
    table_ = proximity_table(ctx_, max_squared_distance(shape), status);
    return table_ ? kOk : status;
}

int Pipeline::set_occupancy(const std::uint8_t* d_occupancy)
{
    cudaStream_t st = ctx_->stream;
    const long long cells = static_cast<long long>(E_[0]) * E_[1] * E_[2];
    if (d_occupancy != occ_) {
        cudaMemcpyAsync(occ_, d_occupancy, cells, cudaMemcpyDeviceToDevice, st);
    }
    const std::uint32_t shape[3] = { static_cast<std::uint32_t>(E_[0]), static_cast<std::uint32_t>(E_[1]),
                                     static_cast<std::uint32_t>(E_[2]) };
    int status = edt_squared(ctx_, occ_, d2_, shape, st);
    if (status || (status = edt_tile_max(ctx_, d2_, shape, tile_max_, st))) {
        return status;
    }
    return update_spectrum();
}

int Pipeline::add_occupied(const std::uint8_t* d_occupancy, const std::uint8_t* d_sites, const EdtBox& sites)
{
    cudaStream_t st = ctx_->stream;
    const long long cells = static_cast<long long>(E_[0]) * E_[1] * E_[2];
    if (d_occupancy != occ_) {
        cudaMemcpyAsync(occ_, d_occupancy, cells, cudaMemcpyDeviceToDevice, st);
    }
    const std::uint32_t shape[3] = { static_cast<std::uint32_t>(E_[0]), static_cast<std::uint32_t>(E_[1]),
                                     static_cast<std::uint32_t>(E_[2]) };
    int status = edt_add_sites(ctx_, d_sites, sites, d2_, tile_max_, shape, st);
    if (status) {
        return status;
    }
    return update_spectrum();
}

int Pipeline::update_spectrum()
{
    cudaStream_t st = ctx_->stream;
    int status = kOk;
    const long long grid = static_cast<long long>(L_[0]) * L_[1] * L_[2];
    const bool reg256 = L_[0] == 256 && L_[1] == 256 && L_[2] == 256;
    const int blocks = reg256 ? 256 * 256 / 16 : launch_blocks(grid, 256);
    auto* partial = static_cast<double*>(device_buffer(ctx_, "pipe.norm", blocks * sizeof(double), status));
    if (!partial) {
        return status;
    }
    if (reg256) {
        const auto* tw = twiddle_table<float>(ctx_, 256, status);
        if (!tw) {
            return status;
        }
        env_row256_kernel<<<blocks, 256, 0, st>>>(spectrum_, E_[0], E_[1], E_[2], occ_, d2_, table_, tw, partial);
        env_column256_kernel<<<16 * 256, 256, 0, st>>>(spectrum_, 256, 65536, 1.f, tw);  // y
        env_column256_kernel<<<16 * 256, 256, 0, st>>>(spectrum_, 65536, 256,
                                                       static_cast<float>(1.0 / static_cast<double>(grid)), tw);  // z
        ctx_->launches += 3;
        if (cudaGetLastError() != cudaSuccess) {
            return kCuda;
        }
    }
    else {
        env_pack_kernel<<<blocks, 256, 0, st>>>(spectrum_, L_[0], L_[1], L_[2], E_[0], E_[1], E_[2], occ_, d2_, table_,
                                                 partial);
        ctx_->launches++;
        for (int axis = 0; axis != 3; ++axis) {
            const auto* tw = twiddle_table<float>(ctx_, L_[axis], status);
            if (!tw) {
                return status;
            }
            const float scale = axis == 2 ? static_cast<float>(1.0 / static_cast<double>(grid)) : 1.f;
            if (fft_axis<float>(spectrum_, L_[0], L_[1], L_[2], axis, false, scale, tw, st) != cudaSuccess) {
                return kCuda;
            }
            ctx_->launches++;
        }
    }
    // The partial sums of b^2 + p^2 come back to pinned memory; the host
    // adds them up (finish_norm) only when a page needs the error bound, so
    // nothing here waits for the device.
    auto* host = static_cast<double*>(host_buffer(ctx_, "pipe.norm", blocks * sizeof(double), status));
    if (!host) {
        return status;
    }
    cudaMemcpyAsync(host, partial, blocks * sizeof(double), cudaMemcpyDeviceToHost, st);
    norm_host_ = host;
    norm_blocks_ = blocks;
    norm_stream_ = st;
    norm_pending_ = true;
    return cudaGetLastError() == cudaSuccess ? kOk : kCuda;
}

int Pipeline::finish_norm()
{
    if (!norm_pending_) {
        return kOk;
    }
    if (cudaStreamSynchronize(norm_stream_) != cudaSuccess) {
        cudaGetLastError();
        return kCuda;
    }
    double sum = 0;
    for (int i = 0; i < norm_blocks_; ++i) {
        sum += norm_host_[i];
    }
    z_norm_ = std::sqrt(sum);
    norm_pending_ = false;
    return kOk;
}

int Pipeline::refresh_begin(const std::uint8_t* d_occupancy, const std::uint8_t* d_sites, const EdtBox* sites)
{
    refresh_order();
    if (!side_) {
        if (cudaStreamCreateWithFlags(&side_, cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventCreateWithFlags(&ev_in_, cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreateWithFlags(&ev_done_, cudaEventDisableTiming) != cudaSuccess) {
            cudaGetLastError();
            return kCuda;
        }
    }
    cudaStream_t main = ctx_->stream;
    cudaEventRecord(ev_in_, main);
    cudaStreamWaitEvent(side_, ev_in_, 0);
    // Every launch of the update goes to the side stream while it is queued.
    ctx_->stream = side_;
    const int status = d_sites ? add_occupied(d_occupancy, d_sites, *sites) : set_occupancy(d_occupancy);
    cudaEventRecord(ev_done_, side_);
    ctx_->stream = main;
    pending_ = true;
    return status;
}

void Pipeline::refresh_order()
{
    if (pending_) {
        cudaStreamWaitEvent(ctx_->stream, ev_done_, 0);
        pending_ = false;
    }
}

int Pipeline::add_kernel(std::uint64_t orientation, const std::int64_t* first, const std::uint32_t* shape,
                         const std::uint8_t* cells, double max_z, std::uint64_t& slot_out)
{
    KernelSlot s;
    s.orientation = orientation;
    std::uint64_t n = 1;
    for (int a = 0; a != 3; ++a) {
        s.K[a] = static_cast<int>(shape[a]);
        s.first[a] = first[a];
        s.legal[a] = E_[a] >= s.K[a] ? E_[a] - s.K[a] + 1 : 0;
        n *= shape[a];
    }
    s.max_z = max_z;
    s.host_cells.assign(cells, cells + n);
    std::vector<std::int32_t> ones;
    for (int z = 0; z < s.K[2]; ++z) {
        for (int y = 0; y < s.K[1]; ++y) {
            for (int x = 0; x < s.K[0]; ++x) {
                if (cells[x + static_cast<std::uint64_t>(s.K[0]) * (y + static_cast<std::uint64_t>(s.K[1]) * z)]) {
                    ones.push_back(x + E_[0] * (y + E_[1] * z));
                }
            }
        }
    }
    s.occupied = ones.size();
    const bool fits = s.legal[0] && s.legal[1] && s.legal[2];
    cudaStream_t st = ctx_->stream;
    int status = kOk;
    if (fits && !ones.empty()) {
        // The kernel must fit the FFT period: K <= E <= L always holds here.
        const long long partial_cells = static_cast<long long>(L_[0]) * L_[1] * s.K[2];
        if (cudaMalloc(&s.partial, partial_cells * sizeof(float2)) != cudaSuccess ||
            cudaMalloc(&s.ones, ones.size() * sizeof(std::int32_t)) != cudaSuccess ||
            cudaMalloc(&s.t65, s.legal[2] * sizeof(double)) != cudaSuccess) {
            cudaGetLastError();
            cudaFree(s.partial);
            cudaFree(s.ones);
            cudaFree(s.t65);
            return kAllocation;
        }
        cudaMemcpyAsync(s.ones, ones.data(), ones.size() * sizeof(std::int32_t), cudaMemcpyHostToDevice, st);
        std::vector<double> t65(s.legal[2]);
        for (int zi = 0; zi < s.legal[2]; ++zi) {
            const std::int64_t tz = env_first_[2] - s.first[2] + zi;
            const double world_z = origin_[2] + pitch_ * static_cast<double>(tz);
            const double top = (world_z + max_z - cmin_z_) / height_;
            t65[zi] = .65 * top;
        }
        cudaMemcpyAsync(s.t65, t65.data(), t65.size() * sizeof(double), cudaMemcpyHostToDevice, st);
        auto* d_cells = static_cast<std::uint8_t*>(device_buffer(ctx_, "pipe.kcells", n, status));
        if (!d_cells) {
            return status;
        }
        cudaMemcpyAsync(d_cells, cells, n, cudaMemcpyHostToDevice, st);
        kernel_pack_kernel<<<launch_blocks(partial_cells, 256), 256, 0, st>>>(s.partial, L_[0], L_[1], s.K[0],
                                                                               s.K[1], s.K[2], d_cells);
        ctx_->launches++;
        for (int axis = 0; axis != 2; ++axis) {
            const auto* tw = twiddle_table<float>(ctx_, L_[axis], status);
            if (!tw) {
                return status;
            }
            if (fft_axis<float>(s.partial, L_[0], L_[1], s.K[2], axis, false, 1.f, tw, st) != cudaSuccess) {
                return kCuda;
            }
            ctx_->launches++;
        }
        if (cudaStreamSynchronize(st) != cudaSuccess) {
            return kCuda;
        }
    }
    slot_out = slots_.size();
    slots_.push_back(std::move(s));
    return kOk;
}

double Pipeline::approx_epsilon(const KernelSlot& s) const
{
    // Error bound of the FP32 proximity sum: 2^-14 * log2(N) * |Z|_2 * sqrt(occ) / sqrt(N),
    // checked at run time against every exactly rescored candidate.
    const double n = static_cast<double>(L_[0]) * L_[1] * L_[2];
    const double eps_p = std::ldexp(1.0, -14) * std::log2(n) * z_norm_ * std::sqrt(static_cast<double>(s.occupied)) /
                         std::sqrt(n);
    return .35 * eps_p / static_cast<double>(s.occupied);
}

double Pipeline::epsilon_p(const KernelSlot& s) const
{
    return approx_epsilon(s) * static_cast<double>(s.occupied) / .35;
}

double Pipeline::score(const KernelSlot& s, const std::int64_t* t, double p) const
{
    // spectral_pipeline.cpp:1794-1800, evaluated in the same order.
    const double mean_proximity = p / static_cast<double>(s.occupied);
    const double world_z = origin_[2] + pitch_ * static_cast<double>(t[2]);
    const double top = (world_z + s.max_z - cmin_z_) / height_;
    return .65 * top - .35 * mean_proximity;
}

int Pipeline::run_orientation(const KernelSlot& s, int mode, float target, double threshold, double cursor_floor,
                              unsigned long long* keys, unsigned int* count, unsigned int cap,
                              unsigned long long* tau, unsigned long long* resid)
{
    cudaStream_t st = ctx_->stream;
    int status = kOk;
    const std::size_t inter = static_cast<std::size_t>(L_[0]) * L_[1] * s.legal[2] * sizeof(float2);
    if (inter > inter_bytes_) {
        inter_ = static_cast<float2*>(device_buffer(ctx_, "pipe.inter", inter, status));
        if (!inter_) {
            return status;
        }
        inter_bytes_ = inter;
    }
    static std::once_flag configured[64];
    once_per_device(configured, [] {
        allow_large_smem(pass_a_kernel);
        allow_large_smem(pass_b2_kernel);
    });
    const auto* tw0 = twiddle_table<float>(ctx_, L_[0], status);
    const auto* tw1 = twiddle_table<float>(ctx_, L_[1], status);
    const auto* tw2 = twiddle_table<float>(ctx_, L_[2], status);
    if (!tw0 || !tw1 || !tw2) {
        return status;
    }
    if (L_[0] == 256 && L_[1] == 256 && L_[2] == 256) {
        auto ev = pass_begin(ctx_);
        pass_a256_kernel<<<16 * 256, 256, 0, st>>>(spectrum_, s.partial, inter_, s.K[2], s.legal[2], tw2);
        pass_end(ctx_, 0, ev, pass_a_bytes(s));
        ctx_->launches++;
        return run_b256(s, inter_, mode, target, threshold, cursor_floor, keys, count, cap, tau, resid);
    }
    const std::size_t smem_a = sizeof(float2) * (L_[2] + 2 * kColumnGroup * (L_[2] + 1) + kColumnGroup * L_[2]);
    auto ev = pass_begin(ctx_);
    pass_a_kernel<<<(L_[0] / kColumnGroup) * L_[1], 256, smem_a, st>>>(spectrum_, s.partial, inter_, L_[0], L_[1],
                                                                        L_[2], s.K[2], s.legal[2], tw2);
    pass_end(ctx_, 0, ev);
    ctx_->launches++;
    ev = pass_begin(ctx_);
    if (fft_axis<float>(inter_, L_[0], L_[1], s.legal[2], 1, true, 1.f, tw1, st, s.legal[1]) != cudaSuccess) {
        return kCuda;
    }
    pass_end(ctx_, 1, ev);
    ctx_->launches++;
    const long long rows = static_cast<long long>(s.legal[1]) * s.legal[2];
    const std::size_t smem_b = sizeof(float2) * (L_[0] + 2 * kB2Rows * (L_[0] + 1));
    ev = pass_begin(ctx_);
    pass_b2_kernel<<<static_cast<unsigned>((rows + kB2Rows - 1) / kB2Rows), 32 * kB2Rows, smem_b, st>>>(
        inter_, L_[0], L_[1], s.legal[0], s.legal[1], s.legal[2], tw0, s.t65, 1.0 / static_cast<double>(s.occupied),
        mode, target, threshold, cursor_floor, keys, count, cap, tau, resid);
    pass_end(ctx_, 2, ev);
    ctx_->launches++;
    return cudaGetLastError() == cudaSuccess ? kOk : kCuda;
}

double Pipeline::pass_a_bytes(const KernelSlot& s) const
{
    const double plane = static_cast<double>(L_[0]) * L_[1] * sizeof(float2);
    return plane * L_[2] + plane * (s.K[2] + s.legal[2]);
}

double Pipeline::fill_a256(const KernelSlot* const* slots, int count, float2* const* inter, PassABatch& batch) const
{
    batch = {};
    batch.count = count;
    const double spectrum_bytes = static_cast<double>(L_[0]) * L_[1] * L_[2] * sizeof(float2);
    double bytes = spectrum_bytes;
    for (int i = 0; i < count; ++i) {
        batch.slot[i] = { slots[i]->partial, inter[i], slots[i]->K[2], slots[i]->legal[2] };
        bytes += pass_a_bytes(*slots[i]) - spectrum_bytes;
    }
    return bytes;
}

void Pipeline::fill_b256(const KernelSlot* const* slots, int count, float2* const* inter, const PassBSlot* outputs,
                         PassBBatch& b1, PassBBatch& b2, int& blocks1, int& blocks2, double& bytes1,
                         double& bytes2) const
{
    b1 = {};
    b2 = {};
    b1.count = b2.count = count;
    blocks1 = blocks2 = 0;
    bytes1 = bytes2 = 0.0;
    for (int g = 0; g < count; ++g) {
        const KernelSlot& s = *slots[g];
        PassBSlot slot = outputs[g];
        slot.inter = inter[g];
        slot.t65 = s.t65;
        slot.inv_occ = 1.0 / static_cast<double>(s.occupied);
        slot.legal_x = s.legal[0];
        slot.legal_y = s.legal[1];
        slot.legal_z = s.legal[2];
        slot.first_block = blocks1;
        b1.slot[g] = slot;
        blocks1 += 16 * s.legal[2];
        b2.slot[g] = slot;
        const long long rows = static_cast<long long>(s.legal[1]) * s.legal[2];
        blocks2 += static_cast<int>((rows + 15) / 16);
        const double legal_rows = static_cast<double>(rows);
        bytes1 += 8.0 * L_[0] * L_[1] * s.legal[2] + 8.0 * L_[0] * legal_rows;
        bytes2 += 8.0 * L_[0] * legal_rows;
    }
    // Pass B2 visits the orientations round-robin: each orientation's
    // pruning bound (tau) is lowered by its first blocks to finish, and
    // slot-by-slot order would start every orientation with a full wave of
    // blocks that run before any bound exists.
    int min_blocks = count ? 1 << 30 : 0;
    for (int g = 0; g < count; ++g) {
        const long long rows = static_cast<long long>(slots[g]->legal[1]) * slots[g]->legal[2];
        min_blocks = std::min(min_blocks, static_cast<int>((rows + 15) / 16));
    }
    b2.min_blocks = min_blocks;
    b2.interleaved = count * min_blocks;
    int first = b2.interleaved;
    for (int g = 0; g < count; ++g) {
        const long long rows = static_cast<long long>(slots[g]->legal[1]) * slots[g]->legal[2];
        b2.slot[g].first_block = first;
        first += static_cast<int>((rows + 15) / 16) - min_blocks;
    }
}

int Pipeline::run_a256_batch(const KernelSlot* const* slots, int count, float2* const* inter)
{
    int status = kOk;
    const auto* tw2 = twiddle_table<float>(ctx_, L_[2], status);
    if (!tw2) {
        return status;
    }
    PassABatch batch {};
    const double bytes = fill_a256(slots, count, inter, batch);
    auto ev = pass_begin(ctx_);
    static std::once_flag a_configured[64];
    once_per_device(a_configured, [] {
        cudaFuncSetAttribute(pass_a256_batch_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             static_cast<int>(kPassASmem));
    });
    pass_a256_batch_kernel<<<16 * 256, 256, kPassASmem, ctx_->stream>>>(spectrum_, batch, tw2);
    pass_end(ctx_, 0, ev, bytes);
    ctx_->launches++;
    return cudaGetLastError() == cudaSuccess ? kOk : kCuda;
}

int Pipeline::run_b256_batch(const KernelSlot* const* slots, int count, float2* const* inter,
                             const PassBSlot* outputs)
{
    cudaStream_t st = ctx_->stream;
    int status = kOk;
    const auto* tw0 = twiddle_table<float>(ctx_, L_[0], status);
    const auto* tw1 = twiddle_table<float>(ctx_, L_[1], status);
    if (!tw0 || !tw1) {
        return status;
    }
    PassBBatch b1 {}, b2 {};
    int blocks1 = 0, blocks2 = 0;
    double bytes1 = 0.0, bytes2 = 0.0;
    fill_b256(slots, count, inter, outputs, b1, b2, blocks1, blocks2, bytes1, bytes2);
    auto ev = pass_begin(ctx_);
    pass_b1_256_batch_kernel<<<blocks1, 256, 0, st>>>(b1, tw1);
    pass_end(ctx_, 1, ev, bytes1);
    ev = pass_begin(ctx_);
    pass_b2_256_batch_kernel<<<blocks2, 256, 0, st>>>(b2, tw0);
    pass_end(ctx_, 2, ev, bytes2);
    ctx_->launches += 2;
    return cudaGetLastError() == cudaSuccess ? kOk : kCuda;
}

int Pipeline::run_stages256(const std::vector<StageBatch>& batches, float2* const* inter, std::size_t stride)
{
    int status = kOk;
    const auto* tw = twiddle_table<float>(ctx_, 256, status);
    if (!tw) {
        return status;
    }
    static std::once_flag configured[64];
    once_per_device(configured, [] {
        cudaFuncSetAttribute(pass_stage256_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             static_cast<int>(kPassASmem));
    });
    const std::size_t nb = batches.size();
    // Intermediates of batch k: inter[k % 3] + g * stride for its orientation g.
    auto outs_of = [&](std::size_t k, float2** outs) {
        for (int g = 0; g < batches[k].count; ++g) {
            outs[g] = inter[k % 3] + g * stride;
        }
    };
    for (std::size_t stage = 0; stage < nb + 2; ++stage) {
        PassStage p {};
        p.spectrum = spectrum_;
        double bytes = 0.0;
        int blocks_b1 = 0, blocks_b2 = 0;
        float2* outs[kPassABatch];
        if (stage < nb) {
            outs_of(stage, outs);
            bytes += fill_a256(batches[stage].slots, batches[stage].count, outs, p.a);
            p.blocks_a = 16 * 256;
        }
        if (stage >= 1 && stage - 1 < nb) {
            const StageBatch& sb = batches[stage - 1];
            PassBBatch unused {};
            int unused_blocks = 0;
            double b1_bytes = 0.0, unused_bytes = 0.0;
            outs_of(stage - 1, outs);
            fill_b256(sb.slots, sb.count, outs, sb.outputs, p.b1, unused, blocks_b1, unused_blocks, b1_bytes,
                      unused_bytes);
            bytes += b1_bytes;
        }
        if (stage >= 2) {
            const StageBatch& sb = batches[stage - 2];
            PassBBatch unused {};
            int unused_blocks = 0;
            double b2_bytes = 0.0, unused_bytes = 0.0;
            outs_of(stage - 2, outs);
            fill_b256(sb.slots, sb.count, outs, sb.outputs, unused, p.b2, unused_blocks, blocks_b2, unused_bytes,
                      b2_bytes);
            bytes += b2_bytes;
        }
        p.blocks_b1 = static_cast<unsigned int>(blocks_b1);
        const unsigned int blocks = p.blocks_a + p.blocks_b1 + static_cast<unsigned int>(blocks_b2);
        if (!blocks) {
            continue;
        }
        auto ev = pass_begin(ctx_);
        pass_stage256_kernel<<<blocks, 256, kPassASmem, ctx_->stream>>>(p, tw);
        pass_end(ctx_, 4, ev, bytes);
        ctx_->launches++;
        if (cudaGetLastError() != cudaSuccess) {
            return kCuda;
        }
    }
    return kOk;
}

int Pipeline::run_b256(const KernelSlot& s, float2* inter, int mode, float target, double threshold, double cursor_floor,
                       unsigned long long* keys, unsigned int* count, unsigned int cap, unsigned long long* tau,
                       unsigned long long* resid)
{
    cudaStream_t st = ctx_->stream;
    int status = kOk;
    const auto* tw0 = twiddle_table<float>(ctx_, L_[0], status);
    const auto* tw1 = twiddle_table<float>(ctx_, L_[1], status);
    if (!tw0 || !tw1) {
        return status;
    }
    // Algorithmic bytes: B1 reads the legal-z planes and writes their legal
    // rows; B2 reads those rows (its keys are a few KB).  Fused, the planes
    // are read once and nothing else crosses HBM.
    const double legal_rows = static_cast<double>(s.legal[1]) * s.legal[2];
    if (fused_b_) {
        static std::once_flag configured[64];
        once_per_device(configured, [] {
            cudaFuncSetAttribute(pass_b_fused_256_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(kFusedSmem));
        });
        auto ev = pass_begin(ctx_);
        pass_b_fused_256_kernel<<<kFusedCluster * s.legal[2], 256, kFusedSmem, st>>>(
            inter, s.legal[0], s.legal[1], tw1, s.t65, 1.0 / static_cast<double>(s.occupied), mode, target, threshold,
            cursor_floor, keys, count, cap, tau, resid);
        pass_end(ctx_, 2, ev, 8.0 * L_[0] * L_[1] * s.legal[2]);
        ctx_->launches++;
        return cudaGetLastError() == cudaSuccess ? kOk : kCuda;
    }
    auto ev = pass_begin(ctx_);
    pass_b1_256_kernel<<<16 * s.legal[2], 256, 0, st>>>(inter, s.legal[1], tw1);
    pass_end(ctx_, 1, ev, 8.0 * L_[0] * L_[1] * s.legal[2] + 8.0 * L_[0] * legal_rows);
    const long long rows = static_cast<long long>(s.legal[1]) * s.legal[2];
    ev = pass_begin(ctx_);
    pass_b2_256_kernel<<<static_cast<unsigned>((rows + 15) / 16), 256, 0, st>>>(
        inter, s.legal[0], s.legal[1], s.legal[2], tw0, s.t65, 1.0 / static_cast<double>(s.occupied), mode, target,
        threshold, cursor_floor, keys, count, cap, tau, resid);
    pass_end(ctx_, 2, ev, 8.0 * L_[0] * legal_rows);
    ctx_->launches += 2;
    return cudaGetLastError() == cudaSuccess ? kOk : kCuda;
}

int Pipeline::pages(const std::vector<PageRequest>& requests, std::vector<PageOutcome>& out, bool full)
{
    refresh_order();
    if (int status = finish_norm()) {
        return status;
    }
    std::vector<std::size_t> ordinary;
    for (std::size_t r = 0; r < requests.size(); ++r) {
        if (!requests[r].low_overlap) {
            ordinary.push_back(r);
        }
    }
    if (ordinary.size() == requests.size()) {
        return ordinary_pages(requests, out, full);
    }
    out.assign(requests.size(), {});
    if (!ordinary.empty()) {
        std::vector<PageRequest> sub;
        for (std::size_t r : ordinary) {
            sub.push_back(requests[r]);
        }
        std::vector<PageOutcome> sub_out;
        if (int status = ordinary_pages(sub, sub_out, full)) {
            return status;
        }
        for (std::size_t i = 0; i < ordinary.size(); ++i) {
            out[ordinary[i]] = std::move(sub_out[i]);
        }
    }
    for (std::size_t r = 0; r < requests.size(); ++r) {
        if (requests[r].low_overlap) {
            if (int status = low_overlap_page(requests[r], out[r])) {
                return status;
            }
        }
    }
    return kOk;
}

// A low-overlap page (spectral_pipeline.cpp:1758-1824, mode low_overlap):
// the 32 legal translations after the cursor that are smallest by
// (rounded overlap count, score, z, y, x), over every legal translation, with
// no recount (direct_zero_overlap stays false).  A histogram pass counts the
// translations per rounded overlap; then, from the cursor's count upward,
// each count with translations contributes its certified ordinary-style page
// (candidates: overlap == that count) until 32 entries are gathered.  Counts
// of kOverlapBins - 1 and above share the last bin; a page that would need
// them fails with SPK_SCRATCH_LIMIT.
int Pipeline::low_overlap_page(const PageRequest& req, PageOutcome& out)
{
    out = {};
    const auto& s = slots_[req.slot];
    if (!s.legal[0] || !s.legal[1] || !s.legal[2]) {
        out.certified = true;
        return kOk;
    }
    if (!s.occupied) {
        out.status = kEmptyKernel;
        return kOk;
    }
    constexpr unsigned int kOverlapBins = 4096;
    cudaStream_t st = ctx_->stream;
    int status = kOk;
    auto* hist = static_cast<unsigned int*>(device_buffer(ctx_, "pipe.overlap_hist", kOverlapBins * 4, status));
    auto* meta = static_cast<unsigned long long*>(device_buffer(ctx_, "pipe.overlap_meta", 24, status));
    if (!hist || !meta) {
        return status;
    }
    cudaMemsetAsync(hist, 0, kOverlapBins * 4, st);
    cudaMemsetAsync(meta, 0, 24, st);
    if ((status = run_orientation(s, 2, 0.f, 0.0, -INFINITY, reinterpret_cast<unsigned long long*>(hist),
                                  reinterpret_cast<unsigned int*>(meta + 2), kOverlapBins, meta, meta + 1))) {
        return status;
    }
    std::vector<unsigned int> h(kOverlapBins);
    unsigned long long h_meta[3] {};
    cudaMemcpyAsync(h.data(), hist, kOverlapBins * 4, cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(h_meta, meta, 24, cudaMemcpyDeviceToHost, st);
    if (cudaStreamSynchronize(st) != cudaSuccess) {
        cudaGetLastError();
        return kCuda;
    }
    std::uint32_t rbits = static_cast<std::uint32_t>(h_meta[1]);
    float rf;
    std::memcpy(&rf, &rbits, 4);
    out.max_integer_residual = rf;
    if (rf >= 0.25f) {
        out.status = kNumeric;  // correlation.cpp:521-528 residual guard
        return kOk;
    }
    // The cursor's overlap is a rounded count held as a double.
    const std::uint32_t first =
        req.has_cursor ? static_cast<std::uint32_t>(std::max(0.0, std::nearbyint(req.cursor.binary_overlap))) : 0u;
    for (std::uint32_t c = first; c < kOverlapBins && out.page.size() < static_cast<std::size_t>(kPageSize); ++c) {
        if (h[c] == 0) {
            continue;
        }
        if (c == kOverlapBins - 1) {
            out.status = kScratchLimit;  // the counts beyond the histogram are not resolved
            return kOk;
        }
        PageRequest bin = req;
        bin.low_overlap = false;
        bin.overlap = c;
        bin.has_cursor = req.has_cursor && c == first;
        std::vector<PageOutcome> bin_out;
        if ((status = ordinary_pages({ bin }, bin_out, true))) {
            return status;
        }
        if (bin_out[0].status) {
            out.status = bin_out[0].status;
            return kOk;
        }
        out.rescored += bin_out[0].rescored;
        out.max_score_error = std::max(out.max_score_error, bin_out[0].max_score_error);
        for (auto& candidate : bin_out[0].page) {
            if (out.page.size() == static_cast<std::size_t>(kPageSize)) {
                break;
            }
            candidate.direct_zero = false;
            out.page.push_back(candidate);
        }
    }
    out.certified = true;
    out.exact_floor = INFINITY;
    return kOk;
}

int Pipeline::ordinary_pages(const std::vector<PageRequest>& requests, std::vector<PageOutcome>& out, bool full)
{
    const int R = static_cast<int>(requests.size());
    out.assign(R, {});
    if (R == 0) {
        return kOk;
    }
    cudaStream_t st = ctx_->stream;
    int status = kOk;
    const int per = kExactPerOrientation + 1;
    // 256^3 grids: each pass-B2 block emits the keys of its histogram bins up
    // to the one where 64 accumulate (about 64), below the pruning bound, so
    // 64 x 4096 keys cover a request; only heavy exact ties could exceed that,
    // and an overflowing page is then left uncertified and widened.  Other
    // grids keep kKeyCapacity.
    const bool large = L_[0] == 256 && L_[1] == 256 && L_[2] == 256;
    const unsigned int cap = large ? kLargeKeyChunks * kKeyCapacity : kKeyCapacity;
    auto* keys = static_cast<unsigned long long*>(
        device_buffer(ctx_, "pipe.keys", static_cast<std::size_t>(R) * cap * 8, status));
    auto* partial = large ? static_cast<unsigned long long*>(device_buffer(
                                ctx_, "pipe.partial", static_cast<std::size_t>(R) * kLargeKeyChunks * per * 8, status))
                          : nullptr;
    auto* meta = static_cast<unsigned long long*>(device_buffer(ctx_, "pipe.meta", static_cast<std::size_t>(R) * 24,
                                                                status));
    auto* selected = static_cast<unsigned long long*>(
        device_buffer(ctx_, "pipe.selected", static_cast<std::size_t>(R) * per * 8, status));
    auto* jobs = static_cast<ExactJob*>(device_buffer(ctx_, "pipe.jobs", R * sizeof(ExactJob), status));
    auto* counts_out = static_cast<long long*>(
        device_buffer(ctx_, "pipe.ecount", static_cast<std::size_t>(R) * per * 8, status));
    auto* p_out = static_cast<double*>(device_buffer(ctx_, "pipe.ep", static_cast<std::size_t>(R) * per * 8, status));
    auto* range_error = static_cast<int*>(device_buffer(ctx_, "pipe.rangeerr", 16, status));
    if (!keys || !meta || !selected || !jobs || !counts_out || !p_out || !range_error || (large && !partial)) {
        return status;
    }
    // meta layout: tau[R] (u64), resid[R] (u64), count[R] (u32, in the last third as u64 slots)
    unsigned long long* tau = meta;
    unsigned long long* resid = meta + R;
    auto* count = reinterpret_cast<unsigned int*>(meta + 2 * R);
    std::vector<unsigned long long> init(3 * R, 0);
    for (int r = 0; r < R; ++r) {
        init[r] = kEmptyKey;
    }
    cudaMemcpyAsync(meta, init.data(), init.size() * 8, cudaMemcpyHostToDevice, st);
    cudaMemsetAsync(range_error, 0, 16, st);
    std::vector<ExactJob> host_jobs(R);
    std::vector<double> eps_s(R), floor(R);
    std::vector<int> runnable;
    for (int r = 0; r < R; ++r) {
        const auto& s = slots_[requests[r].slot];
        host_jobs[r] = { s.ones, static_cast<int>(s.occupied), std::max(s.legal[0], 1), std::max(s.legal[1], 1) };
        if (!s.legal[0] || !s.legal[1] || !s.legal[2] || !s.occupied) {
            continue;
        }
        eps_s[r] = approx_epsilon(s) + std::ldexp(1.0, -22);
        floor[r] = requests[r].has_cursor ? requests[r].cursor.score - eps_s[r] : -INFINITY;
        runnable.push_back(r);
    }
    // The pipelined schedule holds up to three batches' intermediates at once;
    // where the device memory cap does not allow that, the passes run one
    // launch each on one batch's intermediate.
    const std::size_t stride = static_cast<std::size_t>(L_[0]) * L_[1] * L_[2];
    const std::size_t batch_size = std::min<std::size_t>(kPassABatch, runnable.size());
    const std::size_t batches = (runnable.size() + kPassABatch - 1) / kPassABatch;
    float2* staged_inter = nullptr;
    const std::size_t copies = std::min<std::size_t>(batches, 3);
    if (large && staged_ && !fused_b_ && batches) {
        int alloc_status = kOk;
        staged_inter = static_cast<float2*>(device_buffer(
            ctx_, "pipe.inter_batch", copies * batch_size * stride * sizeof(float2), alloc_status));
    }
    if (staged_inter) {
        std::vector<StageBatch> work(batches);
        for (std::size_t k = 0; k < work.size(); ++k) {
            StageBatch& sb = work[k];
            sb = {};
            sb.count = static_cast<int>(std::min<std::size_t>(kPassABatch, runnable.size() - k * kPassABatch));
            for (int g = 0; g < sb.count; ++g) {
                const int r = runnable[k * kPassABatch + g];
                sb.slots[g] = &slots_[requests[r].slot];
                PassBSlot& t = sb.outputs[g];
                t.keys = keys + static_cast<long long>(r) * cap;
                t.count = count + r;
                t.cap = cap;
                t.tau = tau + r;
                t.resid = resid + r;
                t.target = static_cast<float>(requests[r].overlap);
                t.cursor_floor = floor[r];
            }
        }
        float2* rotation[3] = { nullptr, nullptr, nullptr };
        for (std::size_t c = 0; c < copies; ++c) {
            rotation[c] = staged_inter + c * batch_size * stride;
        }
        if ((status = run_stages256(work, rotation, stride))) {
            return status;
        }
    }
    else if (large) {
        // Pass A in batches of kPassABatch orientations, each batch followed by
        // the batch's B passes.
        auto* inter = static_cast<float2*>(
            device_buffer(ctx_, "pipe.inter_batch", batch_size * stride * sizeof(float2), status));
        if (!inter) {
            return status;
        }
        for (std::size_t i0 = 0; i0 < runnable.size(); i0 += kPassABatch) {
            const int n = static_cast<int>(std::min<std::size_t>(kPassABatch, runnable.size() - i0));
            const KernelSlot* group[kPassABatch];
            float2* outs[kPassABatch];
            for (int g = 0; g < n; ++g) {
                group[g] = &slots_[requests[runnable[i0 + g]].slot];
                outs[g] = inter + g * stride;
            }
            if ((status = run_a256_batch(group, n, outs))) {
                return status;
            }
            if (!fused_b_) {
                PassBSlot targets[kPassABatch] {};
                for (int g = 0; g < n; ++g) {
                    const int r = runnable[i0 + g];
                    targets[g].keys = keys + static_cast<long long>(r) * cap;
                    targets[g].count = count + r;
                    targets[g].cap = cap;
                    targets[g].tau = tau + r;
                    targets[g].resid = resid + r;
                    targets[g].target = static_cast<float>(requests[r].overlap);
                    targets[g].cursor_floor = floor[r];
                }
                if ((status = run_b256_batch(group, n, outs, targets))) {
                    return status;
                }
                continue;
            }
            for (int g = 0; g < n; ++g) {
                const int r = runnable[i0 + g];
                if ((status = run_b256(*group[g], outs[g], 0, static_cast<float>(requests[r].overlap), 0.0, floor[r],
                                       keys + static_cast<long long>(r) * cap, count + r, cap, tau + r,
                                       resid + r))) {
                    return status;
                }
            }
        }
    }
    else {
        for (std::size_t i = 0; i < runnable.size(); ++i) {
            const int r = runnable[i];
            const auto& s = slots_[requests[r].slot];
            if ((status = run_orientation(s, 0, static_cast<float>(requests[r].overlap), 0.0, floor[r],
                                          keys + static_cast<long long>(r) * cap, count + r, cap, tau + r,
                                          resid + r))) {
                return status;
            }
        }
    }
    cudaMemcpyAsync(jobs, host_jobs.data(), R * sizeof(ExactJob), cudaMemcpyHostToDevice, st);
    auto ev = pass_begin(ctx_);
    if (large) {
        merge_chunk_kernel<<<dim3(kLargeKeyChunks, R), 1024, 0, st>>>(keys, cap, count, partial);
        static_assert(kLargeKeyChunks <= 64, "merge_lists_kernel holds one list head per thread of 64");
        merge_lists_kernel<<<R, 64, 0, st>>>(partial, kLargeKeyChunks, per, selected);
        ctx_->launches++;
    }
    else {
        merge_kernel<<<R, 1024, kKeyCapacity * 8, st>>>(keys, cap, count, kKeyCapacity, selected);
    }
    exact_kernel<<<R * per, 256, 0, st>>>(selected, jobs, per, occ_, d2_, table_, E_[0], E_[1], counts_out, p_out,
                                          range_error);
    pass_end(ctx_, 3, ev);
    ctx_->launches += 2;
    std::vector<unsigned long long> h_meta(3 * R), h_sel(static_cast<std::size_t>(R) * per);
    std::vector<long long> h_count(static_cast<std::size_t>(R) * per);
    std::vector<double> h_p(static_cast<std::size_t>(R) * per);
    int h_range = 0;
    cudaMemcpyAsync(h_meta.data(), meta, h_meta.size() * 8, cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(h_sel.data(), selected, h_sel.size() * 8, cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(h_count.data(), counts_out, h_count.size() * 8, cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(h_p.data(), p_out, h_p.size() * 8, cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(&h_range, range_error, 4, cudaMemcpyDeviceToHost, st);
    if (cudaStreamSynchronize(st) != cudaSuccess) {
        cudaGetLastError();
        return kCuda;
    }
    if (h_range) {
        return kNumericRange;
    }
    const auto* h_count32 = reinterpret_cast<const unsigned int*>(h_meta.data() + 2 * R);
    for (int r = 0; r < R; ++r) {
        const auto& req = requests[r];
        const auto& s = slots_[req.slot];
        auto& o = out[r];
        if (!s.legal[0] || !s.legal[1] || !s.legal[2]) {
            o.certified = true;  // kernel wider than the environment: complete, empty page
            continue;
        }
        if (!s.occupied) {
            o.status = kEmptyKernel;
            continue;
        }
        std::uint32_t rbits = static_cast<std::uint32_t>(h_meta[R + r]);
        float rf;
        std::memcpy(&rf, &rbits, 4);
        o.max_integer_residual = rf;
        if (rf >= 0.25f) {
            o.status = kNumeric;  // correlation.cpp:521-528 residual guard
            continue;
        }
        const unsigned int n = h_count32[r];
        const unsigned long long tau_r = h_meta[r];
        std::vector<Candidate> all;
        double max_error = 0;
        const std::int64_t legal_first[3] = { env_first_[0] - s.first[0], env_first_[1] - s.first[1],
                                              env_first_[2] - s.first[2] };
        const int m = static_cast<int>(std::min<unsigned int>(n, kExactPerOrientation));
        for (int i = 0; i < m; ++i) {
            const unsigned long long key = h_sel[static_cast<std::size_t>(r) * per + i];
            const long long overlap = h_count[static_cast<std::size_t>(r) * per + i];
            const double p = h_p[static_cast<std::size_t>(r) * per + i];
            const unsigned int index = static_cast<unsigned int>(key & 0xffffffffULL);
            Candidate c {};
            c.t[0] = legal_first[0] + index % s.legal[0];
            c.t[1] = legal_first[1] + (index / s.legal[0]) % s.legal[1];
            c.t[2] = legal_first[2] + index / (static_cast<unsigned int>(s.legal[0]) * s.legal[1]);
            c.orientation = s.orientation;
            c.score = score(s, c.t, p);
            c.binary_overlap = static_cast<double>(overlap);
            c.direct_zero = overlap == 0;
            const double approx = decode_key_score(key);
            max_error = std::max(max_error, std::fabs(approx - c.score));
            ++o.rescored;
            if (overlap != static_cast<long long>(req.overlap)) {
                continue;  // the reference's FFT rounding never admits these
            }
            if (req.has_cursor && !rank_less(req.cursor, c)) {
                continue;
            }
            all.push_back(c);
        }
        o.max_score_error = max_error;
        if (max_error > eps_s[r]) {
            o.status = kNumeric;  // the FP32 bound did not hold: fail closed
            continue;
        }
        std::sort(all.begin(), all.end(), rank_less);
        if (all.size() > static_cast<std::size_t>(kPageSize)) {
            all.resize(kPageSize);
        }
        unsigned long long excluded = kEmptyKey;
        if (n > cap) {
            excluded = 0;  // overflowed: nothing can be certified
        }
        else {
            if (n > static_cast<unsigned int>(kExactPerOrientation)) {
                excluded = h_sel[static_cast<std::size_t>(r) * per + kExactPerOrientation];
            }
            excluded = std::min(excluded, tau_r);
        }
        bool certified;
        if (excluded == kEmptyKey) {
            certified = true;
        }
        else if (all.size() == static_cast<std::size_t>(kPageSize)) {
            certified = excluded != 0 && decode_key_score(excluded) - eps_s[r] > all.back().score;
        }
        else {
            certified = false;
        }
        o.page = std::move(all);
        o.certified = certified;
        ++stat_pages;
        stat_first_certified += certified ? 1 : 0;
        stat_rescored += o.rescored;
        o.exact_floor = excluded == kEmptyKey ? INFINITY
                        : excluded == 0      ? -INFINITY
                                             : decode_key_score(excluded) - eps_s[r];
        // Starting bound for a threshold pass over a page that is not full:
        // the lowest excluded approximate score, or the last rescored one.
        double start = m > 0 ? decode_key_score(h_sel[static_cast<std::size_t>(r) * per + m - 1]) : -INFINITY;
        if (excluded != kEmptyKey && excluded != 0) {
            start = std::max(start, decode_key_score(excluded));
        }
        o.excluded_score = start;
        if (std::getenv("SPK_DEBUG_PAGES")) {
            std::fprintf(stderr, "page r=%d n=%u tau=%llx m=%d page=%zu certified=%d eps=%g err=%g start=%.17g\n", r,
                         n, tau_r, m, o.page.size(), certified ? 1 : 0, eps_s[r], max_error, start);
        }
    }
    // Threshold passes for every uncertified page (each recomputes that
    // orientation): collect every candidate whose approximate score is <= T,
    // rescore all of them exactly, and widen T until the page is certified.
    for (int r = 0; r < R && full; ++r) {
        auto& o = out[r];
        if (o.status || o.certified) {
            continue;
        }
        const auto& req = requests[r];
        const auto& s = slots_[req.slot];
        const std::int64_t legal_first[3] = { env_first_[0] - s.first[0], env_first_[1] - s.first[1],
                                              env_first_[2] - s.first[2] };
        // Everything left out of a threshold pass has approximate score > T, so
        // exact score > T - eps; T = S32 + 2 eps certifies a page whose 32nd
        // entry did not get worse.
        double threshold = o.page.size() == static_cast<std::size_t>(kPageSize)
                               ? o.page.back().score + 2 * eps_s[r]
                               : o.excluded_score + 2 * eps_s[r];
        double widen = std::max(4 * eps_s[r], 1e-6);
        unsigned int cap = kKeyCapacity;
        for (int attempt = 0; attempt < 24 && !o.certified; ++attempt) {
            auto* tkeys = static_cast<unsigned long long*>(device_buffer(ctx_, "pipe.tkeys", cap * 8ULL, status));
            if (!tkeys) {
                return status;
            }
            unsigned long long zero[3] = { 0, 0, 0 };
            cudaMemcpyAsync(meta, zero, 24, cudaMemcpyHostToDevice, st);
            if ((status = run_orientation(s, 1, static_cast<float>(req.overlap), threshold, floor[r], tkeys,
                                          reinterpret_cast<unsigned int*>(meta + 2), cap, meta, meta + 1))) {
                return status;
            }
            ++stat_threshold_passes;
            unsigned long long h[3];
            cudaMemcpyAsync(h, meta, 24, cudaMemcpyDeviceToHost, st);
            if (cudaStreamSynchronize(st) != cudaSuccess) {
                return kCuda;
            }
            const unsigned int n = static_cast<unsigned int>(h[2] & 0xffffffffULL);
            const unsigned long long total = h[0];
            if (n > cap) {
                cap = n + 1024;
                --attempt;
                continue;
            }
            std::vector<Candidate> all;
            if (n) {
                auto* tcount = static_cast<long long*>(device_buffer(ctx_, "pipe.tcount", n * 8ULL, status));
                auto* tp = static_cast<double*>(device_buffer(ctx_, "pipe.tp", n * 8ULL, status));
                if (!tcount || !tp) {
                    return status;
                }
                ExactJob job { s.ones, static_cast<int>(s.occupied), s.legal[0], s.legal[1] };
                cudaMemcpyAsync(jobs, &job, sizeof(job), cudaMemcpyHostToDevice, st);
                exact_kernel<<<n, 256, 0, st>>>(tkeys, jobs, static_cast<int>(n), occ_, d2_, table_, E_[0], E_[1],
                                                tcount, tp, range_error);
                ctx_->launches++;
                std::vector<unsigned long long> hk(n);
                std::vector<long long> cnt(n);
                std::vector<double> pv(n);
                cudaMemcpyAsync(hk.data(), tkeys, n * 8ULL, cudaMemcpyDeviceToHost, st);
                cudaMemcpyAsync(cnt.data(), tcount, n * 8ULL, cudaMemcpyDeviceToHost, st);
                cudaMemcpyAsync(pv.data(), tp, n * 8ULL, cudaMemcpyDeviceToHost, st);
                if (cudaStreamSynchronize(st) != cudaSuccess) {
                    return kCuda;
                }
                for (unsigned int i = 0; i < n; ++i) {
                    const unsigned int index = static_cast<unsigned int>(hk[i] & 0xffffffffULL);
                    Candidate c {};
                    c.t[0] = legal_first[0] + index % s.legal[0];
                    c.t[1] = legal_first[1] + (index / s.legal[0]) % s.legal[1];
                    c.t[2] = legal_first[2] + index / (static_cast<unsigned int>(s.legal[0]) * s.legal[1]);
                    c.orientation = s.orientation;
                    c.score = score(s, c.t, pv[i]);
                    c.binary_overlap = static_cast<double>(cnt[i]);
                    c.direct_zero = cnt[i] == 0;
                    o.max_score_error = std::max(o.max_score_error, std::fabs(decode_key_score(hk[i]) - c.score));
                    ++o.rescored;
                    if (cnt[i] != static_cast<long long>(req.overlap) || (req.has_cursor && !rank_less(req.cursor, c))) {
                        continue;
                    }
                    all.push_back(c);
                }
            }
            if (o.max_score_error > eps_s[r]) {
                o.status = kNumeric;
                break;
            }
            std::sort(all.begin(), all.end(), rank_less);
            if (all.size() > static_cast<std::size_t>(kPageSize)) {
                all.resize(kPageSize);
            }
            const bool complete = n == total;
            const bool full_page = all.size() == static_cast<std::size_t>(kPageSize);
            o.page = std::move(all);
            o.threshold_pass = true;
            if (complete || (full_page && o.page.back().score < threshold - eps_s[r])) {
                o.certified = true;
                o.exact_floor = complete ? INFINITY : threshold - eps_s[r];
                break;
            }
            if (std::getenv("SPK_DEBUG_PAGES")) {
                std::fprintf(stderr, "threshold r=%d T=%.17g n=%u total=%llu page=%zu\n", r, threshold, n, total,
                             o.page.size());
            }
            threshold = full_page ? std::max(o.page.back().score + 2 * eps_s[r], threshold + widen) : threshold + widen;
            widen *= 4;
        }
        if (!o.certified && !o.status) {
            o.status = kScratchLimit;
        }
    }
    return kOk;
}

}  // namespace spk
