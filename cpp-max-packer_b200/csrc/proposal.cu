// Learned orientation proposal network on the fifth-generation tensor cores.
//
// Every convolution (forward, data gradient, weight gradient) is one
// implicit GEMM D[M x N] = sum_k A[m, k] B[n, k] on tcgen05:
//   forward : m = output voxel, n = cout, k = (tap, cin)   A K-major, B K-major
//   data    : m = input voxel,  n = cin,  k = (tap, cout)  A K-major, B MN-major
//   weight  : m = (tap, cin),   n = cout, k = output voxel A MN-major, B MN-major
// The CTA's 128 threads gather the im2col operand tiles straight from the
// channels-last activations into shared memory (one 16-byte unit = 8 channels
// of one voxel), a single thread issues the MMAs into a TMEM accumulator of
// 128 lanes x N FP32 columns, and tcgen05.commit on a per-stage mbarrier
// releases each of the four shared-memory stages for the next gather.  The
// epilogue reads TMEM with tcgen05.ld: bias + ReLU + BF16 store (forward),
// ReLU mask + BF16 store (data gradient), FP32 partial sums per K split
// (weight gradient; the row after the last (tap, cin) row is all ones, so its
// sums are the bias gradient).
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <vector>

#include "../../include/spk_b200.h"
#include "context.hpp"
#include "proposal.hpp"
#include "umma.cuh"

struct spk_proposal;

namespace spk {

using bf16 = __nv_bfloat16;

namespace {

constexpr int kRows = 128;   // MMA M = TMEM lanes
constexpr int kKC = 32;      // K elements per stage (two MMA K-steps of 16)
constexpr int kStages = 4;
constexpr int kThreads = 128;
constexpr int kStepBytesA = kRows * 16 * 2;  // one K-step block of A: 128 rows x 16 bf16
enum Mode { kFwd = 0, kData = 1, kWeight = 2, kFwdBox = 3 };

int cin_pad(int cin) { return cin < 8 ? 8 : cin; }

struct ConvArgs {
    const bf16* x;       // layer input, [batch][s_in^3][cin]
    const bf16* dy;      // gradient of this layer's pre-activation, [batch][s_out^3][cout]
    const bf16* w;       // [cout][kw], kw = 27 * cin_pad, zero padded channels
    const float* bias;   // [cout]
    bf16* out;           // forward: [batch][s_out^3][cout]; data: [batch][s_in^3][cin]
    float* out_f32;      // forward, when set: the FP32 linear sums (no bias, no ReLU) instead of `out`
    float* partial;      // weight: [split][cout][kw + 1]
    unsigned* error;
    int batch, s_in, s_out, stride, cin, cinp, cout, kw;
    long long m_total;   // GEMM rows
    long long k_total;   // GEMM K
    int chunks_per_split;
    int relu_mask;       // data gradient: multiply by (x > 0)
    // log2 of the power-of-two extents and channel counts (every layer of the
    // network has them), so the gathers index with shifts and masks.
    int lg_s_in, lg_s_out, lg_cin, lg_cinp, lg_cout;
    // Corner-box forward (kFwdBox): `out` / `out_f32` hold the box
    // [0, box_out) of every sample, voxel (x, y, z) of sample n at row
    // n * box_out_vol + (z * box_out[1] + y) * box_out[0] + x.  The GEMM rows
    // are the voxels of the sub-box [region_first, region_first + region) of
    // every sample (row m = n * region_vol + its place in the sub-box, x
    // fastest), each written to its place in the box.  An input voxel inside
    // [0, box_in) is read from x, laid out [n][box_in voxels][cin] the same
    // way; any other input voxel is read from x_shared ([s_in^3][cin], one
    // sample shared by all), or is zero when x_shared is null.
    const bf16* x_shared;
    int box_in[3], box_out[3];
    int box_in_vol, box_out_vol;
    int region_first[3], region[3];
    int region_vol;
};

struct Vox {
    int n, z, y, x;
};

// Voxel of row m of a corner-box GEMM over the sub-box [first, first +
// region) (rows < 2^32).
__device__ __forceinline__ Vox decode_box(unsigned m, const int (&first)[3], const int (&region)[3], int vol)
{
    Vox v;
    v.n = static_cast<int>(m / static_cast<unsigned>(vol));
    const int r = static_cast<int>(m % static_cast<unsigned>(vol));
    v.x = first[0] + r % region[0];
    v.y = first[1] + (r / region[0]) % region[1];
    v.z = first[2] + r / (region[0] * region[1]);
    return v;
}

// Voxel of row m in a batch of cubes of side 2^lg (rows < 2^32).
__device__ __forceinline__ Vox decode_pow2(unsigned m, int lg)
{
    const unsigned mask = (1u << lg) - 1u;
    Vox v;
    v.x = static_cast<int>(m & mask);
    v.y = static_cast<int>((m >> lg) & mask);
    v.z = static_cast<int>((m >> (2 * lg)) & mask);
    v.n = static_cast<int>(m >> (3 * lg));
    return v;
}

// Channel-0 element offset of a voxel of a cube of side 2^lg with 2^lg_c channels.
__device__ __forceinline__ long long voxel_offset(const Vox& v, int iz, int iy, int ix, int lg, int lg_c)
{
    const unsigned cell = ((((static_cast<unsigned>(v.n) << lg | static_cast<unsigned>(iz)) << lg) |
                            static_cast<unsigned>(iy)) << lg) | static_cast<unsigned>(ix);
    return static_cast<long long>(cell) << lg_c;
}

__device__ __forceinline__ uint4 load_channels(const bf16* voxel, int cin, int ci0)
{
    if (cin >= 8) {
        return __ldg(reinterpret_cast<const uint4*>(voxel + ci0));
    }
    const unsigned short* h = reinterpret_cast<const unsigned short*>(voxel);
    unsigned w[4] = { 0u, 0u, 0u, 0u };
    for (int i = 0; i < cin; ++i) {
        w[i >> 1] |= static_cast<unsigned>(__ldg(h + i)) << (16 * (i & 1));
    }
    return make_uint4(w[0], w[1], w[2], w[3]);
}

__device__ __forceinline__ void put(unsigned char* base, std::uint32_t offset, uint4 v)
{
    *reinterpret_cast<uint4*>(base + offset) = v;
}

// Asynchronous 16-byte copy global -> shared; when `valid` is false nothing
// is read and the 16 bytes are zero-filled (src is then any mapped address).
__device__ __forceinline__ void copy16(unsigned char* base, std::uint32_t offset, const void* src, bool valid)
{
    asm volatile("cp.async.ca.shared.global [%0], [%1], 16, %2;"
                 :
                 : "r"(umma::smem_addr(base + offset)), "l"(src), "r"(valid ? 16 : 0)
                 : "memory");
}
__device__ __forceinline__ void copy_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void copy_wait()
{
    asm volatile("cp.async.wait_group %0;" : : "n"(N) : "memory");
}

// Input voxel of output voxel `o` through tap (kz, ky, kx); false outside.
__device__ __forceinline__ bool tap_input(const Vox& o, int tap, int stride, int s_in, int& iz, int& iy, int& ix)
{
    const int kz = tap / 9, ky = (tap / 3) % 3, kx = tap % 3;
    iz = o.z * stride + kz - 1;
    iy = o.y * stride + ky - 1;
    ix = o.x * stride + kx - 1;
    return iz >= 0 && iz < s_in && iy >= 0 && iy < s_in && ix >= 0 && ix < s_in;
}

// Output voxel that reads input voxel `p` through tap; false when none.
__device__ __forceinline__ bool tap_output(const Vox& p, int tap, int stride, int s_out, int& qz, int& qy, int& qx)
{
    const int kz = tap / 9, ky = (tap / 3) % 3, kx = tap % 3;
    const int az = p.z + 1 - kz, ay = p.y + 1 - ky, ax = p.x + 1 - kx;
    if (az < 0 || ay < 0 || ax < 0 || az % stride || ay % stride || ax % stride) {
        return false;
    }
    qz = az / stride;
    qy = ay / stride;
    qx = ax / stride;
    return qz < s_out && qy < s_out && qx < s_out;
}

template <int MODE>
__device__ __forceinline__ void gather_a(const ConvArgs& a, unsigned char* A, long long m0, int chunk, int tid,
                                         const Vox& row_vox, bool row_ok)
{
    if (MODE != kWeight) {
        // K-major: thread tid owns row tid; unit j covers K half (j & 1) of K-step (j >> 1).
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int ks = j >> 1, c = j & 1;
            const long long k = static_cast<long long>(chunk) * kKC + ks * 16 + c * 8;
            const std::uint32_t off = ks * kStepBytesA + umma::unit_offset(tid >> 3, c, tid & 7);
            const void* src = a.w;
            bool valid = false;
            if (row_ok && k < a.k_total) {
                const int kk = static_cast<int>(k);
                if (MODE == kFwd || MODE == kFwdBox) {
                    const int tap = kk >> a.lg_cinp, ci0 = kk & ((1 << a.lg_cinp) - 1);
                    int iz, iy, ix;
                    if (tap < 27 && (a.cin >= 8 || ci0 == 0) && tap_input(row_vox, tap, a.stride, a.s_in, iz, iy, ix)) {
                        const bf16* base = a.x;
                        long long at;
                        if (MODE == kFwd) {
                            at = voxel_offset(row_vox, iz, iy, ix, a.lg_s_in, a.lg_cin);
                        }
                        else if (iz < a.box_in[2] && iy < a.box_in[1] && ix < a.box_in[0]) {
                            at = (static_cast<long long>(row_vox.n) * a.box_in_vol +
                                  (iz * a.box_in[1] + iy) * a.box_in[0] + ix) << a.lg_cin;
                        }
                        else if (a.x_shared) {
                            base = a.x_shared;
                            at = voxel_offset(Vox { 0, 0, 0, 0 }, iz, iy, ix, a.lg_s_in, a.lg_cin);
                        }
                        else {
                            copy16(A, off, src, false);  // zero outside the box
                            continue;
                        }
                        if (a.cin < 8) {
                            put(A, off, load_channels(base + at, a.cin, ci0));
                            continue;
                        }
                        src = base + at + ci0;
                        valid = true;
                    }
                }
                else {
                    const int tap = kk >> a.lg_cout, co0 = kk & ((1 << a.lg_cout) - 1);
                    int qz, qy, qx;
                    if (tap < 27 && tap_output(row_vox, tap, a.stride, a.s_out, qz, qy, qx)) {
                        src = a.dy + voxel_offset(row_vox, qz, qy, qx, a.lg_s_out, a.lg_cout) + co0;
                        valid = true;
                    }
                }
            }
            copy16(A, off, src, valid);
        }
    }
    else {
        // MN-major over rows (tap, cin): unit = 8 channels of one output voxel q.
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int e = tid + kThreads * j;
            const int ks = e >> 8, kk = e & 15, g = (e & 255) >> 4;
            const long long r0 = m0 + 8 * g;
            const long long q = static_cast<long long>(chunk) * kKC + ks * 16 + kk;
            const std::uint32_t off = ks * kStepBytesA + umma::unit_offset(g, kk >> 3, kk & 7);
            const void* src = a.w;
            bool valid = false;
            if (q < a.k_total) {
                if (r0 < a.kw) {
                    const int r = static_cast<int>(r0);
                    const int tap = r >> a.lg_cinp, ci0 = r & ((1 << a.lg_cinp) - 1);
                    const Vox o = decode_pow2(static_cast<unsigned>(q), a.lg_s_out);
                    int iz, iy, ix;
                    if ((a.cin >= 8 || ci0 == 0) && tap_input(o, tap, a.stride, a.s_in, iz, iy, ix)) {
                        const long long at = voxel_offset(o, iz, iy, ix, a.lg_s_in, a.lg_cin);
                        if (a.cin < 8) {
                            put(A, off, load_channels(a.x + at, a.cin, ci0));
                            continue;
                        }
                        src = a.x + at + ci0;
                        valid = true;
                    }
                }
                else if (r0 == a.kw) {
                    put(A, off, make_uint4(0x3F80u, 0u, 0u, 0u));  // bf16 1.0 in row kw: the bias-gradient row
                    continue;
                }
            }
            copy16(A, off, src, valid);
        }
    }
}

template <int MODE>
__device__ __forceinline__ void gather_b(const ConvArgs& a, unsigned char* B, int N, int chunk, int tid)
{
    const int units = 4 * N;  // (N / 8) groups x 2 halves x 8 x 2 K-steps
    for (int e = tid; e < units; e += kThreads) {
        const int ks = e / (2 * N), rem = e % (2 * N);
        const void* src = a.w;
        bool valid = false;
        std::uint32_t off;
        if (MODE == kFwd || MODE == kFwdBox) {
            // K-major rows cout.
            const int c = rem / N, co = rem % N;
            const long long k = static_cast<long long>(chunk) * kKC + ks * 16 + c * 8;
            if (k < a.kw) {
                src = a.w + static_cast<long long>(co) * a.kw + k;
                valid = true;
            }
            off = umma::unit_offset(co >> 3, c, co & 7);
        }
        else {
            // MN-major: unit = 8 consecutive rows at one K index.
            const int kk = rem & 15, g = rem >> 4;
            const long long k = static_cast<long long>(chunk) * kKC + ks * 16 + kk;
            if (MODE == kData) {
                const int tap = static_cast<int>(k) >> a.lg_cout, co = static_cast<int>(k) & ((1 << a.lg_cout) - 1);
                if (k < a.k_total && tap < 27) {
                    src = a.w + static_cast<long long>(co) * a.kw + tap * a.cinp + 8 * g;
                    valid = true;
                }
            }
            else if (k < a.k_total) {
                src = a.dy + k * a.cout + 8 * g;
                valid = true;
            }
            off = umma::unit_offset(g, kk >> 3, kk & 7);
        }
        copy16(B, ks * (N * 32) + off, src, valid);
    }
}

template <int MODE>
__global__ void __launch_bounds__(kThreads) conv_kernel(const ConvArgs a)
{
    extern __shared__ __align__(1024) unsigned char smem[];
    __shared__ __align__(8) unsigned long long bars[kStages];
    __shared__ std::uint32_t tmem_base;

    const int tid = threadIdx.x, warp = tid >> 5;
    const int N = MODE == kData ? a.cin : a.cout;
    const std::uint32_t columns = N <= 32 ? 32u : 64u;
    const int stage_bytes = kRows * kKC * 2 + N * kKC * 2;

    if (warp == 0) {
        umma::tmem_alloc(&tmem_base, columns);
        umma::tmem_relinquish();
    }
    if (tid == 0) {
        for (int s = 0; s < kStages; ++s) {
            umma::bar_init(&bars[s], 1);
        }
        umma::bar_init_fence();
    }
    umma::fence_before();
    __syncthreads();
    umma::fence_after();
    const std::uint32_t tmem = tmem_base;

    const long long m0 = static_cast<long long>(blockIdx.x) * kRows;
    const int chunks = static_cast<int>((a.k_total + kKC - 1) / kKC);
    int c_begin = 0, c_end = chunks;
    if (MODE == kWeight) {
        c_begin = blockIdx.y * a.chunks_per_split;
        c_end = min(chunks, c_begin + a.chunks_per_split);
    }
    Vox row_vox {};
    bool row_ok = false;
    if (MODE != kWeight) {
        const long long m = m0 + tid;
        row_ok = m < a.m_total;
        if (MODE == kFwdBox) {
            row_vox = decode_box(static_cast<unsigned>(row_ok ? m : 0), a.region_first, a.region, a.region_vol);
        }
        else {
            row_vox = decode_pow2(static_cast<unsigned>(row_ok ? m : 0), MODE == kFwd ? a.lg_s_out : a.lg_s_in);
        }
    }
    constexpr bool fwd = MODE == kFwd || MODE == kFwdBox;
    constexpr bool a_mn = MODE == kWeight;
    constexpr bool b_mn = !fwd;
    const std::uint32_t idesc = umma::idesc_bf16(kRows, N, a_mn, b_mn);

    // Gathers run kAhead chunks in front of the MMA as asynchronous copies;
    // every iteration commits one copy group (possibly empty), so waiting
    // for all but the newest kAhead - 1 groups means chunk `it` has landed.
    constexpr int kAhead = kStages - 1;
    const int n_chunks = c_end - c_begin;
    auto gather = [&](int it) {
        unsigned char* A = smem + (it % kStages) * stage_bytes;
        gather_a<MODE>(a, A, m0, c_begin + it, tid, row_vox, row_ok);
        gather_b<MODE>(a, A + kRows * kKC * 2, N, c_begin + it, tid);
    };
    bool ok = true;
    for (int it = 0; it < kAhead; ++it) {
        if (it < n_chunks) {
            gather(it);
        }
        copy_commit();
    }
    for (int it = 0; it < n_chunks; ++it) {
        const int st = it % kStages;
        copy_wait<kAhead - 1>();
        umma::fence_async_smem();
        __syncthreads();
        if (tid == 0) {
            umma::fence_after();
            unsigned char* A = smem + st * stage_bytes;
            unsigned char* B = A + kRows * kKC * 2;
#pragma unroll
            for (int ks = 0; ks < 2; ++ks) {
                const std::uint64_t da = umma::desc(umma::smem_addr(A + ks * kStepBytesA));
                const std::uint64_t db = umma::desc(umma::smem_addr(B + ks * N * 32));
                umma::mma_bf16(tmem, da, db, idesc, (it > 0 || ks > 0) ? 1u : 0u);
            }
            umma::commit(&bars[st]);
        }
        const int next = it + kAhead;
        if (next < n_chunks) {
            // Stage next % kStages was last read by the MMA of chunk it - 1.
            if (it >= 1 && !umma::bar_wait(&bars[(it - 1) % kStages], static_cast<std::uint32_t>(((it - 1) / kStages) & 1))) {
                ok = false;
            }
            gather(next);
        }
        copy_commit();
    }
    const int n_it = c_end - c_begin;
    if (n_it > 0) {
        const int last = n_it - 1;
        if (!umma::bar_wait(&bars[last % kStages], static_cast<std::uint32_t>((last / kStages) & 1))) {
            ok = false;
        }
    }
    umma::fence_after();
    if (!ok && (tid & 31) == 0) {
        atomicOr(a.error, 1u);
    }

    // Epilogue: thread tid holds TMEM lane tid = tile row tid, written to
    // its output row (for kFwdBox, the voxel's place in the box).
    const std::uint32_t lane_addr = tmem + (static_cast<std::uint32_t>(warp * 32) << 16);
    const long long row = m0 + tid;
    const long long out_row =
        MODE == kFwdBox ? static_cast<long long>(row_vox.n) * a.box_out_vol +
                              (row_vox.z * a.box_out[1] + row_vox.y) * a.box_out[0] + row_vox.x
                        : row;
    for (int c0 = 0; c0 < N; c0 += 16) {
        float v[16];
        umma::tmem_load16(lane_addr + static_cast<std::uint32_t>(c0), v);
        if (n_it == 0) {
#pragma unroll
            for (int i = 0; i < 16; ++i) {
                v[i] = 0.f;
            }
        }
        if (fwd && a.out_f32) {
            if (row < a.m_total) {
                float4* dst = reinterpret_cast<float4*>(a.out_f32 + out_row * a.cout + c0);
#pragma unroll
                for (int i = 0; i < 4; ++i) {
                    dst[i] = make_float4(v[4 * i], v[4 * i + 1], v[4 * i + 2], v[4 * i + 3]);
                }
            }
        }
        else if (fwd) {
            if (row < a.m_total) {
                __align__(16) bf16 h[16];
#pragma unroll
                for (int i = 0; i < 16; ++i) {
                    h[i] = __float2bfloat16_rn(fmaxf(v[i] + a.bias[c0 + i], 0.f));
                }
                uint4* dst = reinterpret_cast<uint4*>(a.out + out_row * a.cout + c0);
                dst[0] = reinterpret_cast<const uint4*>(h)[0];
                dst[1] = reinterpret_cast<const uint4*>(h)[1];
            }
        }
        else if (MODE == kData) {
            if (row < a.m_total) {
                __align__(16) bf16 h[16];
                const bf16* xr = a.x + row * a.cin + c0;
#pragma unroll
                for (int i = 0; i < 16; ++i) {
                    float g = v[i];
                    if (a.relu_mask && !(__bfloat162float(xr[i]) > 0.f)) {
                        g = 0.f;
                    }
                    h[i] = __float2bfloat16_rn(g);
                }
                uint4* dst = reinterpret_cast<uint4*>(a.out + row * a.cin + c0);
                dst[0] = reinterpret_cast<const uint4*>(h)[0];
                dst[1] = reinterpret_cast<const uint4*>(h)[1];
            }
        }
        else {
            if (row <= a.kw) {
                float* p = a.partial + static_cast<long long>(blockIdx.y) * a.cout * (a.kw + 1);
#pragma unroll
                for (int i = 0; i < 16; ++i) {
                    p[static_cast<long long>(c0 + i) * (a.kw + 1) + row] = v[i];
                }
            }
        }
    }

    umma::fence_before();
    __syncthreads();
    if (warp == 0) {
        umma::fence_after();
        umma::tmem_dealloc(tmem, columns);
    }
}

// Sums the weight-gradient partials of `splits` K ranges into the flat FP32
// gradient (weights [cout][27][cin], then bias [cout]).
__global__ void reduce_weight_grad_kernel(const float* partial, int splits, int cout, int cin, int cinp, float* grad_w,
                                          float* grad_b)
{
    const int kw = 27 * cinp;
    const int total = cout * 27 * cin + cout;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
        int co, col;
        float* dst;
        if (i < cout * 27 * cin) {
            co = i / (27 * cin);
            const int rest = i % (27 * cin);
            col = (rest / cin) * cinp + rest % cin;
            dst = grad_w + i;
        }
        else {
            co = i - cout * 27 * cin;
            col = kw;
            dst = grad_b + co;
        }
        float s = 0.f;
        for (int sp = 0; sp < splits; ++sp) {
            s += partial[(static_cast<long long>(sp) * cout + co) * (kw + 1) + col];
        }
        *dst = s;
    }
}

// Head: mean over the 64 voxels of the last layer, linear 64 -> 1.  With
// labels it also forms the squared-error loss, its gradient through the head
// and the last layer's ReLU mask, and keeps the pooled features and dpred
// for the head's parameter gradients.  One block of 64 threads per sample.
__global__ void head_kernel(const bf16* act, const float* w, const float* b, int batch, const float* labels,
                            float* pred, float* pooled_out, float* dpred_out, float* loss_terms, bf16* dpre)
{
    const int n = blockIdx.x, c = threadIdx.x;
    if (n >= batch) {
        return;
    }
    __shared__ float part[64];
    __shared__ float shared_dpred;
    const bf16* a = act + static_cast<long long>(n) * 64 * 64;
    float s = 0.f;
    for (int v = 0; v < 64; ++v) {
        s += __bfloat162float(a[v * 64 + c]);
    }
    const float pooled = s * (1.0f / 64.0f);
    part[c] = w[c] * pooled;
    __syncthreads();
    if (c == 0) {
        float t = 0.f;
        for (int i = 0; i < 64; ++i) {
            t += part[i];
        }
        const float p = t + b[0];
        pred[n] = p;
        if (labels) {
            const float d = p - labels[n];
            loss_terms[n] = d * d;
            shared_dpred = 2.0f * d / static_cast<float>(batch);
            dpred_out[n] = shared_dpred;
        }
    }
    if (!labels) {
        return;
    }
    __syncthreads();
    pooled_out[n * 64 + c] = pooled;
    const float g = shared_dpred * w[c] * (1.0f / 64.0f);
    bf16* d = dpre + static_cast<long long>(n) * 64 * 64;
    for (int v = 0; v < 64; ++v) {
        d[v * 64 + c] = __float2bfloat16_rn(__bfloat162float(a[v * 64 + c]) > 0.f ? g : 0.f);
    }
}

// Head parameter gradients and the mean loss (one block of 64 threads).
__global__ void head_grad_kernel(const float* pooled, const float* dpred, const float* loss_terms, int batch,
                                 float* grad_w, float* grad_b, float* loss)
{
    const int c = threadIdx.x;
    float gw = 0.f;
    for (int n = 0; n < batch; ++n) {
        gw += dpred[n] * pooled[n * 64 + c];
    }
    grad_w[c] = gw;
    if (c == 0) {
        float gb = 0.f, l = 0.f;
        for (int n = 0; n < batch; ++n) {
            gb += dpred[n];
            l += loss_terms[n];
        }
        grad_b[0] = gb;
        loss[0] = l / static_cast<float>(batch);
    }
}

__global__ void adam_kernel(float* p, const float* g, float* m, float* v, long long count, float lr, float b1,
                            float b2, float eps, float c1, float c2)
{
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < count;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.f - b1) * gi;
        const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    }
}

// FP32 master weights [cout][27][cin] -> BF16 [cout][27 * cinp], zero padded.
__global__ void pack_weights_kernel(const float* w, int cout, int cin, int cinp, bf16* out)
{
    const int kw = 27 * cinp;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < cout * kw; i += gridDim.x * blockDim.x) {
        const int co = i / kw, col = i % kw, tap = col / cinp, ci = col % cinp;
        out[i] = __float2bfloat16_rn(ci < cin ? w[(co * 27 + tap) * cin + ci] : 0.f);
    }
}

// Network input: sample b = (crop[crop_index[b]], item[item_index[b]]), 2 channels.
__global__ void assemble_kernel(const bf16* crops, const std::uint32_t* crop_index, const bf16* items,
                                const std::uint32_t* item_index, int batch, bf16* x0)
{
    const long long total = static_cast<long long>(batch) * kProposalVoxels;
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < total;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        const int b = static_cast<int>(i / kProposalVoxels), v = static_cast<int>(i % kProposalVoxels);
        const long long crop = crop_index ? crop_index[b] : 0;
        const long long item = item_index ? item_index[b] : b;
        __nv_bfloat162 pair;
        pair.x = crops ? crops[crop * kProposalVoxels + v] : __float2bfloat16_rn(0.f);
        pair.y = items ? items[item * kProposalVoxels + v] : __float2bfloat16_rn(0.f);
        reinterpret_cast<__nv_bfloat162*>(x0)[i] = pair;
    }
}

// First-layer activation from its two linear halves: the item channel's sums
// (per sample) plus the layout channel's sums (shared by every sample).  One
// thread per 8 channels of one voxel (cout is a multiple of 8).  A null
// item_half stands for zero item sums (the voxels no item reaches).
__global__ void combine_first_kernel(const float* __restrict__ item_half, const float* __restrict__ crop_half,
                                     const float* __restrict__ bias, int batch, int cout, bf16* __restrict__ act)
{
    const int groups = cout / 8;
    const long long per = static_cast<long long>(kProposalVoxels) * groups;
    const long long total = per * batch;
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < total;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        const long long j = i % per;
        const int c0 = static_cast<int>(j % groups) * 8;
        const float4* a = reinterpret_cast<const float4*>(item_half + i * 8);
        const float4* c = reinterpret_cast<const float4*>(crop_half + j * 8);
        const float4 zero = make_float4(0.f, 0.f, 0.f, 0.f);
        const float4 a0 = item_half ? __ldcs(a) : zero, a1 = item_half ? __ldcs(a + 1) : zero;
        const float4 b0 = c[0], b1 = c[1];
        const float v[8] = { a0.x + b0.x, a0.y + b0.y, a0.z + b0.z, a0.w + b0.w,
                             a1.x + b1.x, a1.y + b1.y, a1.z + b1.z, a1.w + b1.w };
        __align__(16) bf16 h[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            h[k] = __float2bfloat16_rn(fmaxf(v[k] + bias[c0 + k], 0.f));
        }
        reinterpret_cast<uint4*>(act)[i] = *reinterpret_cast<const uint4*>(h);
    }
}

// The corner box that holds every non-zero voxel of `batch` pooled item
// channels ([batch][32^3], x fastest): support[a] = 1 + the largest
// coordinate along axis a of a non-zero voxel (0 when every voxel is zero).
__global__ void item_support_kernel(const bf16* __restrict__ items, int batch, unsigned* __restrict__ support)
{
    unsigned hi[3] = { 0u, 0u, 0u };
    const long long total = static_cast<long long>(batch) * kProposalVoxels;
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < total;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        if (__bfloat162float(items[i]) != 0.f) {
            const int v = static_cast<int>(i % kProposalVoxels);
            hi[0] = max(hi[0], static_cast<unsigned>(v % kProposalGrid) + 1u);
            hi[1] = max(hi[1], static_cast<unsigned>((v / kProposalGrid) % kProposalGrid) + 1u);
            hi[2] = max(hi[2], static_cast<unsigned>(v / (kProposalGrid * kProposalGrid)) + 1u);
        }
    }
    for (int a = 0; a < 3; ++a) {
        for (int o = 16; o > 0; o >>= 1) {
            hi[a] = max(hi[a], __shfl_xor_sync(0xffffffffu, hi[a], o));
        }
        if ((threadIdx.x & 31) == 0 && hi[a]) {
            atomicMax(support + a, hi[a]);
        }
    }
}

// Network inputs of the item channels inside a corner box: x[b][v] =
// (0, items[b][voxel v of the box]), 2 channels, box voxels x fastest.
__global__ void assemble_box_kernel(const bf16* __restrict__ items, int batch, int b0, int b1, int b2,
                                    bf16* __restrict__ x)
{
    const int vol = b0 * b1 * b2;
    const long long total = static_cast<long long>(batch) * vol;
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < total;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        const long long b = i / vol;
        const int r = static_cast<int>(i % vol);
        const int vx = r % b0, vy = (r / b0) % b1, vz = r / (b0 * b1);
        __nv_bfloat162 pair;
        pair.x = __float2bfloat16_rn(0.f);
        pair.y = items[b * kProposalVoxels + (vz * kProposalGrid + vy) * kProposalGrid + vx];
        reinterpret_cast<__nv_bfloat162*>(x)[i] = pair;
    }
}

// First-layer activations of the corner box from the item channel's sums
// over the box ([batch][box voxels][cout]) and the layout channel's sums
// ([32^3][cout]), with the expression of combine_first_kernel.
__global__ void combine_box_kernel(const float* __restrict__ item_box, const float* __restrict__ crop_half,
                                   const float* __restrict__ bias, int batch, int cout, int b0, int b1, int b2,
                                   int f0, int f1, int f2, int r0, int r1, int r2, bf16* __restrict__ act)
{
    // Voxels of the sub-box [f, f + r) of the box [0, b) of every sample.
    const int groups = cout / 8;
    const int vol = b0 * b1 * b2;
    const int rvol = r0 * r1 * r2;
    const long long total = static_cast<long long>(batch) * rvol * groups;
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < total;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        const int g = static_cast<int>(i % groups);
        const int r = static_cast<int>((i / groups) % rvol);
        const long long n = i / (static_cast<long long>(groups) * rvol);
        const int vx = f0 + r % r0, vy = f1 + (r / r0) % r1, vz = f2 + r / (r0 * r1);
        const long long voxel = (vz * kProposalGrid + vy) * kProposalGrid + vx;
        const long long at = (n * vol + (vz * b1 + vy) * b0 + vx) * groups + g;  // 8-channel group in the box
        const int c0 = g * 8;
        const float4* a = reinterpret_cast<const float4*>(item_box + at * 8);
        const float4* c = reinterpret_cast<const float4*>(crop_half + voxel * cout + c0);
        const float4 a0 = a[0], a1 = a[1], q0 = c[0], q1 = c[1];
        const float v[8] = { a0.x + q0.x, a0.y + q0.y, a0.z + q0.z, a0.w + q0.w,
                             a1.x + q1.x, a1.y + q1.y, a1.z + q1.z, a1.w + q1.w };
        __align__(16) bf16 h[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            h[k] = __float2bfloat16_rn(fmaxf(v[k] + bias[c0 + k], 0.f));
        }
        reinterpret_cast<uint4*>(act)[at] = *reinterpret_cast<const uint4*>(h);
    }
}

// Bounding range of the voxels where two pooled layouts differ (bitwise):
// box[0..2] = lowest x, y, z and box[3..5] = highest, updated atomically.
__global__ void crop_dirty_kernel(const bf16* __restrict__ a, const bf16* __restrict__ b, int* __restrict__ box)
{
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= kProposalVoxels) {
        return;
    }
    if (__bfloat16_as_ushort(a[v]) != __bfloat16_as_ushort(b[v])) {
        const int x = v % kProposalGrid, y = (v / kProposalGrid) % kProposalGrid, z = v / (kProposalGrid * kProposalGrid);
        atomicMin(box, x);
        atomicMin(box + 1, y);
        atomicMin(box + 2, z);
        atomicMax(box + 3, x);
        atomicMax(box + 4, y);
        atomicMax(box + 5, z);
    }
}

// Last-layer activations of every sample ([batch][side^3][c]) from the shared
// ones ([side^3][c]) and the corner box's ([batch][box voxels][c]).
__global__ void expand_box_kernel(const bf16* __restrict__ shared, const bf16* __restrict__ box, int batch, int side,
                                  int c, int b0, int b1, int b2, bf16* __restrict__ act)
{
    const int groups = c / 8;
    const int voxels = side * side * side;
    const int vol = b0 * b1 * b2;
    const long long total = static_cast<long long>(batch) * voxels * groups;
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < total;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        const int g = static_cast<int>(i % groups);
        const int v = static_cast<int>((i / groups) % voxels);
        const long long n = i / (static_cast<long long>(groups) * voxels);
        const int x = v % side, y = (v / side) % side, z = v / (side * side);
        const uint4* src;
        if (x < b0 && y < b1 && z < b2) {
            src = reinterpret_cast<const uint4*>(box + ((n * vol + (z * b1 + y) * b0 + x) * c)) + g;
        }
        else {
            src = reinterpret_cast<const uint4*>(shared + static_cast<long long>(v) * c) + g;
        }
        reinterpret_cast<uint4*>(act)[i] = *src;
    }
}

__global__ void to_bf16_kernel(const float* in, long long count, bf16* out)
{
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < count;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        out[i] = __float2bfloat16_rn(in[i]);
    }
}

// Pools a u8 field (X-fastest, shape[0..2]) into 32^3 fractions with block
// edge f per axis; cells outside the field count as `outside`.
__global__ void pool_kernel(const std::uint8_t* field, int s0, int s1, int s2, int f0, int f1, int f2,
                            float outside, bf16* out)
{
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= kProposalVoxels) {
        return;
    }
    const int x = v % kProposalGrid, y = (v / kProposalGrid) % kProposalGrid, z = v / (kProposalGrid * kProposalGrid);
    float sum = 0.f;
    for (int dz = 0; dz < f2; ++dz) {
        const int cz = z * f2 + dz;
        for (int dy = 0; dy < f1; ++dy) {
            const int cy = y * f1 + dy;
            for (int dx = 0; dx < f0; ++dx) {
                const int cx = x * f0 + dx;
                if (cx < s0 && cy < s1 && cz < s2) {
                    sum += field[(static_cast<long long>(cz) * s1 + cy) * s0 + cx] ? 1.f : 0.f;
                }
                else {
                    sum += outside;
                }
            }
        }
    }
    out[v] = __float2bfloat16_rn(sum / static_cast<float>(f0 * f1 * f2));
}

template <int MODE>
void set_smem_attribute()
{
    static std::once_flag flag[64];
    once_per_device(flag, [] {
        cudaFuncSetAttribute(conv_kernel<MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             kStages * (kRows * kKC * 2 + 64 * kKC * 2));
    });
}

std::uint64_t splitmix(std::uint64_t& s)
{
    std::uint64_t z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

double uniform01(std::uint64_t& s) { return (static_cast<double>(splitmix(s) >> 11) + 0.5) * (1.0 / 9007199254740992.0); }

}  // namespace

struct ProposalNet {
    int device {};
    std::uint64_t count {};
    std::uint64_t w_off[kProposalLayers] {}, b_off[kProposalLayers] {}, head_w {}, head_b {};
    float* params {};
    float* grads {};
    float* adam_m {};
    float* adam_v {};
    std::uint64_t adam_t {};
    bf16* w[kProposalLayers] {};
    // batch buffers
    std::uint32_t capacity {};
    bf16* x0 {};
    bf16* act[kProposalLayers] {};
    bf16* dpre[kProposalLayers] {};
    float* pred {};
    float* labels {};
    float* pooled {};
    float* dpred {};
    float* loss_terms {};
    float* loss {};
    float* partial {};
    std::size_t partial_bytes {};
    unsigned* error {};
    // Parameter version (bumped whenever the parameters change) and the cached
    // first-layer sums of a fixed set of item channels (the session path).
    std::uint64_t version { 1 };
    float* item_half {};
    std::size_t item_half_capacity {};
    std::uint64_t item_half_tag {};
    std::uint32_t item_half_batch {};
    std::uint64_t item_half_version {};
    float* crop_half {};
    bool item_half_box {};  // item_half holds the corner-box layout below
    // Corner-box trunk of the session path (proposal_predict): the item
    // channels' support, each layer's output box, the per-sample box
    // activations and the activations shared by every sample.
    unsigned* support {};
    int box[kProposalLayers][3] {};
    int item_box[3] {};
    bf16* x_item {};
    std::size_t x_item_capacity {};
    bf16* x_crop {};
    bf16* act_box[kProposalLayers] {};
    std::size_t act_box_capacity[kProposalLayers] {};
    bf16* act_shared[kProposalLayers] {};
    bf16* box_last {};
    std::size_t box_last_capacity {};
    // The layout channel the kept activations were computed from, and the
    // changed-voxel range found against it.
    bf16* prev_crop {};
    int* dirty {};
    bool trunk_valid {};
    // The layout-only layers run on a stream of their own, ahead of the
    // per-sample boxes that read them (one event per layer).
    cudaStream_t side {};
    cudaEvent_t layer_done[kProposalLayers] {};
    std::vector<void*> owned;
};

namespace {

int out_side(const ProposalLayer& l) { return l.s_in / l.stride; }

constexpr bool pow2(int v) { return v > 0 && (v & (v - 1)) == 0; }
constexpr bool shapes_are_pow2()
{
    for (const ProposalLayer& l : kProposalSpec) {
        if (!pow2(l.cin) || !pow2(l.cout) || !pow2(l.s_in) || !pow2(l.s_in / l.stride)) {
            return false;
        }
    }
    return true;
}
static_assert(shapes_are_pow2(), "the convolution gathers index power-of-two extents and channel counts");

template <typename T>
int alloc(ProposalNet* net, T*& p, std::size_t count)
{
    void* raw {};
    if (cudaMalloc(&raw, sizeof(T) * (count ? count : 1)) != cudaSuccess) {
        cudaGetLastError();
        return kAllocation;
    }
    net->owned.push_back(raw);
    p = static_cast<T*>(raw);
    return kOk;
}

template <typename T>
void release(ProposalNet* net, T*& p)
{
    if (!p) {
        return;
    }
    cudaFree(p);
    net->owned.erase(std::remove(net->owned.begin(), net->owned.end(), static_cast<void*>(p)), net->owned.end());
    p = nullptr;
}

int ensure_batch(ProposalNet* net, std::uint32_t batch)
{
    if (batch <= net->capacity) {
        return kOk;
    }
    release(net, net->x0);
    for (int l = 0; l < kProposalLayers; ++l) {
        release(net, net->act[l]);
        release(net, net->dpre[l]);
    }
    release(net, net->pred);
    release(net, net->labels);
    release(net, net->pooled);
    release(net, net->dpred);
    release(net, net->loss_terms);
    net->capacity = 0;
    int s = alloc(net, net->x0, static_cast<std::size_t>(batch) * kProposalVoxels * 2);
    for (int l = 0; l < kProposalLayers && !s; ++l) {
        const int so = out_side(kProposalSpec[l]);
        const std::size_t n = static_cast<std::size_t>(batch) * so * so * so * kProposalSpec[l].cout;
        s = alloc(net, net->act[l], n);
        if (!s) {
            s = alloc(net, net->dpre[l], n);
        }
    }
    if (!s) s = alloc(net, net->pred, batch);
    if (!s) s = alloc(net, net->labels, batch);
    if (!s) s = alloc(net, net->pooled, static_cast<std::size_t>(batch) * 64);
    if (!s) s = alloc(net, net->dpred, batch);
    if (!s) s = alloc(net, net->loss_terms, batch);
    if (s) {
        return s;
    }
    net->capacity = batch;
    return kOk;
}

// Grows a device buffer to at least `count` elements (contents discarded).
template <typename T>
int reserve(ProposalNet* net, T*& p, std::size_t& capacity, std::size_t count)
{
    if (p && count <= capacity) {
        return kOk;
    }
    release(net, p);
    capacity = 0;
    if (int status = alloc(net, p, count)) {
        return status;
    }
    capacity = count;
    return kOk;
}

int grid_for(long long n, int threads = 256)
{
    const long long g = (n + threads - 1) / threads;
    return static_cast<int>(std::min<long long>(std::max<long long>(g, 1), 148LL * 32));
}

ConvArgs layer_args(ProposalNet* net, int l, std::uint32_t batch)
{
    const ProposalLayer& L = kProposalSpec[l];
    ConvArgs a {};
    a.x = l == 0 ? net->x0 : net->act[l - 1];
    a.dy = net->dpre[l];
    a.w = net->w[l];
    a.bias = net->params + net->b_off[l];
    a.error = net->error;
    a.batch = static_cast<int>(batch);
    a.s_in = L.s_in;
    a.s_out = out_side(L);
    a.stride = L.stride;
    a.cin = L.cin;
    a.cinp = cin_pad(L.cin);
    a.cout = L.cout;
    a.kw = 27 * a.cinp;
    a.lg_s_in = ilog2(static_cast<unsigned>(a.s_in));
    a.lg_s_out = ilog2(static_cast<unsigned>(a.s_out));
    a.lg_cin = ilog2(static_cast<unsigned>(a.cin));
    a.lg_cinp = ilog2(static_cast<unsigned>(a.cinp));
    a.lg_cout = ilog2(static_cast<unsigned>(a.cout));
    return a;
}

void launch_conv_forward(spk_context* ctx, ProposalNet* net, int l, std::uint32_t batch, const bf16* x, bf16* out,
                         float* out_f32, cudaStream_t stream = nullptr)
{
    ConvArgs a = layer_args(net, l, batch);
    a.x = x;
    a.out = out;
    a.out_f32 = out_f32;
    a.m_total = static_cast<long long>(batch) * a.s_out * a.s_out * a.s_out;
    a.k_total = a.kw;
    const int blocks = static_cast<int>((a.m_total + kRows - 1) / kRows);
    const int smem = kStages * (kRows * kKC * 2 + a.cout * kKC * 2);
    conv_kernel<kFwd><<<blocks, kThreads, smem, stream ? stream : ctx->stream>>>(a);
    ctx->launches++;
}

// Forward layer l over the corner box `box_out` of every sample (kFwdBox).
void launch_conv_box(spk_context* ctx, ProposalNet* net, int l, std::uint32_t batch, const bf16* x,
                     const int (&box_in)[3], const bf16* x_shared, const int (&box_out)[3], bf16* out,
                     float* out_f32, const int (&region_first)[3], const int (&region)[3],
                     cudaStream_t stream = nullptr)
{
    ConvArgs a = layer_args(net, l, batch);
    a.x = x;
    a.x_shared = x_shared;
    a.out = out;
    a.out_f32 = out_f32;
    a.box_in_vol = 1;
    a.box_out_vol = 1;
    a.region_vol = 1;
    for (int i = 0; i < 3; ++i) {
        a.box_in[i] = box_in[i];
        a.box_out[i] = box_out[i];
        a.box_in_vol *= box_in[i];
        a.box_out_vol *= box_out[i];
        a.region_first[i] = region_first[i];
        a.region[i] = region[i];
        a.region_vol *= region[i];
    }
    a.m_total = static_cast<long long>(batch) * a.region_vol;
    a.k_total = a.kw;
    if (a.m_total == 0) {
        return;
    }
    const int blocks = static_cast<int>((a.m_total + kRows - 1) / kRows);
    const int smem = kStages * (kRows * kKC * 2 + a.cout * kKC * 2);
    conv_kernel<kFwdBox><<<blocks, kThreads, smem, stream ? stream : ctx->stream>>>(a);
    ctx->launches++;
}

int launch_forward(spk_context* ctx, ProposalNet* net, std::uint32_t batch, int first = 0)
{
    set_smem_attribute<kFwd>();
    for (int l = first; l < kProposalLayers; ++l) {
        launch_conv_forward(ctx, net, l, batch, l == 0 ? net->x0 : net->act[l - 1], net->act[l], nullptr);
    }
    return cudaGetLastError() == cudaSuccess ? kOk : kCuda;
}

// Forward + backward for `batch` samples already in x0 with labels in
// net->labels; leaves the flat gradient in net->grads and the loss in net->loss.
int launch_gradients(spk_context* ctx, ProposalNet* net, std::uint32_t batch)
{
    int status = launch_forward(ctx, net, batch);
    if (status) {
        return status;
    }
    head_kernel<<<batch, 64, 0, ctx->stream>>>(net->act[3], net->params + net->head_w, net->params + net->head_b,
                                                static_cast<int>(batch), net->labels, net->pred, net->pooled,
                                                net->dpred, net->loss_terms, net->dpre[3]);
    head_grad_kernel<<<1, 64, 0, ctx->stream>>>(net->pooled, net->dpred, net->loss_terms, static_cast<int>(batch),
                                                net->grads + net->head_w, net->grads + net->head_b, net->loss);
    ctx->launches += 2;
    set_smem_attribute<kData>();
    set_smem_attribute<kWeight>();
    for (int l = kProposalLayers - 1; l >= 0; --l) {
        ConvArgs a = layer_args(net, l, batch);
        // weight gradient
        {
            ConvArgs g = a;
            g.k_total = static_cast<long long>(batch) * a.s_out * a.s_out * a.s_out;
            g.m_total = a.kw + 1;
            const int m_tiles = static_cast<int>((a.kw + 1 + kRows - 1) / kRows);
            const int chunks = static_cast<int>((g.k_total + kKC - 1) / kKC);
            int splits = std::max(1, std::min((2 * 148 * 2 + m_tiles - 1) / m_tiles, chunks / 4));
            g.chunks_per_split = (chunks + splits - 1) / splits;
            splits = (chunks + g.chunks_per_split - 1) / g.chunks_per_split;
            const std::size_t need = static_cast<std::size_t>(splits) * a.cout * (a.kw + 1) * sizeof(float);
            if (need > net->partial_bytes) {
                release(net, net->partial);
                net->partial_bytes = 0;
                if ((status = alloc(net, net->partial, need / sizeof(float)))) {
                    return status;
                }
                net->partial_bytes = need;
            }
            g.partial = net->partial;
            const int smem = kStages * (kRows * kKC * 2 + a.cout * kKC * 2);
            conv_kernel<kWeight><<<dim3(m_tiles, splits), kThreads, smem, ctx->stream>>>(g);
            reduce_weight_grad_kernel<<<grid_for(a.cout * 27 * a.cin + a.cout), 256, 0, ctx->stream>>>(
                net->partial, splits, a.cout, a.cin, a.cinp, net->grads + net->w_off[l], net->grads + net->b_off[l]);
            ctx->launches += 2;
        }
        // data gradient into the previous layer's pre-activation gradient
        if (l > 0) {
            ConvArgs d = a;
            d.out = net->dpre[l - 1];
            d.m_total = static_cast<long long>(batch) * a.s_in * a.s_in * a.s_in;
            d.k_total = 27LL * a.cout;
            d.relu_mask = 1;
            const int blocks = static_cast<int>((d.m_total + kRows - 1) / kRows);
            const int smem = kStages * (kRows * kKC * 2 + a.cin * kKC * 2);
            conv_kernel<kData><<<blocks, kThreads, smem, ctx->stream>>>(d);
            ctx->launches++;
        }
    }
    return cudaGetLastError() == cudaSuccess ? kOk : kCuda;
}

int pack_all(spk_context* ctx, ProposalNet* net)
{
    for (int l = 0; l < kProposalLayers; ++l) {
        const ProposalLayer& L = kProposalSpec[l];
        pack_weights_kernel<<<grid_for(L.cout * 27 * cin_pad(L.cin)), 256, 0, ctx->stream>>>(
            net->params + net->w_off[l], L.cout, L.cin, cin_pad(L.cin), net->w[l]);
        ctx->launches++;
    }
    return cudaGetLastError() == cudaSuccess ? kOk : kCuda;
}

// The bounded wait's expiry path on its own: one CTA initialises an
// mbarrier that expects one arrival, which never comes, and waits on it with
// bar_wait for `spins` polls.  The expired wait sets *error; the barrier is
// invalidated before the CTA exits.
__global__ void bounded_wait_check_kernel(std::uint32_t spins, unsigned* __restrict__ error)
{
    __shared__ __align__(8) unsigned long long bar;
    if (threadIdx.x == 0) {
        umma::bar_init(&bar, 1);
        umma::bar_init_fence();
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        if (!umma::bar_wait(&bar, 0, spins)) {
            atomicOr(error, 1u);
        }
        asm volatile("mbarrier.inval.shared::cta.b64 [%0];" : : "r"(umma::smem_addr(&bar)) : "memory");
    }
}

int check_error(spk_context* ctx, ProposalNet* net)
{
    unsigned err = 0;
    if (cudaMemcpyAsync(&err, net->error, sizeof(err), cudaMemcpyDeviceToHost, ctx->stream) != cudaSuccess ||
        cudaStreamSynchronize(ctx->stream) != cudaSuccess) {
        cudaGetLastError();
        return kCuda;
    }
    if (err) {
        cudaMemsetAsync(net->error, 0, sizeof(unsigned), ctx->stream);
        return kKernelWait;
    }
    return kOk;
}

int upload_inputs(spk_context* ctx, ProposalNet* net, std::uint32_t batch, const float* inputs)
{
    const long long n = static_cast<long long>(batch) * kProposalVoxels * 2;
    int status = kOk;
    float* staging = static_cast<float*>(device_buffer(ctx, "proposal_inputs", sizeof(float) * n, status));
    if (!staging) {
        return status;
    }
    if (cudaMemcpyAsync(staging, inputs, sizeof(float) * n, cudaMemcpyHostToDevice, ctx->stream) != cudaSuccess) {
        cudaGetLastError();
        return kCuda;
    }
    to_bf16_kernel<<<grid_for(n), 256, 0, ctx->stream>>>(staging, n, net->x0);
    ctx->launches++;
    return kOk;
}

}  // namespace

std::uint64_t proposal_parameter_count()
{
    std::uint64_t n = 0;
    for (const ProposalLayer& l : kProposalSpec) {
        n += static_cast<std::uint64_t>(l.cout) * 27 * l.cin + l.cout;
    }
    return n + 64 + 1;
}

namespace {

// One layout scored against a fixed set of items, by the corner-box trunk.
// Each item channel is zero outside a corner box of the 32^3 grid (the
// pooled item is corner aligned and small), so every layer's output is the
// same for all samples outside a corner box of its own: a voxel of layer l
// depends on the item only if its 3^3 window, at its stride, reaches the
// box of layer l - 1.  The layers therefore run once on the layout alone
// (one sample, item sums zero) and, per sample, only over their boxes,
// reading the layout-only activations wherever a window leaves the box.
//
// Between calls only the layout channel changes (a session places a copy),
// and the activations of both kinds are kept: a call compares the layout
// with the previous one, and each layer recomputes only the voxels whose
// window reaches the previous layer's changed voxels (a box per layer,
// grown by the window and shrunk by the stride).  An unchanged layout
// recomputes nothing before the head.
//
// Every output row is the same dot product in the same K order as in the
// full forward, so the predictions equal the full split forward's.
int predict_box(spk_context* ctx, ProposalNet* net, std::uint32_t batch, const bf16* crops, const bf16* items,
                std::uint64_t items_tag, float* pred)
{
    set_smem_attribute<kFwd>();
    set_smem_attribute<kFwdBox>();
    const int c1 = kProposalSpec[0].cout;
    int status = kOk;
    if (net->item_half_tag != items_tag || net->item_half_batch != batch || net->item_half_version != net->version ||
        !net->item_half_box) {
        if (!net->support && (status = alloc(net, net->support, 3))) {
            return status;
        }
        cudaMemsetAsync(net->support, 0, 3 * sizeof(unsigned), ctx->stream);
        item_support_kernel<<<grid_for(static_cast<long long>(batch) * kProposalVoxels), 256, 0, ctx->stream>>>(
            items, static_cast<int>(batch), net->support);
        unsigned support[3] {};
        if (cudaMemcpyAsync(support, net->support, sizeof(support), cudaMemcpyDeviceToHost, ctx->stream) !=
                cudaSuccess ||
            cudaStreamSynchronize(ctx->stream) != cudaSuccess) {
            cudaGetLastError();
            return kCuda;
        }
        ctx->launches++;
        for (int a = 0; a < 3; ++a) {
            net->item_box[a] = static_cast<int>(support[a]);
            int r = net->item_box[a];
            for (int l = 0; l < kProposalLayers; ++l) {
                const ProposalLayer& L = kProposalSpec[l];
                r = std::min(r / L.stride + 1, out_side(L));  // output o reads o * stride - 1 .. o * stride + 1
                net->box[l][a] = r;
            }
        }
        const std::size_t item_vol = static_cast<std::size_t>(net->item_box[0]) * net->item_box[1] * net->item_box[2];
        const std::size_t vol0 = static_cast<std::size_t>(net->box[0][0]) * net->box[0][1] * net->box[0][2];
        if ((status = reserve(net, net->x_item, net->x_item_capacity, batch * item_vol * 2)) ||
            (status = reserve(net, net->item_half, net->item_half_capacity, batch * vol0 * c1))) {
            return status;
        }
        if (item_vol) {
            assemble_box_kernel<<<grid_for(static_cast<long long>(batch * item_vol)), 256, 0, ctx->stream>>>(
                items, static_cast<int>(batch), net->item_box[0], net->item_box[1], net->item_box[2], net->x_item);
            ctx->launches++;
        }
        const int origin[3] = { 0, 0, 0 };
        launch_conv_box(ctx, net, 0, batch, net->x_item, net->item_box, nullptr, net->box[0], nullptr, net->item_half,
                        origin, net->box[0]);
        net->item_half_tag = items_tag;
        net->item_half_batch = batch;
        net->item_half_version = net->version;
        net->item_half_box = true;
        net->trunk_valid = false;
    }
    if ((!net->x_crop && (status = alloc(net, net->x_crop, static_cast<std::size_t>(kProposalVoxels) * 2))) ||
        (!net->crop_half && (status = alloc(net, net->crop_half, static_cast<std::size_t>(kProposalVoxels) * c1))) ||
        (!net->prev_crop && (status = alloc(net, net->prev_crop, static_cast<std::size_t>(kProposalVoxels)))) ||
        (!net->dirty && (status = alloc(net, net->dirty, 6)))) {
        return status;
    }
    for (int l = 0; l < kProposalLayers; ++l) {
        const ProposalLayer& L = kProposalSpec[l];
        const std::size_t so = static_cast<std::size_t>(out_side(L));
        const std::size_t vol = static_cast<std::size_t>(net->box[l][0]) * net->box[l][1] * net->box[l][2];
        if ((!net->act_shared[l] && (status = alloc(net, net->act_shared[l], so * so * so * L.cout))) ||
            (status = reserve(net, net->act_box[l], net->act_box_capacity[l], batch * vol * L.cout))) {
            return status;
        }
    }
    const int s3 = out_side(kProposalSpec[kProposalLayers - 1]);
    const int c3 = kProposalSpec[kProposalLayers - 1].cout;
    if ((status = reserve(net, net->box_last, net->box_last_capacity,
                          static_cast<std::size_t>(batch) * s3 * s3 * s3 * c3))) {
        return status;
    }
    if (!net->side) {
        if (cudaStreamCreateWithFlags(&net->side, cudaStreamNonBlocking) != cudaSuccess) {
            cudaGetLastError();
            net->side = nullptr;
            return kCuda;
        }
        for (auto& e : net->layer_done) {
            if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) {
                cudaGetLastError();
                return kCuda;
            }
        }
    }
    // The layout voxels that changed since the activations were computed:
    // lo / hi per axis, inclusive (hi < lo: none).
    int lo[3] = { 0, 0, 0 }, hi[3] = { kProposalGrid - 1, kProposalGrid - 1, kProposalGrid - 1 };
    if (net->trunk_valid) {
        const int init[6] = { kProposalGrid, kProposalGrid, kProposalGrid, -1, -1, -1 };
        int found[6] {};
        cudaMemcpyAsync(net->dirty, init, sizeof(init), cudaMemcpyHostToDevice, ctx->stream);
        crop_dirty_kernel<<<kProposalVoxels / 256, 256, 0, ctx->stream>>>(crops, net->prev_crop, net->dirty);
        ctx->launches++;
        if (cudaMemcpyAsync(found, net->dirty, sizeof(found), cudaMemcpyDeviceToHost, ctx->stream) != cudaSuccess ||
            cudaStreamSynchronize(ctx->stream) != cudaSuccess) {
            cudaGetLastError();
            return kCuda;
        }
        for (int a = 0; a < 3; ++a) {
            lo[a] = found[a];
            hi[a] = found[3 + a];
        }
    }
    const bool changed = hi[0] >= lo[0] && hi[1] >= lo[1] && hi[2] >= lo[2];
    if (changed) {
        cudaMemcpyAsync(net->prev_crop, crops, sizeof(bf16) * kProposalVoxels, cudaMemcpyDeviceToDevice,
                        ctx->stream);
        // A layer's layout-only activations are read only where its box does
        // not cover it (boxes never shrink back once they cover their layer).
        bool shared_needed[kProposalLayers];
        for (int l = 0; l < kProposalLayers; ++l) {
            const int so = out_side(kProposalSpec[l]);
            shared_needed[l] = net->box[l][0] < so || net->box[l][1] < so || net->box[l][2] < so;
        }
        // Changed output voxels per layer: window o * stride - 1 .. o * stride
        // + 1 meets the previous layer's changed range.
        int first[kProposalLayers][3], region[kProposalLayers][3], box_first[kProposalLayers][3],
            box_region[kProposalLayers][3];
        for (int l = 0; l < kProposalLayers; ++l) {
            const ProposalLayer& L = kProposalSpec[l];
            const int so = out_side(L);
            for (int a = 0; a < 3; ++a) {
                const int pl = l == 0 ? lo[a] : first[l - 1][a];
                const int ph = l == 0 ? hi[a] : first[l - 1][a] + region[l - 1][a] - 1;
                int ol = (pl - 1 + L.stride - 1) / L.stride;  // ceil((pl - 1) / stride), pl >= 0
                if (pl - 1 < 0) {
                    ol = 0;
                }
                const int oh = std::min((ph + 1) / L.stride, so - 1);
                first[l][a] = ol;
                region[l][a] = std::max(0, oh - ol + 1);
                box_first[l][a] = ol;
                box_region[l][a] = std::max(0, std::min(oh, net->box[l][a] - 1) - ol + 1);
            }
        }
        // The layout's first-layer sums (one sample, item channel zero).
        assemble_kernel<<<grid_for(kProposalVoxels), 256, 0, ctx->stream>>>(crops, nullptr, nullptr, nullptr, 1,
                                                                            net->x_crop);
        launch_conv_forward(ctx, net, 0, 1, net->x_crop, nullptr, net->crop_half);
        const float* bias0 = net->params + net->b_off[0];
        combine_first_kernel<<<grid_for(static_cast<long long>(kProposalVoxels) * c1 / 8), 256, 0, ctx->stream>>>(
            nullptr, net->crop_half, bias0, 1, c1, net->act_shared[0]);
        ctx->launches += 2;
        cudaEventRecord(net->layer_done[0], ctx->stream);
        cudaStreamWaitEvent(net->side, net->layer_done[0], 0);
        const int zero[3] = { 0, 0, 0 };
        for (int l = 1; l < kProposalLayers; ++l) {
            if (shared_needed[l]) {
                const int so = out_side(kProposalSpec[l]);
                const int whole[3] = { so, so, so };
                launch_conv_box(ctx, net, l, 1, nullptr, zero, net->act_shared[l - 1], whole, net->act_shared[l],
                                nullptr, first[l], region[l], net->side);
            }
            cudaEventRecord(net->layer_done[l], net->side);
        }
        const long long box0 = static_cast<long long>(batch) * box_region[0][0] * box_region[0][1] * box_region[0][2];
        if (box0) {
            combine_box_kernel<<<grid_for(box0 * c1 / 8), 256, 0, ctx->stream>>>(
                net->item_half, net->crop_half, bias0, static_cast<int>(batch), c1, net->box[0][0], net->box[0][1],
                net->box[0][2], box_first[0][0], box_first[0][1], box_first[0][2], box_region[0][0],
                box_region[0][1], box_region[0][2], net->act_box[0]);
            ctx->launches++;
        }
        for (int l = 1; l < kProposalLayers; ++l) {
            if (l >= 2) {
                cudaStreamWaitEvent(ctx->stream, net->layer_done[l - 1], 0);
            }
            launch_conv_box(ctx, net, l, batch, net->act_box[l - 1], net->box[l - 1],
                            shared_needed[l - 1] ? net->act_shared[l - 1] : nullptr, net->box[l], net->act_box[l],
                            nullptr, box_first[l], box_region[l]);
        }
        // Joins the side stream (the next call rewrites what it read).
        cudaStreamWaitEvent(ctx->stream, net->layer_done[kProposalLayers - 1], 0);
        const int* b3 = net->box[kProposalLayers - 1];
        expand_box_kernel<<<grid_for(static_cast<long long>(batch) * s3 * s3 * s3 * c3 / 8), 256, 0, ctx->stream>>>(
            net->act_shared[kProposalLayers - 1], net->act_box[kProposalLayers - 1], static_cast<int>(batch), s3,
            c3, b3[0], b3[1], b3[2], net->box_last);
        ctx->launches++;
        net->trunk_valid = true;
    }
    head_kernel<<<batch, 64, 0, ctx->stream>>>(net->box_last, net->params + net->head_w, net->params + net->head_b,
                                                static_cast<int>(batch), nullptr, pred, nullptr, nullptr, nullptr,
                                                nullptr);
    ctx->launches++;
    return cudaGetLastError() == cudaSuccess ? kOk : kCuda;
}

// SPK_PROPOSAL_TRUNK=full scores the session path with the full split forward
// (every voxel of every sample), kept to check the corner-box trunk against.
bool full_trunk()
{
    const char* v = std::getenv("SPK_PROPOSAL_TRUNK");
    return v && std::strcmp(v, "full") == 0;
}

}  // namespace

int proposal_predict(spk_context* ctx, ProposalNet* net, std::uint32_t batch, const bf16* crops,
                     const std::uint32_t* crop_index, const bf16* items, const std::uint32_t* item_index,
                     std::uint64_t items_tag, float* pred)
{
    if (batch == 0 || batch > (1u << 16)) {
        return kInvalidArgument;  // row indices of the gathers are 32-bit
    }
    if (!crop_index && !item_index && crops && items && items_tag && !full_trunk()) {
        return predict_box(ctx, net, batch, crops, items, items_tag, pred);
    }
    int status = ensure_batch(net, batch);
    if (status) {
        return status;
    }
    const int grid1 = kProposalGrid;  // first-layer output side (stride 1)
    const int c1 = kProposalSpec[0].cout;
    if (!crop_index && !item_index && crops && items && items_tag) {
        // One layout scored against fixed items: the first convolution is
        // linear in its two input channels, so the item channel's sums are
        // computed once per (items, batch, parameters) and only the layout
        // channel's sums (one sample) are computed per call.
        set_smem_attribute<kFwd>();
        const std::size_t half = static_cast<std::size_t>(batch) * grid1 * grid1 * grid1 * c1;
        if (net->item_half_tag != items_tag || net->item_half_batch != batch ||
            net->item_half_version != net->version || net->item_half_box) {
            if (half > net->item_half_capacity) {
                release(net, net->item_half);
                net->item_half_capacity = 0;
                if ((status = alloc(net, net->item_half, half))) {
                    return status;
                }
                net->item_half_capacity = half;
            }
            assemble_kernel<<<grid_for(static_cast<long long>(batch) * kProposalVoxels), 256, 0, ctx->stream>>>(
                nullptr, nullptr, items, nullptr, static_cast<int>(batch), net->x0);
            launch_conv_forward(ctx, net, 0, batch, net->x0, nullptr, net->item_half);
            ctx->launches++;
            net->item_half_tag = items_tag;
            net->item_half_batch = batch;
            net->item_half_version = net->version;
            net->item_half_box = false;
        }
        if (!net->crop_half && (status = alloc(net, net->crop_half, static_cast<std::size_t>(kProposalVoxels) * c1))) {
            return status;
        }
        assemble_kernel<<<grid_for(kProposalVoxels), 256, 0, ctx->stream>>>(crops, nullptr, nullptr, nullptr, 1,
                                                                            net->x0);
        launch_conv_forward(ctx, net, 0, 1, net->x0, nullptr, net->crop_half);
        combine_first_kernel<<<grid_for(static_cast<long long>(half / 8)), 256, 0, ctx->stream>>>(
            net->item_half, net->crop_half, net->params + net->b_off[0], static_cast<int>(batch), c1, net->act[0]);
        ctx->launches += 2;
        if ((status = launch_forward(ctx, net, batch, 1))) {
            return status;
        }
    }
    else {
        assemble_kernel<<<grid_for(static_cast<long long>(batch) * kProposalVoxels), 256, 0, ctx->stream>>>(
            crops, crop_index, items, item_index, static_cast<int>(batch), net->x0);
        ctx->launches++;
        if ((status = launch_forward(ctx, net, batch))) {
            return status;
        }
    }
    head_kernel<<<batch, 64, 0, ctx->stream>>>(net->act[3], net->params + net->head_w, net->params + net->head_b,
                                                static_cast<int>(batch), nullptr, pred, nullptr, nullptr, nullptr,
                                                nullptr);
    ctx->launches++;
    return cudaGetLastError() == cudaSuccess ? kOk : kCuda;
}

int pool_occupancy(spk_context* ctx, const std::uint8_t* occupancy, const int* shape, bf16* out)
{
    int f[3];
    for (int a = 0; a < 3; ++a) {
        f[a] = std::max(1, (shape[a] + kProposalGrid - 1) / kProposalGrid);
    }
    pool_kernel<<<kProposalVoxels / 256, 256, 0, ctx->stream>>>(occupancy, shape[0], shape[1], shape[2], f[0], f[1],
                                                                 f[2], 1.0f, out);
    ctx->launches++;
    return cudaGetLastError() == cudaSuccess ? kOk : kCuda;
}

int pool_item(spk_context* ctx, const std::uint8_t* cells, const int* shape, bf16* out)
{
    const int m = std::max(shape[0], std::max(shape[1], shape[2]));
    const int f = std::max(1, (m + kProposalGrid - 1) / kProposalGrid);
    pool_kernel<<<kProposalVoxels / 256, 256, 0, ctx->stream>>>(cells, shape[0], shape[1], shape[2], f, f, f, 0.0f,
                                                                 out);
    ctx->launches++;
    return cudaGetLastError() == cudaSuccess ? kOk : kCuda;
}

}  // namespace spk

using spk::ProposalNet;

struct spk_proposal {
    ProposalNet net;
};

namespace {

ProposalNet* net_of(spk_proposal* p) { return p ? &p->net : nullptr; }

}  // namespace

extern "C" {

uint64_t spk_proposal_parameter_count(void) { return spk::proposal_parameter_count(); }

int spk_check_bounded_wait(spk_context* ctx, uint32_t spins)
{
    if (!ctx) {
        return spk::kNotReady;
    }
    if (spins == 0 || spins > (1u << 22)) {
        return spk::kInvalidArgument;
    }
    int status = spk::kOk;
    auto* error = static_cast<unsigned*>(spk::device_buffer(ctx, "wait.check", sizeof(unsigned), status));
    if (!error) {
        return status;
    }
    unsigned host = 0;
    cudaMemsetAsync(error, 0, sizeof(unsigned), ctx->stream);
    spk::bounded_wait_check_kernel<<<1, 32, 0, ctx->stream>>>(spins, error);
    ctx->launches++;
    if (cudaMemcpyAsync(&host, error, sizeof(unsigned), cudaMemcpyDeviceToHost, ctx->stream) != cudaSuccess ||
        cudaStreamSynchronize(ctx->stream) != cudaSuccess) {
        cudaGetLastError();
        return spk::kCuda;
    }
    return host ? spk::fail(ctx, spk::kKernelWait, "A bounded device wait expired.") : spk::kOk;
}

int spk_proposal_create(spk_context* ctx, uint64_t seed, spk_proposal** out)
{
    try {
        if (!ctx || !out) {
            return spk::kInvalidArgument;
        }
        *out = nullptr;
        if (cudaSetDevice(ctx->device) != cudaSuccess) {
            return spk::kCuda;
        }
        auto* p = new spk_proposal();
        ProposalNet* net = &p->net;
        net->device = ctx->device;
        net->count = spk::proposal_parameter_count();
        std::vector<float> host(net->count, 0.f);
        std::uint64_t off = 0, state = seed ^ 0x5EED5EED5EEDull;
        for (int l = 0; l < spk::kProposalLayers; ++l) {
            const spk::ProposalLayer& L = spk::kProposalSpec[l];
            net->w_off[l] = off;
            const std::uint64_t nw = static_cast<std::uint64_t>(L.cout) * 27 * L.cin;
            const double sd = std::sqrt(2.0 / (27.0 * L.cin));  // He initialisation for ReLU
            for (std::uint64_t i = 0; i < nw; ++i) {
                const double u1 = spk::uniform01(state), u2 = spk::uniform01(state);
                host[off + i] = static_cast<float>(sd * std::sqrt(-2.0 * std::log(u1)) *
                                                   std::cos(6.283185307179586 * u2));
            }
            off += nw;
            net->b_off[l] = off;
            off += L.cout;
        }
        net->head_w = off;
        for (int c = 0; c < 64; ++c) {
            const double u1 = spk::uniform01(state), u2 = spk::uniform01(state);
            host[off + c] = static_cast<float>(0.125 * std::sqrt(-2.0 * std::log(u1)) *
                                               std::cos(6.283185307179586 * u2));
        }
        off += 64;
        net->head_b = off;
        int s = spk::alloc(net, net->params, net->count);
        if (!s) s = spk::alloc(net, net->grads, net->count);
        if (!s) s = spk::alloc(net, net->adam_m, net->count);
        if (!s) s = spk::alloc(net, net->adam_v, net->count);
        if (!s) s = spk::alloc(net, net->loss, 1);
        if (!s) s = spk::alloc(net, net->error, 1);
        for (int l = 0; l < spk::kProposalLayers && !s; ++l) {
            const spk::ProposalLayer& L = spk::kProposalSpec[l];
            s = spk::alloc(net, net->w[l], static_cast<std::size_t>(L.cout) * 27 * spk::cin_pad(L.cin));
        }
        if (s) {
            for (void* q : net->owned) {
                cudaFree(q);
            }
            delete p;
            return s;
        }
        cudaMemcpyAsync(net->params, host.data(), sizeof(float) * net->count, cudaMemcpyHostToDevice, ctx->stream);
        cudaMemsetAsync(net->adam_m, 0, sizeof(float) * net->count, ctx->stream);
        cudaMemsetAsync(net->adam_v, 0, sizeof(float) * net->count, ctx->stream);
        cudaMemsetAsync(net->grads, 0, sizeof(float) * net->count, ctx->stream);
        cudaMemsetAsync(net->error, 0, sizeof(unsigned), ctx->stream);
        if ((s = spk::pack_all(ctx, net)) || cudaStreamSynchronize(ctx->stream) != cudaSuccess) {
            cudaGetLastError();
            for (void* q : net->owned) {
                cudaFree(q);
            }
            delete p;
            return s ? s : spk::kCuda;
        }
        *out = p;
        return spk::kOk;
    }
    catch (...) {
        return spk::kAllocation;
    }
}

void spk_proposal_destroy(spk_proposal* p)
{
    if (!p) {
        return;
    }
    cudaSetDevice(p->net.device);
    if (p->net.side) {
        cudaStreamSynchronize(p->net.side);
        for (auto& e : p->net.layer_done) {
            if (e) {
                cudaEventDestroy(e);
            }
        }
        cudaStreamDestroy(p->net.side);
    }
    for (void* q : p->net.owned) {
        cudaFree(q);
    }
    delete p;
}

int spk_proposal_get_parameters(spk_context* ctx, spk_proposal* p, float* out)
{
    ProposalNet* net = net_of(p);
    if (!ctx || !net || !out) {
        return spk::kInvalidArgument;
    }
    if (cudaMemcpyAsync(out, net->params, sizeof(float) * net->count, cudaMemcpyDeviceToHost, ctx->stream) !=
            cudaSuccess ||
        cudaStreamSynchronize(ctx->stream) != cudaSuccess) {
        cudaGetLastError();
        return spk::kCuda;
    }
    return spk::kOk;
}

int spk_proposal_set_parameters(spk_context* ctx, spk_proposal* p, const float* in)
{
    ProposalNet* net = net_of(p);
    if (!ctx || !net || !in) {
        return spk::kInvalidArgument;
    }
    if (cudaMemcpyAsync(net->params, in, sizeof(float) * net->count, cudaMemcpyHostToDevice, ctx->stream) !=
        cudaSuccess) {
        cudaGetLastError();
        return spk::kCuda;
    }
    cudaMemsetAsync(net->adam_m, 0, sizeof(float) * net->count, ctx->stream);
    cudaMemsetAsync(net->adam_v, 0, sizeof(float) * net->count, ctx->stream);
    net->adam_t = 0;
    net->version++;
    int s = spk::pack_all(ctx, net);
    if (!s && cudaStreamSynchronize(ctx->stream) != cudaSuccess) {
        cudaGetLastError();
        s = spk::kCuda;
    }
    return s;
}

int spk_proposal_forward(spk_context* ctx, spk_proposal* p, uint64_t batch, const float* inputs, float* predictions)
{
    try {
        ProposalNet* net = net_of(p);
        if (!ctx || !net || !inputs || !predictions || batch == 0 || batch > (1u << 16)) {
            return spk::kInvalidArgument;
        }
        const auto b = static_cast<std::uint32_t>(batch);
        int s = spk::ensure_batch(net, b);
        if (!s) s = spk::upload_inputs(ctx, net, b, inputs);
        if (!s) s = spk::launch_forward(ctx, net, b);
        if (s) {
            return s;
        }
        spk::head_kernel<<<b, 64, 0, ctx->stream>>>(net->act[3], net->params + net->head_w,
                                                     net->params + net->head_b, static_cast<int>(b), nullptr,
                                                     net->pred, nullptr, nullptr, nullptr, nullptr);
        ctx->launches++;
        if (cudaMemcpyAsync(predictions, net->pred, sizeof(float) * b, cudaMemcpyDeviceToHost, ctx->stream) !=
            cudaSuccess) {
            cudaGetLastError();
            return spk::kCuda;
        }
        return spk::check_error(ctx, net);
    }
    catch (...) {
        return spk::kAllocation;
    }
}

int spk_proposal_gradients(spk_context* ctx, spk_proposal* p, uint64_t batch, const float* inputs,
                           const float* labels, float* loss, float* gradients)
{
    try {
        ProposalNet* net = net_of(p);
        if (!ctx || !net || !inputs || !labels || !loss || !gradients || batch == 0 || batch > (1u << 16)) {
            return spk::kInvalidArgument;
        }
        const auto b = static_cast<std::uint32_t>(batch);
        int s = spk::ensure_batch(net, b);
        if (!s) s = spk::upload_inputs(ctx, net, b, inputs);
        if (s) {
            return s;
        }
        cudaMemcpyAsync(net->labels, labels, sizeof(float) * b, cudaMemcpyHostToDevice, ctx->stream);
        if ((s = spk::launch_gradients(ctx, net, b))) {
            return s;
        }
        cudaMemcpyAsync(loss, net->loss, sizeof(float), cudaMemcpyDeviceToHost, ctx->stream);
        cudaMemcpyAsync(gradients, net->grads, sizeof(float) * net->count, cudaMemcpyDeviceToHost, ctx->stream);
        return spk::check_error(ctx, net);
    }
    catch (...) {
        return spk::kAllocation;
    }
}

int spk_proposal_train(spk_context* ctx, spk_proposal* p, const spk_proposal_dataset* data, uint32_t batch,
                       uint32_t steps, float learning_rate, uint64_t seed, float* losses)
{
    try {
        ProposalNet* net = net_of(p);
        if (!ctx || !net || !data || !data->crops || !data->items || !data->sample_crop || !data->sample_item ||
            !data->sample_label || data->sample_count == 0 || batch == 0 || batch > (1u << 14)) {
            return spk::kInvalidArgument;
        }
        for (std::uint64_t i = 0; i < data->sample_count; ++i) {
            if (data->sample_crop[i] >= data->crop_count || data->sample_item[i] >= data->item_count) {
                return spk::kInvalidArgument;
            }
        }
        int s = spk::ensure_batch(net, batch);
        if (s) {
            return s;
        }
        const std::uint64_t nc = data->crop_count * spk::kProposalVoxels;
        const std::uint64_t ni = data->item_count * spk::kProposalVoxels;
        float* staging =
            static_cast<float*>(spk::device_buffer(ctx, "proposal_inputs", sizeof(float) * std::max(nc, ni), s));
        spk::bf16* crops = static_cast<spk::bf16*>(spk::device_buffer(ctx, "proposal_crops", sizeof(spk::bf16) * nc, s));
        spk::bf16* items = static_cast<spk::bf16*>(spk::device_buffer(ctx, "proposal_items", sizeof(spk::bf16) * ni, s));
        auto* index = static_cast<std::uint32_t*>(
            spk::device_buffer(ctx, "proposal_index", sizeof(std::uint32_t) * 2 * batch, s));
        auto* host_index = static_cast<std::uint32_t*>(
            spk::host_buffer(ctx, "proposal_index_host", sizeof(std::uint32_t) * 2 * batch * steps, s));
        auto* host_labels =
            static_cast<float*>(spk::host_buffer(ctx, "proposal_labels_host", sizeof(float) * batch * steps, s));
        if (!staging || !crops || !items || !index || !host_index || !host_labels) {
            return s ? s : spk::kAllocation;
        }
        cudaMemcpyAsync(staging, data->crops, sizeof(float) * nc, cudaMemcpyHostToDevice, ctx->stream);
        spk::to_bf16_kernel<<<spk::grid_for(nc), 256, 0, ctx->stream>>>(staging, nc, crops);
        cudaMemcpyAsync(staging, data->items, sizeof(float) * ni, cudaMemcpyHostToDevice, ctx->stream);
        spk::to_bf16_kernel<<<spk::grid_for(ni), 256, 0, ctx->stream>>>(staging, ni, items);
        ctx->launches += 2;
        std::uint64_t state = seed;
        for (std::uint32_t t = 0; t < steps; ++t) {
            for (std::uint32_t b = 0; b < batch; ++b) {
                const std::uint64_t pick = spk::splitmix(state) % data->sample_count;
                host_index[2 * batch * t + b] = data->sample_crop[pick];
                host_index[2 * batch * t + batch + b] = data->sample_item[pick];
                host_labels[batch * t + b] = data->sample_label[pick];
            }
        }
        const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
        for (std::uint32_t t = 0; t < steps; ++t) {
            cudaMemcpyAsync(index, host_index + 2 * batch * t, sizeof(std::uint32_t) * 2 * batch,
                            cudaMemcpyHostToDevice, ctx->stream);
            cudaMemcpyAsync(net->labels, host_labels + batch * t, sizeof(float) * batch, cudaMemcpyHostToDevice,
                            ctx->stream);
            spk::assemble_kernel<<<spk::grid_for(static_cast<long long>(batch) * spk::kProposalVoxels), 256, 0,
                                   ctx->stream>>>(crops, index, items, index + batch, static_cast<int>(batch),
                                                  net->x0);
            ctx->launches++;
            if ((s = spk::launch_gradients(ctx, net, batch))) {
                return s;
            }
            net->adam_t += 1;
            net->version++;
            const float c1 = 1.f - std::pow(b1, static_cast<float>(net->adam_t));
            const float c2 = 1.f - std::pow(b2, static_cast<float>(net->adam_t));
            spk::adam_kernel<<<spk::grid_for(static_cast<long long>(net->count)), 256, 0, ctx->stream>>>(
                net->params, net->grads, net->adam_m, net->adam_v, static_cast<long long>(net->count), learning_rate,
                b1, b2, eps, c1, c2);
            ctx->launches++;
            if ((s = spk::pack_all(ctx, net))) {
                return s;
            }
            if (losses) {
                cudaMemcpyAsync(losses + t, net->loss, sizeof(float), cudaMemcpyDeviceToHost, ctx->stream);
            }
        }
        return spk::check_error(ctx, net);
    }
    catch (...) {
        return spk::kAllocation;
    }
}

}  // extern "C"

namespace spk {
ProposalNet* proposal_net(spk_proposal* p) { return p ? &p->net : nullptr; }
}  // namespace spk
