// Kernels of the surrogate charge model (a 1D Fourier neural operator used
// to start the self-consistent loop): a BF16 tensor-core GEMM with FP32
// accumulation and the elementwise / reduction kernels of its training and
// inference.  The reference engine has no counterpart.
//
// GEMM: C[b] (M x N, FP32) = A[b] (M x K) * B[b] (K x N), BF16 operands in any
// of the four layouts (A row- or column-major, B row- or column-major), with
// strided batches; optional accumulation into C and an optional BF16 copy of
// the result.  CTA tile 128 x 128 x 32, 8 warps (2 x 4), warp tile 64 x 32 of
// mma.sync m16n8k16 (BF16 in, FP32 accumulate).  Tiles go global -> registers
// -> shared memory (k-contiguous rows, padded to 40 elements so that the
// fragment loads of a warp hit distinct banks); the next tile is loaded while
// the current one is multiplied.  Every global access is bounds-checked, so
// M, N, K need not be tile multiples.

#include <cuda.h>
#include <cuda_bf16.h>

#include <algorithm>
#include <cstdint>

#include "negf_internal.h"

namespace negf {
namespace {

constexpr int BM = 128, BN = 128, BK = 32, PAD = 40, NT = 256;

__device__ __forceinline__ unsigned pack2(const __nv_bfloat16* p) { return *reinterpret_cast<const unsigned*>(p); }

__device__ __forceinline__ void mma_bf16(float (&d)[4], const unsigned (&a)[4], const unsigned (&b)[2]) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// Element (m, k) of A and (k, n) of B for the four layouts.
template <bool AT>
__device__ __forceinline__ size_t a_off(int m, int k, int lda) {
    return AT ? (size_t)k * lda + m : (size_t)m * lda + k;
}
template <bool BT>
__device__ __forceinline__ size_t b_off(int k, int n, int ldb) {
    return BT ? (size_t)n * ldb + k : (size_t)k * ldb + n;
}

// splits > 1: blockIdx.z = batch * splits + split; the split covers K
// elements [split * kchunk, min(K, (split + 1) * kchunk)) and writes its
// partial product to the workspace (C = workspace, ldc = N, sC = M * N per z),
// summed by splitk_reduce_kernel in split order.
template <bool AT, bool BT>
__global__ void __launch_bounds__(NT) gemm_bf16_kernel(int M, int N, int K, const __nv_bfloat16* __restrict__ A,
                                                       int lda, long long sA, const __nv_bfloat16* __restrict__ B,
                                                       int ldb, long long sB, float* __restrict__ C, int ldc,
                                                       long long sC, __nv_bfloat16* __restrict__ Cb, int accumulate,
                                                       int splits, int kchunk) {
    __shared__ __align__(16) __nv_bfloat16 As[2][BM][PAD];
    __shared__ __align__(16) __nv_bfloat16 Bs[2][BN][PAD];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int wm = warp >> 2, wn = warp & 3;  // warp tile: rows wm*64, cols wn*32
    const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
    const long long bz = blockIdx.z / splits;
    const int split = blockIdx.z % splits;
    const int kbeg = split * kchunk;
    const int kend = min(K, kbeg + kchunk);
    A += bz * sA;
    B += bz * sB;
    C += splits > 1 ? (long long)blockIdx.z * sC : bz * sC;
    if (Cb) Cb += bz * sC;
    const __nv_bfloat16 zero = __float2bfloat16(0.0f);

    // staging: 16 elements of A and 16 of B per thread per k-tile.  Tiles that
    // lie inside the matrix with 16-byte aligned rows go through two 16-byte
    // vector loads per operand (fast path); edge tiles through bounds-checked
    // element loads, index i = tid + NT * j.
    const bool alignA = ((reinterpret_cast<uintptr_t>(A) & 15) == 0) && (lda % 8 == 0);
    const bool alignB = ((reinterpret_cast<uintptr_t>(B) & 15) == 0) && (ldb % 8 == 0);
    __nv_bfloat16 ra[16], rb[16];
    uint4 va[2], vb[2];
    bool fa = false, fb = false;
    auto load_tile = [&](int k0) {
        fa = alignA && m0 + BM <= M && k0 + BK <= kend;
        fb = alignB && n0 + BN <= N && k0 + BK <= kend;
        if (fa) {
            const uint4* p = AT ? reinterpret_cast<const uint4*>(A + (size_t)(k0 + (tid >> 3)) * lda + m0 + (tid & 7) * 16)
                                : reinterpret_cast<const uint4*>(A + (size_t)(m0 + (tid >> 1)) * lda + k0 + (tid & 1) * 16);
            va[0] = p[0];
            va[1] = p[1];
        }
        if (fb) {
            const uint4* p = BT ? reinterpret_cast<const uint4*>(B + (size_t)(n0 + (tid >> 1)) * ldb + k0 + (tid & 1) * 16)
                                : reinterpret_cast<const uint4*>(B + (size_t)(k0 + (tid >> 3)) * ldb + n0 + (tid & 7) * 16);
            vb[0] = p[0];
            vb[1] = p[1];
        }
#pragma unroll
        for (int j = 0; j < 16; ++j) {
            const int i = tid + NT * j;
            // A: the contiguous dimension varies fastest across threads
            int m, k;
            if (AT) {
                k = i / BM;
                m = i % BM;
            } else {
                m = i / BK;
                k = i % BK;
            }
            const int gm = m0 + m, gk = k0 + k;
            if (!fa) ra[j] = (gm < M && gk < kend) ? A[a_off<AT>(gm, gk, lda)] : zero;
            int n, kb;
            if (BT) {
                n = i / BK;
                kb = i % BK;
            } else {
                kb = i / BN;
                n = i % BN;
            }
            const int gn = n0 + n, gkb = k0 + kb;
            if (!fb) rb[j] = (gn < N && gkb < kend) ? B[b_off<BT>(gkb, gn, ldb)] : zero;
        }
    };
    auto store_tile = [&](int buf) {
        if (fa) {
            if (AT) {  // 16 consecutive m of one k: transpose into the k-contiguous rows
                const __nv_bfloat16* e = reinterpret_cast<const __nv_bfloat16*>(va);
                const int k = tid >> 3, mh = (tid & 7) * 16;
#pragma unroll
                for (int q = 0; q < 16; ++q) As[buf][mh + q][k] = e[q];
            } else {
                const int m = tid >> 1, kh = (tid & 1) * 16;
                *reinterpret_cast<uint4*>(&As[buf][m][kh]) = va[0];
                *reinterpret_cast<uint4*>(&As[buf][m][kh + 8]) = va[1];
            }
        }
        if (fb) {
            if (BT) {
                const int n = tid >> 1, kh = (tid & 1) * 16;
                *reinterpret_cast<uint4*>(&Bs[buf][n][kh]) = vb[0];
                *reinterpret_cast<uint4*>(&Bs[buf][n][kh + 8]) = vb[1];
            } else {
                const __nv_bfloat16* e = reinterpret_cast<const __nv_bfloat16*>(vb);
                const int k = tid >> 3, nh = (tid & 7) * 16;
#pragma unroll
                for (int q = 0; q < 16; ++q) Bs[buf][nh + q][k] = e[q];
            }
        }
#pragma unroll
        for (int j = 0; j < 16; ++j) {
            const int i = tid + NT * j;
            if (!fa) {
                int m, k;
                if (AT) {
                    k = i / BM;
                    m = i % BM;
                } else {
                    m = i / BK;
                    k = i % BK;
                }
                As[buf][m][k] = ra[j];
            }
            if (!fb) {
                int n, kb;
                if (BT) {
                    n = i / BK;
                    kb = i % BK;
                } else {
                    kb = i / BN;
                    n = i % BN;
                }
                Bs[buf][n][kb] = rb[j];
            }
        }
    };

    float acc[4][4][4];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b)
#pragma unroll
            for (int c = 0; c < 4; ++c) acc[a][b][c] = 0.0f;

    const int g = lane >> 2, t = lane & 3;
    const int ktiles = (kend - kbeg + BK - 1) / BK;
    load_tile(kbeg);
    store_tile(0);
    __syncthreads();
    for (int kt = 0; kt < ktiles; ++kt) {
        const int buf = kt & 1;
        if (kt + 1 < ktiles) load_tile(kbeg + (kt + 1) * BK);
#pragma unroll
        for (int kk = 0; kk < BK; kk += 16) {
            unsigned af[4][4], bf[4][2];
#pragma unroll
            for (int im = 0; im < 4; ++im) {
                const int r = wm * 64 + im * 16 + g;
                af[im][0] = pack2(&As[buf][r][kk + 2 * t]);
                af[im][1] = pack2(&As[buf][r + 8][kk + 2 * t]);
                af[im][2] = pack2(&As[buf][r][kk + 2 * t + 8]);
                af[im][3] = pack2(&As[buf][r + 8][kk + 2 * t + 8]);
            }
#pragma unroll
            for (int in = 0; in < 4; ++in) {
                const int c = wn * 32 + in * 8 + g;
                bf[in][0] = pack2(&Bs[buf][c][kk + 2 * t]);
                bf[in][1] = pack2(&Bs[buf][c][kk + 2 * t + 8]);
            }
#pragma unroll
            for (int im = 0; im < 4; ++im)
#pragma unroll
                for (int in = 0; in < 4; ++in) mma_bf16(acc[im][in], af[im], bf[in]);
        }
        if (kt + 1 < ktiles) {
            store_tile(buf ^ 1);  // the other buffer: last read one iteration ago, before the barrier below
        }
        __syncthreads();
    }
    // epilogue: c0,c1 at (row g, cols 2t, 2t+1); c2,c3 at (row g+8, same cols)
#pragma unroll
    for (int im = 0; im < 4; ++im)
#pragma unroll
        for (int in = 0; in < 4; ++in)
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int row = m0 + wm * 64 + im * 16 + g + 8 * h;
                if (row >= M) continue;
#pragma unroll
                for (int q = 0; q < 2; ++q) {
                    const int col = n0 + wn * 32 + in * 8 + 2 * t + q;
                    if (col >= N) continue;
                    float v = acc[im][in][2 * h + q];
                    float* p = C + (size_t)row * ldc + col;
                    if (splits > 1) {
                        *p = v;
                        continue;
                    }
                    if (accumulate) v += *p;
                    *p = v;
                    if (Cb) Cb[(size_t)row * ldc + col] = __float2bfloat16(v);
                }
            }
}

// ---------------------------------------------------------------------------
// The same GEMM on the 5th-generation tensor cores (tcgen05).  One CTA of 128
// threads computes a 128 x 128 tile of C with the FP32 accumulator in tensor
// memory: per k-tile of 64, the four warps stage the A and B tiles in shared
// memory in the UMMA canonical no-swizzle layout (8 x 16-byte core matrices),
// thread 0 issues four tcgen05.mma (M 128, N 128, K 16, BF16 in, FP32 out)
// and commits them to an mbarrier, and the next k-tile is staged in the other
// buffer while they run.  Operands whose contiguous dimension is K use the
// K-major descriptor, the others the MN-major one, so every staged chunk is
// one 16-byte store.  The epilogue reads the accumulator with tcgen05.ld (warp
// w owns rows 32w .. 32w + 31) and writes C as the mma.sync kernel does
// (bounds, accumulation, BF16 copy, split-K partials).
// Descriptor encodings (sm_100 UMMA):
//   shared-memory descriptor: start >> 4 in bits [0,14), leading byte offset
//   (between the two 8-element K groups of one K-16 step) >> 4 in [16,30),
//   stride byte offset (between 8-row MN groups) >> 4 in [32,46), version 1
//   in [46,48), layout 0 (no swizzle) in [61,64);
//   instruction descriptor (kind::f16): D F32 (1 << 4), A BF16 (1 << 7),
//   B BF16 (1 << 10), A MN-major (1 << 15), B MN-major (1 << 16), N >> 3 in
//   [17,23), M >> 4 in [24,29).
// Waits are bounded: a wait that runs out sets tc_error and the CTA writes
// NaN into its tile instead of results.
constexpr int TC_BM = 128, TC_BN = 128, TC_BK = 64, TC_NT = 128;
constexpr int TC_TILE_BYTES = TC_BM * TC_BK * 2;            // one operand tile per stage (16 KB)
constexpr int TC_SMEM = 2 * 2 * TC_TILE_BYTES + 64;         // 2 stages x (A, B) + barriers and the TMEM address
constexpr uint32_t TC_SBO = (TC_BK / 8) * 128;              // bytes between 8-row MN groups
constexpr uint32_t TC_LBO = 128;                            // bytes between 8-element K groups
constexpr long long TC_SPIN_LIMIT = 1LL << 28;

__device__ int tc_error;

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr) {
    return (uint64_t)((saddr >> 4) & 0x3FFF) | ((uint64_t)((TC_LBO >> 4) & 0x3FFF) << 16) |
           ((uint64_t)((TC_SBO >> 4) & 0x3FFF) << 32) | (1ull << 46);
}
template <bool AMN, bool BMN>
__device__ __forceinline__ uint32_t umma_idesc() {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((AMN ? 1u : 0u) << 15) | ((BMN ? 1u : 0u) << 16) |
           ((uint32_t)(TC_BN >> 3) << 17) | ((uint32_t)(TC_BM >> 4) << 24);
}
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
    for (long long i = 0; i < TC_SPIN_LIMIT; ++i) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(bar), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

// Chunk c (0 .. 1023) of a 128 x 64 operand tile: 8 contiguous elements
// starting at row r, column k.  A warp's 32 chunks cover 8 consecutive
// core-matrix rows x 4 consecutive 16-byte columns, so its global loads are
// 64-byte runs and its 16-byte shared stores hit 8 distinct bank groups
// (no conflicts in the no-swizzle core-matrix layout).
template <bool KCONTIG>
__device__ __forceinline__ void tc_chunk(int c, int& r, int& k) {
    const int lo = c & 7, mid = (c >> 3) & 3, rest = c >> 5;
    if (KCONTIG) {  // core rows are rows r; 8 K-groups of 8
        r = (rest & 15) * 8 + lo;
        k = ((rest >> 4) * 4 + mid) * 8;
    } else {  // core rows are k; 16 row-groups of 8
        k = (rest >> 2) * 8 + lo;
        r = ((rest & 3) * 4 + mid) * 8;
    }
}

// Stage one 128 x 64 operand tile (rows = the M or N dimension) into shared
// memory.  KCONTIG: the operand's contiguous dimension is K (element (r, k) at
// P[r * ld + k]), else it is the row dimension (element (r, k) at P[k * ld + r]).
// 1024 chunks of 8 contiguous elements, 8 per thread; a chunk inside the
// matrix with a 16-byte aligned address is one vector load, the rest are
// bounds-checked element loads (zero outside).
template <bool KCONTIG>
__device__ __forceinline__ void tc_load(const __nv_bfloat16* __restrict__ P, int ld, int r0, int rows, int k0,
                                        int kend, bool aligned, int tid, uint4 (&v)[8]) {
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const int c = tid + TC_NT * i;
        int r, k;
        tc_chunk<KCONTIG>(c, r, k);
        const int gr = r0 + r, gk = k0 + k;
        const bool full = KCONTIG ? (gr < rows && gk + 8 <= kend) : (gk < kend && gr + 8 <= rows);
        if (full && aligned) {
            const __nv_bfloat16* src = KCONTIG ? P + (size_t)gr * ld + gk : P + (size_t)gk * ld + gr;
            v[i] = *reinterpret_cast<const uint4*>(src);
        } else {
            __align__(16) __nv_bfloat16 e[8];
#pragma unroll
            for (int q = 0; q < 8; ++q) {
                const int rr = KCONTIG ? gr : gr + q, kk = KCONTIG ? gk + q : gk;
                e[q] = (rr < rows && kk < kend) ? P[KCONTIG ? (size_t)rr * ld + kk : (size_t)kk * ld + rr]
                                                : __float2bfloat16(0.0f);
            }
            v[i] = *reinterpret_cast<const uint4*>(e);
        }
    }
}
template <bool KCONTIG>
__device__ __forceinline__ void tc_store(unsigned char* tile, int tid, const uint4 (&v)[8]) {
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const int c = tid + TC_NT * i;
        int r, k;
        tc_chunk<KCONTIG>(c, r, k);
        uint32_t off;
        if (KCONTIG)  // K-major core matrix: row r % 8, 16 bytes of K
            off = (r >> 3) * TC_SBO + (k >> 3) * TC_LBO + (r & 7) * 16;
        else  // MN-major core matrix: row k % 8, 16 bytes of MN
            off = (r >> 3) * TC_SBO + (k >> 3) * TC_LBO + (k & 7) * 16;
        *reinterpret_cast<uint4*>(tile + off) = v[i];
    }
}

// Epilogue of both tcgen05 kernels: 16 accumulator columns of one row of C
// (bounds, accumulation, BF16 copy, split-K partials; NaN when a wait ran out).
__device__ __forceinline__ void tc_write16(float* __restrict__ C, int ldc, __nv_bfloat16* __restrict__ Cb, int row,
                                           int col0, int M, int N, const uint32_t (&r)[16], bool ok, bool vec_c,
                                           int splits, int accumulate) {
    if (row >= M) return;
    if (ok && col0 + 16 <= N && vec_c) {
        // 16 consecutive columns of one row: four 16-byte stores (whole sectors)
        float* p = C + (size_t)row * ldc + col0;
        float v[16];
#pragma unroll
        for (int q = 0; q < 16; ++q) v[q] = __uint_as_float(r[q]);
        if (splits == 1 && accumulate) {
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const float4 o = reinterpret_cast<const float4*>(p)[q];
                v[4 * q] += o.x;
                v[4 * q + 1] += o.y;
                v[4 * q + 2] += o.z;
                v[4 * q + 3] += o.w;
            }
        }
#pragma unroll
        for (int q = 0; q < 4; ++q)
            reinterpret_cast<float4*>(p)[q] = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
        if (splits == 1 && Cb) {
            __align__(16) __nv_bfloat16 hb[16];
#pragma unroll
            for (int q = 0; q < 16; ++q) hb[q] = __float2bfloat16(v[q]);
            uint4* pb = reinterpret_cast<uint4*>(Cb + (size_t)row * ldc + col0);
            pb[0] = reinterpret_cast<const uint4*>(hb)[0];
            pb[1] = reinterpret_cast<const uint4*>(hb)[1];
        }
        return;
    }
#pragma unroll
    for (int q = 0; q < 16; ++q) {
        const int col = col0 + q;
        if (col >= N) continue;
        float v = ok ? __uint_as_float(r[q]) : __int_as_float(0x7fc00000);
        float* p = C + (size_t)row * ldc + col;
        if (splits > 1) {
            *p = v;
            continue;
        }
        if (accumulate) v += *p;
        *p = v;
        if (Cb) Cb[(size_t)row * ldc + col] = __float2bfloat16(v);
    }
}

template <bool AT, bool BT>
__global__ void __launch_bounds__(TC_NT) gemm_tc_kernel(int M, int N, int K, const __nv_bfloat16* __restrict__ A,
                                                        int lda, long long sA, const __nv_bfloat16* __restrict__ B,
                                                        int ldb, long long sB, float* __restrict__ C, int ldc,
                                                        long long sC, __nv_bfloat16* __restrict__ Cb, int accumulate,
                                                        int splits, int kchunk) {
    // A (M x K): K contiguous unless AT; B (K x N): N contiguous unless BT
    constexpr bool AK = !AT, BK_ = BT;
    extern __shared__ __align__(1024) unsigned char tc_smem[];
    unsigned char* tiles = tc_smem;
    uint64_t* bars = reinterpret_cast<uint64_t*>(tc_smem + 4 * TC_TILE_BYTES);
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(tc_smem + 4 * TC_TILE_BYTES + 16);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int m0 = blockIdx.y * TC_BM, n0 = blockIdx.x * TC_BN;
    const long long bz = blockIdx.z / splits;
    const int split = blockIdx.z % splits;
    const int kbeg = split * kchunk;
    const int kend = min(K, kbeg + kchunk);
    A += bz * sA;
    B += bz * sB;
    C += splits > 1 ? (long long)blockIdx.z * sC : bz * sC;
    if (Cb) Cb += bz * sC;
    const bool alignA = ((reinterpret_cast<uintptr_t>(A) & 15) == 0) && (lda % 8 == 0);
    const bool alignB = ((reinterpret_cast<uintptr_t>(B) & 15) == 0) && (ldb % 8 == 0);
    // vector epilogue: rows of C (and of its BF16 copy) 16-byte aligned at every 16th column
    const bool vec_c = ((reinterpret_cast<uintptr_t>(C) & 15) == 0) && (ldc % 8 == 0) &&
                       (splits > 1 || !Cb || (reinterpret_cast<uintptr_t>(Cb) & 15) == 0);

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(TC_BN));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&bars[0])));
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&bars[1])));
        asm volatile("fence.mbarrier_init.release.cluster;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    const uint32_t tmem = *tmem_slot;

    const int ktiles = (kend - kbeg + TC_BK - 1) / TC_BK;
    uint32_t phase[2] = {0u, 0u};
    bool ok = true;
    for (int kt = 0; kt < ktiles && ok; ++kt) {
        const int s = kt & 1;
        const int k0 = kbeg + kt * TC_BK;
        uint4 va[8], vb[8];
        tc_load<AK>(A, lda, m0, M, k0, kend, alignA, tid, va);
        tc_load<BK_>(B, ldb, n0, N, k0, kend, alignB, tid, vb);
        if (kt >= 2) {  // the MMAs of k-tile kt - 2 read this buffer
            ok = mbar_wait(smem_u32(&bars[s]), phase[s]);
            phase[s] ^= 1u;
        }
        unsigned char* ta = tiles + (2 * s) * TC_TILE_BYTES;
        unsigned char* tb = tiles + (2 * s + 1) * TC_TILE_BYTES;
        tc_store<AK>(ta, tid, va);
        tc_store<BK_>(tb, tid, vb);
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        if (!__syncthreads_and(ok)) {
            ok = false;
            break;
        }
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;");
            const uint32_t idesc = umma_idesc<!AK, !BK_>();
#pragma unroll
            for (int ks = 0; ks < TC_BK / 16; ++ks) {
                const uint64_t da = umma_desc(smem_u32(ta) + ks * 2 * TC_LBO);
                const uint64_t db = umma_desc(smem_u32(tb) + ks * 2 * TC_LBO);
                const uint32_t acc = (kt > 0 || ks > 0) ? 1u : 0u;
                asm volatile(
                    "{\n\t.reg .pred p;\n\t"
                    "setp.ne.b32 p, %4, 0;\n\t"
                    "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
                    :
                    : "r"(tmem), "l"(da), "l"(db), "r"(idesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                             smem_u32(&bars[s]))
                         : "memory");
        }
    }
    if (ok && ktiles > 0) {  // the last commit covers every MMA issued before it
        const int sl = (ktiles - 1) & 1;
        ok = mbar_wait(smem_u32(&bars[sl]), phase[sl]);
    }
    ok = __syncthreads_and(ok) != 0;
    asm volatile("tcgen05.fence::after_thread_sync;");
    if (!ok && tid == 0) atomicExch(&tc_error, 1);
    // epilogue: warp w reads accumulator rows 32w .. 32w + 31 (its TMEM lanes), 16 columns at a time
    const int row = m0 + warp * 32 + lane;
#pragma unroll 1
    for (int c0 = 0; c0 < TC_BN; c0 += 16) {
        uint32_t r[16];
        if (ktiles > 0) {
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
                "%14, %15}, [%16];\n"
                : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                  "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
                  "=r"(r[15])
                : "r"(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        } else {
#pragma unroll
            for (int q = 0; q < 16; ++q) r[q] = 0u;
        }
        tc_write16(C, ldc, Cb, row, n0 + c0, M, N, r, ok, vec_c, splits, accumulate);
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TC_BN));
}

// ---------------------------------------------------------------------------
// The tcgen05 GEMM fed by the Tensor Memory Accelerator.  Same tile and
// accumulator as gemm_tc_kernel, but the operand tiles arrive by
// cp.async.bulk.tensor (one elected thread issues them) into the 128-byte
// swizzled UMMA layout, through a ring of TMA_STAGES k-tile buffers with a
// "full" mbarrier (transaction bytes) and an "empty" mbarrier (the commit of
// the MMAs that read the buffer) per stage: warp 0 produces, warp 1 issues
// the MMAs, all four warps run the epilogue.  Tiles past the matrix edges
// arrive zero-filled (out-of-bounds fill), so edge tiles need no special path.
//   K-major operand (K contiguous): one box of 64 K x 128 rows per stage,
//   rows of 128 bytes, 8-row swizzle atoms 1024 bytes apart (SBO); a K-16
//   step advances the descriptor's start by 32 bytes inside the atom.
//   MN-major operand (M or N contiguous): two boxes of 64 MN x 64 K, rows
//   (one K each) of 128 bytes; 8-row K groups 1024 bytes apart (SBO), the two
//   64-wide MN halves 8 KB apart (LBO); a K-16 step advances 2048 bytes.
// Descriptor layout type 2 = 128-byte swizzle (bits [61,64)).
// ring of ST stages + alignment slack + barriers; 4 stages for long K, 2 (three CTAs per SM) for K <= 128
constexpr int tma_smem(int st) { return st * 2 * TC_TILE_BYTES + 1024 + 128; }

__device__ __forceinline__ uint64_t umma_desc_sw128(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((saddr >> 4) & 0x3FFF) | ((uint64_t)((lbo >> 4) & 0x3FFF) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFF) << 32) | (1ull << 46) | (2ull << 61);
}
__device__ __forceinline__ void tma_load_3d(uint32_t dst, const CUtensorMap* map, uint32_t bar, int c0, int c1,
                                            int c2) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5}], "
        "[%2];" ::"r"(dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(bar), "r"(c0), "r"(c1), "r"(c2)
        : "memory");
}

template <bool AK, bool BKC, int TMA_STAGES>
__global__ void __launch_bounds__(TC_NT) gemm_tma_kernel(const __grid_constant__ CUtensorMap tmA,
                                                         const __grid_constant__ CUtensorMap tmB, int M, int N,
                                                         int K, float* __restrict__ C, int ldc, long long sC,
                                                         __nv_bfloat16* __restrict__ Cb, int accumulate, int splits,
                                                         int kchunk, int a_batched, int b_batched) {
    extern __shared__ unsigned char tma_smem_raw[];
    // 1024-byte aligned ring (the swizzle atoms' alignment)
    const uint32_t raw = smem_u32(tma_smem_raw);
    const uint32_t ring = (raw + 1023u) & ~1023u;
    unsigned char* ring_ptr = tma_smem_raw + (ring - raw);
    uint64_t* full = reinterpret_cast<uint64_t*>(ring_ptr + TMA_STAGES * 2 * TC_TILE_BYTES);
    uint64_t* empty = full + TMA_STAGES;
    uint64_t* done = empty + TMA_STAGES;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(done + 1);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int m0 = blockIdx.y * TC_BM, n0 = blockIdx.x * TC_BN;
    const int bz = blockIdx.z / splits;
    const int split = blockIdx.z % splits;
    const int kbeg = split * kchunk;
    const int kend = min(K, kbeg + kchunk);
    C += splits > 1 ? (long long)blockIdx.z * sC : (long long)bz * sC;
    if (Cb) Cb += (long long)bz * sC;
    const bool vec_c = ((reinterpret_cast<uintptr_t>(C) & 15) == 0) && (ldc % 8 == 0) &&
                       (splits > 1 || !Cb || (reinterpret_cast<uintptr_t>(Cb) & 15) == 0);

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(TC_BN));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 32) {
        for (int i = 0; i < TMA_STAGES; ++i) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&full[i])));
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&empty[i])));
        }
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(done)));
        asm volatile("fence.mbarrier_init.release.cluster;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    const uint32_t tmem = *tmem_slot;
    const int ktiles = (kend - kbeg + TC_BK - 1) / TC_BK;
    const int za = a_batched ? bz : 0, zb = b_batched ? bz : 0;
    bool ok = true;

    if (tid == 0) {  // producer
        for (int kt = 0; kt < ktiles && ok; ++kt) {
            const int s = kt % TMA_STAGES;
            if (kt >= TMA_STAGES) ok = mbar_wait(smem_u32(&empty[s]), (uint32_t)((kt / TMA_STAGES - 1) & 1));
            if (!ok) break;
            const uint32_t bar = smem_u32(&full[s]);
            asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(2 * TC_TILE_BYTES)
                         : "memory");
            const uint32_t ta = ring + (2 * s) * TC_TILE_BYTES, tb = ring + (2 * s + 1) * TC_TILE_BYTES;
            const int k0 = kbeg + kt * TC_BK;
            if (AK) {
                tma_load_3d(ta, &tmA, bar, k0, m0, za);
            } else {
                tma_load_3d(ta, &tmA, bar, m0, k0, za);
                tma_load_3d(ta + TC_TILE_BYTES / 2, &tmA, bar, m0 + 64, k0, za);
            }
            if (BKC) {
                tma_load_3d(tb, &tmB, bar, k0, n0, zb);
            } else {
                tma_load_3d(tb, &tmB, bar, n0, k0, zb);
                tma_load_3d(tb + TC_TILE_BYTES / 2, &tmB, bar, n0 + 64, k0, zb);
            }
        }
    } else if (tid == 32) {  // MMA issuer
        const uint32_t idesc = umma_idesc<!AK, !BKC>();
        for (int kt = 0; kt < ktiles && ok; ++kt) {
            const int s = kt % TMA_STAGES;
            ok = mbar_wait(smem_u32(&full[s]), (uint32_t)((kt / TMA_STAGES) & 1));
            if (!ok) break;
            asm volatile("tcgen05.fence::after_thread_sync;");
            const uint32_t ta = ring + (2 * s) * TC_TILE_BYTES, tb = ring + (2 * s + 1) * TC_TILE_BYTES;
#pragma unroll
            for (int ks = 0; ks < TC_BK / 16; ++ks) {
                const uint64_t da = AK ? umma_desc_sw128(ta + ks * 32, 16, 1024)
                                       : umma_desc_sw128(ta + ks * 2048, TC_TILE_BYTES / 2, 1024);
                const uint64_t db = BKC ? umma_desc_sw128(tb + ks * 32, 16, 1024)
                                        : umma_desc_sw128(tb + ks * 2048, TC_TILE_BYTES / 2, 1024);
                const uint32_t acc = (kt > 0 || ks > 0) ? 1u : 0u;
                asm volatile(
                    "{\n\t.reg .pred p;\n\t"
                    "setp.ne.b32 p, %4, 0;\n\t"
                    "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
                    :
                    : "r"(tmem), "l"(da), "l"(db), "r"(idesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                             smem_u32(&empty[s]))
                         : "memory");
        }
        if (ok && ktiles > 0)
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                             smem_u32(done))
                         : "memory");
    }
    ok = __syncthreads_and(ok) != 0;
    if (ok && ktiles > 0) ok = mbar_wait(smem_u32(done), 0u);
    ok = __syncthreads_and(ok) != 0;
    asm volatile("tcgen05.fence::after_thread_sync;");
    if (!ok && tid == 0) atomicExch(&tc_error, 1);
    const int row = m0 + warp * 32 + lane;
#pragma unroll 1
    for (int c0 = 0; c0 < TC_BN; c0 += 16) {
        uint32_t r[16];
        if (ktiles > 0) {
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
                "%14, %15}, [%16];\n"
                : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                  "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
                  "=r"(r[15])
                : "r"(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        } else {
#pragma unroll
            for (int q = 0; q < 16; ++q) r[q] = 0u;
        }
        tc_write16(C, ldc, Cb, row, n0 + c0, M, N, r, ok, vec_c, splits, accumulate);
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TC_BN));
}

// C[b][m][n] (+)= sum over splits (in order) of W[b * splits + s][m][n]
__global__ void splitk_reduce_kernel(int M, int N, int batch, int splits, const float* __restrict__ W,
                                     float* __restrict__ C, int ldc, long long sC, __nv_bfloat16* __restrict__ Cb,
                                     int accumulate) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long MN = (long long)M * N;
    if (i >= MN * batch) return;
    const long long b = i / MN, r = i % MN;
    const int m = (int)(r / N), n = (int)(r % N);
    float v = 0.0f;
    for (int s = 0; s < splits; ++s) v += W[(b * splits + s) * MN + r];
    float* p = C + b * sC + (size_t)m * ldc + n;
    if (accumulate) v += *p;
    *p = v;
    if (Cb) Cb[b * sC + (size_t)m * ldc + n] = __float2bfloat16(v);
}

__device__ __forceinline__ float gelu(float x) {
    const float k0 = 0.7978845608028654f, k1 = 0.044715f;
    return 0.5f * x * (1.0f + tanhf(k0 * (x + k1 * x * x * x)));
}
__device__ __forceinline__ float gelu_grad(float x) {
    const float k0 = 0.7978845608028654f, k1 = 0.044715f;
    const float u = k0 * (x + k1 * x * x * x), th = tanhf(u);
    return 0.5f * (1.0f + th) + 0.5f * x * (1.0f - th * th) * k0 * (1.0f + 3.0f * k1 * x * x);
}

// pre[r][c] = a[r][c] + b[r][c] + bias[c]; out = gelu(pre) (FP32 and BF16)
__global__ void gelu_fwd_kernel(long long rows, int cols, const float* __restrict__ a, const float* __restrict__ b,
                                const float* __restrict__ bias, float* __restrict__ pre, float* __restrict__ out,
                                __nv_bfloat16* __restrict__ outb, int act) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= rows * cols) return;
    const int c = (int)(i % cols);
    const float x = a[i] + (b ? b[i] : 0.0f) + (bias ? bias[c] : 0.0f);
    if (pre) pre[i] = x;
    const float y = act ? gelu(x) : x;
    if (out) out[i] = y;
    if (outb) outb[i] = __float2bfloat16(y);
}

// d[i] = dy[i] * gelu'(pre[i]) (FP32 and BF16 copies)
__global__ void gelu_bwd_kernel(long long n, const float* __restrict__ dy, const float* __restrict__ pre,
                                float* __restrict__ d, __nv_bfloat16* __restrict__ db) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float v = dy[i] * gelu_grad(pre[i]);
    if (d) d[i] = v;
    if (db) db[i] = __float2bfloat16(v);
}

// out[c] (+)= sum_r x[r][c], one block per 32 columns, fixed order.
__global__ void colsum_kernel(long long rows, int cols, const float* __restrict__ x, float* __restrict__ out,
                              int accumulate) {
    __shared__ float sh[8][33];
    const int c = blockIdx.x * 32 + threadIdx.x;
    float s = 0.0f;
    if (c < cols)
        for (long long r = threadIdx.y; r < rows; r += 8) s += x[r * cols + c];
    sh[threadIdx.y][threadIdx.x] = s;
    __syncthreads();
    if (threadIdx.y == 0 && c < cols) {
        float t = 0.0f;
        for (int y = 0; y < 8; ++y) t += sh[y][threadIdx.x];
        out[c] = accumulate ? out[c] + t : t;
    }
}

__global__ void cast_bf16_kernel(long long n, const float* __restrict__ x, __nv_bfloat16* __restrict__ y) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) y[i] = __float2bfloat16(x[i]);
}

// Adam on FP32 master weights, refreshed BF16 copy.
__global__ void adam_kernel(long long n, float* __restrict__ w, const float* __restrict__ g, float* __restrict__ m,
                            float* __restrict__ v, __nv_bfloat16* __restrict__ wb, float lr, float b1, float b2,
                            float eps, float c1, float c2, float wd) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i] + wd * w[i];
    const float mi = b1 * m[i] + (1.0f - b1) * gi;
    const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    const float wi = w[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    w[i] = wi;
    if (wb) wb[i] = __float2bfloat16(wi);
}

// Per row r: q[r] = sum_c h[r][c] w[c] + b (one warp per row)
__global__ void rowdot_kernel(long long rows, int cols, const float* __restrict__ h, const float* __restrict__ w,
                              const float* __restrict__ b, float* __restrict__ q) {
    const long long r = (long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (r >= rows) return;
    float s = 0.0f;
    for (int c = lane; c < cols; c += 32) s += h[r * cols + c] * w[c];
#pragma unroll
    for (int o = 16; o >= 1; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) q[r] = s + (b ? *b : 0.0f);
}

// dh[r][c] = dq[r] * w[c] (FP32 and BF16)
__global__ void outer_kernel(long long rows, int cols, const float* __restrict__ dq, const float* __restrict__ w,
                             float* __restrict__ dh, __nv_bfloat16* __restrict__ dhb) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= rows * cols) return;
    const float v = dq[i / cols] * w[i % cols];
    if (dh) dh[i] = v;
    if (dhb) dhb[i] = __float2bfloat16(v);
}

// Squared-error loss: d[i] = 2 (q[i] - y[i]) / n; per-block partial sums of (q - y)^2.
__global__ void mse_kernel(long long n, const float* __restrict__ q, const float* __restrict__ y, float* __restrict__ d,
                           float* __restrict__ part) {
    __shared__ float sh[256];
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    float e = 0.0f;
    if (i < n) {
        const float r = q[i] - y[i];
        d[i] = 2.0f * r / (float)n;
        e = r * r;
    }
    sh[threadIdx.x] = e;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s) sh[threadIdx.x] += sh[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = sh[0];
}

}  // namespace

// Tensor maps of the TMA path.  An operand is described as a 3-d tensor
// (contiguous dimension, the other matrix dimension, batch) with 128-byte
// swizzle; boxes of 64 x 128 (K contiguous) or 64 x 64 (M or N contiguous).
// cudaErrorNotSupported: the operand's layout cannot be described (16-byte
// alignment of the base and the leading dimension, batches that overlap) and
// the caller takes the register-staged kernel.
using EncodeTiled = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                 const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                 CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
static EncodeTiled encode_tiled() {
    static EncodeTiled fn = nullptr;
    static bool tried = false;
    if (!tried) {
        tried = true;
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiled>(p);
    }
    return fn;
}
// inner: the contiguous extent, outer: the other extent, ld: elements between
// rows of outer, sb: elements between batches (0: shared by every batch)
static bool make_map(CUtensorMap* m, const __nv_bfloat16* base, long long inner, long long outer, int ld, long long sb,
                     int batch, bool k_contig, int* batched) {
    EncodeTiled enc = encode_tiled();
    if (!enc) return false;
    if ((reinterpret_cast<uintptr_t>(base) & 15) != 0 || ld % 8 != 0 || ld < inner) return false;
    const bool use_batch = batch > 1 && sb != 0;
    if (use_batch && (sb % 8 != 0 || sb < (long long)ld * outer)) return false;
    *batched = use_batch ? 1 : 0;
    const cuuint64_t dims[3] = {(cuuint64_t)inner, (cuuint64_t)outer, (cuuint64_t)(use_batch ? batch : 1)};
    const cuuint64_t strides[2] = {(cuuint64_t)ld * 2, (cuuint64_t)(use_batch ? sb : (long long)ld * outer) * 2};
    const cuuint32_t box[3] = {64, (cuuint32_t)(k_contig ? 128 : 64), 1};
    const cuuint32_t estr[3] = {1, 1, 1};
    return enc(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 3, const_cast<__nv_bfloat16*>(base), dims, strides, box, estr,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}
template <bool AK, bool BKC, int ST>
static cudaError_t launch_tma_st(int M, int N, int K, int batch, const __nv_bfloat16* a, int lda, long long sA,
                              const __nv_bfloat16* b, int ldb, long long sB, float* out, int ldo, long long so,
                              __nv_bfloat16* cb, int accumulate, int splits, int kchunk, dim3 grid, cudaStream_t s) {
    CUtensorMap ta, tb;
    int ab = 0, bb = 0;
    // A (M x K): K contiguous when AK; B (K x N): K contiguous when BKC
    if (!make_map(&ta, a, AK ? K : M, AK ? M : K, lda, sA, batch, AK, &ab)) return cudaErrorNotSupported;
    if (!make_map(&tb, b, BKC ? K : N, BKC ? N : K, ldb, sB, batch, BKC, &bb)) return cudaErrorNotSupported;
    static bool attr = false;
    if (!attr) {
        cudaFuncSetAttribute(gemm_tma_kernel<AK, BKC, ST>, cudaFuncAttributeMaxDynamicSharedMemorySize, tma_smem(ST));
        attr = true;
    }
    gemm_tma_kernel<AK, BKC, ST><<<grid, TC_NT, tma_smem(ST), s>>>(ta, tb, M, N, K, out, ldo, so, cb, accumulate,
                                                                  splits, kchunk, ab, bb);
    return cudaGetLastError();
}
template <bool AK, bool BKC>
static cudaError_t launch_tma(int M, int N, int K, int batch, const __nv_bfloat16* a, int lda, long long sA,
                              const __nv_bfloat16* b, int ldb, long long sB, float* out, int ldo, long long so,
                              __nv_bfloat16* cb, int accumulate, int splits, int kchunk, dim3 grid, cudaStream_t s) {
    if (std::min(K, kchunk) <= 2 * TC_BK)
        return launch_tma_st<AK, BKC, 2>(M, N, K, batch, a, lda, sA, b, ldb, sB, out, ldo, so, cb, accumulate, splits,
                                         kchunk, grid, s);
    return launch_tma_st<AK, BKC, 4>(M, N, K, batch, a, lda, sA, b, ldb, sB, out, ldo, so, cb, accumulate, splits,
                                     kchunk, grid, s);
}

cudaError_t nn_gemm(int at, int bt, int M, int N, int K, int batch, const void* A, int lda, long long sA,
                    const void* B, int ldb, long long sB, float* C, int ldc, long long sC, void* Cb, int accumulate,
                    cudaStream_t s, int path) {
    if (M <= 0 || N <= 0 || K <= 0 || batch <= 0) return cudaSuccess;
    const int tiles = ((N + BN - 1) / BN) * ((M + BM - 1) / BM) * batch;
    // split K when the output has too few tiles to fill the GPU (deterministic: partials + ordered sum)
    // (k-chunks in whole 64-element tiles, so that a tensor-core k-tile never straddles two splits)
    const int kg = path == kNnGemmMmaSync ? BK : TC_BK;
    int splits = 1;
    const int kt = (K + kg - 1) / kg;
    if (tiles < 296 && kt >= 8) splits = std::min(std::min(296 / tiles + 1, kt / 4), 64);
    if (splits < 1) splits = 1;
    const int kchunk = ((kt + splits - 1) / splits) * kg;
    splits = (K + kchunk - 1) / kchunk;
    static float* ws = nullptr;
    static size_t ws_bytes = 0;
    float* out = C;
    int ldo = ldc;
    long long so = sC;
    if (splits > 1) {
        const size_t need = sizeof(float) * (size_t)M * N * batch * splits;
        if (need > ws_bytes) {
            if (ws) cudaFree(ws);
            ws = nullptr;
            ws_bytes = 0;
            cudaError_t e = cudaMalloc(&ws, need);
            if (e != cudaSuccess) return e;
            ws_bytes = need;
        }
        out = ws;
        ldo = N;
        so = (long long)M * N;
    }
    dim3 grid((N + BN - 1) / BN, (M + BM - 1) / BM, batch * splits);
    const auto* a = static_cast<const __nv_bfloat16*>(A);
    const auto* b = static_cast<const __nv_bfloat16*>(B);
    auto* cb = splits > 1 ? nullptr : static_cast<__nv_bfloat16*>(Cb);
    if (path != kNnGemmMmaSync && path != kNnGemmTcgen05Staged) {
        cudaError_t e = cudaErrorNotSupported;
        if (at == 0 && bt == 0)
            e = launch_tma<true, false>(M, N, K, batch, a, lda, sA, b, ldb, sB, out, ldo, so, cb, accumulate, splits,
                                        kchunk, grid, s);
        else if (at == 0 && bt == 1)
            e = launch_tma<true, true>(M, N, K, batch, a, lda, sA, b, ldb, sB, out, ldo, so, cb, accumulate, splits,
                                       kchunk, grid, s);
        else if (at == 1 && bt == 0)
            e = launch_tma<false, false>(M, N, K, batch, a, lda, sA, b, ldb, sB, out, ldo, so, cb, accumulate, splits,
                                         kchunk, grid, s);
        else
            e = launch_tma<false, true>(M, N, K, batch, a, lda, sA, b, ldb, sB, out, ldo, so, cb, accumulate, splits,
                                        kchunk, grid, s);
        if (e == cudaSuccess) {
            if (splits == 1) return cudaSuccess;
            const long long n = (long long)M * N * batch;
            splitk_reduce_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(M, N, batch, splits, ws, C, ldc, sC,
                                                                             static_cast<__nv_bfloat16*>(Cb),
                                                                             accumulate);
            return cudaGetLastError();
        }
        if (e != cudaErrorNotSupported) return e;
        // operands TMA cannot describe: the register-staged tcgen05 kernel
    }
    if (path != kNnGemmMmaSync) {
        static bool attr_set = false;
        if (!attr_set) {
            cudaFuncSetAttribute(gemm_tc_kernel<false, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, TC_SMEM);
            cudaFuncSetAttribute(gemm_tc_kernel<false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, TC_SMEM);
            cudaFuncSetAttribute(gemm_tc_kernel<true, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, TC_SMEM);
            cudaFuncSetAttribute(gemm_tc_kernel<true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, TC_SMEM);
            attr_set = true;
        }
        static_assert(TC_BM == BM && TC_BN == BN, "the two GEMM paths share the tiling of C");
        if (!at && !bt)
            gemm_tc_kernel<false, false><<<grid, TC_NT, TC_SMEM, s>>>(M, N, K, a, lda, sA, b, ldb, sB, out, ldo, so,
                                                                      cb, accumulate, splits, kchunk);
        else if (!at && bt)
            gemm_tc_kernel<false, true><<<grid, TC_NT, TC_SMEM, s>>>(M, N, K, a, lda, sA, b, ldb, sB, out, ldo, so,
                                                                     cb, accumulate, splits, kchunk);
        else if (at && !bt)
            gemm_tc_kernel<true, false><<<grid, TC_NT, TC_SMEM, s>>>(M, N, K, a, lda, sA, b, ldb, sB, out, ldo, so,
                                                                     cb, accumulate, splits, kchunk);
        else
            gemm_tc_kernel<true, true><<<grid, TC_NT, TC_SMEM, s>>>(M, N, K, a, lda, sA, b, ldb, sB, out, ldo, so,
                                                                    cb, accumulate, splits, kchunk);
    } else if (!at && !bt)
        gemm_bf16_kernel<false, false><<<grid, NT, 0, s>>>(M, N, K, a, lda, sA, b, ldb, sB, out, ldo, so, cb,
                                                           accumulate, splits, kchunk);
    else if (!at && bt)
        gemm_bf16_kernel<false, true><<<grid, NT, 0, s>>>(M, N, K, a, lda, sA, b, ldb, sB, out, ldo, so, cb,
                                                          accumulate, splits, kchunk);
    else if (at && !bt)
        gemm_bf16_kernel<true, false><<<grid, NT, 0, s>>>(M, N, K, a, lda, sA, b, ldb, sB, out, ldo, so, cb,
                                                          accumulate, splits, kchunk);
    else
        gemm_bf16_kernel<true, true><<<grid, NT, 0, s>>>(M, N, K, a, lda, sA, b, ldb, sB, out, ldo, so, cb,
                                                         accumulate, splits, kchunk);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess || splits == 1) return e;
    const long long n = (long long)M * N * batch;
    splitk_reduce_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(M, N, batch, splits, ws, C, ldc, sC,
                                                                     static_cast<__nv_bfloat16*>(Cb), accumulate);
    return cudaGetLastError();
}

static unsigned blocks_for(long long n, int t) { return (unsigned)((n + t - 1) / t); }

cudaError_t nn_gelu_fwd(long long rows, int cols, const float* a, const float* b, const float* bias, float* pre,
                        float* out, void* outb, int act, cudaStream_t s) {
    const long long n = rows * cols;
    if (n <= 0) return cudaSuccess;
    gelu_fwd_kernel<<<blocks_for(n, 256), 256, 0, s>>>(rows, cols, a, b, bias, pre, out,
                                                       static_cast<__nv_bfloat16*>(outb), act);
    return cudaGetLastError();
}
cudaError_t nn_gelu_bwd(long long n, const float* dy, const float* pre, float* d, void* db, cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    gelu_bwd_kernel<<<blocks_for(n, 256), 256, 0, s>>>(n, dy, pre, d, static_cast<__nv_bfloat16*>(db));
    return cudaGetLastError();
}
cudaError_t nn_colsum(long long rows, int cols, const float* x, float* out, int accumulate, cudaStream_t s) {
    if (cols <= 0) return cudaSuccess;
    colsum_kernel<<<(cols + 31) / 32, dim3(32, 8), 0, s>>>(rows, cols, x, out, accumulate);
    return cudaGetLastError();
}
cudaError_t nn_cast_bf16(long long n, const float* x, void* y, cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    cast_bf16_kernel<<<blocks_for(n, 256), 256, 0, s>>>(n, x, static_cast<__nv_bfloat16*>(y));
    return cudaGetLastError();
}
cudaError_t nn_adam(long long n, float* w, const float* g, float* m, float* v, void* wb, float lr, float b1, float b2,
                    float eps, int step, float wd, cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    const float c1 = 1.0f - powf(b1, (float)step), c2 = 1.0f - powf(b2, (float)step);
    adam_kernel<<<blocks_for(n, 256), 256, 0, s>>>(n, w, g, m, v, static_cast<__nv_bfloat16*>(wb), lr, b1, b2, eps, c1,
                                                   c2, wd);
    return cudaGetLastError();
}
cudaError_t nn_rowdot(long long rows, int cols, const float* h, const float* w, const float* b, float* q,
                      cudaStream_t s) {
    if (rows <= 0) return cudaSuccess;
    rowdot_kernel<<<blocks_for(rows, 8), 256, 0, s>>>(rows, cols, h, w, b, q);
    return cudaGetLastError();
}
cudaError_t nn_outer(long long rows, int cols, const float* dq, const float* w, float* dh, void* dhb, cudaStream_t s) {
    const long long n = rows * cols;
    if (n <= 0) return cudaSuccess;
    outer_kernel<<<blocks_for(n, 256), 256, 0, s>>>(rows, cols, dq, w, dh, static_cast<__nv_bfloat16*>(dhb));
    return cudaGetLastError();
}
cudaError_t nn_mse(long long n, const float* q, const float* y, float* d, float* part, cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    mse_kernel<<<blocks_for(n, 256), 256, 0, s>>>(n, q, y, d, part);
    return cudaGetLastError();
}

}  // namespace negf
