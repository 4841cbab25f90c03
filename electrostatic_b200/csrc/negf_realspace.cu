// Real-space ring-block RGF of a zigzag (m,0) tube (FP64, or mixed FP32/FP64).
//
// Blocks of two rings (2m atoms, m <= 16): ring a = 2k and ring b = 2k+1 are
// joined by the double bond (atom j of a to atoms j and j+1 mod m of b:
// E - H has -gamma C with C[j][j] = C[j][j+1] = 1), ring b of block k and
// ring a of block k+1 by the single bond (atom j to atom j, -gamma I).  In
// mode space these are beta_J = 2 gamma cos(pi J/m) and gamma
// (CNT.cpp:288-336), so a ring-uniform potential reproduces the sum of the m
// mode chains.  The dense 2m x 2m block is
//     M_k = [[A, -gamma C], [-gamma C^T, D]],
// A = diag(E - U_a) - Sigma_a, D = diag(E - U_b) - Sigma_b, where the
// self-energies of the neighbours touch one ring each.  The block algebra
// works on m x m ring corners with Schur complements instead of 2m x 2m
// inversions:
//   forward  (Sigma_b = 0, D diagonal): X_k = g_L[a][a] = S^-1 with
//            S = A - gamma^2 C D^-1 C^T (C D^-1 C^T has three diagonals);
//            g_L[b][b] = D^-1 + gamma^2 Y^T X Y and g_L[a][b] = gamma X Y,
//            Y = C D^-1, follow from X with O(m^2) work; X_k is kept.
//   backward G_kk = g_L + gamma^2 g_L[:, b] G_{k+1}[a][a] g_L[b, :] gives
//            G[a][a] = X + gamma^4 X (Y G' Y^T) X  and
//            tr G[b][b] = tr g_L[b][b] + gamma^2 tr(g_L[b][b] G' g_L[b][b])
//            with G' = G_{k+1}[a][a]: three m x m products per block.  The
//            right lead enters through G_K[a][a] = (I - gamma^2 s_R
//            g_L[b][b])^-1 s_R of its first ring.
// One block update costs one m x m inversion and three m x m products
// instead of three 2m x 2m inversions (about 10x fewer operations).
//
// Leads: a lead is uniform (the contact potential on every atom), so the
// ring Fourier modes decouple it into the mode chains of the mode-space pass;
// the ring corner of its surface Green's function is the circulant of the
// per-mode surface values (rs_lead_kernel).

// Kernels (one warp per energy; m x m complex tiles in shared memory,
// row-major; m x m products on the FP64 tensor cores, mma.sync m8n8k4, with
// the results staged in registers so that outputs may alias inputs):
//   rs_lead_kernel   both lead corners s_L = g[b][b], s_R = g[a][a] (ring
//                    Fourier modes, per-mode surface values);
//   rs_chain_kernel  forward sweep (X_k to global scratch), backward sweep
//                    with the ring sums of c G_jj written per energy;
//   rs_chain_neq_kernel  the same sweeps at a real-axis energy of a biased
//                    tube, carrying the source and drain columns of G in
//                    ring corners: ring sums of the contact spectral
//                    functions (the non-equilibrium term, FP64);
//   rs_reduce_kernel sum over energies per ring in a fixed order (Kahan).
// The energies of the U = 0 pass (Rho0) run in the same launches with
// negated coefficients, so one reduction gives the induced charge.
// Inversions: Gauss-Jordan on [S | I] (lane = column), on the diagonal
// pivots with a fall-back to partial pivoting when a pivot is small.
//
// Mixed precision: the chain of an energy runs in FP32 when its tube is in
// mixed mode and the point lies at least mixed_fp64_band above the real axis
// (the rule of the mode-space pass); the leads, the other energies, the ring
// sums per energy and their Kahan sum stay FP64.  In FP32 the m x m
// products run on the tensor cores: mma.sync m16n8k8 TF32 with each operand
// split into a TF32 high part and a TF32 remainder (three products per
// pair, about FP32 accuracy) and the complex product in the three-multiply
// form Re = ArBr - AiBi, Im = (Ar + Ai)(Br + Bi) - ArBr - AiBi; the
// inversion runs on the FP32 cores.  One launch holds both precisions (the
// FP64 energies first).

#include "negf_internal.h"

namespace negf {
namespace {

constexpr int kMaxM = 16;  // atoms per ring: [S | I] has one lane per column

#include "negf_sgf.cuh"  // cd, sgf_analytic, sgf_decimation (lead mode chains)

template <typename R>
struct __align__(2 * sizeof(R)) cplx {
    R x, y;
};
using cplxd = cplx<double>;
using cplxf = cplx<float>;
template <typename R>
__device__ __forceinline__ cplx<R> cmk(R a, R b) {
    return {a, b};
}
template <typename R>
__device__ __forceinline__ cplx<R> cadd(cplx<R> a, cplx<R> b) {
    return {a.x + b.x, a.y + b.y};
}
template <typename R>
__device__ __forceinline__ cplx<R> csub(cplx<R> a, cplx<R> b) {
    return {a.x - b.x, a.y - b.y};
}
template <typename R>
__device__ __forceinline__ cplx<R> cscale(cplx<R> a, R s) {
    return {a.x * s, a.y * s};
}
template <typename R>
__device__ __forceinline__ cplx<R> cmul(cplx<R> a, cplx<R> b) {
    return {fma(a.x, b.x, -a.y * b.y), fma(a.x, b.y, a.y * b.x)};
}
// acc + a b
template <typename R>
__device__ __forceinline__ cplx<R> cfma(cplx<R> a, cplx<R> b, cplx<R> acc) {
    return {fma(a.x, b.x, fma(-a.y, b.y, acc.x)), fma(a.x, b.y, fma(a.y, b.x, acc.y))};
}
// acc - a b
template <typename R>
__device__ __forceinline__ cplx<R> cfms(cplx<R> a, cplx<R> b, cplx<R> acc) {
    return {fma(-a.x, b.x, fma(a.y, b.y, acc.x)), fma(-a.x, b.y, fma(-a.y, b.x, acc.y))};
}
// Reciprocal: hardware approximation y0 = rcp.approx.ftz(x) with relative
// error e = 1 - x y0 (|e| <= 2^-20 or better), corrected by the truncated
// series 1/x = y0 (1 + e + e^2 + ...) to a relative error of order e^3 (FP64)
// or e^2 (FP32).  Arguments are squared moduli of pivots and of E - U.
__device__ __forceinline__ double rcp_r(double x) {
    double y;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
    const double e = fma(-x, y, 1.0);
    return fma(y, fma(e, e, e), y);
}
__device__ __forceinline__ float rcp_r(float x) {
    float y;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return fmaf(y, fmaf(-x, y, 1.0f), y);
}
// 1 / b = conj(b) / |b|^2
template <typename R>
__device__ __forceinline__ cplx<R> crcp(cplx<R> b) {
    const R q = rcp_r(fma(b.x, b.x, b.y * b.y));
    return {b.x * q, -b.y * q};
}

// Complex tile, row-major with compile-time leading dimension LD
template <int LD, typename R>
struct Mat {
    cplx<R>* a;
    __device__ __forceinline__ cplx<R>& at(int r, int c) const { return a[r * LD + c]; }
};

template <int M>
__device__ __forceinline__ int wrap(int i) { return i < 0 ? i + M : (i >= M ? i - M : i); }

// Lane layout of every tile operation: column c = lane & 15, rows h, h + 2,
// ..., h = lane >> 4 (lanes of a half-warp share the row operands).  The
// body sees r and c.
#define RS_FOR_ENTRIES(m, lane, ...)                           \
    {                                                          \
        const int c_ = (lane) & 15, h_ = (lane) >> 4;          \
        if (c_ < (m)) {                                        \
            _Pragma("unroll") for (int i_ = 0; i_ < 8; ++i_) { \
                const int r_ = h_ + 2 * i_;                    \
                if (r_ < (m)) {                                \
                    const int r = r_, c = c_;                  \
                    __VA_ARGS__                                \
                }                                              \
            }                                                  \
        }                                                      \
    }

// FP64 tensor-core product D += A B of an 8 x 8 x 4 tile (mma.sync m8n8k4,
// FP64).  Fragments, g = lane / 4, t = lane % 4: a = A[g][t]; b = B[t][g];
// d = D[g][2t], D[g][2t+1].
__device__ __forceinline__ void dmma(double (&d)[2], double a, double b) {
    asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
        : "+d"(d[0]), "+d"(d[1])
        : "d"(a), "d"(b));
}

// C = s op(A) op(B) (+ D when ADD) in FP64 on the tensor cores: the m x m
// tiles are read as zero-padded 16 x 16 operands (2 x 2 output tiles of
// 8 x 8, k in steps of 4), complex products in the three-multiply form
// Re = ArBr - AiBi, Im = (Ar + Ai)(Br + Bi) - ArBr - AiBi.  C may alias any
// operand: the products are staged in registers.
template <int m, bool TA, bool TB, bool ADD>
__device__ __forceinline__ void mm(Mat<m, double> C, Mat<m, double> A, Mat<m, double> B, Mat<m, double> D, double s,
                                   int lane) {
    const int g = lane >> 2, t = lane & 3;
    constexpr int NT = (m + 7) / 8;  // 8 x 8 output tiles per dimension
    double p1[NT][NT][2], p2[NT][NT][2], p3[NT][NT][2];  // Ar Br, Ai Bi, (Ar + Ai)(Br + Bi)
#pragma unroll
    for (int i = 0; i < NT; ++i)
#pragma unroll
        for (int j = 0; j < NT; ++j)
#pragma unroll
            for (int q = 0; q < 2; ++q) p1[i][j][q] = p2[i][j][q] = p3[i][j][q] = 0.0;
#pragma unroll
    for (int k0 = 0; k0 < m; k0 += 4) {
        const int k = k0 + t;
        cplxd a[NT], b[NT];
#pragma unroll
        for (int i = 0; i < NT; ++i) {
            const int r = 8 * i + g;
            a[i] = cmk(0.0, 0.0);
            if (r < m && k < m) a[i] = TA ? A.at(k, r) : A.at(r, k);
            b[i] = cmk(0.0, 0.0);
            if (k < m && r < m) b[i] = TB ? B.at(r, k) : B.at(k, r);  // column 8 i + g of B
        }
#pragma unroll
        for (int i = 0; i < NT; ++i) {
            const double as = a[i].x + a[i].y;
#pragma unroll
            for (int j = 0; j < NT; ++j) {
                dmma(p1[i][j], a[i].x, b[j].x);
                dmma(p2[i][j], a[i].y, b[j].y);
                dmma(p3[i][j], as, b[j].x + b[j].y);
            }
        }
    }
    __syncwarp();
#pragma unroll
    for (int i = 0; i < NT; ++i)
#pragma unroll
        for (int j = 0; j < NT; ++j)
#pragma unroll
            for (int q = 0; q < 2; ++q) {
                const int r = 8 * i + g, c = 8 * j + 2 * t + q;
                if (r < m && c < m) {
                    const double re = p1[i][j][q] - p2[i][j][q], im = p3[i][j][q] - p1[i][j][q] - p2[i][j][q];
                    cplxd v = cmk(re * s, im * s);
                    if (ADD) v = cadd(v, D.at(r, c));
                    C.at(r, c) = v;
                }
            }
    __syncwarp();
}

// TF32 tensor-core product D += A B of a 16 x 8 x 8 tile (mma.sync
// m16n8k8, FP32 accumulate).  Fragments, g = lane / 4, t = lane % 4:
// a = A[g][t], A[g+8][t], A[g][t+4], A[g+8][t+4]; b = B[t][g], B[t+4][g];
// d = D[g][2t], D[g][2t+1], D[g+8][2t], D[g+8][2t+1].
__device__ __forceinline__ void mma_tf32(float (&d)[4], const unsigned (&a)[4], const unsigned (&b)[2]) {
    asm("mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, "
        "{%0, %1, %2, %3};"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}
// x = hi + lo with hi the TF32 rounding of x and lo the TF32 rounding of the rest
__device__ __forceinline__ void split_tf32(float x, unsigned& hi, unsigned& lo) {
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(hi) : "f"(x));
    const float rest = x - __uint_as_float(hi);
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(lo) : "f"(rest));
}
// D += A B in three tensor-core products: lo hi + hi lo + hi hi
__device__ __forceinline__ void mma3(float (&d)[4], const unsigned (&ah)[4], const unsigned (&al)[4],
                                     const unsigned (&bh)[2], const unsigned (&bl)[2]) {
    mma_tf32(d, al, bh);
    mma_tf32(d, ah, bl);
    mma_tf32(d, ah, bh);
}

// C = s op(A) op(B) (+ D when ADD) in FP32 on the tensor cores: the m x m
// tiles are read as zero-padded 16 x 16 operands, the complex product in
// the three-multiply form.  C may alias any operand.
template <int m, bool TA, bool TB, bool ADD>
__device__ __forceinline__ void mm(Mat<m, float> C, Mat<m, float> A, Mat<m, float> B, Mat<m, float> D, float s,
                                   int lane) {
    const int g = lane >> 2, t = lane & 3;
    float t1[2][4], t2[2][4], t3[2][4];  // Ar Br, Ai Bi, (Ar + Ai)(Br + Bi) per 8-column tile
#pragma unroll
    for (int n = 0; n < 2; ++n)
#pragma unroll
        for (int q = 0; q < 4; ++q) t1[n][q] = t2[n][q] = t3[n][q] = 0.0f;
#pragma unroll
    for (int k0 = 0; k0 < m; k0 += 8) {
        unsigned arh[4], arl[4], aih[4], ail[4], ash[4], asl[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int r = g + ((q & 1) ? 8 : 0), k = k0 + t + ((q & 2) ? 4 : 0);
            cplxf v = cmk(0.0f, 0.0f);
            if (r < m && k < m) v = TA ? A.at(k, r) : A.at(r, k);
            split_tf32(v.x, arh[q], arl[q]);
            split_tf32(v.y, aih[q], ail[q]);
            split_tf32(v.x + v.y, ash[q], asl[q]);
        }
#pragma unroll
        for (int n = 0; n < 2; ++n) {
            if (8 * n < m) {
                unsigned brh[2], brl[2], bih[2], bil[2], bsh[2], bsl[2];
#pragma unroll
                for (int q = 0; q < 2; ++q) {
                    const int k = k0 + t + 4 * q, c = 8 * n + g;
                    cplxf v = cmk(0.0f, 0.0f);
                    if (k < m && c < m) v = TB ? B.at(c, k) : B.at(k, c);
                    split_tf32(v.x, brh[q], brl[q]);
                    split_tf32(v.y, bih[q], bil[q]);
                    split_tf32(v.x + v.y, bsh[q], bsl[q]);
                }
                mma3(t1[n], arh, arl, brh, brl);
                mma3(t2[n], aih, ail, bih, bil);
                mma3(t3[n], ash, asl, bsh, bsl);
            }
        }
    }
    __syncwarp();
#pragma unroll
    for (int n = 0; n < 2; ++n) {
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int r = g + ((q & 2) ? 8 : 0), c = 8 * n + 2 * t + (q & 1);
            if (r < m && c < m) {
                cplxf v = cmk((t1[n][q] - t2[n][q]) * s, (t3[n][q] - t1[n][q] - t2[n][q]) * s);
                if (ADD) v = cadd(v, D.at(r, c));
                C.at(r, c) = v;
            }
        }
    }
    __syncwarp();
}

// max(|Re|, |Im|)
template <typename R>
__device__ __forceinline__ R cmaxabs(cplx<R> a) {
    return fmax(fabs(a.x), fabs(a.y));
}

// out = S^-1 by Gauss-Jordan with partial pivoting (largest |.|^2 over the
// rows below, lowest row on ties).  Lane c < 2m holds column c of [S | I] in
// registers; the pivot column reaches every lane through buf (m complex in
// shared memory), every lane finds the pivot row by a tournament over it.
// out may alias S.  Returns false on a zero pivot.
template <int m, typename R>
__device__ __noinline__ bool invert_pivoted(Mat<m, R> out, Mat<m, R> S, cplx<R>* buf, int lane) {
    constexpr int n2 = 2 * m;
    __syncwarp();  // S complete
    cplx<R> col[m];
#pragma unroll
    for (int r = 0; r < m; ++r) col[r] = lane < m ? S.at(r, lane) : cmk<R>(lane - m == r ? R(1) : R(0), R(0));
    bool ok = true;
#pragma unroll
    for (int p = 0; p < m; ++p) {
        __syncwarp();  // every lane is done with buf (and with S on the first pivot)
        if (lane == p) {
#pragma unroll
            for (int r = 0; r < m; ++r) buf[r] = col[r];
        }
        __syncwarp();
        R bv[m];
        int bi[m];
#pragma unroll
        for (int r = 0; r < m; ++r) {
            bi[r] = r;
            bv[r] = R(-1);
            if (r >= p) {
                const cplx<R> x = buf[r];
                bv[r] = fma(x.x, x.x, x.y * x.y);
            }
        }
#pragma unroll
        for (int st = 1; st < m; st *= 2) {
#pragma unroll
            for (int r = 0; r + st < m; r += 2 * st) {
                if (bv[r + st] > bv[r]) {
                    bv[r] = bv[r + st];
                    bi[r] = bi[r + st];
                }
            }
        }
        const int idx = bi[0];
        if (!(bv[0] > R(0))) ok = false;
        if (idx != p) {
#pragma unroll
            for (int r = p + 1; r < m; ++r) {
                if (r == idx) {
                    const cplx<R> t = col[r];
                    col[r] = col[p];
                    col[p] = t;
                }
            }
        }
        // multiplier of row r after the swap: buf[r], but buf[p] for row idx
        const cplx<R> rp = cmul(col[p], crcp(buf[idx]));
#pragma unroll
        for (int r = 0; r < m; ++r) {
            if (r == 8) asm volatile("" ::: "memory");  // two batches of multiplier loads
            if (r != p) col[r] = cfms(buf[r == idx ? p : r], rp, col[r]);
        }
        col[p] = rp;
    }
    __syncwarp();
    if (lane >= m && lane < n2) {
#pragma unroll
        for (int r = 0; r < m; ++r) out.at(r, lane - m) = col[r];
    }
    __syncwarp();
    return ok;
}

// out = S^-1 by Gauss-Jordan on the diagonal pivots, falling back to partial
// pivoting (invert_pivoted, from S, which stays untouched until the result
// is written) when any pivot is small: max(|Re|, |Im|) of a pivot below tau
// (1e-3 in FP64, 1e-2 in FP32) times the largest such value of the entries
// of S.  For E - H - Sigma with Im E > 0, S is complex symmetric with a
// positive definite imaginary part, so its leading minors never vanish and
// the diagonal pivots are the usual case; the search and the row swaps of
// partial pivoting (about half the cost of the inversion) leave the common
// path.  Lane c < 2m holds column c of [S | I] in registers, the pivot
// column reaches every lane through buf.  out may alias S.  Returns false on
// a zero pivot.
template <int m, typename R>
__device__ __forceinline__ bool invert(Mat<m, R> out, Mat<m, R> S, cplx<R>* buf, int lane) {
    constexpr int n2 = 2 * m;
    const R tau = sizeof(R) == 8 ? R(1e-3) : R(1e-2);
    __syncwarp();  // S complete
    cplx<R> col[m];
    R smax = R(0), pmin;
#pragma unroll
    for (int r = 0; r < m; ++r) {
        col[r] = lane < m ? S.at(r, lane) : cmk<R>(lane - m == r ? R(1) : R(0), R(0));
        if (lane < m) smax = fmax(smax, cmaxabs(col[r]));
    }
#pragma unroll
    for (int p = 0; p < m; ++p) {
        __syncwarp();  // every lane is done with buf
        if (lane == p) {
#pragma unroll
            for (int r = 0; r < m; ++r) buf[r] = col[r];
        }
        __syncwarp();
        const cplx<R> piv = buf[p];
        pmin = p == 0 ? cmaxabs(piv) : fmin(pmin, cmaxabs(piv));
        const cplx<R> rp = cmul(col[p], crcp(piv));
#pragma unroll
        for (int r = 0; r < m; ++r) {
            if (r == 8) asm volatile("" ::: "memory");  // two batches of multiplier loads
            if (r != p) col[r] = cfms(buf[r], rp, col[r]);
        }
        col[p] = rp;
    }
#pragma unroll
    for (int o = 16; o >= 1; o >>= 1) smax = fmax(smax, __shfl_xor_sync(0xffffffffu, smax, o));
    if (!(pmin >= tau * smax)) return invert_pivoted<m, R>(out, S, buf, lane);
    __syncwarp();
    if (lane >= m && lane < n2) {
#pragma unroll
        for (int r = 0; r < m; ++r) out.at(r, lane - m) = col[r];
    }
    __syncwarp();
    return true;
}

__device__ __forceinline__ cplxd warp_sum(cplxd v) {
#pragma unroll
    for (int o = 16; o >= 1; o >>= 1) {
        v.x += __shfl_xor_sync(0xffffffffu, v.x, o);
        v.y += __shfl_xor_sync(0xffffffffu, v.y, o);
    }
    return v;
}

// Asynchronous global -> shared copy of one complex value (cp.async, 8 or 16
// bytes, both addresses aligned to the size) and the wait for all of them.
template <typename T>
__device__ __forceinline__ void cp_async(T* smem_dst, const T* gsrc) {
    static_assert(sizeof(T) == 8 || sizeof(T) == 16, "cp.async copies 8 or 16 bytes here");
    const unsigned d = (unsigned)__cvta_generic_to_shared(smem_dst);
    if constexpr (sizeof(T) == 16)
        asm volatile("cp.async.ca.shared.global [%0], [%1], 16;" ::"r"(d), "l"(gsrc) : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(d), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// Energy flags: kRsFP32 runs the chain in FP32, kRsZeroU takes U = 0 on the
// atoms and the contacts (the Rho0 pass).
constexpr int kRsFP32 = 1, kRsZeroU = 2;

// Lead kernel: block e -> energy e, lanes 0-15 the left lead, 16-31 the
// right one.  A lead is uniform (the contact potential u on every atom), so
// the Fourier vectors of a ring, v_k[j] = exp(2 pi i k j / m) / sqrt(m),
// decouple it: C v_k = (1 + exp(2 pi i k / m)) v_k, and with a gauge phase
// per ring mode k is the chain of alternating hoppings
// beta_k = 2 gamma cos(pi k / m) (the double bond) and gamma (the single
// bond), the surface ring's first bond being beta_k on both sides (left:
// surface ring b bonded to ring a of its cell; right: surface ring a bonded
// to ring b).  These are the mode chains of the mode-space pass
// (CNT.cpp:288-336), so the ring corner of the lead's surface Green's
// function is the circulant
//   s[j][l] = (1/m) sum_k cos(2 pi k (j - l) / m) s_k,
// s_k the mode chain's surface value by the mode-space formula
// (sgf_analytic, CNT.cpp:354-393, or the reference's decimation when the
// tube uses it).  Exact in O(m^2) per energy and lead, with no matrix
// iteration (an iterated decimation on the 2m-atom cell loses accuracy on
// the real axis, where its Schur complements divide by E - u).
// corners[e][side] = g_surface[s][s] (m x m, row-major).
template <int m>
__global__ void __launch_bounds__(32) rs_lead_kernel(double gamma, const double* __restrict__ Ere,
                                                     const double* __restrict__ Eim, int num_e,
                                                     const int* __restrict__ flags, double Uc0, double Uc1,
                                                     int use_decimation, int dec_layers, int dec_iters,
                                                     cplxd* __restrict__ corners) {
    __shared__ cd sk[2][kMaxM], cdiff[2][kMaxM];
    const int lane = threadIdx.x;
    const int e = blockIdx.x;
    if (e >= num_e) return;
    const int side = lane >> 4, k = lane & 15;
    const double u = (flags[e] & kRsZeroU) ? 0.0 : (side == 0 ? Uc0 : Uc1);
    const cd EmU = {Ere[e] - u, Eim[e]};
    if (k < m) {
        const double beta = 2.0 * gamma * cospi((double)k / m);
        sk[side][k] = use_decimation ? sgf_decimation(EmU, beta, gamma, dec_layers, dec_iters)
                                     : sgf_analytic(EmU, beta, gamma);
    }
    __syncwarp();
    if (k < m) {  // circulant value of ring-index difference d = k
        cd acc = {0.0, 0.0};
        for (int q = 0; q < m; ++q) acc = cadd(acc, cscale(cospi(2.0 * (double)((q * k) % m) / m), sk[side][q]));
        cdiff[side][k] = cscale(1.0 / m, acc);
    }
    __syncwarp();
    cplxd* out = corners + ((size_t)e * 2 + side) * m * m;
    for (int i = k; i < m * m; i += 16) {
        const int j = i / m, l = i % m;
        const cd v = cdiff[side][j >= l ? j - l : j - l + m];
        out[i] = cmk(v.x, v.y);
    }
}

// Gamma = i (Sigma - Sigma^dagger) = -2 gamma^2 Im s of a contact (s: the
// lead's surface corner, complex symmetric), factored as L L^T by Cholesky
// with diagonal pivoting (Gamma is real symmetric positive semidefinite);
// columns past the numerical rank (pivots below 1e-13 of the largest
// diagonal entry) stay zero.  One lane, once per energy and contact; L times
// `scale` into a complex tile (imaginary parts zero).
template <int m>
__device__ __noinline__ void gamma_factor(const cplxd* __restrict__ s, double g2, double scale, Mat<m, double> L,
                                          int lane) {
    if (lane == 0) {
        double a[m][m];
        int perm[m];
        double dmax = 0.0;
        for (int i = 0; i < m; ++i) {
            perm[i] = i;
            for (int j = 0; j < m; ++j) a[i][j] = -g2 * (s[i * m + j].y + s[j * m + i].y);
            dmax = fmax(dmax, a[i][i]);
        }
        int rank = 0;
        for (int p = 0; p < m; ++p) {
            int q = p;
            for (int i = p + 1; i < m; ++i)
                if (a[i][i] > a[q][q]) q = i;
            if (!(a[q][q] > 1e-13 * dmax)) break;
            if (q != p) {
                for (int j = 0; j < m; ++j) {
                    const double t = a[p][j];
                    a[p][j] = a[q][j];
                    a[q][j] = t;
                }
                for (int i = 0; i < m; ++i) {
                    const double t = a[i][p];
                    a[i][p] = a[i][q];
                    a[i][q] = t;
                }
                const int t = perm[p];
                perm[p] = perm[q];
                perm[q] = t;
            }
            const double l = sqrt(a[p][p]), il = 1.0 / l;
            a[p][p] = l;
            for (int i = p + 1; i < m; ++i) a[i][p] *= il;
            for (int j = p + 1; j < m; ++j)
                for (int i = j; i < m; ++i) {
                    a[i][j] -= a[i][p] * a[j][p];
                    a[j][i] = a[i][j];
                }
            rank = p + 1;
        }
        for (int i = 0; i < m * m; ++i) L.a[i] = cmk(0.0, 0.0);
        for (int p = 0; p < rank; ++p)
            for (int i = p; i < m; ++i) L.at(perm[i], p) = cmk(a[i][p] * scale, 0.0);
    }
    __syncwarp();
}

// One energy's chain in precision R (warp e): atom potentials Ua, lead
// corners (FP64, m x m, row-major), scratch myX for X_k (K m^2 complex R),
// row of 2K ring sums Im(c sum_j G_jj) written in FP64.  The potentials of
// the next block are loaded while the current block is computed.
//
// NEQ (a real-axis energy, FP64): the row holds instead the ring sums of the
// contact spectral functions, b0 A^L + b1 A^R with (b0, b1) = cc and
// A^c_ring = sum_{n in ring} [G_{n,c} Gamma_c G_{n,c}^dagger]_nn
// = || G_{ring,c} L_c ||_F^2 (Gamma_c = L_c L_c^T).  The contact columns of
// G are carried through the sweeps in ring corners:
//   source (ring a of block 0): Q_k = g_L[k]_{b_k, a_0} L_L with
//     Q_{-1} = L_L / gamma, Q_k = gamma^2 Y^T (X_k Q_{k-1}) (forward, kept in
//     myQ); G_{k,0}[a] L_L = gamma G_kk[a][a] Q_{k-1} and
//     G_{k,0}[b] L_L = (I + gamma^2 g_L[b][b] G') Q_k (backward);
//   drain (ring b of block K-1): T_k = G_{k,c}[a] L_R with
//     T_K = (I + gamma^2 G'_K g_L[b][b]) L_R / gamma (G'_K of the right lead),
//     T_k = gamma^2 X_k (Y T_{k+1}) and G_{k,c}[b] L_R = gamma g_L[b][b] T_{k+1}.
// Four more m x m products per block in the backward sweep and one in the
// forward sweep; no G_jj sums (the real-axis energies carry no contour term).
template <int m, typename R, bool NEQ = false>
__device__ __forceinline__ bool rs_chain(int K, R gamma, cplx<R> E, cplxd cc, const double* __restrict__ Ua,
                                         const cplxd* __restrict__ sL, const cplxd* __restrict__ sR,
                                         cplx<R>* __restrict__ myX, cplx<R>* __restrict__ myQ,
                                         double* __restrict__ row, cplx<R>* sh, int lane) {
    static_assert(!NEQ || sizeof(R) == 8, "the non-equilibrium chains run in FP64");
    using C = cplx<R>;
    constexpr int mm2 = m * m;
    constexpr int tiles = NEQ ? 9 : 5;
    const R g2 = gamma * gamma, g4 = g2 * g2;
    const R zero(0), one(1);
    const Mat<m, R> X{sh}, Gbb{sh + mm2}, Gn{sh + 2 * mm2}, Z{sh + 3 * mm2}, W{sh + 4 * mm2};
    // NEQ: source columns (current / previous block), drain column, product tile
    const Mat<m, R> Qa{sh + 5 * mm2}, Qb{sh + 6 * mm2}, T{sh + 7 * mm2}, P{sh + 8 * mm2};
    C* dv = sh + tiles * mm2;  // D^-1 of the current ring b
    C* da = dv + kMaxM;        // E - U of the current ring a
    C* buf = da + kMaxM;       // pivot column
    bool ok = true;
    if constexpr (NEQ) {
        gamma_factor<m>(sL, g2, one / gamma, Qa, lane);  // Q_{-1}
        gamma_factor<m>(sR, g2, one, T, lane);           // L_R
        for (int i = lane; i < mm2; i += 32) myQ[i] = Qa.a[i];
    }
    // lane j < m: potentials of atom j on rings a and b of the next block
    R ua_n = zero, ub_n = zero;
    auto fetch_u = [&](int k) {
        if (lane < m) {
            ua_n = (R)__ldg(Ua + (size_t)(2 * k) * m + lane);
            ub_n = (R)__ldg(Ua + (size_t)(2 * k + 1) * m + lane);
        }
    };
    // g_L[b][b] = D^-1 + gamma^2 Y^T X Y into Gbb
    auto form_gbb = [&](Mat<m, R> Xt) {
        RS_FOR_ENTRIES(m, lane, {
            const int r0 = wrap<m>(r - 1), c0 = wrap<m>(c - 1);
            const C q = cadd(cadd(Xt.at(r, c), Xt.at(r, c0)), cadd(Xt.at(r0, c), Xt.at(r0, c0)));
            C v = cscale(cmul(cmul(dv[r], dv[c]), q), g2);
            if (r == c) v = cadd(v, dv[r]);
            Gbb.at(r, c) = v;
        })
        __syncwarp();
    };
    // left lead corner as g_L[b][b] of block -1
    for (int i = lane; i < mm2; i += 32) Gbb.a[i] = cmk((R)sL[i].x, (R)sL[i].y);
    fetch_u(0);
    for (int k = 0; k < K; ++k) {
        if (lane < m) {
            dv[lane] = crcp(cmk(E.x - ub_n, E.y));
            da[lane] = cmk(E.x - ua_n, E.y);
        }
        if (k + 1 < K) fetch_u(k + 1);
        __syncwarp();
        // S = diag(E - U_a) - gamma^2 g_L[b][b]_{k-1} - gamma^2 C D^-1 C^T
        RS_FOR_ENTRIES(m, lane, {
            const int r1 = wrap<m>(r + 1), c1 = wrap<m>(c + 1);
            C cd = cmk(zero, zero);
            if (r == c) cd = cadd(cd, dv[r]);
            if (r == c1) cd = cadd(cd, dv[r]);
            if (r1 == c) cd = cadd(cd, dv[r1]);
            if (r1 == c1) cd = cadd(cd, dv[r1]);
            C v = cscale(cadd(Gbb.at(r, c), cd), -g2);
            if (r == c) v = cadd(v, da[r]);
            X.at(r, c) = v;
        })
        ok = invert<m>(X, X, buf, lane) && ok;
        C* dst = myX + (size_t)k * mm2;
        for (int i = lane; i < mm2; i += 32) dst[i] = X.a[i];
        if constexpr (NEQ) {
            // Q_k = gamma^2 Y^T (X_k Q_{k-1}), (Y^T M)[r][c] = D^-1_r (M[r][c] + M[r-1][c])
            mm<m, false, false, false>(P, X, Qa, P, one, lane);
            RS_FOR_ENTRIES(m, lane, {
                const int r0 = wrap<m>(r - 1);
                Qa.at(r, c) = cscale(cmul(dv[r], cadd(P.at(r, c), P.at(r0, c))), g2);
            })
            __syncwarp();
            C* qd = myQ + (size_t)(k + 1) * mm2;
            for (int i = lane; i < mm2; i += 32) qd[i] = Qa.a[i];
        }
        form_gbb(X);
    }
    // G_K[a][a] of the right lead's first ring: (I - gamma^2 s_R g_L[b][b])^-1 s_R
    for (int i = lane; i < mm2; i += 32) X.a[i] = cmk((R)sR[i].x, (R)sR[i].y);
    __syncwarp();
    mm<m, false, false, false>(Gn, X, Gbb, Gn, -g2, lane);
    if (lane < m) Gn.at(lane, lane) = cadd(Gn.at(lane, lane), cmk(one, zero));
    ok = invert<m>(Gn, Gn, buf, lane) && ok;
    mm<m, false, false, false>(Gn, Gn, X, Gn, one, lane);
    if constexpr (NEQ) {
        // T_K = (L_R + gamma^2 G'_K (g_L[b][b] L_R)) / gamma
        mm<m, false, false, false>(P, Gbb, T, P, one, lane);
        mm<m, false, false, true>(T, Gn, P, T, g2, lane);
        RS_FOR_ENTRIES(m, lane, { T.at(r, c) = cscale(T.at(r, c), one / gamma); })
        __syncwarp();
    }
    fetch_u(K - 1);
    // Backward.  X_{k-1} is copied into the tile that held the product W of
    // step k (free once tr G[b][b] is formed) while the last two products of
    // step k run; the two tiles swap roles every step.
    Mat<m, R> Xc = X, Wc = W;
    // NEQ: Qc = Q_k, Qp = Q_{k-1}; Q_{k-2} is copied into Qc once Q_k is used
    Mat<m, R> Qc = Qa, Qp = Qb;
    {
        const C* src = myX + (size_t)(K - 1) * mm2;
        for (int i = lane; i < mm2; i += 32) Xc.a[i] = src[i];
        if constexpr (NEQ) {
            for (int i = lane; i < mm2; i += 32) {
                Qc.a[i] = myQ[(size_t)K * mm2 + i];
                Qp.a[i] = myQ[(size_t)(K - 1) * mm2 + i];
            }
        }
    }
    for (int k = K - 1; k >= 0; --k) {
        cp_async_wait_all();  // X_k (and Q_{k-1}), issued during step k + 1, have landed
        if (lane < m) dv[lane] = crcp(cmk(E.x - ub_n, E.y));
        if (k > 0) fetch_u(k - 1);
        __syncwarp();
        form_gbb(Xc);
        double tRa = 0.0, tRb = 0.0, tLa = 0.0, tLb = 0.0;
        if constexpr (NEQ) {
            // drain column, ring b: gamma g_L[b][b] T_{k+1}; then Y T_{k+1} into P
            mm<m, false, false, false>(P, Gbb, T, P, gamma, lane);
            RS_FOR_ENTRIES(m, lane, {
                const C v = P.at(r, c);
                tRb = fma(v.x, v.x, fma(v.y, v.y, tRb));
                const int r1 = wrap<m>(r + 1);
                P.at(r, c) = cadd(cmul(dv[r], T.at(r, c)), cmul(dv[r1], T.at(r1, c)));
            })
            __syncwarp();
            // ring a: T_k = gamma^2 X_k (Y T_{k+1})
            mm<m, false, false, false>(T, Xc, P, T, g2, lane);
            RS_FOR_ENTRIES(m, lane, {
                const C v = T.at(r, c);
                tRa = fma(v.x, v.x, fma(v.y, v.y, tRa));
            })
        }
        // Z = Y G' Y^T = C (D^-1 G' D^-1) C^T, Y = C D^-1: H = D^-1 G' D^-1 in the
        // free tile Wc, then four neighbours of H per entry
        RS_FOR_ENTRIES(m, lane, { Wc.at(r, c) = cmul(cmul(dv[r], Gn.at(r, c)), dv[c]); })
        __syncwarp();
        RS_FOR_ENTRIES(m, lane, {
            const int r1 = wrap<m>(r + 1), c1 = wrap<m>(c + 1);
            Z.at(r, c) = cadd(cadd(Wc.at(r, c), Wc.at(r, c1)), cadd(Wc.at(r1, c), Wc.at(r1, c1)));
        })
        __syncwarp();
        // W = g_L[b][b] G'; tr G[b][b] = tr g_L[b][b] + gamma^2 sum_rc W[r][c] g_L[b][b][c][r]
        mm<m, false, false, false>(Wc, Gbb, Gn, Wc, one, lane);
        cplxd tb = cmk(0.0, 0.0);
        if constexpr (NEQ) {
            // source column, ring b: (I + gamma^2 W) Q_k
            mm<m, false, false, true>(P, Wc, Qc, Qc, g2, lane);
            RS_FOR_ENTRIES(m, lane, {
                const C v = P.at(r, c);
                tLb = fma(v.x, v.x, fma(v.y, v.y, tLb));
            })
        } else {
            RS_FOR_ENTRIES(m, lane, {
                const C w = cmul(cscale(Wc.at(r, c), g2), Gbb.at(c, r));
                tb = cadd(tb, cmk((double)w.x, (double)w.y));
                if (r == c) tb = cadd(tb, cmk((double)Gbb.at(r, r).x, (double)Gbb.at(r, r).y));
            })
        }
        __syncwarp();  // every lane is done with Wc (and Qc)
        if (k > 0) {
            const C* src = myX + (size_t)(k - 1) * mm2;
            for (int i = lane; i < mm2; i += 32) cp_async(Wc.a + i, src + i);
            if constexpr (NEQ) {
                const C* qs = myQ + (size_t)(k - 1) * mm2;  // Q_{k-2}
                for (int i = lane; i < mm2; i += 32) cp_async(Qc.a + i, qs + i);
            }
            cp_async_commit();
        }
        // G[a][a] = X + gamma^4 (X Z) X
        mm<m, false, false, false>(Z, Xc, Z, Z, one, lane);
        mm<m, false, false, true>(Gn, Z, Xc, Xc, g4, lane);
        {
            const Mat<m, R> tt = Xc;
            Xc = Wc;
            Wc = tt;
        }
        if constexpr (NEQ) {
            // source column, ring a: gamma G_kk[a][a] Q_{k-1}
            mm<m, false, false, false>(P, Gn, Qp, P, gamma, lane);
            RS_FOR_ENTRIES(m, lane, {
                const C v = P.at(r, c);
                tLa = fma(v.x, v.x, fma(v.y, v.y, tLa));
            })
            const Mat<m, R> tt = Qc;
            Qc = Qp;
            Qp = tt;
            const cplxd sa = warp_sum(cmk(tLa, tRa)), sb = warp_sum(cmk(tLb, tRb));
            if (lane == 0) {
                row[2 * k] = fma(cc.x, sa.x, cc.y * sa.y);
                row[2 * k + 1] = fma(cc.x, sb.x, cc.y * sb.y);
            }
        } else {
            cplxd ta = cmk(0.0, 0.0);
            if (lane < m) ta = cmk((double)Gn.at(lane, lane).x, (double)Gn.at(lane, lane).y);
            ta = warp_sum(ta);
            tb = warp_sum(tb);
            if (lane == 0) {
                row[2 * k] = fma(cc.x, ta.y, cc.y * ta.x);      // Im(c tr G[a][a])
                row[2 * k + 1] = fma(cc.x, tb.y, cc.y * tb.x);  // Im(c tr G[b][b])
            }
        }
    }
    return ok;
}

// Chain kernel: warp e -> energy e in the precision and with the potentials
// its flags give (Uatoms, or Uzero for the U = 0 pass).
// gX: [num_e][K][m*m] FP64-complex slots (an FP32 chain uses the first half
// of its slot); rows: [num_e][N].
template <int m>
__global__ void __launch_bounds__(32, 16) rs_chain_kernel(int K, double gamma, const double* __restrict__ Ere,
                                                          const double* __restrict__ Eim,
                                                          const double* __restrict__ cre,
                                                          const double* __restrict__ cim, int num_e,
                                                          const int* __restrict__ flags,
                                                          const double* __restrict__ Uatoms,
                                                          const double* __restrict__ Uzero,
                                                          const cplxd* __restrict__ corners, cplxd* __restrict__ gX,
                                                          double* __restrict__ rows, int* __restrict__ status) {
    extern __shared__ cplxd sh[];
    const int lane = threadIdx.x;
    const int e = blockIdx.x;
    if (e >= num_e) return;
    constexpr int mm2 = m * m;
    const int fl = flags[e];
    const double* __restrict__ Ua = (fl & kRsZeroU) ? Uzero : Uatoms;
    const cplxd* sL = corners + (size_t)e * 2 * mm2;
    const cplxd* sR = sL + mm2;
    cplxd* myX = gX + (size_t)e * K * mm2;
    double* row = rows + (size_t)e * 2 * K;
    const cplxd cc = cmk(cre[e], cim[e]);
    bool ok;
    if (!(fl & kRsFP32))
        ok = rs_chain<m, double>(K, gamma, cmk(Ere[e], Eim[e]), cc, Ua, sL, sR, myX, nullptr, row, sh, lane);
    else
        ok = rs_chain<m, float>(K, (float)gamma, cmk((float)Ere[e], (float)Eim[e]), cc, Ua, sL, sR,
                                reinterpret_cast<cplxf*>(myX), nullptr, row, reinterpret_cast<cplxf*>(sh), lane);
    if (!ok && lane == 0) atomicExch(status, 1);
}

// Non-equilibrium chain kernel: warp i -> real-axis energy e = e_off + i in
// FP64 with the atom potentials and coefficients (b0, b1) = (cre, cim)[e].
// gXn: [num][2K + 1][m*m] FP64-complex (X_k, then Q_{-1} ... Q_{K-1});
// rows: [e][2K] as for the other energies.
template <int m>
__global__ void __launch_bounds__(32, 8) rs_chain_neq_kernel(int K, double gamma, const double* __restrict__ Ere,
                                                             const double* __restrict__ Eim,
                                                             const double* __restrict__ cre,
                                                             const double* __restrict__ cim, int e_off, int num,
                                                             const double* __restrict__ Uatoms,
                                                             const cplxd* __restrict__ corners,
                                                             cplxd* __restrict__ gXn, double* __restrict__ rows,
                                                             int* __restrict__ status) {
    extern __shared__ cplxd sh[];
    const int lane = threadIdx.x;
    const int i = blockIdx.x;
    if (i >= num) return;
    constexpr int mm2 = m * m;
    const int e = e_off + i;
    const cplxd* sL = corners + (size_t)e * 2 * mm2;
    const cplxd* sR = sL + mm2;
    cplxd* myX = gXn + (size_t)i * (2 * K + 1) * mm2;
    cplxd* myQ = myX + (size_t)K * mm2;
    double* row = rows + (size_t)e * 2 * K;
    const bool ok = rs_chain<m, double, true>(K, gamma, cmk(Ere[e], Eim[e]), cmk(cre[e], cim[e]), Uatoms, sL, sR,
                                              myX, myQ, row, sh, lane);
    if (!ok && lane == 0) atomicExch(status, 1);
}

// Self-test of the tile primitives: warp w takes matrix w (inversion) or the
// pair (A, B) w (product) from in (complex, re/im interleaved, row-major
// m x m, FP64), computes in precision R and writes the m x m result to out.
template <int m, typename R>
__global__ void __launch_bounds__(32) rs_selftest_kernel(int product, int count, const double* __restrict__ in,
                                                         double* __restrict__ out) {
    __shared__ cplx<R> sh[3 * m * m + kMaxM];
    const int lane = threadIdx.x, w = blockIdx.x;
    if (w >= count) return;
    constexpr int mm2 = m * m;
    const Mat<m, R> A{sh}, B{sh + mm2}, C{sh + 2 * mm2};
    cplx<R>* buf = sh + 3 * mm2;
    const double* src = in + (size_t)w * (product ? 2 : 1) * 2 * mm2;
    for (int i = lane; i < mm2; i += 32) {
        A.a[i] = cmk((R)src[2 * i], (R)src[2 * i + 1]);
        if (product) B.a[i] = cmk((R)src[2 * mm2 + 2 * i], (R)src[2 * mm2 + 2 * i + 1]);
    }
    __syncwarp();
    bool ok = true;
    if (product)
        mm<m, false, false, false>(C, A, B, C, R(1), lane);
    else
        ok = invert<m>(C, A, buf, lane);
    double* dst = out + (size_t)w * 2 * mm2;
    for (int i = lane; i < mm2; i += 32) {
        dst[2 * i] = ok ? (double)C.a[i].x : NAN;
        dst[2 * i + 1] = ok ? (double)C.a[i].y : NAN;
    }
}

// Q[r] = sum over energies of rows[e][r] (minus sub[r]): block = 32 rings x kRsGroups
// energy groups; each thread sums energies g, g + kRsGroups, ... (Kahan),
// then the groups are combined in a fixed order (deterministic).
constexpr int kRsGroups = 8;
__global__ void __launch_bounds__(32 * kRsGroups) rs_reduce_kernel(const double* __restrict__ rows, int num_e, int N,
                                                                   const double* __restrict__ sub,
                                                                   double* __restrict__ Q) {
    __shared__ double sh_s[kRsGroups][32], sh_c[kRsGroups][32];
    const int r = blockIdx.x * 32 + threadIdx.x, g = threadIdx.y;
    double s = 0.0, comp = 0.0;
    if (r < N) {
        for (int e = g; e < num_e; e += kRsGroups) {
            const double y = rows[(size_t)e * N + r] - comp;
            const double t = s + y;
            comp = (t - s) - y;
            s = t;
        }
    }
    sh_s[g][threadIdx.x] = s;
    sh_c[g][threadIdx.x] = comp;
    __syncthreads();
    if (g == 0 && r < N) {
        double tot = 0.0, c = 0.0;
        for (int i = 0; i < kRsGroups; ++i) {
            const double y = (sh_s[i][threadIdx.x] - sh_c[i][threadIdx.x]) - c;
            const double t = tot + y;
            c = (t - tot) - y;
            tot = t;
        }
        Q[r] = sub ? tot - sub[r] : tot;
    }
}

// Uatoms[r][j] = U[r] (ring-uniform potential on the atoms).
__global__ void rs_expand_kernel(const double* __restrict__ U, int N, int m, double* __restrict__ Ua) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < N * m) Ua[i] = U[i / m];
}

size_t rs_chain_smem_bytes(int m) { return sizeof(cplxd) * (5 * m * m + 3 * kMaxM); }
size_t rs_chain_neq_smem_bytes(int m) { return sizeof(cplxd) * (9 * m * m + 3 * kMaxM); }

}  // namespace

cudaError_t rs_expand(const double* d_U, int N, int m, double* d_Ua, cudaStream_t stream) {
    if (N * m <= 0) return cudaSuccess;
    rs_expand_kernel<<<(N * m + 255) / 256, 256, 0, stream>>>(d_U, N, m, d_Ua);
    return cudaGetLastError();
}

int rs_max_atoms_per_block() { return 2 * kMaxM; }

cudaError_t rs_selftest(int which, int m, int count, const double* d_in, double* d_out, cudaStream_t stream) {
    if (count <= 0) return cudaSuccess;
    const int product = which >= 4;
    const bool fp32 = which == 3 || which == 5;
#define RS_ST(M)                                                                                                   \
    case M:                                                                                                        \
        if (fp32)                                                                                                  \
            rs_selftest_kernel<M, float><<<count, 32, 0, stream>>>(product, count, d_in, d_out);                   \
        else                                                                                                       \
            rs_selftest_kernel<M, double><<<count, 32, 0, stream>>>(product, count, d_in, d_out);                  \
        break;
    switch (m) {
        RS_ST(4) RS_ST(13) RS_ST(16)
        default:
            return cudaErrorInvalidValue;
    }
#undef RS_ST
    return cudaGetLastError();
}

namespace {
template <int m>
cudaError_t launch_rs(int K, double gamma, const double* d_Ere, const double* d_Eim, const double* d_cre,
                      const double* d_cim, int num_e, int num_neq, const int* d_flags, const double* d_Uatoms,
                      const double* d_Uzero, double Uc0, double Uc1, const RsLeads& leads, void* d_corners,
                      void* d_gL,
                      void* d_gLn, double* d_rows, double* d_Q, const double* d_sub, int* d_status,
                      cudaStream_t stream) {
    cudaError_t e = cudaFuncSetAttribute(rs_chain_kernel<m>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)rs_chain_smem_bytes(m));
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(rs_chain_neq_kernel<m>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)rs_chain_neq_smem_bytes(m));
    if (e != cudaSuccess) return e;
    const int num_eq = num_e - num_neq;
    if (num_e > 0) {
        rs_lead_kernel<m><<<num_e, 32, 0, stream>>>(gamma, d_Ere, d_Eim, num_e, d_flags, Uc0, Uc1,
                                                    leads.use_decimation, leads.dec_layers, leads.dec_iters,
                                                    static_cast<cplxd*>(d_corners));
        e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    if (num_neq > 0) {
        // the longer chains first
        rs_chain_neq_kernel<m><<<num_neq, 32, rs_chain_neq_smem_bytes(m), stream>>>(
            K, gamma, d_Ere, d_Eim, d_cre, d_cim, num_eq, num_neq, d_Uatoms, static_cast<const cplxd*>(d_corners),
            static_cast<cplxd*>(d_gLn), d_rows, d_status);
        e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    if (num_eq > 0) {
        rs_chain_kernel<m><<<num_eq, 32, rs_chain_smem_bytes(m), stream>>>(
            K, gamma, d_Ere, d_Eim, d_cre, d_cim, num_eq, d_flags, d_Uatoms, d_Uzero,
            static_cast<const cplxd*>(d_corners), static_cast<cplxd*>(d_gL), d_rows, d_status);
        e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    const int N = 2 * K;
    rs_reduce_kernel<<<(N + 31) / 32, dim3(32, kRsGroups), 0, stream>>>(d_rows, num_e, N, d_sub, d_Q);
    return cudaGetLastError();
}
}  // namespace

cudaError_t launch_realspace(int m, int K, double gamma, const double* d_Ere, const double* d_Eim,
                             const double* d_cre, const double* d_cim, int num_e, int num_neq, const int* d_flags,
                             const double* d_Uatoms, const double* d_Uzero, double Uc0, double Uc1,
                             const RsLeads& leads,
                             void* d_corners, void* d_gL, void* d_gLn, double* d_rows, double* d_Q,
                             const double* d_sub, int* d_status, cudaStream_t stream) {
    if (num_e < 0 || num_neq < 0 || num_neq > num_e || K < 1) return cudaErrorInvalidValue;
#define RS_CASE(M)                                                                                                 \
    case M:                                                                                                        \
        return launch_rs<M>(K, gamma, d_Ere, d_Eim, d_cre, d_cim, num_e, num_neq, d_flags, d_Uatoms, d_Uzero, Uc0,  \
                            Uc1, leads, d_corners, d_gL, d_gLn, d_rows, d_Q, d_sub, d_status, stream);
    switch (m) {
        RS_CASE(1) RS_CASE(2) RS_CASE(3) RS_CASE(4) RS_CASE(5) RS_CASE(6) RS_CASE(7) RS_CASE(8)
        RS_CASE(9) RS_CASE(10) RS_CASE(11) RS_CASE(12) RS_CASE(13) RS_CASE(14) RS_CASE(15) RS_CASE(16)
        default:
            return cudaErrorInvalidValue;
    }
#undef RS_CASE
}

}  // namespace negf
