// Real-space ring-block RGF of a zigzag (m,0) tube (FP64).
//
// Blocks of two rings (n = 2m atoms, m <= 16 so that one lane owns one row):
// rings 2k and 2k+1 are joined by the double bond (atom j to atoms j and
// j+1 mod m), ring 2k+1 to ring 2k+2 by the single bond (atom j to atom j),
// hopping gamma; in mode space these are beta_J = 2 gamma cos(pi J/m) and
// gamma (CNT.cpp:288-336), so a ring-uniform potential reproduces the sum of
// the m mode chains.  The self-energies of neighbouring blocks and of the
// leads touch one m x m corner only (gamma^2 g_bb on ring a, gamma^2 g_aa on
// ring b).
//
// Kernels (one warp per energy, rows of the working matrices owned by lanes,
// column-major shared-memory tiles so that lanes read consecutive words):
//   rs_lead_kernel   surface Green's functions of the two semi-infinite
//                    leads by the Lopez Sancho-Sancho-Rubio decimation,
//                    fixed iteration count -> corners sL[b][b], sR[a][a];
//   rs_chain_kernel  forward sweep (left-connected g_L, corner [b][b] kept in
//                    global memory per block), backward sweep (right-connected
//                    g_R in shared memory) with G_kk = (E - H_kk - S_L - S_R)^-1
//                    and the ring sums of c G_jj written to the energy's row;
//   rs_reduce_kernel sum over energies per ring in a fixed order (Kahan).
// Every inversion is Gauss-Jordan with partial pivoting on the augmented
// [M | I] tile (n x 2n complex).

#include "negf_internal.h"

namespace negf {
namespace {

constexpr int kMaxN = 32;

struct cplxd {
    double x, y;
};
__device__ __forceinline__ cplxd cmk(double a, double b) { return {a, b}; }
__device__ __forceinline__ cplxd cadd(cplxd a, cplxd b) { return {a.x + b.x, a.y + b.y}; }
__device__ __forceinline__ cplxd csub(cplxd a, cplxd b) { return {a.x - b.x, a.y - b.y}; }
__device__ __forceinline__ cplxd cmul(cplxd a, cplxd b) { return {fma(a.x, b.x, -a.y * b.y), fma(a.x, b.y, a.y * b.x)}; }
// a - f b
__device__ __forceinline__ cplxd cfnms(cplxd f, cplxd b, cplxd a) {
    return {fma(-f.x, b.x, fma(f.y, b.y, a.x)), fma(-f.x, b.y, fma(-f.y, b.x, a.y))};
}
// 1 / b, Smith (1962)
__device__ __forceinline__ cplxd cinvd(cplxd b) {
    if (fabs(b.x) >= fabs(b.y)) {
        const double r = b.y / b.x, d = b.x + r * b.y;
        return {1.0 / d, -r / d};
    }
    const double r = b.x / b.y, d = b.y + r * b.x;
    return {r / d, -1.0 / d};
}

// Tile: column-major, leading dimension ld (= n, the block size).
struct Tile {
    cplxd* a;
    int ld;
    __device__ cplxd& at(int r, int c) const { return a[c * ld + r]; }
};

// Gauss-Jordan: on entry columns [0, n) hold M, columns [n, 2n) are set to I
// here; on exit columns [n, 2n) hold M^-1.  Returns false if a pivot is 0.
__device__ bool gj_invert(Tile T, int n, int lane) {
    for (int c = 0; c < n; ++c)
        if (lane < n) T.at(lane, n + c) = cmk(lane == c ? 1.0 : 0.0, 0.0);
    __syncwarp();
    bool ok = true;
    for (int p = 0; p < n; ++p) {
        // pivot: largest |M[r][p]| over r >= p (lowest row on ties)
        double v = -1.0;
        if (lane >= p && lane < n) {
            const cplxd x = T.at(lane, p);
            v = x.x * x.x + x.y * x.y;
        }
        int idx = lane;
#pragma unroll
        for (int o = 16; o >= 1; o >>= 1) {
            const double ov = __shfl_xor_sync(0xffffffffu, v, o);
            const int oi = __shfl_xor_sync(0xffffffffu, idx, o);
            if (ov > v || (ov == v && oi < idx)) {
                v = ov;
                idx = oi;
            }
        }
        if (!(v > 0.0)) ok = false;
        const int piv = idx;
        if (piv != p) {  // swap rows p and piv, lanes over columns
            for (int c = lane; c < 2 * n; c += 32) {
                const cplxd t = T.at(p, c);
                T.at(p, c) = T.at(piv, c);
                T.at(piv, c) = t;
            }
        }
        __syncwarp();
        const cplxd inv = cinvd(T.at(p, p));
        __syncwarp();
        for (int c = lane; c < 2 * n; c += 32)
            if (c > p) T.at(p, c) = cmul(T.at(p, c), inv);
        if (lane == 0) T.at(p, p) = cmk(1.0, 0.0);
        __syncwarp();
        if (lane < n && lane != p) {
            const cplxd f = T.at(lane, p);
            for (int c = p + 1; c < 2 * n; ++c) T.at(lane, c) = cfnms(f, T.at(p, c), T.at(lane, c));
            T.at(lane, p) = cmk(0.0, 0.0);
        }
        __syncwarp();
    }
    return ok;
}

// E - H of one block into columns [0, n) of T (rows = lanes).
__device__ void build_block(Tile T, int m, double gamma, cplxd E, const double* __restrict__ U, int lane) {
    const int n = 2 * m;
    if (lane < n) {
        for (int c = 0; c < n; ++c) T.at(lane, c) = cmk(0.0, 0.0);
        T.at(lane, lane) = cmk(E.x - U[lane], E.y);
    }
    __syncwarp();
    if (lane < m) {  // double bond: ring a atom j <-> ring b atoms j, j+1
        const int a = lane, b1 = m + lane, b2 = m + (lane + 1) % m;
        T.at(a, b1).x -= gamma;
        T.at(b1, a).x -= gamma;
        T.at(a, b2).x -= gamma;
        T.at(b2, a).x -= gamma;
    }
    __syncwarp();
}

// C = A B for n x n tiles (columns [0, n)); lane = row of C.
__device__ void tile_gemm(Tile C, Tile A, Tile B, int n, int lane) {
    if (lane < n)
        for (int j = 0; j < n; ++j) {
            cplxd s = cmk(0.0, 0.0);
            for (int k = 0; k < n; ++k) s = cadd(s, cmul(A.at(lane, k), B.at(k, j)));
            C.at(lane, j) = s;
        }
    __syncwarp();
}


// Lead kernel: warp w -> energy w / 2, lead w % 2 (0 left, 1 right).
__global__ void __launch_bounds__(32) rs_lead_kernel(int m, double gamma, const double* __restrict__ Ere,
                                                     const double* __restrict__ Eim, int num_e, double Uc0, double Uc1,
                                                     int iters, cplxd* __restrict__ corners, int* __restrict__ status) {
    extern __shared__ cplxd sh[];
    const int lane = threadIdx.x;
    const int w = blockIdx.x;
    if (w >= 2 * num_e) return;
    const int e = w / 2, side = w % 2;
    const bool left = side == 0;
    const int n = 2 * m;
    const cplxd E = cmk(Ere[e], Eim[e]);
    const int sq = n * n;  // one n x n tile; the augmented tile is two
    Tile aug{sh, n}, eps{sh + 2 * sq, n}, epss{sh + 3 * sq, n}, al{sh + 4 * sq, n}, be{sh + 5 * sq, n},
        t1{sh + 6 * sq, n}, t2{sh + 7 * sq, n};
    // eps = eps_s = E - H00 at the contact potential
    {
        const double u = left ? Uc0 : Uc1;
        if (lane < n) {
            for (int c = 0; c < n; ++c) eps.at(lane, c) = cmk(0.0, 0.0);
            eps.at(lane, lane) = cmk(E.x - u, E.y);
        }
        __syncwarp();
        if (lane < m) {
            const int a = lane, b1 = m + lane, b2 = m + (lane + 1) % m;
            eps.at(a, b1).x -= gamma;
            eps.at(b1, a).x -= gamma;
            eps.at(a, b2).x -= gamma;
            eps.at(b2, a).x -= gamma;
        }
        __syncwarp();
        if (lane < n)
            for (int c = 0; c < n; ++c) {
                epss.at(lane, c) = eps.at(lane, c);
                // tau (ring b of a cell -> ring a of the next): -gamma at (m + j, j); tau^dagger at (j, m + j)
                const bool tb = (lane >= m && c == lane - m), td = (lane < m && c == lane + m);
                const cplxd tau = cmk(tb ? -gamma : 0.0, 0.0), taud = cmk(td ? -gamma : 0.0, 0.0);
                al.at(lane, c) = left ? taud : tau;
                be.at(lane, c) = left ? tau : taud;
            }
        __syncwarp();
    }
    bool ok = true;
    const Tile T0{sh, n};          // columns [0, n) of aug: free once g is formed
    const Tile g{sh + sq, n};      // columns [n, 2n) of aug: eps^-1 after the inversion
    for (int it = 0; it < iters; ++it) {
        if (lane < n)
            for (int c = 0; c < n; ++c) aug.at(lane, c) = eps.at(lane, c);
        __syncwarp();
        ok = gj_invert(aug, n, lane) && ok;
        tile_gemm(t1, al, g, n, lane);  // a g
        tile_gemm(t2, t1, be, n, lane);  // a g b
        if (lane < n)
            for (int c = 0; c < n; ++c) {
                epss.at(lane, c) = csub(epss.at(lane, c), t2.at(lane, c));
                eps.at(lane, c) = csub(eps.at(lane, c), t2.at(lane, c));
            }
        __syncwarp();
        tile_gemm(T0, be, g, n, lane);   // b g
        tile_gemm(t2, T0, al, n, lane);  // b g a
        if (lane < n)
            for (int c = 0; c < n; ++c) eps.at(lane, c) = csub(eps.at(lane, c), t2.at(lane, c));
        __syncwarp();
        tile_gemm(t2, t1, al, n, lane);  // a g a
        tile_gemm(t1, T0, be, n, lane);  // b g b
        if (lane < n)
            for (int c = 0; c < n; ++c) {
                al.at(lane, c) = t2.at(lane, c);
                be.at(lane, c) = t1.at(lane, c);
            }
        __syncwarp();
    }
    if (lane < n)
        for (int c = 0; c < n; ++c) aug.at(lane, c) = epss.at(lane, c);
    __syncwarp();
    ok = gj_invert(aug, n, lane) && ok;
    // corner: left lead -> g[b][b], right lead -> g[a][a]; stored column-major m x m
    const int off = left ? m : 0;
    cplxd* out = corners + ((size_t)e * 2 + side) * m * m;
    if (lane < m)
        for (int c = 0; c < m; ++c) out[c * m + lane] = aug.at(off + lane, n + off + c);
    if (!ok && lane == 0) atomicExch(status, 1);
}

// Chain kernel: warp e -> energy e.  gL: [num_e][K][m*m] scratch; rows:
// [num_e][N] ring sums of c G_jj (imaginary part).
__global__ void __launch_bounds__(32) rs_chain_kernel(int m, int K, double gamma, const double* __restrict__ Ere,
                                                      const double* __restrict__ Eim, const double* __restrict__ cre,
                                                      const double* __restrict__ cim, int num_e,
                                                      const double* __restrict__ Uatoms,
                                                      const cplxd* __restrict__ corners, cplxd* __restrict__ gL,
                                                      double* __restrict__ rows, int* __restrict__ status) {
    extern __shared__ cplxd sh[];
    const int lane = threadIdx.x;
    const int e = blockIdx.x;
    if (e >= num_e) return;
    const int n = 2 * m, mm = m * m, N = 2 * K;
    const cplxd E = cmk(Ere[e], Eim[e]);
    const cplxd cc = cmk(cre[e], cim[e]);
    const double g2 = gamma * gamma;
    Tile aug{sh, n};
    cplxd* gR = sh + 2 * n * n;  // m x m corner [a][a] of the right-connected g_R of block k+1
    const cplxd* sL = corners + (size_t)e * 2 * mm;
    const cplxd* sR = sL + mm;
    cplxd* myL = gL + (size_t)e * K * mm;
    double* row = rows + (size_t)e * N;
    bool ok = true;
    // forward: g_L[k] corner [b][b]
    for (int k = 0; k < K; ++k) {
        build_block(aug, m, gamma, E, Uatoms + (size_t)k * n, lane);
        const cplxd* c = k == 0 ? sL : myL + (size_t)(k - 1) * mm;
        if (lane < m)
            for (int j = 0; j < m; ++j) {
                const cplxd v = c[j * m + lane];
                aug.at(lane, j) = cmk(fma(-g2, v.x, aug.at(lane, j).x), fma(-g2, v.y, aug.at(lane, j).y));
            }
        __syncwarp();
        ok = gj_invert(aug, n, lane) && ok;
        if (lane < m)
            for (int j = 0; j < m; ++j) myL[(size_t)k * mm + j * m + lane] = aug.at(m + lane, n + m + j);
        __syncwarp();
    }
    // backward: g_R[k] and G_kk
    for (int k = K - 1; k >= 0; --k) {
        const cplxd* cr = k == K - 1 ? sR : gR;
        const cplxd* cl = k == 0 ? sL : myL + (size_t)(k - 1) * mm;
        // G_kk
        build_block(aug, m, gamma, E, Uatoms + (size_t)k * n, lane);
        if (lane < m)
            for (int j = 0; j < m; ++j) {
                const cplxd vl = cl[j * m + lane], vr = cr[j * m + lane];
                cplxd& a = aug.at(lane, j);
                a = cmk(fma(-g2, vl.x, a.x), fma(-g2, vl.y, a.y));
                cplxd& b = aug.at(m + lane, m + j);
                b = cmk(fma(-g2, vr.x, b.x), fma(-g2, vr.y, b.y));
            }
        __syncwarp();
        ok = gj_invert(aug, n, lane) && ok;
        {
            // ring sums of the diagonal: lanes [0, m) ring a, [m, 2m) ring b
            cplxd d = lane < n ? aug.at(lane, n + lane) : cmk(0.0, 0.0);
            double sa_x = lane < m ? d.x : 0.0, sa_y = lane < m ? d.y : 0.0;
            double sb_x = (lane >= m && lane < n) ? d.x : 0.0, sb_y = (lane >= m && lane < n) ? d.y : 0.0;
#pragma unroll
            for (int o = 16; o >= 1; o >>= 1) {
                sa_x += __shfl_xor_sync(0xffffffffu, sa_x, o);
                sa_y += __shfl_xor_sync(0xffffffffu, sa_y, o);
                sb_x += __shfl_xor_sync(0xffffffffu, sb_x, o);
                sb_y += __shfl_xor_sync(0xffffffffu, sb_y, o);
            }
            if (lane == 0) {
                row[2 * k] = fma(cc.x, sa_y, cc.y * sa_x);      // Im(c s_a)
                row[2 * k + 1] = fma(cc.x, sb_y, cc.y * sb_x);  // Im(c s_b)
            }
        }
        __syncwarp();
        if (k == 0) break;
        // g_R[k]: corner [a][a] for block k-1
        build_block(aug, m, gamma, E, Uatoms + (size_t)k * n, lane);
        if (lane < m)
            for (int j = 0; j < m; ++j) {
                const cplxd vr = cr[j * m + lane];
                cplxd& b = aug.at(m + lane, m + j);
                b = cmk(fma(-g2, vr.x, b.x), fma(-g2, vr.y, b.y));
            }
        __syncwarp();
        ok = gj_invert(aug, n, lane) && ok;
        if (lane < m)
            for (int j = 0; j < m; ++j) gR[j * m + lane] = aug.at(lane, n + j);
        __syncwarp();
    }
    if (!ok && lane == 0) atomicExch(status, 1);
}

// Q[r] (+)= sum over energies of rows[e][r], Kahan, energies in order.
__global__ void rs_reduce_kernel(const double* __restrict__ rows, int num_e, int N, double sign,
                                 double* __restrict__ Q, int accumulate) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= N) return;
    double s = 0.0, comp = 0.0;
    for (int e = 0; e < num_e; ++e) {
        const double y = rows[(size_t)e * N + r] - comp;
        const double t = s + y;
        comp = (t - s) - y;
        s = t;
    }
    Q[r] = accumulate ? Q[r] + sign * s : sign * s;
}

// Uatoms[r][j] = U[r] (ring-uniform potential on the atoms).
__global__ void rs_expand_kernel(const double* __restrict__ U, int N, int m, double* __restrict__ Ua) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < N * m) Ua[i] = U[i / m];
}

}  // namespace

cudaError_t rs_expand(const double* d_U, int N, int m, double* d_Ua, cudaStream_t stream) {
    if (N * m <= 0) return cudaSuccess;
    rs_expand_kernel<<<(N * m + 255) / 256, 256, 0, stream>>>(d_U, N, m, d_Ua);
    return cudaGetLastError();
}

size_t rs_lead_smem_bytes(int n) { return sizeof(cplxd) * 8 * n * n; }
size_t rs_chain_smem_bytes(int n) { return sizeof(cplxd) * (2 * n * n + n * n / 4 + 1); }
int rs_max_atoms_per_block() { return kMaxN; }

cudaError_t launch_realspace(int m, int K, double gamma, const double* d_Ere, const double* d_Eim,
                             const double* d_cre, const double* d_cim, int num_e, const double* d_Uatoms, double Uc0,
                             double Uc1, int lead_iters, void* d_corners, void* d_gL, double* d_rows, double* d_Q,
                             double sign, int accumulate, int* d_status, cudaStream_t stream) {
    if (num_e <= 0) return cudaSuccess;
    const int n = 2 * m;
    if (n > kMaxN) return cudaErrorInvalidValue;
    cudaError_t e = cudaFuncSetAttribute(rs_lead_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)rs_lead_smem_bytes(kMaxN));
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(rs_chain_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)rs_chain_smem_bytes(kMaxN));
    if (e != cudaSuccess) return e;
    rs_lead_kernel<<<2 * num_e, 32, rs_lead_smem_bytes(n), stream>>>(m, gamma, d_Ere, d_Eim, num_e, Uc0, Uc1,
                                                                     lead_iters, static_cast<cplxd*>(d_corners),
                                                                     d_status);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    rs_chain_kernel<<<num_e, 32, rs_chain_smem_bytes(n), stream>>>(
        m, K, gamma, d_Ere, d_Eim, d_cre, d_cim, num_e, d_Uatoms, static_cast<const cplxd*>(d_corners),
        static_cast<cplxd*>(d_gL), d_rows, d_status);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    const int N = 2 * K;
    rs_reduce_kernel<<<(N + 127) / 128, 128, 0, stream>>>(d_rows, num_e, N, sign, d_Q, accumulate);
    return cudaGetLastError();
}

}  // namespace negf
