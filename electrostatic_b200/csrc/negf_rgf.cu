// Mode-space recursive Green's function (RGF) sweeps on sm_100a.
//
// Reference path replaced: the per-energy host recursion plus per-site
// device kernels of Source/Solver/Transport/NEGF/NEGF_Common.cpp
//   Compute_RhoEq      :3581-3781 (kernel :3742-3754)
//   Compute_GR_atPoles :3784-3954 (kernel :3937-3948)
//   Compute_Rho0       :3957-4092 (kernel :4073-4084)
//   Compute_RhoNonEq   :3115-3578 (kernel :3377-3497)
// and the analytic / decimation lead surface Green's function
//   CNT.cpp:354-393, NEGF_Common.cpp:1436-1508, 4095-4177.
//
// Work decomposition: one lane = one (tube, mode, energy) chain of N sites;
// one warp = 32 chains of the same tube, kind (contour/pole vs real axis)
// and precision.  Per chain:
//   forward  : Y_0 = 0, Y_{n+1} = h_n^2 / (alpha_n - Y_n)
//              lambda_{n+1} = lambda_n |h_n / (alpha_n - Y_n)|^2      (real axis)
//   backward : X_{N-1} = 0, X_{n-1} = h_{n-1}^2 / (alpha_n - X_n)
//              rho_{n-1} = rho_n |h_{n-1} / (alpha_n - X_n)|^2          (real axis)
//   G_nn = 1 / (alpha_n - X_n - Y_n)
//   |G_{n,0}|^2 = |G_nn|^2 lambda_n,  |G_{n,N-1}|^2 = |G_nn|^2 rho_n
// The last line uses the symmetry of (E - H - Sigma) (Hb = Hc in
// CNT.cpp:322-335): G_{n,0} = G_nn prod_{i=1..n}(-Ytil_i) equals the
// reference's per-site walk G_00 prod_{m<n}(-Xtil_m), so the O(N) walk per
// site (O(N^2) per energy) becomes two running products.
//
// The forward sweep stores (Y, lambda) every kSeg sites; the backward sweep
// recomputes each segment into registers and walks it in reverse, so the
// per-site state never goes to HBM (kSeg x fewer scratch bytes).  Each
// segment's per-lane contributions are summed over the 32 lanes with a
// butterfly reduce-scatter (one shuffle per site) and written as one
// coalesced row segment; a second kernel sums the rows per site in a fixed
// order (deterministic).

#include "negf_internal.h"

namespace negf {
namespace {

constexpr unsigned kFull = 0xffffffffu;

__device__ __forceinline__ double rcp(double x) { return __drcp_rn(x); }
__device__ __forceinline__ float rcp(float x) { return __frcp_rn(x); }

struct cd {
    double x, y;
};
__device__ __forceinline__ cd cadd(cd a, cd b) { return {a.x + b.x, a.y + b.y}; }
__device__ __forceinline__ cd csub(cd a, cd b) { return {a.x - b.x, a.y - b.y}; }
__device__ __forceinline__ cd cmul(cd a, cd b) { return {a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x}; }
__device__ __forceinline__ cd cscale(double s, cd a) { return {s * a.x, s * a.y}; }
__device__ __forceinline__ cd cconj(cd a) { return {a.x, -a.y}; }
__device__ __forceinline__ cd cinv(cd a) {
    const double r = rcp(a.x * a.x + a.y * a.y);
    return {a.x * r, -a.y * r};
}
// Principal square root: with m = |z|, t = sqrt((m + |Re z|)/2),
// sqrt(z) = (t, Im z / 2t) for Re z >= 0 and (|Im z| / 2t, copysign(t, Im z)) otherwise.
__device__ __forceinline__ cd csqrt_principal(cd z) {
    if (z.x == 0.0 && z.y == 0.0) return {0.0, z.y};
    const double m = hypot(z.x, z.y);
    const double t = sqrt(0.5 * (m + fabs(z.x)));
    if (z.x >= 0.0) return {t, z.y / (2.0 * t)};
    return {fabs(z.y) / (2.0 * t), copysign(t, z.y)};
}

// CNT.cpp:354-393: g = (F +- sqrt(F^2 - 4 (E-U)^2 gamma^2)) / (2 gamma^2 (E-U)),
// F = (E-U)^2 + gamma^2 - beta^2, root with Im g < 0 (first (F+S)/D, then
// (F-S)/D); when neither qualifies g keeps its zero initial value.
__device__ cd sgf_analytic(cd EmU, double beta, double gamma) {
    const cd e2 = cmul(EmU, EmU);
    const double g2 = gamma * gamma;
    const cd F = {e2.x + g2 - beta * beta, e2.y};
    const cd S = csqrt_principal(csub(cmul(F, F), cscale(4.0 * g2, e2)));
    const cd Di = cinv(cscale(2.0 * g2, EmU));
    const cd v1 = cmul(cadd(F, S), Di);
    if (v1.y < 0.0) return v1;
    const cd v2 = cmul(csub(F, S), Di);
    if (v2.y < 0.0) return v2;
    return {0.0, 0.0};
}

// NEGF_Common.cpp:1436-1508 + 4095-4153 on one mode of the diagonal block:
// condensed P-layer lead, then the decimation iterations.  The reference's
// tolerance is an int holding 1e-5, i.e. 0, so it always runs `iters`
// (= decimation_max_iter + 2) iterations; a zero update leaves the result
// unchanged, which makes the fixed count exact.
__device__ cd sgf_decimation(cd EmU, double beta, double gamma, int P, int iters) {
    constexpr int kMaxP = 64;
    cd Ht[kMaxP];
    const double Hb[2] = {-beta, -gamma};
    Ht[P - 1] = cinv(EmU);
    cd HtkP = Ht[P - 1];
    for (int k = P - 2; k >= 1; --k) {
        const double h = Hb[k % 2];
        Ht[k] = cinv(csub(EmU, cscale(h * h, Ht[k + 1])));
        HtkP = cscale(h, cmul(Ht[k], HtkP));
    }
    cd C = Ht[1];
    for (int k = 2; k < P; ++k) {
        const double h = Hb[(k - 1) % 2];
        C = cadd(Ht[k], cscale(h * h, cmul(cmul(Ht[k], C), Ht[k])));
    }
    const int id = (P - 1) % 2;
    const cd Xi_s = cscale(Hb[0] * Hb[0], Ht[1]);
    const cd Xi = cadd(Xi_s, cscale(Hb[id] * Hb[id], C));
    const cd Pi = cscale(Hb[0] * Hb[id], HtkP);
    const cd nu0i = cinv(csub(EmU, Xi));
    const cd g0d = cconj(Pi);
    const cd t1 = cmul(Pi, nu0i), t2 = cmul(t1, g0d), t3 = cmul(g0d, nu0i);
    cd mu = csub(csub(EmU, Xi_s), t2);
    cd nu = csub(csub(csub(EmU, Xi), t2), cmul(t3, Pi));
    cd ga = cmul(t1, Pi), ze = cmul(t3, g0d);
    for (int i = 0; i < iters; ++i) {
        const cd nui = cinv(nu);
        const cd a = cmul(cmul(ze, nui), ga), b = cmul(cmul(ga, nui), ze);
        mu = csub(mu, a);
        nu = csub(csub(nu, a), b);
        ga = cmul(cmul(ga, nui), ga);
        ze = cmul(cmul(ze, nui), ze);
    }
    return cinv(mu);
}

// Sigma_c = tau g tau^dagger with tau = gamma (CNT.cpp:338-352, NEGF_Common.cpp:4165-4177).
__device__ cd sigma_contact(cd E, double Uc, double beta, const TubeDev& T) {
    const cd EmU = {E.x - Uc, E.y};
    const cd g = T.use_decimation ? sgf_decimation(EmU, beta, T.gamma, T.dec_layers, T.dec_iters)
                                  : sgf_analytic(EmU, beta, T.gamma);
    return cscale(T.gamma * T.gamma, g);
}

// Butterfly reduce-scatter of K per-lane values over the 32 lanes: returns
// the sum over lanes of element j = lane >> (5 - log2 K).  K - 1 + log2(32/K)
// shuffles in total, fixed order (deterministic).
template <int K>
__device__ __forceinline__ double warp_reduce_scatter(double (&a)[K], int lane) {
    static_assert(K == 8 || K == 16 || K == 32, "K");
#pragma unroll
    for (int half = K / 2, bit = 16; half >= 1; half >>= 1, bit >>= 1) {
        const bool up = (lane & bit) != 0;
#pragma unroll
        for (int i = 0; i < half; ++i) {
            const double send = up ? a[i] : a[i + half];
            const double keep = up ? a[i + half] : a[i];
            a[i] = keep + __shfl_xor_sync(kFull, send, bit);
        }
    }
    constexpr int rest = (K == 8) ? 2 : (K == 16 ? 1 : 0);
#pragma unroll
    for (int r = 0, bit = (K == 8 ? 2 : 1); r < rest; ++r, bit >>= 1) a[0] += __shfl_xor_sync(kFull, a[0], bit);
    return a[0];
}

// One warp of chains.  R: recursion precision.  RA: real-axis (non-equilibrium) chains.
template <typename R, bool RA>
__device__ __forceinline__ void rgf_warp(const TubeDev* __restrict__ tubes, const ChainRec& c, const WarpRec& wr,
                                         double* __restrict__ prow, R* __restrict__ ck, int lane) {
    constexpr int K = kSeg;
    constexpr int NC = RA ? 3 : 2;  // checkpoint components: Y.re, Y.im (, lambda)
    const TubeDev& T = tubes[wr.tube];
    const int N = T.N;
    const double* __restrict__ U = T.U;
    const bool valid = c.mode >= 0;
    const int mode = valid ? c.mode : 0;
    const double beta = T.beta[mode];
    const double deg = valid ? T.degen[mode] : 0.0;

    // Lead self-energies in FP64 (both precisions).
    const cd E = {c.Er, c.Ei};
    const cd S0 = sigma_contact(E, T.Uc0, beta, T);
    const cd S1 = sigma_contact(E, T.Uc1, beta, T);

    const R Er = (R)c.Er, Ei = (R)c.Ei;
    const R s0r = (R)S0.x, s0i = (R)S0.y, s1r = (R)S1.x, s1i = (R)S1.y;
    const R hb2 = (R)(beta * beta), hg2 = (R)(T.gamma * T.gamma);
    const double cr = c.cr * deg, ci = c.ci * deg;
    // Gamma_k = i (Sigma_k - Sigma_k^dagger) = -2 Im Sigma_k
    const double k0 = RA ? (-2.0 * S0.y) * c.b0 * deg : 0.0;
    const double k1 = RA ? (-2.0 * S1.y) * c.b1 * deg : 0.0;
    const int nseg = (N + K - 1) / K;

    // ---- pass 1: forward sweep with checkpoints at segment starts
    {
        R yr = 0, yi = 0, lam = 1;
        for (int s = 0; s < nseg; ++s) {
            R* cks = ck + (size_t)s * NC * kWarp + lane;
            cks[0] = yr;
            cks[kWarp] = yi;
            if (RA) cks[2 * kWarp] = lam;
            const int n0 = s * K;
            R u[K];
#pragma unroll
            for (int j = 0; j < K; ++j) u[j] = (n0 + j < N) ? (R)__ldg(U + n0 + j) : (R)0;
#pragma unroll
            for (int j = 0; j < K; ++j) {
                const int n = n0 + j;
                if (n >= N - 1) break;
                R ar = Er - u[j], ai = Ei;
                if (n == 0) {
                    ar -= s0r;
                    ai -= s0i;
                }
                const R dr = ar - yr, di = ai - yi;
                const R inv = rcp(dr * dr + di * di);
                const R h2 = (n & 1) ? hg2 : hb2;
                yr = h2 * dr * inv;
                yi = -h2 * di * inv;
                if (RA) lam = lam * (h2 * inv);
            }
        }
    }

    // ---- pass 2: backward sweep, segment by segment
    R xr = 0, xi = 0, rho = 1;
    for (int s = nseg - 1; s >= 0; --s) {
        const int n0 = s * K;
        const R* cks = ck + (size_t)s * NC * kWarp + lane;
        R u[K], Yr[K], Yi[K], L[K];
#pragma unroll
        for (int j = 0; j < K; ++j) u[j] = (n0 + j < N) ? (R)__ldg(U + n0 + j) : (R)0;
        Yr[0] = cks[0];
        Yi[0] = cks[kWarp];
        L[0] = RA ? cks[2 * kWarp] : (R)1;
#pragma unroll
        for (int j = 0; j < K - 1; ++j) {
            const int n = n0 + j;
            if (n >= N - 1) break;
            R ar = Er - u[j], ai = Ei;
            if (n == 0) {
                ar -= s0r;
                ai -= s0i;
            }
            const R dr = ar - Yr[j], di = ai - Yi[j];
            const R inv = rcp(dr * dr + di * di);
            const R h2 = (n & 1) ? hg2 : hb2;
            Yr[j + 1] = h2 * dr * inv;
            Yi[j + 1] = -h2 * di * inv;
            if (RA) L[j + 1] = L[j] * (h2 * inv);
        }
        double acc[K];
#pragma unroll
        for (int j = K - 1; j >= 0; --j) {
            const int n = n0 + j;
            acc[j] = 0.0;
            if (n < N) {
                R ar = Er - u[j], ai = Ei;
                if (n == 0) {
                    ar -= s0r;
                    ai -= s0i;
                }
                if (n == N - 1) {
                    ar -= s1r;
                    ai -= s1i;
                }
                const R er = ar - xr, ei = ai - xi;  // alpha_n - X_n
                const R gr = er - Yr[j], gi = ei - Yi[j];
                const R ginv = rcp(gr * gr + gi * gi);  // = |G_nn|^2
                const double Gr = (double)(gr * ginv), Gi = (double)(-gi * ginv);
                double v = cr * Gi + ci * Gr;  // Im(c G)
                if (RA) v += (double)ginv * ((double)L[j] * k0 + (double)rho * k1);
                acc[j] = valid ? v : 0.0;
                if (n > 0) {
                    const R einv = rcp(er * er + ei * ei);
                    const R h2 = ((n - 1) & 1) ? hg2 : hb2;
                    xr = h2 * er * einv;
                    xi = -h2 * ei * einv;
                    if (RA) rho = rho * (h2 * einv);
                }
            }
        }
        const double tot = warp_reduce_scatter<K>(acc, lane);
        constexpr int shift = (K == 16) ? 1 : (K == 8 ? 2 : 0);
        const int j = lane >> shift;
        if ((lane & ((1 << shift) - 1)) == 0 && n0 + j < N) prow[n0 + j] = tot;
    }
}

__global__ void __launch_bounds__(128) rgf_kernel(const TubeDev* __restrict__ tubes,
                                                  const ChainRec* __restrict__ chains,
                                                  const WarpRec* __restrict__ warps, int num_warps,
                                                  double* __restrict__ partial, double* __restrict__ scratch) {
    const int lane = threadIdx.x & 31;
    const int w = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (w >= num_warps) return;
    const WarpRec wr = warps[w];
    const ChainRec c = chains[(size_t)w * kWarp + lane];
    double* prow = partial + wr.row_off;
    if (wr.fp32) {
        float* ck = reinterpret_cast<float*>(scratch + wr.ck_off);
        if (wr.kind == kRealAxis)
            rgf_warp<float, true>(tubes, c, wr, prow, ck, lane);
        else
            rgf_warp<float, false>(tubes, c, wr, prow, ck, lane);
    } else {
        double* ck = scratch + wr.ck_off;
        if (wr.kind == kRealAxis)
            rgf_warp<double, true>(tubes, c, wr, prow, ck, lane);
        else
            rgf_warp<double, false>(tubes, c, wr, prow, ck, lane);
    }
}

// Q[q_off + n] = sum_w partial[row_base + w N + n] (Kahan, fixed order) - rho0[n]
__global__ void reduce_kernel(const ReduceTube* __restrict__ rts, const double* __restrict__ partial,
                              double* __restrict__ Q) {
    const ReduceTube r = rts[blockIdx.y];
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= r.N) return;
    const double* p = partial + r.row_base + n;
    double s = 0.0, comp = 0.0;
    for (int w = 0; w < r.num_rows; ++w) {
        const double y = p[(size_t)w * r.N] - comp;
        const double t = s + y;
        comp = (t - s) - y;
        s = t;
    }
    if (r.rho0) s -= r.rho0[n];
    Q[r.q_off + n] = s;
}

}  // namespace

long long rgf_scratch_doubles(int N, int kind, int fp32) {
    const long long nseg = (N + kSeg - 1) / kSeg;
    const long long nc = (kind == kRealAxis) ? 3 : 2;
    const long long bytes = nseg * nc * kWarp * (fp32 ? 4 : 8);
    return (bytes + 15) / 16 * 2;  // 16-byte granules
}

int rgf_kernel_regs() {
    cudaFuncAttributes a;
    if (cudaFuncGetAttributes(&a, rgf_kernel) != cudaSuccess) return 0;
    return a.numRegs;
}

cudaError_t launch_rgf(const TubeDev* d_tubes, const ChainRec* d_chains, const WarpRec* d_warps, int num_warps,
                       double* d_partial, void* d_scratch, int warps_per_block, cudaStream_t stream) {
    if (num_warps <= 0) return cudaSuccess;
    if (warps_per_block < 1 || warps_per_block > 4) warps_per_block = 4;
    const int threads = warps_per_block * kWarp;
    const int blocks = (num_warps + warps_per_block - 1) / warps_per_block;
    rgf_kernel<<<blocks, threads, 0, stream>>>(d_tubes, d_chains, d_warps, num_warps, d_partial,
                                               static_cast<double*>(d_scratch));
    return cudaGetLastError();
}

cudaError_t launch_reduce(const ReduceTube* d_rt, int num_tubes, int max_N, const double* d_partial, double* d_Q,
                          cudaStream_t stream) {
    if (num_tubes <= 0 || max_N <= 0) return cudaSuccess;
    dim3 grid((max_N + 127) / 128, num_tubes);
    reduce_kernel<<<grid, 128, 0, stream>>>(d_rt, d_partial, d_Q);
    return cudaGetLastError();
}

}  // namespace negf
