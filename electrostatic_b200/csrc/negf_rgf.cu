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
// Pass 1 (one warp per 32 chains) runs the forward and the backward
// recursions together -- they are independent, so each lane carries two
// dependency chains -- and stores (Y, lambda) at every kSeg-site segment
// start and (X, rho) at every segment end.  With both boundary states known,
// the segments are independent: pass 2 launches one warp per (32 chains,
// group of kSegsPerUnit segments), recomputes Y forward inside a segment,
// walks X backward through it and forms the site contributions, so the
// per-site state never goes to HBM and the GPU is filled with
// throughput-bound warps instead of N-long latency-bound chains.  Each
// segment's per-lane contributions are summed over the 32 lanes with a
// butterfly reduce-scatter and written as one coalesced row segment; a third
// kernel sums the rows per site in a fixed order (deterministic).

#include <type_traits>

#include "negf_internal.h"

namespace negf {
namespace {

constexpr unsigned kFull = 0xffffffffu;

// Reciprocal: hardware approximation y0 = rcp.approx.ftz(x) with relative
// error e = 1 - x y0 (|e| <= 2^-20 or better), corrected by the truncated
// series 1/x = y0 / (1 - e) = y0 (1 + e + e^2 + ...): keeping e^2 leaves a
// relative error of order e^3 (< 2^-60) in FP64; FP32 keeps e (order e^2).
// Inputs here are squared moduli in [1e-30, 1e30]; x = 0 or inf is not handled.
__device__ __forceinline__ double rcp(double x) {
    double y;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
    const double e = fma(-x, y, 1.0);
    return fma(y, fma(e, e, e), y);
}
// Cache hint: bring the line holding p into L1 (every caller passes an
// address inside its buffer).
__device__ __forceinline__ void prefetch_l1(const void* p) { asm volatile("prefetch.global.L1 [%0];" ::"l"(p)); }

__device__ __forceinline__ float rcp(float x) {
    float y;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return fmaf(y, fmaf(-x, y, 1.0f), y);
}

#include "negf_sgf.cuh"  // cd, sgf_analytic, sgf_decimation

// Sigma_c = tau g tau^dagger with tau = gamma (CNT.cpp:338-352, NEGF_Common.cpp:4165-4177).
__device__ cd sigma_contact(cd E, double Uc, double beta, const TubeDev& T) {
    const cd EmU = {E.x - Uc, E.y};
    const cd g = T.use_decimation ? sgf_decimation(EmU, beta, T.gamma, T.dec_layers, T.dec_iters)
                                  : sgf_analytic(EmU, beta, T.gamma);
    return cscale(T.gamma * T.gamma, g);
}

// Accumulator of the per-site contributions before the 32-lane sum: FP64 for
// every chain (default), or the chains' precision when NEGF_FP32_LANE_SUMS is
// set (FP32 chains then sum their lanes in FP32: half the shuffles, about 5%
// faster, but at a biased self-consistent state of the 16-tube batch the
// mixed charge moved from 1.65e-5 to 2.6e-5 of the FP64 one).
#ifndef NEGF_FP32_LANE_SUMS
#define NEGF_FP32_LANE_SUMS 0
#endif
template <typename R>
using AccOf = typename std::conditional<(NEGF_FP32_LANE_SUMS != 0) || (sizeof(R) == 8), R, double>::type;

// Butterfly reduce-scatter of K per-lane values over the 32 lanes: returns
// the sum over lanes of element j = lane >> (5 - log2 K).  Fixed order, in
// the chains' precision (FP32 chains sum their 32 lanes in FP32; the rows
// are added up in FP64 afterwards).
template <int K, typename T>
__device__ __forceinline__ T warp_reduce_scatter(T (&a)[K], int lane) {
    static_assert(K == 8 || K == 16, "K");
#pragma unroll
    for (int half = K / 2, bit = 16; half >= 1; half >>= 1, bit >>= 1) {
        const bool up = (lane & bit) != 0;
#pragma unroll
        for (int i = 0; i < half; ++i) {
            const T send = up ? a[i] : a[i + half];
            const T keep = up ? a[i + half] : a[i];
            a[i] = keep + __shfl_xor_sync(kFull, send, bit);
        }
    }
    if (K == 8) {
        a[0] += __shfl_xor_sync(kFull, a[0], 2);
        a[0] += __shfl_xor_sync(kFull, a[0], 1);
    } else {
        a[0] += __shfl_xor_sync(kFull, a[0], 1);
    }
    return a[0];
}

template <typename R>
struct Chain {
    int N;
    R Er, Ei, s0r, s0i, s1r, s1i, hb2, hg2;
    double cr, ci, k0, k1;
    bool valid;
};

template <typename R, bool RA>
__device__ __forceinline__ Chain<R> make_chain(const TubeDev& T, const ChainRec& cr, double s0r, double s0i,
                                               double s1r, double s1i) {
    const bool valid = cr.mode >= 0;
    const int mode = valid ? cr.mode : 0;
    const double beta = T.beta[mode];
    const double deg = valid ? T.degen[mode] : 0.0;
    Chain<R> c;
    c.N = T.N;
    c.Er = (R)cr.Er;
    c.Ei = (R)cr.Ei;
    c.s0r = (R)s0r;
    c.s0i = (R)s0i;
    c.s1r = (R)s1r;
    c.s1i = (R)s1i;
    c.hb2 = (R)(beta * beta);
    c.hg2 = (R)(T.gamma * T.gamma);
    c.cr = cr.cr * deg;
    c.ci = cr.ci * deg;
    // Gamma_k = i (Sigma_k - Sigma_k^dagger) = -2 Im Sigma_k
    c.k0 = RA ? (-2.0 * s0i) * cr.b0 * deg : 0.0;
    c.k1 = RA ? (-2.0 * s1i) * cr.b1 * deg : 0.0;
    c.valid = valid;
    return c;
}

// Checkpoint record of segment s (per lane): Y_start (2), lambda_start,
// X_end (2), rho_end for real-axis warps; Y_start, X_end for contour warps.
template <bool RA>
struct CkLayout {
    static constexpr int NC = RA ? 6 : 4;
    static constexpr int Y = 0, L = 2, X = RA ? 3 : 2, RHO = 5;
};

// Projective form of the two recursions used by pass 1.  With
// Y_n = P_n / Q_n the forward map Y_{n+1} = h_n^2 / (alpha_n - Y_n) is the
// linear update (P, Q) <- (h_n^2 Q, alpha_n Q - P), and
// lambda_n = lambda_{n0} prod_{m=n0}^{n-1} h_m^2 / |Q_n|^2 when Q_{n0} = 1
// (the moduli |alpha_m - Y_m| = |Q_{m+1} / Q_m| telescope).  Likewise
// X_n = R_n / S_n with (R, S) <- (h_{n-1}^2 S, alpha_n S - R) going down.
// Im(alpha_n - Y_n) >= Im E > 0, so Q never vanishes; renormalising to
// Q = 1 once per segment keeps |P|, |Q| < (max |alpha|)^kSeg.
template <typename R>
struct Proj {
    R pr, pi, qr, qi;  // P, Q (scaled projective state)
    R lam;             // lambda (or rho) at the last segment boundary
    R H;               // product of h^2 since the last segment boundary
    R rq;              // 1 / |Q|^2 at the last segment boundary
};

// Linear step with hopping square h2 at a site of potential u (interior
// site: the caller accounts for the product of h^2); proj_step_edge adds
// the contact self-energy sr + i si to alpha and tracks the product.
template <typename R>
__device__ __forceinline__ void proj_step_int(const Chain<R>& c, Proj<R>& p, R u, R h2) {
    const R ar = c.Er - u;
    const R npr = h2 * p.qr, npi = h2 * p.qi;
    const R nqr = fma(ar, p.qr, fma(-c.Ei, p.qi, -p.pr));
    const R nqi = fma(ar, p.qi, fma(c.Ei, p.qr, -p.pi));
    p.pr = npr;
    p.pi = npi;
    p.qr = nqr;
    p.qi = nqi;
}
template <typename R>
__device__ __forceinline__ void proj_step(const Chain<R>& c, Proj<R>& p, R u, R h2) {
    const R ar = c.Er - u;
    const R npr = h2 * p.qr, npi = h2 * p.qi;
    const R nqr = fma(ar, p.qr, fma(-c.Ei, p.qi, -p.pr));
    const R nqi = fma(ar, p.qi, fma(c.Ei, p.qr, -p.pi));
    p.pr = npr;
    p.pi = npi;
    p.qr = nqr;
    p.qi = nqi;
    p.H *= h2;
}
template <typename R>
__device__ __forceinline__ void proj_step_edge(const Chain<R>& c, Proj<R>& p, R u, R h2, R sr, R si) {
    const R ar = c.Er - u - sr, ai = c.Ei - si;
    const R npr = h2 * p.qr, npi = h2 * p.qi;
    const R nqr = ar * p.qr - ai * p.qi - p.pr;
    const R nqi = ar * p.qi + ai * p.qr - p.pi;
    p.pr = npr;
    p.pi = npi;
    p.qr = nqr;
    p.qi = nqi;
    p.H *= h2;
}
// Segment boundary, off the recurrence's critical path: the checkpoint
// Y = P / Q and lambda from a snapshot of the state; the running state is
// rescaled by rq = 1 / |Q_b|^2 half a segment later.  With that scaling the
// telescoped moduli give lambda_{b+K} = lambda_b prod(h^2) rq_b rq_{b+K}.
// FP32 renormalises at the boundary itself (state := (Y, 1)): the deferred
// scaling lets |Q| swing to |Q_b|^-2 between boundaries, which can leave the
// FP32 range when |alpha - Y| is near its floor Im E.
template <typename R, bool RA>
__device__ __forceinline__ void proj_boundary(Proj<R>& p, R& yr, R& yi) {
    const R rq = rcp(p.qr * p.qr + p.qi * p.qi);
    yr = (p.pr * p.qr + p.pi * p.qi) * rq;
    yi = (p.pi * p.qr - p.pr * p.qi) * rq;
    if constexpr (sizeof(R) == 4) {
        if (RA) p.lam = p.lam * (p.H * rq);
        p.pr = yr;
        p.pi = yi;
        p.qr = 1;
        p.qi = 0;
    } else {
        if (RA) p.lam = p.lam * (p.H * p.rq * rq);
        p.rq = rq;
    }
    p.H = 1;
}
template <typename R>
__device__ __forceinline__ void proj_scale(Proj<R>& p) {
    if constexpr (sizeof(R) == 8) {
        p.pr *= p.rq;
        p.pi *= p.rq;
        p.qr *= p.rq;
        p.qi *= p.rq;
    }
}

// One block of pass 1: checkpoint both sweeps at their segment boundaries,
// prefetch the potentials of the next block (forward segment fs+1, backward
// segment bs-1) into (nf, nb) when has_next, then advance the forward sweep
// through segment fs and the backward sweep through segment bs.  INTERIOR:
// the caller guarantees that both segments are full and hold no contact site
// and that a next block exists.
// Checkpoint record of the fused schedule: one per segment, (Y, lambda) at
// the start of a segment the forward sweep crosses first, (X, rho) at the end
// of one the backward sweep crosses first.
template <bool RA>
struct CkCompact {
    static constexpr int NC = RA ? 3 : 2;
};

template <typename R, bool RA, bool INTERIOR, bool COMPACT = false>
__device__ __forceinline__ void pass1_block(const Chain<R>& c, Proj<R>& f, Proj<R>& b, int fs, int bs, bool has_next,
                                            const double* __restrict__ U, R* __restrict__ ck, const R (&uf)[kSeg],
                                            const R (&ub)[kSeg], R (&nf)[kSeg], R (&nb)[kSeg], R hfull) {
    constexpr int K = kSeg;
    using CL = CkLayout<RA>;
    const int N = c.N;
    const int f0 = fs * K;                  // forward segment start
    const int be = min(bs * K + K, N) - 1;  // backward segment end
    {
        R yr, yi, xr, xi;
        proj_boundary<R, RA>(f, yr, yi);
        proj_boundary<R, RA>(b, xr, xi);
        if (COMPACT) {
            constexpr int NC = CkCompact<RA>::NC;
            R* p = ck + (size_t)fs * NC * kWarp;
            p[0] = yr;
            p[kWarp] = yi;
            if (RA) p[2 * kWarp] = f.lam;
            R* q = ck + (size_t)bs * NC * kWarp;
            q[0] = xr;
            q[kWarp] = xi;
            if (RA) q[2 * kWarp] = b.lam;
        } else {
            R* p = ck + (size_t)fs * CL::NC * kWarp;
            p[CL::Y * kWarp] = yr;
            p[(CL::Y + 1) * kWarp] = yi;
            if (RA) p[CL::L * kWarp] = f.lam;
            R* q = ck + (size_t)bs * CL::NC * kWarp;
            q[CL::X * kWarp] = xr;
            q[(CL::X + 1) * kWarp] = xi;
            if (RA) q[CL::RHO * kWarp] = b.lam;
        }
    }
    if (INTERIOR || has_next) {
        // next forward segment fs+1 and next backward segment bs-1 (full, bs >= 1):
        // 16-byte aligned, inside the padded buffer
        const double2* pf = reinterpret_cast<const double2*>(U + f0 + K);
        const double2* pb = reinterpret_cast<const double2*>(U + (bs - 1) * K);
#pragma unroll
        for (int k = 0; k < K / 2; ++k) {
            const double2 vf = __ldg(pf + k), vb = __ldg(pb + k);
            nf[2 * k] = (R)vf.x;
            nf[2 * k + 1] = (R)vf.y;
            nb[K - 1 - 2 * k] = (R)vb.x;
            nb[K - 2 - 2 * k] = (R)vb.y;
        }
    }
    const bool interior =
        INTERIOR || ((f0 > 0) && (f0 + K < N) && (be < N - 1) && (bs > 0) && (be == bs * K + K - 1));
    if (interior) {
        // forward sites f0 + j (parity of j since f0 is even); backward sites
        // be - j use h_{be-j-1}, parity of j since be - 1 is even.
#pragma unroll
        for (int j = 0; j < K; ++j) {
            if (j == K / 2) {
                proj_scale(f);
                proj_scale(b);
            }
            const R h2 = (j & 1) ? c.hg2 : c.hb2;
            proj_step_int(c, f, uf[j], h2);
            proj_step_int(c, b, ub[j], h2);
        }
        f.H = hfull;
        b.H = hfull;
    } else {
#pragma unroll
        for (int j = 0; j < K; ++j) {
            const int n = f0 + j;
            const int m = be - j;  // backward step at site m gives X_{m-1}
            if (j == K / 2) {
                proj_scale(f);
                proj_scale(b);
            }
            if (n < N - 1) {
                const R h2 = (n & 1) ? c.hg2 : c.hb2;
                if (n == 0)
                    proj_step_edge(c, f, uf[j], h2, c.s0r, c.s0i);
                else
                    proj_step(c, f, uf[j], h2);
            }
            if (m >= bs * K && m >= 1) {
                const R h2 = ((m - 1) & 1) ? c.hg2 : c.hb2;
                if (m == N - 1)
                    proj_step_edge(c, b, ub[j], h2, c.s1r, c.s1i);
                else
                    proj_step(c, b, ub[j], h2);
            }
        }
    }
}

// Initial sweep states of one piece of a chain (FP64): forward (Y, lambda)
// at the piece's first site, backward (X, rho) at its last site.
struct PieceState {
    double yr, yi, lam, xr, xi, rho;
};

// Pass 1 over segments [s0, s1) of a chain: lead self-energies (FP64; the
// piece holding site 0 stores them for pass 2), then the forward (Y, lambda)
// and backward (X, rho) sweeps run together (they are independent), in
// projective form, from the piece's initial states, storing the state at
// every segment start (forward) and segment end (backward).  The whole chain
// is the single piece [0, nseg) with Y_0 = 0, lambda_0 = 1, X_{N-1} = 0,
// rho_{N-1} = 1.
template <typename R, bool RA>
__device__ __forceinline__ void pass1_chain(const TubeDev* __restrict__ tubes, const ChainRec& cr, int tube,
                                            double* __restrict__ wscratch, int lane, int s0, int s1,
                                            const PieceState& st) {
    constexpr int K = kSeg;
    static_assert(K % 2 == 0, "segment length must be even");
    const TubeDev& T = tubes[tube];
    const int N = T.N;
    const int nseg = (N + K - 1) / K;
    if (s1 <= s0) return;
    const double* __restrict__ U = T.U;
    const bool valid = cr.mode >= 0;
    const double beta = T.beta[valid ? cr.mode : 0];
    const cd E = {cr.Er, cr.Ei};
    cd S0 = {0.0, 0.0}, S1 = {0.0, 0.0};
    if (s0 == 0 || s1 == nseg) {  // the contact sites lie in the first and the last piece
        // U_contact = U at the end sites (Nanostructure.cpp:500-504) when read on the device
        const double Uc0 = T.uc_from_U ? U[0] : T.Uc0, Uc1 = T.uc_from_U ? U[N - 1] : T.Uc1;
        S0 = sigma_contact(E, Uc0, beta, T);
        S1 = sigma_contact(E, Uc1, beta, T);
    }
    if (s0 == 0) {
        wscratch[0 * kWarp + lane] = S0.x;
        wscratch[1 * kWarp + lane] = S0.y;
        wscratch[2 * kWarp + lane] = S1.x;
        wscratch[3 * kWarp + lane] = S1.y;
    }
    const Chain<R> c = make_chain<R, RA>(T, cr, S0.x, S0.y, S1.x, S1.y);
    R* __restrict__ ck = reinterpret_cast<R*>(wscratch + 4 * kWarp) + lane;
    Proj<R> f{(R)st.yr, (R)st.yi, 1, 0, (R)st.lam, 1, 1};
    Proj<R> b{(R)st.xr, (R)st.xi, 1, 0, (R)st.rho, 1, 1};
    R hfull = 1;  // prod of h^2 over a full segment
#pragma unroll
    for (int j = 0; j < K / 2; ++j) hfull *= c.hb2 * c.hg2;
    const int nb = s1 - s0;
    const int e = min(s1 * K, N) - 1;  // the piece's last site
    // potentials of the first block: forward segment s0, backward segment s1-1
    // (the buffer has kPadLo zeros before site 0 and kPadHi after site N-1)
    R ua_f[K], ua_b[K], ub_f[K], ub_b[K];
#pragma unroll
    for (int j = 0; j < K; ++j) {
        ua_f[j] = (R)__ldg(U + s0 * K + j);
        ua_b[j] = (R)__ldg(U + e - j);
    }
    // Block k advances forward segment s0+k and backward segment s1-1-k.
    // Blocks 1 .. nb-2 never touch the contact segments and run in a
    // branch-free loop, two blocks per trip with the potential buffers
    // alternating; the first and last blocks decide at run time.
    pass1_block<R, RA, false>(c, f, b, s0, s1 - 1, nb > 1, U, ck, ua_f, ua_b, ub_f, ub_b, hfull);
    if (nb == 1) return;
    int k = 1;
    for (; k + 2 <= nb - 1; k += 2) {
        pass1_block<R, RA, true>(c, f, b, s0 + k, s1 - 1 - k, true, U, ck, ub_f, ub_b, ua_f, ua_b, hfull);
        pass1_block<R, RA, true>(c, f, b, s0 + k + 1, s1 - 2 - k, true, U, ck, ua_f, ua_b, ub_f, ub_b, hfull);
    }
    if (k < nb - 1) {
        pass1_block<R, RA, true>(c, f, b, s0 + k, s1 - 1 - k, true, U, ck, ub_f, ub_b, ua_f, ua_b, hfull);
        pass1_block<R, RA, false>(c, f, b, s1 - 1, s0, false, U, ck, ua_f, ua_b, ub_f, ub_b, hfull);
    } else {
        pass1_block<R, RA, false>(c, f, b, s1 - 1, s0, false, U, ck, ub_f, ub_b, ua_f, ua_b, hfull);
    }
}

// Pass 2 segment in projective form (FP64).  From (P, Q) = (Y_{n0}, 1) the
// forward recurrence gives P_n, Q_n and Q_{n+1} = alpha_n Q_n - P_n; from
// (R, S) = (X_e, 1) the backward one gives R_n, S_n.  Then
//   D_n = alpha_n Q_n S_n - R_n Q_n - P_n S_n = S_n Q_{n+1} - R_n Q_n,
//   G_nn = Q_n S_n / D_n,
//   |G_nn|^2 lambda_n = lambda_{n0} prod_{n0<=m<n} h_m^2 |S_n|^2 / |D_n|^2,
//   |G_nn|^2 rho_n    = rho_e prod_{n<=m<e} h_m^2 |Q_n|^2 / |D_n|^2,
// with only short linear dependency chains.  D_n does not depend on n inside
// a segment, so full segments take one reciprocal in all.
template <typename R>
struct CkVals {  // one lane's checkpoint of a segment
    R yr, yi, lam, xr, xi, rho;
};
template <typename R, bool RA>
__device__ __forceinline__ CkVals<R> load_ck(const R* __restrict__ p) {
    using CL = CkLayout<RA>;
    CkVals<R> v;
    v.yr = p[CL::Y * kWarp];
    v.yi = p[(CL::Y + 1) * kWarp];
    v.lam = RA ? p[CL::L * kWarp] : (R)1;
    v.xr = p[CL::X * kWarp];
    v.xi = p[(CL::X + 1) * kWarp];
    v.rho = RA ? p[CL::RHO * kWarp] : (R)1;
    return v;
}

// Sweep state at a segment boundary (normalised: (Y, 1) with lambda).
template <typename R>
struct Bnd {
    R yr, yi, lam;
};

// State of one segment between its forward part (recompute of (P, Q) from
// the start record, D and the folded coefficients) and its backward part
// (walk of (R, S) from the end record with the site contributions).
template <typename R>
struct SegWork {
    R qr[kSeg + 1], qi[kSeg + 1], lm[kSeg];
    R Rr, Ri, rh, cgr, cgi;
};

template <typename R, bool RA, bool EDGE, bool NEXT = false>
__device__ __forceinline__ void seg_fwd(const Chain<R>& c, int n0, const CkVals<R>& ckv, const R (&u)[kSeg],
                                        SegWork<R>& w, Bnd<R>* next = nullptr) {
    constexpr int K = kSeg;
    const int N = c.N;
    R pr = ckv.yr, pi = ckv.yi;
    w.qr[0] = 1;
    w.qi[0] = 0;
    w.lm[0] = ckv.lam;
    w.Rr = ckv.xr;
    w.Ri = ckv.xi;
    w.rh = ckv.rho;
#pragma unroll
    for (int j = 0; j < K; ++j) {
        const int n = n0 + j;
        R ar = c.Er - u[j], ai = c.Ei;
        if (EDGE) {
            if (n >= N) break;
            if (n == 0) {
                ar -= c.s0r;
                ai -= c.s0i;
            }
            if (n == N - 1) {
                ar -= c.s1r;
                ai -= c.s1i;
            }
        }
        w.qr[j + 1] = fma(ar, w.qr[j], fma(-ai, w.qi[j], -pr));
        w.qi[j + 1] = fma(ar, w.qi[j], fma(ai, w.qr[j], -pi));
        if (j + 1 < K) {
            const R h2 = EDGE ? ((n & 1) ? c.hg2 : c.hb2) : ((j & 1) ? c.hg2 : c.hb2);
            pr = h2 * w.qr[j];
            pi = h2 * w.qi[j];
            if (RA) w.lm[j + 1] = w.lm[j] * h2;
        }
    }
    if constexpr (NEXT) {
        // forward state at the next segment start (interior segments, K even:
        // the last hopping of the segment is gamma): Y = h^2 Q_{K-1} / Q_K,
        // lambda = lambda_{n0} prod h^2 / |Q_K|^2 with Q_{n0} = 1
        static_assert(!EDGE, "next boundary of interior segments only");
        const R rq = rcp(fma(w.qr[K], w.qr[K], w.qi[K] * w.qi[K]));
        const R tr = fma(w.qr[K - 1], w.qr[K], w.qi[K - 1] * w.qi[K]);
        const R ti = fma(w.qi[K - 1], w.qr[K], -w.qr[K - 1] * w.qi[K]);
        next->yr = c.hg2 * tr * rq;
        next->yi = c.hg2 * ti * rq;
        next->lam = RA ? w.lm[K - 1] * c.hg2 * rq : (R)1;
    }
    // Interior segment: D_n is the same at every site of the segment (the
    // discrete Wronskian: with S_{n-1} = alpha_n S_n - h_n^2 S_{n+1} and
    // Q_{n+1} = alpha_n Q_n - h_{n-1}^2 Q_{n-1}, D_{n-1} = D_n), so it is
    // formed once at the segment end, where S = 1 and R = X_e, and folded
    // into the per-segment coefficients.
    // D, |D|^2 and the folded coefficients in FP64 once per segment; the
    // per-site products then run in the chain's precision
    w.cgr = 0;
    w.cgi = 0;  // contour: c conj(D) / |D|^2
    if (!EDGE) {
        const double dr =
            fma(-(double)w.Rr, (double)w.qr[K - 1], fma((double)w.Ri, (double)w.qi[K - 1], (double)w.qr[K]));
        const double di =
            fma(-(double)w.Rr, (double)w.qi[K - 1], fma(-(double)w.Ri, (double)w.qr[K - 1], (double)w.qi[K]));
        const double inv = rcp(fma(dr, dr, di * di));
        if (RA) {
            const R fa = (R)(c.k0 * inv), fb = (R)(c.k1 * inv);
#pragma unroll
            for (int j = 0; j < K; ++j) w.lm[j] *= fa;
            w.rh *= fb;
        } else {
            w.cgr = (R)(fma(c.cr, dr, c.ci * di) * inv);
            w.cgi = (R)(fma(c.ci, dr, -c.cr * di) * inv);
        }
    }
}

template <typename R, bool RA, bool EDGE>
__device__ __forceinline__ void seg_bwd(const Chain<R>& c, int n0, const R (&u)[kSeg], SegWork<R>& w,
                                        AccOf<R> (&acc)[kSeg]) {
    constexpr int K = kSeg;
    const int N = c.N;
    R Rr = w.Rr, Ri = w.Ri, Sr = 1, Si = 0, rh = w.rh;
#pragma unroll
    for (int j = K - 1; j >= 0; --j) {
        const int n = n0 + j;
        acc[j] = 0;
        if (EDGE && n >= N) continue;
        if (!EDGE) {
            R v;
            if (RA) {  // |G|^2 (lambda k0 + rho k1) = lm |S|^2 + rh |Q|^2, 1/|D|^2 folded in
                const R s2 = fma(Sr, Sr, Si * Si), q2 = fma(w.qr[j], w.qr[j], w.qi[j] * w.qi[j]);
                v = fma(w.lm[j], s2, rh * q2);
            } else {  // Im(c Q S / D)
                const R tr = fma(w.qr[j], Sr, -w.qi[j] * Si), ti = fma(w.qr[j], Si, w.qi[j] * Sr);
                v = fma(w.cgr, ti, w.cgi * tr);
            }
            acc[j] = c.valid ? (AccOf<R>)v : (AccOf<R>)0;
        } else {
            double v;
            // D = S Q_{n+1} - R Q_n, per site (the segment may be partial), in FP64
            const double Sd = Sr, Sid = Si, Rd = Rr, Rid = Ri;
            const double q1r = w.qr[j + 1], q1i = w.qi[j + 1], q0r = w.qr[j], q0i = w.qi[j];
            const double dr = fma(Sd, q1r, fma(-Sid, q1i, fma(-Rd, q0r, Rid * q0i)));
            const double di = fma(Sd, q1i, fma(Sid, q1r, fma(-Rd, q0i, -Rid * q0r)));
            const double inv = rcp(fma(dr, dr, di * di));
            if (RA) {  // real-axis chains carry no contour coefficient (c = 0)
                const double s2 = fma(Sd, Sd, Sid * Sid), q2 = fma(q0r, q0r, q0i * q0i);
                v = inv * fma((double)w.lm[j] * s2, c.k0, (double)rh * q2 * c.k1);
            } else {  // Im(c T conj(D)) / |D|^2 with T = Q S
                const double tr = fma(q0r, Sd, -q0i * Sid), ti = fma(q0r, Sid, q0i * Sd);
                const double ur = fma(tr, dr, ti * di), ui = fma(ti, dr, -tr * di);
                v = fma(c.cr, ui, c.ci * ur) * inv;
            }
            acc[j] = c.valid ? (AccOf<R>)v : (AccOf<R>)0;
        }
        if (j > 0) {  // (R, S) at site n - 1
            R ar = c.Er - u[j], ai = c.Ei;
            if (EDGE) {
                if (n == N - 1) {
                    ar -= c.s1r;
                    ai -= c.s1i;
                }
            }
            const R h2 = EDGE ? (((n - 1) & 1) ? c.hg2 : c.hb2) : (((j - 1) & 1) ? c.hg2 : c.hb2);
            const R nrr = h2 * Sr, nri = h2 * Si;
            const R nsr = fma(ar, Sr, fma(-ai, Si, -Rr));
            const R nsi = fma(ar, Si, fma(ai, Sr, -Ri));
            Rr = nrr;
            Ri = nri;
            Sr = nsr;
            Si = nsi;
            if (RA) rh *= h2;
        }
    }
}

template <typename R, bool RA, bool EDGE, bool NEXT = false>
__device__ __forceinline__ void segment_proj(const Chain<R>& c, int n0, const CkVals<R>& ckv, const R (&u)[kSeg],
                                             AccOf<R> (&acc)[kSeg], Bnd<R>* next = nullptr) {
    SegWork<R> w;
    seg_fwd<R, RA, EDGE, NEXT>(c, n0, ckv, u, w, next);
    seg_bwd<R, RA, EDGE>(c, n0, u, w, acc);
}

// Pass 2: segments [seg0, seg1) of one warp's chains.  Per segment: forward
// recompute of Y (and lambda) from the start checkpoint, then the backward
// walk of X (and rho) from the end checkpoint with the site contributions,
// a 32-lane reduce-scatter and one coalesced row write.
template <typename R, bool RA>
__device__ __forceinline__ void pass2_unit(const TubeDev* __restrict__ tubes, const ChainRec& cr, const WarpRec& wr,
                                           const SegUnit& su, const double* __restrict__ wscratch,
                                           double* __restrict__ prow, int lane) {
    constexpr int K = kSeg;
    using CL = CkLayout<RA>;
    const TubeDev& T = tubes[wr.tube];
    const int N = T.N;
    const double* __restrict__ U = T.U;
    const double s0r = wscratch[0 * kWarp + lane], s0i = wscratch[1 * kWarp + lane];
    const double s1r = wscratch[2 * kWarp + lane], s1i = wscratch[3 * kWarp + lane];
    const R* __restrict__ ck = reinterpret_cast<const R*>(wscratch + 4 * kWarp) + lane;
    const Chain<R> c = make_chain<R, RA>(T, cr, s0r, s0i, s1r, s1i);

    {
        // the unit's potentials (at most 256 sites, 17 lines) into L1, one line per lane
        const int first = su.seg0 * K, last = min(su.seg1 * K, N), off = lane * 16;
        if (off < last - first + 16) prefetch_l1(U + min(first + off, last - 1));
    }
    // the next segment's checkpoint is loaded while this one is computed,
    // the one after next is brought into L1
    CkVals<R> cur = load_ck<R, RA>(ck + (size_t)su.seg0 * CL::NC * kWarp);
    for (int s = su.seg0; s < su.seg1; ++s) {
        const int n0 = s * K;
        if (s + 2 < su.seg1) {
            const R* q = ck + (size_t)(s + 2) * CL::NC * kWarp;
#pragma unroll
            for (int k = 0; k < CL::NC; ++k) prefetch_l1(q + k * kWarp);
        }
        CkVals<R> nxt = cur;
        if (s + 1 < su.seg1) nxt = load_ck<R, RA>(ck + (size_t)(s + 1) * CL::NC * kWarp);
        R u[K];
        AccOf<R> acc[K];
        const bool interior = n0 > 0 && n0 + K < N;
        if (interior) {
            const double2* u2 = reinterpret_cast<const double2*>(U + n0);  // n0 even, U 16-byte aligned
#pragma unroll
            for (int k = 0; k < K / 2; ++k) {
                const double2 v = __ldg(u2 + k);
                u[2 * k] = (R)v.x;
                u[2 * k + 1] = (R)v.y;
            }
            segment_proj<R, RA, false>(c, n0, cur, u, acc);
        } else {
#pragma unroll
            for (int k = 0; k < K; ++k) u[k] = (n0 + k < N) ? (R)__ldg(U + n0 + k) : (R)0;
            segment_proj<R, RA, true>(c, n0, cur, u, acc);
        }
        cur = nxt;
        const double tot = (double)warp_reduce_scatter<K>(acc, lane);
        constexpr int shift = (K == 16) ? 1 : 2;
        const int j = lane >> shift;
        if ((lane & ((1 << shift) - 1)) == 0 && n0 + j < N) prow[n0 + j] = tot;
    }
}

// K forward projective steps through an interior segment from the
// normalised state (Y, 1), lambda: the normalised state at the next segment
// start.  The same routine advances the backward sweep when given the
// segment's potentials in reverse order (the hopping parities of an aligned
// segment read the same both ways).
template <typename R, bool RA>
__device__ __forceinline__ Bnd<R> sweep_segment(const Chain<R>& c, const Bnd<R>& in, const R (&u)[kSeg]) {
    constexpr int K = kSeg;
    R pr = in.yr, pi = in.yi, qr = 1, qi = 0, H = 1;
#pragma unroll
    for (int j = 0; j < K; ++j) {
        const R h2 = (j & 1) ? c.hg2 : c.hb2;
        const R ar = c.Er - u[j];
        const R nqr = fma(ar, qr, fma(-c.Ei, qi, -pr));
        const R nqi = fma(ar, qi, fma(c.Ei, qr, -pi));
        pr = h2 * qr;
        pi = h2 * qi;
        qr = nqr;
        qi = nqi;
        H *= h2;
    }
    // Y = h^2 Q_{K-1} / Q_K (pr, pi = h^2 Q_{K-1}), lambda * prod h^2 / |Q_K|^2
    const R rq = rcp(fma(qr, qr, qi * qi));
    Bnd<R> o;
    o.yr = fma(pr, qr, pi * qi) * rq;
    o.yi = fma(pi, qr, -pr * qi) * rq;
    o.lam = RA ? in.lam * H * rq : (R)1;
    return o;
}

// Sum of a segment's per-lane contributions over the warp, one coalesced
// row-segment write (sites n0 .. n0 + K - 1 below N).
template <typename T>
__device__ __forceinline__ void write_segment(T (&acc)[kSeg], int n0, int N, double* __restrict__ prow, int lane) {
    const double tot = (double)warp_reduce_scatter<kSeg>(acc, lane);
    const int j = lane >> 2;
    if ((lane & 3) == 0 && n0 + j < N) prow[n0 + j] = tot;
}

template <typename R>
__device__ __forceinline__ void load_seg(const double* __restrict__ U, int n0, R (&u)[kSeg]) {
    const double2* u2 = reinterpret_cast<const double2*>(U + n0);  // n0 even, U 16-byte aligned
#pragma unroll
    for (int k = 0; k < kSeg / 2; ++k) {
        const double2 v = __ldg(u2 + k);
        u[2 * k] = (R)v.x;
        u[2 * k + 1] = (R)v.y;
    }
}
template <typename R>
__device__ __forceinline__ void load_seg_reversed(const double* __restrict__ U, int n0, R (&u)[kSeg]) {
    const double2* u2 = reinterpret_cast<const double2*>(U + n0);
#pragma unroll
    for (int k = 0; k < kSeg / 2; ++k) {
        const double2 v = __ldg(u2 + k);
        u[kSeg - 1 - 2 * k] = (R)v.x;
        u[kSeg - 2 - 2 * k] = (R)v.y;
    }
}
template <typename R>
__device__ __forceinline__ void load_seg_edge(const double* __restrict__ U, int n0, int N, R (&u)[kSeg]) {
#pragma unroll
    for (int k = 0; k < kSeg; ++k) u[k] = (n0 + k < N) ? (R)__ldg(U + n0 + k) : (R)0;
}

// ---- Packed FP32 pairs (sm_100 FFMA2 / FMUL2 / FADD2).  The fused schedule
// runs two independent recurrences per chain side by side -- the forward
// sweep and the backward sweep (the chain read from the drain end) -- with
// the same operations on different data, so an FP32 chain carries both in
// one float2: .x forward, .y backward, and every step of the interior loops
// issues one packed instruction for the two.  The states keep -P (and -R)
// so that no step needs a negation: with a = E - U and the hopping square h2,
//   Q' = a Q - i Ei Q ... written out: qr' = a qr - Ei qi - pr,
//   qi' = a qi + Ei qr - pi, and -P' = -h2 Q.
struct F2 {
    float2 v;
};
__device__ __forceinline__ F2 f2(float x, float y) { return {make_float2(x, y)}; }
__device__ __forceinline__ F2 f2b(float x) { return {make_float2(x, x)}; }
__device__ __forceinline__ F2 add2(F2 a, F2 b) { return {__fadd2_rn(a.v, b.v)}; }
__device__ __forceinline__ F2 mul2(F2 a, F2 b) { return {__fmul2_rn(a.v, b.v)}; }
__device__ __forceinline__ F2 fma2(F2 a, F2 b, F2 c) { return {__ffma2_rn(a.v, b.v, c.v)}; }

// -U of an aligned interior segment (forward order) and of another read in
// reverse, as pairs: mu[j] = (-U[nf + j], -U[nb + K - 1 - j]).
__device__ __forceinline__ void load_seg_pair(const double* __restrict__ U, int nf, int nb, F2 (&mu)[kSeg]) {
#pragma unroll
    for (int k = 0; k < kSeg / 2; ++k) {
        // nf, nb and K even, U 16-byte aligned
        const double2 va = __ldg(reinterpret_cast<const double2*>(U + nf + 2 * k));
        const double2 vb = __ldg(reinterpret_cast<const double2*>(U + nb + kSeg - 2 - 2 * k));
        mu[2 * k] = f2(-(float)va.x, -(float)vb.y);
        mu[2 * k + 1] = f2(-(float)va.y, -(float)vb.x);
    }
}

// Pass-1 state of both sweeps of a chain: -P, Q, lambda and the product of
// h^2 since the last boundary, per direction.
struct Proj2 {
    F2 mpr, mpi, qr, qi, lam, H;
};

// One interior block of phase A for an FP32 chain (pass1_block with
// INTERIOR and COMPACT, both sweeps packed): boundary records of the forward
// sweep at segment fs and of the backward sweep at segment bs, the next
// block's potentials into mun, then K packed steps over whole segments
// (the product of h^2 at the next boundary is hfull for each direction).
template <bool RA>
__device__ __forceinline__ void pass1_interior2(const Chain<float>& c, Proj2& p, int fs, int bs,
                                                const double* __restrict__ U, float* __restrict__ ck,
                                                const F2 (&mu)[kSeg], F2 (&mun)[kSeg], float hfull) {
    constexpr int K = kSeg;
    constexpr int NC = CkCompact<RA>::NC;
    {
        // boundary (per direction, as proj_boundary's FP32 form): Y = P / Q, state := (Y, 1)
        const float q2x = fmaf(p.qr.v.x, p.qr.v.x, p.qi.v.x * p.qi.v.x);
        const float q2y = fmaf(p.qr.v.y, p.qr.v.y, p.qi.v.y * p.qi.v.y);
        const F2 rq = f2(rcp(q2x), rcp(q2y));
        // P = -mP: Y = P conj(Q) / |Q|^2
        const F2 tr = fma2(p.mpr, p.qr, mul2(p.mpi, p.qi));  // -(pr qr + pi qi)
        const F2 ti = fma2(p.mpi, p.qr, mul2(f2(-p.mpr.v.x, -p.mpr.v.y), p.qi));  // -(pi qr - pr qi)
        const F2 myr = mul2(tr, rq), myi = mul2(ti, rq);  // -Y
        if (RA) p.lam = mul2(p.lam, mul2(p.H, rq));
        p.H = f2b(hfull);
        float* pf = ck + (size_t)fs * NC * kWarp;
        pf[0] = -myr.v.x;
        pf[kWarp] = -myi.v.x;
        if (RA) pf[2 * kWarp] = p.lam.v.x;
        float* pb = ck + (size_t)bs * NC * kWarp;
        pb[0] = -myr.v.y;
        pb[kWarp] = -myi.v.y;
        if (RA) pb[2 * kWarp] = p.lam.v.y;
        p.mpr = myr;
        p.mpi = myi;
        p.qr = f2b(1.0f);
        p.qi = f2b(0.0f);
    }
    load_seg_pair(U, fs * K + K, (bs - 1) * K, mun);
    const F2 Er = f2b(c.Er), Ei = f2b(c.Ei), mEi = f2b(-c.Ei);
    const F2 mhb = f2b(-c.hb2), mhg = f2b(-c.hg2);
#pragma unroll
    for (int j = 0; j < K; ++j) {
        const F2 mh2 = (j & 1) ? mhg : mhb;
        const F2 ar = add2(Er, mu[j]);
        const F2 nqr = fma2(ar, p.qr, fma2(mEi, p.qi, p.mpr));
        const F2 nqi = fma2(ar, p.qi, fma2(Ei, p.qr, p.mpi));
        p.mpr = mul2(mh2, p.qr);
        p.mpi = mul2(mh2, p.qi);
        p.qr = nqr;
        p.qi = nqi;
    }
}

// Phase-B segment pair of an FP32 chain: the forward sweep's interior segment
// at nf (chain c, live state vf, backward record at its end) and the
// backward sweep's at nb read in reverse (chain cr with the contacts'
// roles swapped, live state vb, forward record at its start), as seg_fwd
// (with the next boundary) followed by seg_bwd for each, packed.  Returns
// the contributions of both (accb in reversed site order) and the live
// states at the next segments.
template <bool RA>
__device__ __forceinline__ void segment_pair2(const Chain<float>& c, const Chain<float>& cr,
                                              const CkVals<float>& vf, const CkVals<float>& vb,
                                              const F2 (&mu)[kSeg], AccOf<float> (&accf)[kSeg],
                                              AccOf<float> (&accr)[kSeg],
                                              Bnd<float>& nf, Bnd<float>& nb) {
    constexpr int K = kSeg;
    const F2 Er = f2b(c.Er), Ei = f2b(c.Ei), mEi = f2b(-c.Ei);
    const F2 hb = f2b(c.hb2), hg = f2b(c.hg2), mhb = f2b(-c.hb2), mhg = f2b(-c.hg2);
    F2 qr[K + 1], qi[K + 1], lm[K];
    // forward recompute of Q from (Y, 1) at the segment start
    F2 mpr = f2(-vf.yr, -vb.yr), mpi = f2(-vf.yi, -vb.yi);
    qr[0] = f2b(1.0f);
    qi[0] = f2b(0.0f);
    lm[0] = f2(vf.lam, vb.lam);
#pragma unroll
    for (int j = 0; j < K; ++j) {
        const F2 ar = add2(Er, mu[j]);
        qr[j + 1] = fma2(ar, qr[j], fma2(mEi, qi[j], mpr));
        qi[j + 1] = fma2(ar, qi[j], fma2(Ei, qr[j], mpi));
        if (j + 1 < K) {
            const F2 mh2 = (j & 1) ? mhg : mhb;
            mpr = mul2(mh2, qr[j]);
            mpi = mul2(mh2, qi[j]);
            if (RA) lm[j + 1] = mul2(lm[j], (j & 1) ? hg : hb);
        }
    }
    // next boundary per direction: Y = h^2 Q_{K-1} conj(Q_K) / |Q_K|^2 (the last hopping is gamma)
    {
        const float ax = fmaf(qr[K].v.x, qr[K].v.x, qi[K].v.x * qi[K].v.x);
        const float ay = fmaf(qr[K].v.y, qr[K].v.y, qi[K].v.y * qi[K].v.y);
        const F2 rq = f2(rcp(ax), rcp(ay));
        const F2 tr = fma2(qr[K - 1], qr[K], mul2(qi[K - 1], qi[K]));
        const F2 ti = fma2(qi[K - 1], qr[K], mul2(f2(-qr[K - 1].v.x, -qr[K - 1].v.y), qi[K]));
        const F2 g = mul2(hg, rq);
        const F2 yr = mul2(tr, g), yi = mul2(ti, g);
        nf.yr = yr.v.x;
        nf.yi = yi.v.x;
        nb.yr = yr.v.y;
        nb.yi = yi.v.y;
        if (RA) {
            const F2 l = mul2(lm[K - 1], g);
            nf.lam = l.v.x;
            nb.lam = l.v.y;
        } else {
            nf.lam = 1.0f;
            nb.lam = 1.0f;
        }
    }
    // D = S_e Q_{K} - R_e Q_{K-1} with S_e = 1, R_e = X_e, in FP64 once per segment and direction,
    // folded into the per-site coefficients
    F2 rh = f2(vf.rho, vb.rho), cg_r = f2b(0.0f), cg_i = f2b(0.0f), mcg_i = f2b(0.0f);
    {
        double dr[2], di[2];
        const float Rr[2] = {vf.xr, vb.xr}, Ri[2] = {vf.xi, vb.xi};
        const float q1r[2] = {qr[K].v.x, qr[K].v.y}, q1i[2] = {qi[K].v.x, qi[K].v.y};
        const float q0r[2] = {qr[K - 1].v.x, qr[K - 1].v.y}, q0i[2] = {qi[K - 1].v.x, qi[K - 1].v.y};
        float fa[2], fb[2], gr[2], gi[2];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const Chain<float>& ch = h ? cr : c;
            dr[h] = fma(-(double)Rr[h], (double)q0r[h], fma((double)Ri[h], (double)q0i[h], (double)q1r[h]));
            di[h] = fma(-(double)Rr[h], (double)q0i[h], fma(-(double)Ri[h], (double)q0r[h], (double)q1i[h]));
            const double inv = rcp(fma(dr[h], dr[h], di[h] * di[h]));
            if (RA) {
                fa[h] = (float)(ch.k0 * inv);
                fb[h] = (float)(ch.k1 * inv);
            } else {
                gr[h] = (float)(fma(ch.cr, dr[h], ch.ci * di[h]) * inv);
                gi[h] = (float)(fma(ch.ci, dr[h], -ch.cr * di[h]) * inv);
            }
        }
        if (RA) {
            const F2 f = f2(fa[0], fa[1]);
#pragma unroll
            for (int j = 0; j < K; ++j) lm[j] = mul2(lm[j], f);
            rh = mul2(rh, f2(fb[0], fb[1]));
        } else {
            cg_r = f2(gr[0], gr[1]);
            cg_i = f2(gi[0], gi[1]);
            mcg_i = f2(-gi[0], -gi[1]);
        }
    }
    // backward walk of (R, S) from (X_e, 1) with the site contributions
    F2 mRr = f2(-vf.xr, -vb.xr), mRi = f2(-vf.xi, -vb.xi), Sr = f2b(1.0f), Si = f2b(0.0f);
#pragma unroll
    for (int j = K - 1; j >= 0; --j) {
        F2 v;
        if (RA) {  // lm |S|^2 + rh |Q|^2 (1/|D|^2 folded in)
            const F2 s2 = fma2(Sr, Sr, mul2(Si, Si)), q2 = fma2(qr[j], qr[j], mul2(qi[j], qi[j]));
            v = fma2(lm[j], s2, mul2(rh, q2));
        } else {  // Im(c Q S / D) = qr (cg_r Si + cg_i Sr) + qi (cg_r Sr - cg_i Si)
            const F2 a = fma2(cg_r, Si, mul2(cg_i, Sr)), b = fma2(cg_r, Sr, mul2(mcg_i, Si));
            v = fma2(qr[j], a, mul2(qi[j], b));
        }
        accf[j] = c.valid ? v.v.x : 0.0f;
        accr[j] = c.valid ? v.v.y : 0.0f;
        if (j > 0) {
            const F2 ar = add2(Er, mu[j]);
            const F2 mh2 = ((j - 1) & 1) ? mhg : mhb;
            const F2 nsr = fma2(ar, Sr, fma2(mEi, Si, mRr));
            const F2 nsi = fma2(ar, Si, fma2(Ei, Sr, mRi));
            mRr = mul2(mh2, Sr);
            mRi = mul2(mh2, Si);
            Sr = nsr;
            Si = nsi;
            if (RA) rh = mul2(rh, ((j - 1) & 1) ? hg : hb);
        }
    }
}

// Fused schedule: one warp carries 32 whole chains.  With A = nseg / 2,
// phase A runs the forward sweep through segments [0, A) and the backward
// sweep through [nseg - A, nseg) together (as pass 1), each storing its own
// boundary record at those segments only.  The middle segment of an odd
// count is then integrated from both live states.  Phase B continues each
// sweep into the other half: the forward sweep forms the contributions of
// segment s from its live state at the segment start and the backward record
// at the segment end (the segment recompute of pass 2, whose forward part is
// now the sweep itself), the backward sweep does the mirror image on the
// segment read in reverse.  Every site is crossed twice instead of three
// times, each record is written once and read once, and no second kernel
// runs.  The contact segments take the per-site (edge) form.
template <typename R, bool RA>
__device__ __forceinline__ void fused_chain(const TubeDev* __restrict__ tubes, const ChainRec& cr, int tube,
                                            R* __restrict__ ck_warp, double* __restrict__ prow, int lane) {
    constexpr int K = kSeg;
    constexpr int NC = CkCompact<RA>::NC;
    const TubeDev& T = tubes[tube];
    const int N = T.N;
    const int nseg = (N + K - 1) / K;
    const double* __restrict__ U = T.U;
    const bool valid = cr.mode >= 0;
    const double beta = T.beta[valid ? cr.mode : 0];
    const cd E = {cr.Er, cr.Ei};
    // U_contact = U at the end sites (Nanostructure.cpp:500-504) when read on the device
    const double Uc0 = T.uc_from_U ? U[0] : T.Uc0, Uc1 = T.uc_from_U ? U[N - 1] : T.Uc1;
    const cd S0 = sigma_contact(E, Uc0, beta, T);
    const cd S1 = sigma_contact(E, Uc1, beta, T);
    const Chain<R> c = make_chain<R, RA>(T, cr, S0.x, S0.y, S1.x, S1.y);
    Chain<R> crev = c;  // the chain read from the drain end: the two contacts' roles swap
    crev.k0 = c.k1;
    crev.k1 = c.k0;
    R* __restrict__ ck = ck_warp + lane;
    auto rec = [&](int seg) -> Bnd<R> {
        const R* p = ck + (size_t)seg * NC * kWarp;
        return {p[0], p[kWarp], RA ? p[2 * kWarp] : (R)1};
    };
    const int A = nseg / 2;
    Proj<R> f{0, 0, 1, 0, 1, 1, 1};  // Y_0 = 0, lambda_0 = 1
    Proj<R> b{0, 0, 1, 0, 1, 1, 1};  // X_{N-1} = 0, rho_{N-1} = 1
    // ---- phase A
    if (A > 0) {
        R hfull = 1;  // prod of h^2 over a full segment
#pragma unroll
        for (int j = 0; j < K / 2; ++j) hfull *= c.hb2 * c.hg2;
        R ua_f[K], ua_b[K], ub_f[K], ub_b[K];
#pragma unroll
        for (int j = 0; j < K; ++j) {
            ua_f[j] = (R)__ldg(U + j);
            ua_b[j] = (R)__ldg(U + N - 1 - j);  // kPadLo zeros before site 0 cover N < K
        }
        pass1_block<R, RA, false, true>(c, f, b, 0, nseg - 1, A > 1, U, ck, ua_f, ua_b, ub_f, ub_b, hfull);
        if constexpr (std::is_same<R, float>::value) {
            // interior blocks with both sweeps packed (FFMA2)
            if (A > 1) {
                Proj2 p2;
                p2.mpr = f2(-f.pr, -b.pr);
                p2.mpi = f2(-f.pi, -b.pi);
                p2.qr = f2(f.qr, b.qr);
                p2.qi = f2(f.qi, b.qi);
                p2.lam = f2(f.lam, b.lam);
                p2.H = f2(f.H, b.H);
                F2 m0[K], m1[K];
#pragma unroll
                for (int j = 0; j < K; ++j) m0[j] = f2(-ub_f[j], -ub_b[j]);
                int k = 1;
                for (; k + 2 <= A; k += 2) {
                    pass1_interior2<RA>(c, p2, k, nseg - 1 - k, U, ck, m0, m1, hfull);
                    pass1_interior2<RA>(c, p2, k + 1, nseg - 2 - k, U, ck, m1, m0, hfull);
                }
                if (k < A) pass1_interior2<RA>(c, p2, k, nseg - 1 - k, U, ck, m0, m1, hfull);
                f.pr = -p2.mpr.v.x;
                f.pi = -p2.mpi.v.x;
                f.qr = p2.qr.v.x;
                f.qi = p2.qi.v.x;
                f.lam = p2.lam.v.x;
                f.H = p2.H.v.x;
                b.pr = -p2.mpr.v.y;
                b.pi = -p2.mpi.v.y;
                b.qr = p2.qr.v.y;
                b.qi = p2.qi.v.y;
                b.lam = p2.lam.v.y;
                b.H = p2.H.v.y;
            }
        } else {
            int k = 1;
            for (; k + 2 <= A; k += 2) {
                pass1_block<R, RA, true, true>(c, f, b, k, nseg - 1 - k, true, U, ck, ub_f, ub_b, ua_f, ua_b, hfull);
                pass1_block<R, RA, true, true>(c, f, b, k + 1, nseg - 2 - k, true, U, ck, ua_f, ua_b, ub_f, ub_b,
                                               hfull);
            }
            if (k < A)
                pass1_block<R, RA, true, true>(c, f, b, k, nseg - 1 - k, true, U, ck, ub_f, ub_b, ua_f, ua_b, hfull);
        }
    }
    Bnd<R> fw, bw;  // forward state at the start of segment nseg - A - (nseg odd), backward at the end of segment A - 1 + (nseg odd)
    proj_boundary<R, RA>(f, fw.yr, fw.yi);
    fw.lam = f.lam;
    proj_boundary<R, RA>(b, bw.yr, bw.yi);
    bw.lam = b.lam;
    // ---- middle segment of an odd count, from both live states
    if (nseg & 1) {
        const int n0 = A * K;
        const CkVals<R> v{fw.yr, fw.yi, fw.lam, bw.yr, bw.yi, bw.lam};
        AccOf<R> acc[K];
        R u[K];
        if (nseg == 1) {
            load_seg_edge(U, 0, N, u);
            segment_proj<R, RA, true>(c, 0, v, u, acc);
            write_segment(acc, 0, N, prow, lane);
            return;
        }
        load_seg(U, n0, u);
        Bnd<R> nf;
        segment_proj<R, RA, false, true>(c, n0, v, u, acc, &nf);
        write_segment(acc, n0, N, prow, lane);
        R ur[K];
        load_seg_reversed(U, n0, ur);
        bw = sweep_segment<R, RA>(c, bw, ur);  // X and rho at the end of segment A - 1
        fw = nf;                               // Y and lambda at the start of segment A + 1
    }
    // ---- phase B: forward through [nseg - A, nseg), backward through [0, A) downwards.
    // The records of iteration k + 1 are loaded into registers during
    // iteration k and those of k + 2 brought into L1 (they were written long
    // before and sit in DRAM); interior iterations issue the forward parts of
    // both directions' segments before their backward parts, two independent
    // dependency chains.
    auto prefetch_rec = [&](int k) {
        if (k < A) {
            const R* pf = ck + (size_t)(nseg - A + k) * NC * kWarp;
            const R* pb = ck + (size_t)(A - 1 - k) * NC * kWarp;
#pragma unroll
            for (int q = 0; q < NC; ++q) {
                prefetch_l1(pf + q * kWarp);
                prefetch_l1(pb + q * kWarp);
            }
        }
    };
    Bnd<R> xn = {0, 0, 1}, yn = {0, 0, 1};
    if (A > 0) {
        xn = rec(nseg - A);
        yn = rec(A - 1);
    }
    prefetch_rec(1);
    for (int k = 0; k < A; ++k) {
        const int sf = nseg - A + k, sb = A - 1 - k;
        const int nf = sf * K, nb = sb * K;
        const bool last = k == A - 1;  // the contact segments nseg - 1 and 0
        const Bnd<R> x = xn, y = yn;
        if (!last) {
            xn = rec(sf + 1);
            yn = rec(sb - 1);
        }
        prefetch_rec(k + 2);
        AccOf<R> accf[K], accb[K];
        if (!last) {
            const CkVals<R> vf{fw.yr, fw.yi, fw.lam, x.yr, x.yi, x.lam};
            const CkVals<R> vb{bw.yr, bw.yi, bw.lam, y.yr, y.yi, y.lam};
            AccOf<R> accr[K];
            if constexpr (std::is_same<R, float>::value) {
                F2 mu[K];
                load_seg_pair(U, nf, nb, mu);
                segment_pair2<RA>(c, crev, vf, vb, mu, accf, accr, fw, bw);
            } else {
                R uf[K], ub[K];
                load_seg(U, nf, uf);
                load_seg_reversed(U, nb, ub);
                SegWork<R> wf, wb;
                seg_fwd<R, RA, false, true>(c, nf, vf, uf, wf, &fw);
                seg_fwd<R, RA, false, true>(crev, nb, vb, ub, wb, &bw);
                seg_bwd<R, RA, false>(c, nf, uf, wf, accf);
                seg_bwd<R, RA, false>(crev, nb, ub, wb, accr);
            }
#pragma unroll
            for (int j = 0; j < K; ++j) accb[j] = accr[K - 1 - j];
        } else {
            R uf[K], ub[K];
            load_seg_edge(U, nf, N, uf);
            load_seg_edge(U, nb, N, ub);
            const CkVals<R> vf{fw.yr, fw.yi, fw.lam, x.yr, x.yi, x.lam};
            const CkVals<R> vb{y.yr, y.yi, y.lam, bw.yr, bw.yi, bw.lam};
            segment_proj<R, RA, true>(c, nf, vf, uf, accf);
            segment_proj<R, RA, true>(c, nb, vb, ub, accb);
        }
        write_segment(accf, nf, N, prow, lane);
        write_segment(accb, nb, N, prow, lane);
    }
}

// Segments [s0, s1) of piece p of P on a tube of nseg segments.
__device__ __forceinline__ void piece_range(int nseg, int P, int p, int& s0, int& s1) {
    s0 = (int)((long long)p * nseg / P);
    s1 = (int)((long long)(p + 1) * nseg / P);
}

// One warp (32 chains, one piece of them) per block: the latency-bound
// sweeps spread evenly over the SMs.  pieces > 1: block u = warp * pieces +
// piece, initial states from states[warp][piece][component][lane].
__global__ void __launch_bounds__(32) rgf_pass1_kernel(const TubeDev* __restrict__ tubes,
                                                       const ChainRec* __restrict__ chains,
                                                       const WarpRec* __restrict__ warps, int num_warps,
                                                       double* __restrict__ scratch, const int* __restrict__ skip,
                                                       int pieces, const double* __restrict__ states) {
    if (skip && *skip) return;
    const int lane = threadIdx.x & 31;
    const int w = blockIdx.x / pieces, p = blockIdx.x % pieces;
    if (w >= num_warps) return;
    const WarpRec wr = warps[w];
    const ChainRec c = chains[(size_t)w * kWarp + lane];
    double* ws = scratch + wr.ck_off;
    const int nseg = (tubes[wr.tube].N + kSeg - 1) / kSeg;
    int s0 = 0, s1 = nseg;
    PieceState st{0.0, 0.0, 1.0, 0.0, 0.0, 1.0};
    if (pieces > 1) {
        piece_range(nseg, pieces, p, s0, s1);
        const double* q = states + ((size_t)w * pieces + p) * 6 * kWarp + lane;
        st = PieceState{q[0], q[kWarp], q[2 * kWarp], q[3 * kWarp], q[4 * kWarp], q[5 * kWarp]};
    }
    if (wr.fp32) {
        if (wr.kind == kRealAxis)
            pass1_chain<float, true>(tubes, c, wr.tube, ws, lane, s0, s1, st);
        else
            pass1_chain<float, false>(tubes, c, wr.tube, ws, lane, s0, s1, st);
    } else {
        if (wr.kind == kRealAxis)
            pass1_chain<double, true>(tubes, c, wr.tube, ws, lane, s0, s1, st);
        else
            pass1_chain<double, false>(tubes, c, wr.tube, ws, lane, s0, s1, st);
    }
}

// 2 x 2 complex matrix, row-major: (a b; c d)
struct M2 {
    cd a, b, c, d;
};
__device__ __forceinline__ cd cmulz(cd x, cd y) { return {fma(x.x, y.x, -x.y * y.y), fma(x.x, y.y, x.y * y.x)}; }
// (0 h2; -1 al) * M
__device__ __forceinline__ M2 step_left(double h2, cd al, const M2& m) {
    M2 r;
    r.a = {h2 * m.c.x, h2 * m.c.y};
    r.b = {h2 * m.d.x, h2 * m.d.y};
    const cd ac = cmulz(al, m.c), ad = cmulz(al, m.d);
    r.c = {ac.x - m.a.x, ac.y - m.a.y};
    r.d = {ad.x - m.b.x, ad.y - m.b.y};
    return r;
}
// Scale m by a power of two so that its largest |re| + |im| lies in [1, 2);
// the exponent goes to e (exact: no rounding from the rescaling).
__device__ __forceinline__ void normalise(M2& m, int& e) {
    const double s = fmax(fmax(fabs(m.a.x) + fabs(m.a.y), fabs(m.b.x) + fabs(m.b.y)),
                          fmax(fabs(m.c.x) + fabs(m.c.y), fabs(m.d.x) + fabs(m.d.y)));
    const int be = (int)((__double_as_longlong(s) >> 52) & 0x7ff);  // biased exponent of s
    if (be == 0 || be == 0x7ff) return;                              // zero, subnormal, inf or NaN: leave as is
    const double f = __longlong_as_double((long long)(2046 - be) << 52);  // 2^-(be - 1023)
    m.a = {m.a.x * f, m.a.y * f};
    m.b = {m.b.x * f, m.b.y * f};
    m.c = {m.c.x * f, m.c.y * f};
    m.d = {m.d.x * f, m.d.y * f};
    e += be - 1023;
}

// Transfer matrices of one piece of a chain (FP64): forward
// (P, Q)_{piece end} = Mf (P, Q)_{piece start} with (P, Q) <- (h_n^2 Q,
// alpha_n Q - P) for every forward step of the piece, and backward
// (R, S)_{before the piece} = Mb (R, S)_{piece end} with (R, S) <-
// (h_{m-1}^2 S, alpha_m S - R).  Block k advances the forward product
// through segment s0+k and the backward one through segment s1-1-k (the two
// are independent and interleave), with the next block's potentials loaded
// ahead; both are rescaled by powers of two every segment.
// out[warp][piece][18][lane]: Mf (8), log2 scale of Mf, Mb (8), log2 scale of Mb.
__global__ void __launch_bounds__(32) rgf_piece_transfer_kernel(const TubeDev* __restrict__ tubes,
                                                                const ChainRec* __restrict__ chains,
                                                                const WarpRec* __restrict__ warps, int num_warps,
                                                                int pieces, double* __restrict__ out,
                                                                const int* __restrict__ skip) {
    if (skip && *skip) return;
    constexpr int K = kSeg;
    const int lane = threadIdx.x & 31;
    const int w = blockIdx.x / pieces, p = blockIdx.x % pieces;
    if (w >= num_warps) return;
    const WarpRec wr = warps[w];
    const ChainRec cr = chains[(size_t)w * kWarp + lane];
    const TubeDev& T = tubes[wr.tube];
    const int N = T.N, nseg = (N + K - 1) / K;
    int s0, s1;
    piece_range(nseg, pieces, p, s0, s1);
    const int nb = s1 - s0;
    const bool valid = cr.mode >= 0;
    const double beta = T.beta[valid ? cr.mode : 0];
    const double hb2 = beta * beta, hg2 = T.gamma * T.gamma;
    const cd E = {cr.Er, cr.Ei};
    const double* __restrict__ U = T.U;
    cd S0 = {0.0, 0.0}, S1 = {0.0, 0.0};
    if (nb > 0 && (s0 == 0 || s1 == nseg)) {
        const double Uc0 = T.uc_from_U ? U[0] : T.Uc0, Uc1 = T.uc_from_U ? U[N - 1] : T.Uc1;
        S0 = sigma_contact(E, Uc0, beta, T);
        S1 = sigma_contact(E, Uc1, beta, T);
    }
    M2 mf{{1.0, 0.0}, {0.0, 0.0}, {0.0, 0.0}, {1.0, 0.0}}, mb = mf;
    int ef = 0, eb = 0;
    double uf[K], ub[K];
    if (nb > 0) {
        const int e = min(s1 * K, N) - 1;  // the piece's last site
#pragma unroll
        for (int j = 0; j < K; ++j) {
            uf[j] = __ldg(U + s0 * K + j);
            ub[j] = __ldg(U + e - j);
        }
    }
    for (int k = 0; k < nb; ++k) {
        const int f0 = (s0 + k) * K;
        const int b0 = (s1 - 1 - k) * K;           // backward segment start
        const int be = min(b0 + K, N) - 1;         // backward segment end
        double nf[K], nbk[K];
        if (k + 1 < nb) {
            // next forward segment and next backward segment (full): 16-byte
            // aligned, inside the padded buffer
            const double2* pf = reinterpret_cast<const double2*>(U + f0 + K);
            const double2* pb = reinterpret_cast<const double2*>(U + b0 - K);
#pragma unroll
            for (int q = 0; q < K / 2; ++q) {
                const double2 vf = __ldg(pf + q), vb = __ldg(pb + q);
                nf[2 * q] = vf.x;
                nf[2 * q + 1] = vf.y;
                nbk[K - 1 - 2 * q] = vb.x;
                nbk[K - 2 - 2 * q] = vb.y;
            }
        }
#pragma unroll
        for (int j = 0; j < K; ++j) {
            const int n = f0 + j;
            if (n < N - 1) {  // forward step at site n
                cd al = {E.x - uf[j], E.y};
                if (n == 0) al = {al.x - S0.x, al.y - S0.y};
                mf = step_left((j & 1) ? hg2 : hb2, al, mf);
            }
            const int m = be - j;
            if (m >= b0 && m >= 1) {  // backward step at site m: M <- S_m M
                cd al = {E.x - ub[j], E.y};
                if (m == N - 1) al = {al.x - S1.x, al.y - S1.y};
                mb = step_left(((m - 1) & 1) ? hg2 : hb2, al, mb);
            }
        }
        normalise(mf, ef);
        normalise(mb, eb);
        if (k + 1 < nb) {
#pragma unroll
            for (int j = 0; j < K; ++j) {
                uf[j] = nf[j];
                ub[j] = nbk[j];
            }
        }
    }
    double* o = out + ((size_t)w * pieces + p) * 18 * kWarp + lane;
    const double v[18] = {mf.a.x, mf.a.y, mf.b.x, mf.b.y, mf.c.x, mf.c.y, mf.d.x, mf.d.y, (double)ef,
                          mb.a.x, mb.a.y, mb.b.x, mb.b.y, mb.c.x, mb.c.y, mb.d.x, mb.d.y, (double)eb};
#pragma unroll
    for (int q = 0; q < 18; ++q) o[q * kWarp] = v[q];
}

// One transfer matrix applied to the state (Z, 1): the new ratio Z' = top /
// bottom and log |bottom| (natural log) including the matrix's scale 2^e.
__device__ __forceinline__ void apply_transfer(const double (&t)[9], cd& Z, double& L) {
    const cd a = {t[0], t[1]}, b = {t[2], t[3]}, c = {t[4], t[5]}, d = {t[6], t[7]};
    const cd az = cmulz(a, Z), cz = cmulz(c, Z);
    const cd top = {az.x + b.x, az.y + b.y}, bot = {cz.x + d.x, cz.y + d.y};
    const double q2 = bot.x * bot.x + bot.y * bot.y;
    L += t[8] * 0.69314718055994530942 + 0.5 * log(q2);
    const double iq = 1.0 / q2;
    Z = {(top.x * bot.x + top.y * bot.y) * iq, (top.y * bot.x - top.x * bot.y) * iq};
}

// Per chain: the forward state (Y, lambda) at each piece's first site and the
// backward state (X, rho) at each piece's last site, from the transfer
// matrices; lambda_n = prod_{m<n} h_m^2 / |Q_n|^2 with Q_0 = 1, rho_n =
// prod_{n<=m<N-1} h_m^2 / |S_n|^2 with S_{N-1} = 1, in logarithms.  The
// forward scan (ascending pieces) and the backward one (descending)
// interleave, the next matrices loaded ahead.
__global__ void __launch_bounds__(32) rgf_piece_prefix_kernel(const TubeDev* __restrict__ tubes,
                                                              const ChainRec* __restrict__ chains,
                                                              const WarpRec* __restrict__ warps, int num_warps,
                                                              int pieces, const double* __restrict__ tm,
                                                              double* __restrict__ states,
                                                              const int* __restrict__ skip) {
    if (skip && *skip) return;
    const int lane = threadIdx.x & 31;
    const int w = blockIdx.x;
    if (w >= num_warps) return;
    const WarpRec wr = warps[w];
    const ChainRec cr = chains[(size_t)w * kWarp + lane];
    const TubeDev& T = tubes[wr.tube];
    const int N = T.N, nseg = (N + kSeg - 1) / kSeg;
    const bool valid = cr.mode >= 0;
    const double beta = T.beta[valid ? cr.mode : 0];
    const double lhb = log(fmax(beta * beta, 1e-300)), lhg = log(T.gamma * T.gamma);
    // sum_{m < n} log h_m^2: sites of even index carry beta
    auto hsum = [&](int n) { return ((n + 1) / 2) * lhb + (n / 2) * lhg; };
    auto clampexp = [](double x) { return exp(fmin(fmax(x, -700.0), 700.0)); };
    const double hall = hsum(N - 1);
    const double* base = tm + (size_t)w * pieces * 18 * kWarp + lane;
    auto load = [&](int p, int half, double (&t)[9]) {
        const double* q = base + ((size_t)p * 18 + half * 9) * kWarp;
#pragma unroll
        for (int i = 0; i < 9; ++i) t[i] = q[i * kWarp];
    };
    cd Y = {0.0, 0.0}, X = {0.0, 0.0};
    double Lf = 0.0, Lb = 0.0;
    double tf[9], tb[9];
    load(0, 0, tf);
    load(pieces - 1, 1, tb);
    for (int i = 0; i < pieces; ++i) {
        const int pf = i, pb = pieces - 1 - i;
        double nf[9], nb[9];
        if (i + 1 < pieces) {
            load(pf + 1, 0, nf);
            load(pb - 1, 1, nb);
        }
        int s0, s1;
        piece_range(nseg, pieces, pf, s0, s1);
        double* st = states + ((size_t)w * pieces + pf) * 6 * kWarp + lane;
        st[0] = Y.x;
        st[kWarp] = Y.y;
        st[2 * kWarp] = valid ? clampexp(hsum(s0 * kSeg) - 2.0 * Lf) : 1.0;
        apply_transfer(tf, Y, Lf);
        piece_range(nseg, pieces, pb, s0, s1);
        const int e = min(s1 * kSeg, N) - 1;
        st = states + ((size_t)w * pieces + pb) * 6 * kWarp + lane;
        st[3 * kWarp] = X.x;
        st[4 * kWarp] = X.y;
        st[5 * kWarp] = valid ? clampexp(hall - hsum(e) - 2.0 * Lb) : 1.0;
        apply_transfer(tb, X, Lb);
        if (i + 1 < pieces) {
#pragma unroll
            for (int q = 0; q < 9; ++q) {
                tf[q] = nf[q];
                tb[q] = nb[q];
            }
        }
    }
}

// Fused schedule: one warp (32 whole chains) per block; records in the
// warp's scratch, per-site sums into the warp's partial row.  One
// instantiation per precision; block b takes warp order[b].  The FP32
// instantiation (both sweeps packed) is held to NEGF_FP32_MIN_BLOCKS
// resident warps per SM (12: about 160 registers, no spills) to hide the
// latency of its dependent recurrences; FP64 needs about 240 registers and
// spills below that.
#ifndef NEGF_FP32_MIN_BLOCKS
#define NEGF_FP32_MIN_BLOCKS 12
#endif
#ifndef NEGF_FP64_MIN_BLOCKS
#define NEGF_FP64_MIN_BLOCKS 1
#endif
template <typename R>
__global__ void __launch_bounds__(32, (sizeof(R) == 4 ? NEGF_FP32_MIN_BLOCKS : NEGF_FP64_MIN_BLOCKS)) rgf_fused_kernel(const TubeDev* __restrict__ tubes,
                                                       const ChainRec* __restrict__ chains,
                                                       const WarpRec* __restrict__ warps, const int* __restrict__ order,
                                                       int count, double* __restrict__ partial,
                                                       double* __restrict__ scratch, const int* __restrict__ skip) {
    if (skip && *skip) return;
    const int lane = threadIdx.x & 31;
    if ((int)blockIdx.x >= count) return;
    const int w = order[blockIdx.x];
    const WarpRec wr = warps[w];
    const ChainRec c = chains[(size_t)w * kWarp + lane];
    double* ws = scratch + wr.ck_off;
    double* prow = partial + wr.row_off;
    if (wr.kind == kRealAxis)
        fused_chain<R, true>(tubes, c, wr.tube, reinterpret_cast<R*>(ws), prow, lane);
    else
        fused_chain<R, false>(tubes, c, wr.tube, reinterpret_cast<R*>(ws), prow, lane);
}

__global__ void __launch_bounds__(128) rgf_pass2_kernel(const TubeDev* __restrict__ tubes,
                                                        const ChainRec* __restrict__ chains,
                                                        const WarpRec* __restrict__ warps,
                                                        const SegUnit* __restrict__ units, int num_units,
                                                        double* __restrict__ partial,
                                                        const double* __restrict__ scratch,
                                                        const int* __restrict__ skip) {
    if (skip && *skip) return;
    const int lane = threadIdx.x & 31;
    const int ui = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (ui >= num_units) return;
    const SegUnit su = units[ui];
    const WarpRec wr = warps[su.warp];
    const ChainRec c = chains[(size_t)su.warp * kWarp + lane];
    const double* ws = scratch + wr.ck_off;
    double* prow = partial + wr.row_off;
    if (wr.fp32) {
        if (wr.kind == kRealAxis)
            pass2_unit<float, true>(tubes, c, wr, su, ws, prow, lane);
        else
            pass2_unit<float, false>(tubes, c, wr, su, ws, prow, lane);
    } else {
        if (wr.kind == kRealAxis)
            pass2_unit<double, true>(tubes, c, wr, su, ws, prow, lane);
        else
            pass2_unit<double, false>(tubes, c, wr, su, ws, prow, lane);
    }
}

__global__ void selftest_kernel(int which, int n, const double* __restrict__ in, double* __restrict__ out) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        out[i] = which == 0 ? rcp(in[i]) : (double)rcp((float)in[i]);
}

// Q[q_off + n] = sum_w partial[row_base + w N + n] - rho0[n].
// Block = 32 sites x kRowGroups row groups; each thread sums rows
// g, g + kRowGroups, ... with Kahan compensation, then the row groups are
// combined in a fixed order (deterministic).  32 row groups: a 4000-site tube
// gives 125 blocks of 32 warps, enough loads in flight to stream the rows
// at HBM rate.
constexpr int kRowGroups = 32;
__global__ void __launch_bounds__(32 * kRowGroups) reduce_kernel(const ReduceTube* __restrict__ rts,
                                                                 const double* __restrict__ partial,
                                                                 double* __restrict__ Q, const int* __restrict__ skip) {
    if (skip && *skip) return;  // uniform over the block
    __shared__ double sh_s[kRowGroups][32], sh_c[kRowGroups][32];
    const ReduceTube r = rts[blockIdx.y];
    const int n = blockIdx.x * 32 + threadIdx.x;
    const int g = threadIdx.y;
    double s = 0.0, comp = 0.0;
    if (n < r.N) {
        const double* p = partial + r.row_base + n;
        int w = g;
        for (; w + 3 * kRowGroups < r.num_rows; w += 4 * kRowGroups) {
            double v[4];
#pragma unroll
            for (int k = 0; k < 4; ++k) v[k] = p[(size_t)(w + k * kRowGroups) * r.N];
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const double y = v[k] - comp;
                const double t = s + y;
                comp = (t - s) - y;
                s = t;
            }
        }
        for (; w < r.num_rows; w += kRowGroups) {
            const double y = p[(size_t)w * r.N] - comp;
            const double t = s + y;
            comp = (t - s) - y;
            s = t;
        }
    }
    sh_s[g][threadIdx.x] = s;
    sh_c[g][threadIdx.x] = comp;
    __syncthreads();
    if (g == 0 && n < r.N) {
        double tot = 0.0, cc = 0.0;
        for (int k = 0; k < kRowGroups; ++k) {
            const double y = (sh_s[k][threadIdx.x] - sh_c[k][threadIdx.x]) - cc;
            const double t = tot + y;
            cc = (t - tot) - y;
            tot = t;
        }
        if (r.rho0) tot -= r.rho0[n];
        Q[r.q_off + n] = tot;
    }
}


// ====================================================== transport characteristics
// Spectral terms of one segment (FP64, per-site D as in edge segments):
// a_n = deg Gamma_0 |G_n0|^2 and b_n = deg Gamma_1 |G_n,N-1|^2 for chains
// whose real-axis coefficients are b0 = b1 = 1, so that deg A_nn = a_n + b_n
// (A = sum_k G Gamma_k G^dagger, NEGF_Common.cpp:2654-2726).
__device__ __forceinline__ void segment_spectral(const Chain<double>& c, int n0, const CkVals<double>& ckv,
                                                 const double (&u)[kSeg], double (&a)[kSeg], double (&b)[kSeg]) {
    constexpr int K = kSeg;
    const int N = c.N;
    double pr[K], pi[K], qr[K + 1], qi[K + 1], lm[K];
    pr[0] = ckv.yr;
    pi[0] = ckv.yi;
    qr[0] = 1.0;
    qi[0] = 0.0;
    lm[0] = ckv.lam;
    double Rr = ckv.xr, Ri = ckv.xi, Sr = 1.0, Si = 0.0;
    double rh = ckv.rho;
#pragma unroll
    for (int j = 0; j < K; ++j) {
        const int n = n0 + j;
        if (n >= N) break;
        double ar = c.Er - u[j], ai = c.Ei;
        if (n == 0) {
            ar -= c.s0r;
            ai -= c.s0i;
        }
        if (n == N - 1) {
            ar -= c.s1r;
            ai -= c.s1i;
        }
        qr[j + 1] = fma(ar, qr[j], fma(-ai, qi[j], -pr[j]));
        qi[j + 1] = fma(ar, qi[j], fma(ai, qr[j], -pi[j]));
        if (j + 1 < K) {
            const double h2 = (n & 1) ? c.hg2 : c.hb2;
            pr[j + 1] = h2 * qr[j];
            pi[j + 1] = h2 * qi[j];
            lm[j + 1] = lm[j] * h2;
        }
    }
#pragma unroll
    for (int j = K - 1; j >= 0; --j) {
        const int n = n0 + j;
        a[j] = 0.0;
        b[j] = 0.0;
        if (n >= N) continue;
        const double dr = fma(Sr, qr[j + 1], fma(-Si, qi[j + 1], fma(-Rr, qr[j], Ri * qi[j])));
        const double di = fma(Sr, qi[j + 1], fma(Si, qr[j + 1], fma(-Rr, qi[j], -Ri * qr[j])));
        const double inv = rcp(fma(dr, dr, di * di));
        const double s2 = fma(Sr, Sr, Si * Si), q2 = fma(qr[j], qr[j], qi[j] * qi[j]);
        a[j] = c.valid ? inv * (lm[j] * s2) * c.k0 : 0.0;
        b[j] = c.valid ? inv * (rh * q2) * c.k1 : 0.0;
        if (j > 0) {
            double ar = c.Er - u[j], ai = c.Ei;
            if (n == N - 1) {
                ar -= c.s1r;
                ai -= c.s1i;
            }
            const double h2 = ((n - 1) & 1) ? c.hg2 : c.hb2;
            const double nrr = h2 * Sr, nri = h2 * Si;
            const double nsr = fma(ar, Sr, fma(-ai, Si, -Rr));
            const double nsi = fma(ar, Si, fma(ai, Sr, -Ri));
            Rr = nrr;
            Ri = nri;
            Sr = nsr;
            Si = nsi;
            rh *= h2;
        }
    }
}

// One unit (32 segments of one warp's chains) after pass 1 of real-axis FP64
// chains with b0 = b1 = 1 and (cr, ci) = (Re f_0(E), Re f_1(E)).  Per lane:
// the sum of deg A_nn over the unit's sites -> part[unit][lane]; per chain
// (chain_out[chain][7]): deg Gamma_0 Gamma_1 |G_0,N-1|^2 from the source end,
// the same from the drain end, deg Re(Gn_nn) = a f_0 + b f_1 at n = N/2,
// else 0, else N-1 (the current's probes, NEGF_Common.cpp:4684-4714), and at
// n = N/4, else 3N/4 after N/2 (the charge integrand's probes, :3467-3496);
// optionally deg A_nn per site into site_out[n * site_stride + chain].
__global__ void __launch_bounds__(32) rgf_transport_kernel(const TubeDev* __restrict__ tubes,
                                                           const ChainRec* __restrict__ chains,
                                                           const WarpRec* __restrict__ warps,
                                                           const SegUnit* __restrict__ units, int num_units,
                                                           const double* __restrict__ scratch, double* __restrict__ part,
                                                           double* __restrict__ chain_out,
                                                           double* __restrict__ site_out, long long site_stride) {
    constexpr int K = kSeg;
    using CL = CkLayout<true>;
    const int lane = threadIdx.x & 31;
    if ((int)blockIdx.x >= num_units) return;
    const SegUnit su = units[blockIdx.x];
    const WarpRec wr = warps[su.warp];
    const long long ci = (long long)su.warp * kWarp + lane;
    const ChainRec cr = chains[ci];
    const TubeDev& T = tubes[wr.tube];
    const int N = T.N;
    const double* __restrict__ U = T.U;
    const double* __restrict__ ws = scratch + wr.ck_off;
    const double s0r = ws[0 * kWarp + lane], s0i = ws[1 * kWarp + lane];
    const double s1r = ws[2 * kWarp + lane], s1i = ws[3 * kWarp + lane];
    const Chain<double> c = make_chain<double, true>(T, cr, s0r, s0i, s1r, s1i);
    const double* __restrict__ ck = ws + 4 * kWarp + lane;
    const double f0 = cr.cr, f1 = cr.ci;
    double* out = chain_out + ci * 7;
    double sum = 0.0;
    for (int s = su.seg0; s < su.seg1; ++s) {
        const int n0 = s * K;
        const CkVals<double> ckv = load_ck<double, true>(ck + (size_t)s * CL::NC * kWarp);
        double u[K], a[K], b[K];
#pragma unroll
        for (int k = 0; k < K; ++k) u[k] = (n0 + k < N) ? __ldg(U + n0 + k) : 0.0;
        segment_spectral(c, n0, ckv, u, a, b);
#pragma unroll
        for (int j = 0; j < K; ++j) {
            const int n = n0 + j;
            if (n >= N) break;
            sum += a[j] + b[j];
            if (site_out) site_out[(long long)n * site_stride + ci] = a[j] + b[j];
            if (n == 0) out[0] = (-2.0 * s0i) * b[j];
            if (n == N - 1) out[1] = (-2.0 * s1i) * a[j];
            const double v = fma(a[j], f0, b[j] * f1);
            if (n == N / 2)
                out[2] = v;
            else if (n == 0)
                out[3] = v;
            else if (n == N - 1)
                out[4] = v;
            if (n != N / 2) {
                if (n == N / 4)
                    out[5] = v;
                else if (n == (N * 3) / 4)
                    out[6] = v;
            }
        }
    }
    part[(long long)blockIdx.x * kWarp + lane] = sum;
}

// Per energy e (chains e*M .. e*M+M-1, units w*upw .. w*upw+upw-1 of warp
// w): out[e][8] = (sum deg A_nn over sites, T from the source end, T from the
// drain end, probes at N/2, 0, N-1, N/4, 3N/4), summed over modes in order.
__global__ void transport_reduce_kernel(const double* __restrict__ part, const double* __restrict__ chain_out,
                                        int num_e, int M, int upw, double* __restrict__ out) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= num_e) return;
    double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (int m = 0; m < M; ++m) {
        const long long c = (long long)e * M + m;
        const long long w = c / kWarp, lane = c % kWarp;
        for (int j = 0; j < upw; ++j) acc[0] += part[(w * upw + j) * kWarp + lane];
        for (int k = 0; k < 7; ++k) acc[k + 1] += chain_out[c * 7 + k];
    }
    for (int k = 0; k < 8; ++k) out[(long long)e * 8 + k] = acc[k];
}

// LDOS_n(E_e) = sum_m deg A_nn / 2 pi -> out[e][n].
__global__ void ldos_reduce_kernel(const double* __restrict__ site, long long stride, int num_e, int M, int N,
                                   double* __restrict__ out) {
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (long long)num_e * N) return;
    const int e = (int)(idx / N), n = (int)(idx % N);
    double v = 0.0;
    for (int m = 0; m < M; ++m) v += site[(long long)n * stride + (long long)e * M + m];
    out[idx] = v / (2.0 * 3.14159265358979323846);
}
}  // namespace

long long rgf_scratch_doubles(int N, int kind, int fp32) {
    const long long nseg = (N + kSeg - 1) / kSeg;
    const long long nc = (kind == kRealAxis) ? 6 : 4;
    const long long bytes = nseg * nc * kWarp * (fp32 ? 4 : 8);
    return 4 * kWarp + (bytes + 15) / 16 * 2;  // self-energies, then 16-byte granules
}

int rgf_kernel_regs() {
    cudaFuncAttributes a;
    if (cudaFuncGetAttributes(&a, rgf_pass2_kernel) != cudaSuccess) return 0;
    return a.numRegs;
}

cudaError_t launch_rgf(const TubeDev* d_tubes, const ChainRec* d_chains, const WarpRec* d_warps, int num_warps,
                       const SegUnit* d_units, int num_units, double* d_partial, void* d_scratch,
                       int warps_per_block, cudaStream_t stream, cudaEvent_t mid_event, const int* skip, int pieces,
                       double* d_piece_work, int schedule, const FusedOrder* fo) {
    if (num_warps <= 0) return cudaSuccess;
    if (schedule == kScheduleFused && pieces <= 1 && fo && fo->order) {
        // one warp per block: whole chains spread evenly over the SMs; the FP32
        // warps run on the side stream alongside the FP64 ones when both exist
        double* scr = static_cast<double*>(d_scratch);
        const bool fork = fo->n64 > 0 && fo->n32 > 0 && fo->side && fo->fork && fo->join;
        cudaError_t e = cudaSuccess;
        if (fork) {
            e = cudaEventRecord(fo->fork, stream);
            if (e == cudaSuccess) e = cudaStreamWaitEvent(fo->side, fo->fork, 0);
            if (e != cudaSuccess) return e;
        }
        if (fo->n64 > 0)
            rgf_fused_kernel<double><<<fo->n64, kWarp, 0, stream>>>(d_tubes, d_chains, d_warps, fo->order, fo->n64,
                                                                    d_partial, scr, skip);
        e = cudaGetLastError();
        if (e != cudaSuccess) return e;
        if (fo->n32 > 0)
            rgf_fused_kernel<float><<<fo->n32, kWarp, 0, fork ? fo->side : stream>>>(
                d_tubes, d_chains, d_warps, fo->order + fo->n64, fo->n32, d_partial, scr, skip);
        e = cudaGetLastError();
        if (e != cudaSuccess) return e;
        if (fork) {
            e = cudaEventRecord(fo->join, fo->side);
            if (e == cudaSuccess) e = cudaStreamWaitEvent(stream, fo->join, 0);
            if (e != cudaSuccess) return e;
        }
        if (mid_event) e = cudaEventRecord(mid_event, stream);
        return e;
    }
    if (warps_per_block < 1 || warps_per_block > 4) warps_per_block = 4;
    double* states = nullptr;
    if (pieces > 1) {
        // parallel in length: transfer matrices per piece, prefix per chain, then the pieces' sweeps
        double* tm = d_piece_work;
        states = d_piece_work + (size_t)num_warps * pieces * 18 * kWarp;
        rgf_piece_transfer_kernel<<<num_warps * pieces, kWarp, 0, stream>>>(d_tubes, d_chains, d_warps, num_warps,
                                                                            pieces, tm, skip);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
        rgf_piece_prefix_kernel<<<num_warps, kWarp, 0, stream>>>(d_tubes, d_chains, d_warps, num_warps, pieces, tm,
                                                                 states, skip);
        e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    } else {
        pieces = 1;
    }
    // pass 1 is latency-bound: one warp per block spreads the chains evenly over the SMs
    rgf_pass1_kernel<<<num_warps * pieces, kWarp, 0, stream>>>(d_tubes, d_chains, d_warps, num_warps,
                                                                 static_cast<double*>(d_scratch), skip, pieces,
                                                                 states);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    if (mid_event) cudaEventRecord(mid_event, stream);
    rgf_pass2_kernel<<<(num_units + warps_per_block - 1) / warps_per_block, warps_per_block * kWarp, 0, stream>>>(
        d_tubes, d_chains, d_warps, d_units, num_units, d_partial, static_cast<const double*>(d_scratch), skip);
    return cudaGetLastError();
}

cudaError_t selftest(int which, int n, const double* d_in, double* d_out, cudaStream_t stream) {
    if (n <= 0) return cudaSuccess;
    selftest_kernel<<<(n + 255) / 256, 256, 0, stream>>>(which, n, d_in, d_out);
    return cudaGetLastError();
}

cudaError_t launch_reduce(const ReduceTube* d_rt, int num_tubes, int max_N, const double* d_partial, double* d_Q,
                          cudaStream_t stream, const int* skip) {
    if (num_tubes <= 0 || max_N <= 0) return cudaSuccess;
    dim3 grid((max_N + 31) / 32, num_tubes);
    dim3 block(32, kRowGroups);
    reduce_kernel<<<grid, block, 0, stream>>>(d_rt, d_partial, d_Q, skip);
    return cudaGetLastError();
}

cudaError_t launch_transport(const TubeDev* d_tubes, const ChainRec* d_chains, const WarpRec* d_warps, int num_warps,
                             const SegUnit* d_units, int num_units, void* d_scratch, double* d_part,
                             double* d_chain_out, double* d_site, long long site_stride, int num_e, int M, int upw,
                             double* d_red, double* d_ldos, int N, cudaStream_t stream) {
    if (num_warps <= 0) return cudaSuccess;
    rgf_pass1_kernel<<<num_warps, kWarp, 0, stream>>>(d_tubes, d_chains, d_warps, num_warps,
                                                        static_cast<double*>(d_scratch), nullptr, 1, nullptr);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    rgf_transport_kernel<<<num_units, kWarp, 0, stream>>>(d_tubes, d_chains, d_warps, d_units, num_units,
                                                           static_cast<const double*>(d_scratch), d_part,
                                                           d_chain_out, d_site, site_stride);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    transport_reduce_kernel<<<(num_e + 127) / 128, 128, 0, stream>>>(d_part, d_chain_out, num_e, M, upw, d_red);
    e = cudaGetLastError();
    if (e != cudaSuccess || !d_site) return e;
    const long long tot = (long long)num_e * N;
    ldos_reduce_kernel<<<(unsigned)((tot + 255) / 256), 256, 0, stream>>>(d_site, site_stride, num_e, M, N, d_ldos);
    return cudaGetLastError();
}

}  // namespace negf
