// Internal declarations shared by the host layer (negf_api.cpp) and the
// CUDA translation units (negf_rgf.cu, negf_broyden.cu).  Not part of the
// public C-ABI.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>

namespace negf {

constexpr int kMaxModes = 32;   // distinct modes per tube kept on the device
constexpr int kSeg = 8;         // sites per checkpoint segment of the RGF sweeps
constexpr int kWarp = 32;
constexpr int kPadLo = kSeg;      // zero doubles before a tube's potential buffer
constexpr int kPadHi = 2 * kSeg;  // zero doubles after it

// Per-tube record read by the RGF kernel (one per tube of a launch).
struct __align__(16) TubeDev {
    const double* U;   // site potential [N] (device), kPadLo / kPadHi zeros around it
    int N;             // sites
    int num_modes;
    double gamma;      // hopping [eV]
    double Uc0, Uc1;   // contact potentials [eV]
    int use_decimation, dec_iters, dec_layers;
    int uc_from_U;     // 1: contact potentials are U[0] and U[N-1] read on the device
    double beta[kMaxModes];
    double degen[kMaxModes];
};

// One (tube, mode, energy) chain = one lane of a warp.  Kind and precision
// are uniform over the 32 lanes of a warp (the host pads each group).
//   contour/pole lane:  contribution Im(c * G_nn) * degen
//   real-axis lane:     |G_nn|^2 (lambda_n Gamma_0 b0 + rho_n Gamma_1 b1) * degen
struct __align__(16) ChainRec {
    double Er, Ei;  // energy
    double cr, ci;  // complex coefficient of G_nn
    double b0, b1;  // real-axis coefficients Re(c f_k w J)
    int mode;       // mode index (-1 for padding lanes)
    int pad;
};

enum WarpKind : int { kContour = 0, kRealAxis = 1 };

struct __align__(16) WarpRec {
    long long row_off;   // offset of this warp's per-site partial row (doubles)
    long long ck_off;    // offset of this warp's checkpoint scratch (elements of its precision)
    int tube;            // index into TubeDev[]
    int kind;            // WarpKind
    int fp32;            // 1: recursion in complex FP32
    int pad;
};

// Per-tube description of the reduction of warp rows into site charge.
struct __align__(16) ReduceTube {
    long long row_base;  // first partial row of the tube
    long long q_off;     // offset of the tube's sites in Q
    const double* rho0;  // per-site sum over modes of Im Rho0 (device) or null
    int N;
    int num_rows;        // warps of the tube
};

// Pass-2 work unit: segments [seg0, seg1) of the chains of one warp.
struct __align__(16) SegUnit {
    int warp;
    int seg0, seg1;
    int pad;
};
constexpr int kSegsPerUnit = 32;  // segments per pass-2 unit (256 sites)

// RGF launch: pass 1 (one warp per WarpRec, lane = chain: concurrent forward
// and backward sweeps storing boundary checkpoints) then pass 2 (one warp per
// SegUnit: independent segments, per-site contributions into partial rows).
// Transport characteristics of one tube (DOS, transmission, current
// integrand probes, optional LDOS): pass 1 on real-axis FP64 chains with
// b0 = b1 = 1 and (cr, ci) = (Re f_0, Re f_1), then the spectral kernel and
// the per-energy reductions.  d_red: [num_e][8]; d_ldos: [num_e][N] when
// d_site (scratch of N x chains doubles, stride site_stride) is given.
cudaError_t launch_transport(const TubeDev* d_tubes, const ChainRec* d_chains, const WarpRec* d_warps, int num_warps,
                             const SegUnit* d_units, int num_units, void* d_scratch, double* d_part,
                             double* d_chain_out, double* d_site, long long site_stride, int num_e, int M, int upw,
                             double* d_red, double* d_ldos, int N, cudaStream_t stream);
// Real-space ring-block RGF (negf_realspace.cu): leads, chain and reduction
// for num_e >= 0 energies with coefficients c, Q[r] = sum_e Im(c sum_atoms
// G_jj) - d_sub[r] (d_sub may be null).  The last num_neq energies are
// real-axis points whose coefficients (b0, b1) = (c_re, c_im) weight the
// source and drain spectral functions: they add b0 A^L + b1 A^R per ring
// (FP64).
// d_flags[e]: 1 = chain in FP32 (tensor-core products), 2 = U = 0 pass
// (d_Uzero on the atoms and 0 at the contacts; with negated c it subtracts
// Rho0); otherwise the atom potentials d_Uatoms ([2K][m]) and Uc0, Uc1.
// d_corners: num_e * 2 * m^2 complex, d_gL: (num_e - num_neq) * K * m^2
// complex, d_gLn: num_neq * (2K + 1) * m^2 complex, d_rows: num_e * 2K
// doubles; *d_status set to 1 on a zero pivot.
// Leads of the real-space pass: the mode chains' surface values by the
// analytic formula, or by the reference's decimation (dec_layers layers,
// dec_iters iterations) when use_decimation is set.
struct RsLeads {
    int use_decimation = 0, dec_layers = 10, dec_iters = 32;
};
cudaError_t launch_realspace(int m, int K, double gamma, const double* d_Ere, const double* d_Eim,
                             const double* d_cre, const double* d_cim, int num_e, int num_neq, const int* d_flags,
                             const double* d_Uatoms, const double* d_Uzero, double Uc0, double Uc1,
                             const RsLeads& leads, void* d_corners, void* d_gL, void* d_gLn, double* d_rows,
                             double* d_Q, const double* d_sub, int* d_status, cudaStream_t stream);
cudaError_t rs_expand(const double* d_U, int N, int m, double* d_Ua, cudaStream_t stream);
// Self-test of the real-space tile primitives for m in {4, 13, 16}: which 2 / 3
// inverts count m x m complex matrices in FP64 / FP32, which 4 / 5 forms
// count products A B (FP64 CUDA cores / FP32 tensor cores); complex values
// re/im interleaved, row-major.
cudaError_t rs_selftest(int which, int m, int count, const double* d_in, double* d_out, cudaStream_t stream);
int rs_max_atoms_per_block();

// Surrogate-model kernels (negf_surrogate.cu).  BF16 operands as void*.
// path: kNnGemmTcgen05 (5th-generation tensor cores, tensor-memory accumulator; operands by TMA where
// they can be described, else register-staged), kNnGemmTcgen05Staged (register-staged only) or kNnGemmMmaSync
constexpr int kNnGemmTcgen05 = 1, kNnGemmMmaSync = 2, kNnGemmTcgen05Staged = 3;
cudaError_t nn_gemm(int at, int bt, int M, int N, int K, int batch, const void* A, int lda, long long sA,
                    const void* B, int ldb, long long sB, float* C, int ldc, long long sC, void* Cb, int accumulate,
                    cudaStream_t s, int path = kNnGemmTcgen05);
cudaError_t nn_gelu_fwd(long long rows, int cols, const float* a, const float* b, const float* bias, float* pre,
                        float* out, void* outb, int act, cudaStream_t s);
cudaError_t nn_gelu_bwd(long long n, const float* dy, const float* pre, float* d, void* db, cudaStream_t s);
cudaError_t nn_colsum(long long rows, int cols, const float* x, float* out, int accumulate, cudaStream_t s);
cudaError_t nn_cast_bf16(long long n, const float* x, void* y, cudaStream_t s);
cudaError_t nn_adam(long long n, float* w, const float* g, float* m, float* v, void* wb, float lr, float b1, float b2,
                    float eps, int step, float wd, cudaStream_t s);
cudaError_t nn_rowdot(long long rows, int cols, const float* h, const float* w, const float* b, float* q,
                      cudaStream_t s);
cudaError_t nn_outer(long long rows, int cols, const float* dq, const float* w, float* dh, void* dhb, cudaStream_t s);
cudaError_t nn_mse(long long n, const float* q, const float* y, float* d, float* part, cudaStream_t s);

// RGF schedules.  Two-pass: pass 1 (one warp per 32 chains, both sweeps,
// checkpoints at every segment) then pass 2 (one warp per group of segments:
// segment-parallel tiles).  Fused: one kernel, one warp per 32 whole chains,
// meet-in-the-middle sweeps (fewer operations and half the checkpoint bytes;
// it needs enough warps to fill the GPU).  Results agree to rounding.
constexpr int kScheduleTwoPass = 0;
constexpr int kScheduleFused = 1;
// skip (device int, may be null): when nonzero at launch time every block
// returns at entry (device-side early exit of a captured SCF iteration).
// The fused schedule runs with pieces == 1 only (else the two-pass one runs).
// Warp order of the fused schedule: order[0 .. n64) are the FP64 warps,
// order[n64 .. n64 + n32) the FP32 ones (device array); the FP32 kernel runs
// on `side` between the events fork (recorded on the main stream) and join
// (waited by the main stream) when both kinds exist.
struct FusedOrder {
    const int* order;
    int n64, n32;
    cudaStream_t side;
    cudaEvent_t fork, join;
};
cudaError_t launch_rgf(const TubeDev* d_tubes, const ChainRec* d_chains, const WarpRec* d_warps, int num_warps,
                       const SegUnit* d_units, int num_units, double* d_partial, void* d_scratch,
                       int warps_per_block, cudaStream_t stream, cudaEvent_t mid_event,
                       const int* skip = nullptr, int pieces = 1, double* d_piece_work = nullptr,
                       int schedule = kScheduleTwoPass, const FusedOrder* fo = nullptr);
// pieces > 1 (parallel in length): d_piece_work holds num_warps * pieces * 24 * 32 doubles.
// Device self-test of numeric primitives: which = 0 FP64 reciprocal,
// 1 FP32 reciprocal (input/output as doubles), n values, device pointers.
cudaError_t selftest(int which, int n, const double* d_in, double* d_out, cudaStream_t stream);
// Per-site reduction (Kahan) of warp rows, minus Rho0 when rho0 != null.
cudaError_t launch_reduce(const ReduceTube* d_rt, int num_tubes, int max_N, const double* d_partial, double* d_Q,
                          cudaStream_t stream,
                          const int* skip = nullptr);
// Scratch elements (doubles, rounded up) needed per warp for a tube of N sites.
// Scratch of one warp: per-lane lead self-energies (4 x 32 doubles) then the
// segment checkpoints (Y, lambda at segment starts; X, rho at segment ends).
long long rgf_scratch_doubles(int N, int kind, int fp32);
int rgf_kernel_regs();  // registers per thread of the RGF kernel (0 if unknown)

// Launch tables written into caller-provided fixed arrays (used by the
// allocation-free entry point in negf_noalloc.cu).
struct FixedPlan {
    TubeDev* tubes;
    ReduceTube* rts;
    ChainRec* chains;
    WarpRec* warps;
    SegUnit* units;
    int tube_cap;
    size_t chain_cap, warp_cap, unit_cap;
    // outputs
    int num_tubes, max_N;
    size_t num_chains, num_warps, num_units;
    long long partial_doubles, scratch_doubles, total_sites;
};
}  // namespace negf
struct negf_tube;
namespace negf {
// Lock of the host layer: held by every entry point that reads or writes tube
// state or shared host tables.
std::unique_lock<std::mutex> api_lock();
// Callers hold api_lock().  Fails with NEGF_ERR_ARG when a tube is not on the
// current device or the tables overflow the fixed arrays.
int plan_charge_fixed(negf_tube* const* tubes, int num_tubes, FixedPlan& fp);
int report(int code, const char* msg);  // sets negf_last_error, returns code

// Broyden kernels (negf_broyden.cu).
struct BroydenDev {
    int S, max_step, norm_type;
    double fraction, scalar;
    double* n_in;
    double* n_prev;
    double* F;
    double* dF;
    double* norm;
    double* V;        // [max_step][S] (row it = V^T column it)
    double* W;        // [max_step][S]
    double* c;        // [max_step][nseg]
    double* sum;      // [S]
    double* scal;     // [4]: max norm, sum of squares, denominator, spare
    double* part;     // [3 * nblocks] block partials
    int nblocks;
    int* step_dev;    // device int[2]: [0] the step counter (read by device-resident steps),
                      // [1] rows 1..[1] of V, W hold a seeded initial inverse Jacobian (0: none)
    int base;         // host copy of step_dev[1]
    // Segments (per-tube Broyden): the dot products of the secant update run
    // over each segment's sites separately; nseg == 1 is one Broyden over all sites.
    int nseg;
    int* seg_off;     // device int[nseg + 1] (nseg > 1)
    int* seg_of;      // device int[S]: segment of each site (nseg > 1)
    double* dd;       // [nseg]: per-segment dF^T dF
};
cudaError_t broyden_norm(const BroydenDev& b, const double* n_out, cudaStream_t s, const int* flags = nullptr);
cudaError_t broyden_update(const BroydenDev& b, int m, cudaStream_t s, const int* flags = nullptr);
// Device-resident step end: flags int[4] = converged, iterations, error
// (1 MaxStep exceeded, 2 non-finite norm), skip; advances *step_dev.
cudaError_t broyden_finish_step(const BroydenDev& b, double max_norm, double switch_norm, int* flags, cudaStream_t s);
cudaError_t set_int(int* p, int v, cudaStream_t s);
cudaError_t broyden_set(double* p, double v, int n, cudaStream_t s);
cudaError_t affine_potential(const double* K, const double* U0, const double* Q, double* U, int n, cudaStream_t s,
                             const int* skip = nullptr);
cudaError_t affine_toeplitz(const double* tab, int ntab, const int* idx, const double* U0, const double* Q, double* U,
                            int n, cudaStream_t s, const int* skip = nullptr);
struct ToeplitzOp {  // one tube of a batched lattice-distance potential update
    const double* tab;
    const int* idx;
    const double* U0;
    const double* Q;
    double* U;
    int ntab, n;
};
cudaError_t affine_toeplitz_batch(const ToeplitzOp* d_ops, const int2* d_blocks, int num_blocks, cudaStream_t s,
                                  const int* skip = nullptr);

}  // namespace negf
