// Broyden modified-second mixing on the device, with deterministic
// reductions (fixed-shape block trees, fixed-order partial sums).
//
// Reference: Source/Solver/Transport/Broyden_Second_Parallel.cpp:213-486
// (GPU branch; its CPU twin :9-211 defines the same arithmetic) and
// Broyden_Parallel_General.cpp:68-355.  The reference accumulates
// V^T x with one atomic per element (:355-365, :412-422) and finishes the
// norms with atomics (:268-272); here each dot product is one block-level
// tree reduction, so repeated runs are bitwise identical.
//
// Storage: V^T and W as [max_step][S] row-major (row `it` = iteration it),
// so every dot product and row update is a coalesced sweep over sites.

#include "negf_internal.h"

namespace negf {
namespace {

constexpr int kThreads = 256;

// Device-resident iterations (BroydenDev::step_dev set): the iteration index
// m = step - 1 is read on the device and `flags` (int[4]: converged,
// iterations, error, skip) makes every kernel of a finished solve return at
// entry, so a captured sequence of iterations needs no host round trip.
__device__ __forceinline__ bool skipped(const int* flags) { return flags && flags[3]; }
__device__ __forceinline__ int iter_m(const BroydenDev& b, int m_host) {
    return b.step_dev ? *b.step_dev - 1 : m_host;
}
// Seeded rows, read on the device so that captured launches see later seeds.
__device__ __forceinline__ int seeded(const BroydenDev& b) { return b.step_dev ? b.step_dev[1] : b.base; }

// max that keeps a NaN (a non-finite residual must not read as converged)
__device__ __forceinline__ double nanmax(double a, double b) { return (a != a || b != b) ? a + b : fmax(a, b); }

// Block reduction of (max, sum, sum) in a fixed order.
__device__ __forceinline__ void block_reduce3(double& a, double& b, double& c) {
    __shared__ double sh[3][kThreads / 32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o >= 1; o >>= 1) {
        a = nanmax(a, __shfl_xor_sync(0xffffffffu, a, o));
        b += __shfl_xor_sync(0xffffffffu, b, o);
        c += __shfl_xor_sync(0xffffffffu, c, o);
    }
    if (lane == 0) {
        sh[0][wid] = a;
        sh[1][wid] = b;
        sh[2][wid] = c;
    }
    __syncthreads();
    if (wid == 0) {
        const int nw = blockDim.x >> 5;
        a = lane < nw ? sh[0][lane] : 0.0;
        b = lane < nw ? sh[1][lane] : 0.0;
        c = lane < nw ? sh[2][lane] : 0.0;
#pragma unroll
        for (int o = 16; o >= 1; o >>= 1) {
            a = nanmax(a, __shfl_xor_sync(0xffffffffu, a, o));
            b += __shfl_xor_sync(0xffffffffu, b, o);
            c += __shfl_xor_sync(0xffffffffu, c, o);
        }
    }
}

__device__ __forceinline__ double block_sum(double v) {
    __shared__ double sh[kThreads / 32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o >= 1; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0) sh[wid] = v;
    __syncthreads();
    v = 0.0;
    if (wid == 0) {
        const int nw = blockDim.x >> 5;
        v = lane < nw ? sh[lane] : 0.0;
#pragma unroll
        for (int o = 16; o >= 1; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    }
    return v;
}

// Broyden_Second_Parallel.cpp:243-315: F, |F| (or relative), dF, and the
// three scalars (max norm, sum of squares, dF^T dF) as block partials.
__global__ void norm_kernel(BroydenDev b, const double* __restrict__ n_out, const int* flags) {
    if (skipped(flags)) return;
    double mx = 0.0, s1 = 0.0, s2 = 0.0;
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < b.S; s += gridDim.x * blockDim.x) {
        const double nin = b.n_in[s], nout = n_out[s];
        const double Fc = nin - nout;
        double nr, sq;
        if (b.norm_type == 0) {
            nr = fabs(Fc);
            sq = Fc * Fc;
        } else {
            nr = fabs(Fc / (nin + nout));
            sq = nr * nr;
        }
        b.norm[s] = nr;
        const double d = Fc - b.F[s];
        b.dF[s] = d;
        b.F[s] = Fc;
        b.sum[s] = 0.0;
        mx = nanmax(mx, nr);
        s1 += sq;
        s2 += d * d;
    }
    block_reduce3(mx, s1, s2);
    if (threadIdx.x == 0) {
        b.part[3 * blockIdx.x + 0] = mx;
        b.part[3 * blockIdx.x + 1] = s1;
        b.part[3 * blockIdx.x + 2] = s2;
    }
}

__global__ void norm_finalize(BroydenDev b, const int* flags) {
    if (threadIdx.x != 0 || skipped(flags)) return;
    double mx = 0.0, s1 = 0.0, s2 = 0.0;
    for (int i = 0; i < b.nblocks; ++i) {
        mx = nanmax(mx, b.part[3 * i]);
        s1 += b.part[3 * i + 1];
        s2 += b.part[3 * i + 2];
    }
    b.scal[0] = mx;
    b.scal[1] = sqrt(s1);
    b.scal[2] = s2;
}

// c[it] = sum_s V[it][s] x[s] for it = 1..rows (one block per row);
// rows = seeded + m - 1 + which with m from the host or the device (rows
// 1..seeded: a seeded initial inverse Jacobian).  With segments the sum runs
// over each segment's sites separately (blockIdx.y = segment, c[it][g]).
__global__ void dots_kernel(BroydenDev b, const double* __restrict__ x, int m_host, int which, const int* flags) {
    if (skipped(flags)) return;
    const int rows = seeded(b) + iter_m(b, m_host) - 1 + which;
    const int it = blockIdx.x + 1;
    if (it > rows) return;
    const int g = blockIdx.y;
    const int lo = b.nseg > 1 ? b.seg_off[g] : 0, hi = b.nseg > 1 ? b.seg_off[g + 1] : b.S;
    const double* v = b.V + (size_t)it * b.S;
    double acc = 0.0;
    for (int s = lo + threadIdx.x; s < hi; s += blockDim.x) acc += v[s] * x[s];
    acc = block_sum(acc);
    if (threadIdx.x == 0) b.c[(size_t)it * b.nseg + g] = acc;
}

// Per-segment dF^T dF (the denominators of the new V row when segmented).
__global__ void segsq_kernel(BroydenDev b, int m_host, const int* flags) {
    if (skipped(flags) || iter_m(b, m_host) <= 0) return;
    const int g = blockIdx.x;
    double acc = 0.0;
    for (int s = b.seg_off[g] + threadIdx.x; s < b.seg_off[g + 1]; s += blockDim.x) acc += b.dF[s] * b.dF[s];
    acc = block_sum(acc);
    if (threadIdx.x == 0) b.dd[g] = acc;
}

// Broyden_Second_Parallel.cpp:381-403: sum = W c (it < m), new V and W rows at m
// (after the seeded rows).
__global__ void newrow_kernel(BroydenDev b, int m_host, const int* flags) {
    if (skipped(flags)) return;
    const int m = iter_m(b, m_host);
    if (m <= 0) return;
    const int row = seeded(b) + m;
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < b.S; s += gridDim.x * blockDim.x) {
        const int g = b.nseg > 1 ? b.seg_of[s] : 0;
        const double denom = b.nseg > 1 ? b.dd[g] : b.scal[2];
        double acc = 0.0;
        for (int it = 1; it <= row - 1; ++it) acc += b.W[(size_t)it * b.S + s] * b.c[(size_t)it * b.nseg + g];
        const double dF = b.dF[s];
        const double dn = b.n_in[s] - b.n_prev[s];
        // a zero step (identical consecutive residuals) adds no direction: the
        // reference would divide by zero here
        b.V[(size_t)row * b.S + s] = denom > 0.0 ? dF / denom : 0.0;
        b.W[(size_t)row * b.S + s] = -b.fraction * dF + dn - acc;
    }
}

// Broyden_Second_Parallel.cpp:455-481: sum = W c (it <= m, after the seeded
// rows), then the new input.
__global__ void final_kernel(BroydenDev b, int m_host, const int* flags) {
    if (skipped(flags)) return;
    const int rows = seeded(b) + iter_m(b, m_host);
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < b.S; s += gridDim.x * blockDim.x) {
        const int g = b.nseg > 1 ? b.seg_of[s] : 0;
        double acc = 0.0;
        for (int it = 1; it <= rows; ++it) acc += b.W[(size_t)it * b.S + s] * b.c[(size_t)it * b.nseg + g];
        b.sum[s] = acc;
        const double prev = b.n_in[s];
        b.n_prev[s] = prev;
        b.n_in[s] = prev - b.scalar * b.fraction * b.F[s] - b.scalar * acc;
    }
}

// End of a device-resident step: the loop predicate of Transport.cpp:385-505
// (stop when the norm is not above max_norm), the step count, and the
// MaxStep abort of :389-393 as an error flag for the host.
// switch_norm > 0 (precision switching, flags int[8]): until flags[4] is set
// the charge came from the low-precision plan; the first norm below
// switch_norm sets flags[4] and later steps use the FP64 plan, and only an
// FP64 charge can end the solve.  flags[5] / flags[6] are the skip words of
// the low-precision and FP64 plans; flags[7] counts low-precision steps.
__global__ void step_kernel(BroydenDev b, double max_norm, double switch_norm, int* flags) {
    if (flags[3]) return;
    const double nrm = b.scal[0];
    flags[1] += 1;
    const int step = *b.step_dev + 1;
    *b.step_dev = step;
    const int limit = b.max_step - seeded(b);  // seeded rows take history capacity
    const bool fp64_charge = !(switch_norm > 0) || flags[4];
    if (!fp64_charge) flags[7] += 1;  // steps on a low-precision charge
    if (!isfinite(nrm))
        flags[2] = 2;
    else if (fp64_charge && !(nrm > max_norm))
        flags[0] = 1;
    else if (step > limit)
        flags[2] = 1;
    flags[3] = (flags[0] || flags[2]) ? 1 : 0;
    if (switch_norm > 0) {
        if (!flags[4] && nrm < switch_norm) flags[4] = 1;
        flags[5] = (flags[3] || flags[4]) ? 1 : 0;
        flags[6] = (flags[3] || !flags[4]) ? 1 : 0;
    }
}

__global__ void set_int_kernel(int* p, int v) { *p = v; }

__global__ void set_kernel(double* p, double v, int n) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) p[i] = v;
}

// U[i] = U0[i] + sum_j K[i][j] Q[j]: one warp per row, fixed-order lane tree.
__global__ void affine_kernel(const double* __restrict__ K, const double* __restrict__ U0,
                              const double* __restrict__ Q, double* __restrict__ U, int n, const int* skip) {
    if (skip && *skip) return;
    const int lane = threadIdx.x & 31;
    const int row = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (row >= n) return;
    const double* k = K + (size_t)row * n;
    double acc = 0.0;
    for (int j = lane; j < n; j += 32) acc += k[j] * Q[j];
#pragma unroll
    for (int o = 16; o >= 1; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (lane == 0) U[row] = U0[row] + acc;
}

// U[i] = U0[i] + sum_j tab[|idx[i] - idx[j]|] Q[j]: the same operator for a
// kernel that depends on the lattice distance only (a ring lattice: zigzag
// tubes), read from a table instead of an n x n matrix.  One warp per row;
// the block stages idx and Q in shared memory in chunks of 1024 sites, and
// consecutive sites give consecutive table entries (coalesced gathers).
constexpr int kToeChunk = 1024;
__global__ void __launch_bounds__(256) toeplitz_kernel(const double* __restrict__ tab, int ntab,
                                                       const int* __restrict__ idx, const double* __restrict__ U0,
                                                       const double* __restrict__ Q, double* __restrict__ U, int n,
                                                       const int* skip) {
    if (skip && *skip) return;
    __shared__ double sq[kToeChunk];
    __shared__ int si[kToeChunk];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int row = blockIdx.x * (blockDim.x >> 5) + wib;
    const int ir = row < n ? idx[row] : 0;
    double acc = 0.0;
    for (int c0 = 0; c0 < n; c0 += kToeChunk) {
        const int cn = min(kToeChunk, n - c0);
        __syncthreads();
        for (int t = threadIdx.x; t < cn; t += blockDim.x) {
            sq[t] = Q[c0 + t];
            si[t] = idx[c0 + t];
        }
        __syncthreads();
        if (row < n) {
            for (int t = lane; t < cn; t += 32) {
                int d = ir - si[t];
                d = d < 0 ? -d : d;
                acc = fma(d < ntab ? __ldg(tab + d) : 0.0, sq[t], acc);
            }
        }
    }
#pragma unroll
    for (int o = 16; o >= 1; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (row < n && lane == 0) U[row] = U0[row] + acc;
}

// Batched form: every row of every tube in one launch.  Block b covers rows
// [first, first + 8) of tube tube_of[b] (blocks never straddle tubes), so the
// tubes' potentials are formed concurrently instead of one launch each.
__global__ void __launch_bounds__(256) toeplitz_batch_kernel(const ToeplitzOp* __restrict__ ops,
                                                             const int2* __restrict__ blocks, const int* skip) {
    if (skip && *skip) return;
    __shared__ double sq[kToeChunk];
    __shared__ int si[kToeChunk];
    const int2 bt = blocks[blockIdx.x];  // (tube, first row)
    const ToeplitzOp op = ops[bt.x];
    const int n = op.n;
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int row = bt.y + wib;
    const int ir = row < n ? op.idx[row] : 0;
    double acc = 0.0;
    for (int c0 = 0; c0 < n; c0 += kToeChunk) {
        const int cn = min(kToeChunk, n - c0);
        __syncthreads();
        for (int t = threadIdx.x; t < cn; t += blockDim.x) {
            sq[t] = op.Q[c0 + t];
            si[t] = op.idx[c0 + t];
        }
        __syncthreads();
        if (row < n) {
            for (int t = lane; t < cn; t += 32) {
                int d = ir - si[t];
                d = d < 0 ? -d : d;
                acc = fma(d < op.ntab ? __ldg(op.tab + d) : 0.0, sq[t], acc);
            }
        }
    }
#pragma unroll
    for (int o = 16; o >= 1; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (row < n && lane == 0) op.U[row] = op.U0[row] + acc;
}

}  // namespace

cudaError_t affine_toeplitz_batch(const ToeplitzOp* d_ops, const int2* d_blocks, int num_blocks, cudaStream_t s,
                                  const int* skip) {
    if (num_blocks <= 0) return cudaSuccess;
    toeplitz_batch_kernel<<<num_blocks, 256, 0, s>>>(d_ops, d_blocks, skip);
    return cudaGetLastError();
}

cudaError_t affine_toeplitz(const double* tab, int ntab, const int* idx, const double* U0, const double* Q, double* U,
                            int n, cudaStream_t s, const int* skip) {
    if (n <= 0) return cudaSuccess;
    toeplitz_kernel<<<(n + 7) / 8, 256, 0, s>>>(tab, ntab, idx, U0, Q, U, n, skip);
    return cudaGetLastError();
}

cudaError_t broyden_norm(const BroydenDev& b, const double* n_out, cudaStream_t s, const int* flags) {
    norm_kernel<<<b.nblocks, kThreads, 0, s>>>(b, n_out, flags);
    norm_finalize<<<1, 32, 0, s>>>(b, flags);
    return cudaGetLastError();
}

cudaError_t broyden_update(const BroydenDev& b, int m, cudaStream_t s, const int* flags) {
    if (b.step_dev && flags) {
        // device-resident: shapes cover every m up to max_step, rows above m return
        const dim3 g(b.max_step > 1 ? b.max_step : 1, b.nseg);
        dots_kernel<<<g, kThreads, 0, s>>>(b, b.dF, 0, 0, flags);
        if (b.nseg > 1) segsq_kernel<<<b.nseg, kThreads, 0, s>>>(b, 0, flags);
        newrow_kernel<<<b.nblocks, kThreads, 0, s>>>(b, 0, flags);
        dots_kernel<<<g, kThreads, 0, s>>>(b, b.F, 0, 1, flags);
        final_kernel<<<b.nblocks, kThreads, 0, s>>>(b, 0, flags);
        return cudaGetLastError();
    }
    if (m > 0) {
        if (b.base + m - 1 >= 1) dots_kernel<<<dim3(b.base + m - 1, b.nseg), kThreads, 0, s>>>(b, b.dF, m, 0, nullptr);
        if (b.nseg > 1) segsq_kernel<<<b.nseg, kThreads, 0, s>>>(b, m, nullptr);
        newrow_kernel<<<b.nblocks, kThreads, 0, s>>>(b, m, nullptr);
    }
    if (b.base + m >= 1) dots_kernel<<<dim3(b.base + m, b.nseg), kThreads, 0, s>>>(b, b.F, m, 1, nullptr);
    final_kernel<<<b.nblocks, kThreads, 0, s>>>(b, m, nullptr);
    return cudaGetLastError();
}

cudaError_t broyden_finish_step(const BroydenDev& b, double max_norm, double switch_norm, int* flags, cudaStream_t s) {
    step_kernel<<<1, 1, 0, s>>>(b, max_norm, switch_norm, flags);
    return cudaGetLastError();
}

cudaError_t set_int(int* p, int v, cudaStream_t s) {
    set_int_kernel<<<1, 1, 0, s>>>(p, v);
    return cudaGetLastError();
}

cudaError_t broyden_set(double* p, double v, int n, cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    const int blocks = (n + kThreads - 1) / kThreads;
    set_kernel<<<blocks < 1024 ? blocks : 1024, kThreads, 0, s>>>(p, v, n);
    return cudaGetLastError();
}

cudaError_t affine_potential(const double* K, const double* U0, const double* Q, double* U, int n, cudaStream_t s,
                             const int* skip) {
    if (n <= 0) return cudaSuccess;
    const int warps_per_block = 8;
    affine_kernel<<<(n + warps_per_block - 1) / warps_per_block, 32 * warps_per_block, 0, s>>>(K, U0, Q, U, n, skip);
    return cudaGetLastError();
}

}  // namespace negf
