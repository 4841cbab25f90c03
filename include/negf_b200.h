/*
 * negf_b200.h — C-ABI of the B200-native NEGF induced-charge engine.
 *
 * Drop-in boundary for ELEQTRONeX's NEGF/transport interface
 * (Source/Solver/Transport/NEGF/NEGF_Common.H:518-606,
 *  Source/Solver/Transport/Nanostructure.H:15-45,
 *  Source/Solver/Transport/Transport.H:203-208).
 *
 * Conventions
 *   - every function returns an int status: NEGF_OK (0) or a negative code;
 *     negf_last_error() gives the message of the last failure on the calling
 *     thread.  Nothing aborts the process.
 *   - buffers are caller-owned; pointers are plain host or device pointers
 *     as documented per argument; sizes are element counts.
 *   - `stream` is a cudaStream_t passed as void* (NULL = legacy default).
 *   - one handle is not thread-safe; distinct handles are independent.
 *     Charge calls keep their device scratch per (device, stream): calls
 *     on different streams or devices never share scratch, and calls on one
 *     stream reuse it in stream order.  Each stream's scratch grows to the
 *     largest problem seen on it and is held until negf_release_scratch()
 *     or process exit.
 *   - every tube of a call must live on the current device (NEGF_ERR_ARG).
 *   - reductions are deterministic: the same inputs give bitwise-identical
 *     charge on the same GPU and launch configuration.
 *   - the library has no CPU fallback: every compute call needs a CUDA
 *     device and fails with NEGF_ERR_CUDA when none is present.
 */
#ifndef NEGF_B200_H_
#define NEGF_B200_H_

#ifdef __cplusplus
extern "C" {
#endif

#define NEGF_OK 0
#define NEGF_ERR_ARG (-1)
#define NEGF_ERR_CUDA (-2)
#define NEGF_ERR_STATE (-3)
#define NEGF_ERR_NUMERIC (-4)
#define NEGF_ERR_IO (-5)

#define NEGF_PREC_FP64 0  /* complex FP64 recursion throughout */
#define NEGF_PREC_MIXED 1 /* complex FP32 recursion, FP64 lead GF / near-axis points / reduction */

#define NEGF_NORM_ABSOLUTE 0 /* Broyden_norm_type = absolute */
#define NEGF_NORM_RELATIVE 1 /* Broyden_norm_type = relative */

#define NEGF_MAX_NONEQ_PATHS 8

typedef struct negf_tube negf_tube;
typedef struct negf_broyden negf_broyden;

/* Nanotube + NEGF parameters.  Field names follow the reference input keys
 * (NEGF_Common.cpp:288-643, CNT.cpp:13-21).  negf_tube_desc_init() fills the
 * reference defaults. */
typedef struct negf_tube_desc {
    int type_id[2];                /* (m, n) chirality; CNT.cpp:11 default (17, 0) */
    int num_unitcells;             /* NS.num_unitcells */
    int num_modes;                 /* BLOCK_SIZE: lowest distinct modes kept (Code_Definitions.H:9) */
    double acc;                    /* C-C distance [m] (CNT.H:16, 1.42e-10) */
    double gamma;                  /* hopping [eV] (CNT.H:17, 2.5) */
    double contact_T[2];           /* contact_T [K] (NEGF_Common.H:442) */
    double contact_mu[2];          /* contact_mu [eV] (NEGF_Common.cpp:395-407) */
    int eq_integration_pts[3];     /* NEGF_Common.cpp:445-449 */
    int num_noneq_paths;           /* NEGF_Common.cpp:473-497 */
    int noneq_integration_pts[NEGF_MAX_NONEQ_PATHS];
    double noneq_percent_intercuts[NEGF_MAX_NONEQ_PATHS]; /* <0 in [0] = uniform default */
    double E_valence_min;          /* NEGF_Common.H:387 (-14) */
    double E_pole_max;             /* NEGF_Common.H:388 (10) */
    double E_zPlus_imag;           /* NEGF_Common.H:386 (1e-8) */
    double Fermi_tail_factors[2];  /* NEGF_Common.H:395-396 (14, 14) */
    int use_decimation;            /* NEGF_Common.H:469 (CNT default 0: analytic lead GF) */
    int decimation_max_iter;       /* NEGF_Common.H:474 (30) */
    int decimation_layers;         /* NEGF_Common.H:476 (10) */
    /* Optional explicit real-axis window: when realaxis_pts > 0 the equilibrium
     * contour ends at realaxis_min + i*E_zPlus_imag and the non-equilibrium
     * integral runs over [realaxis_min, realaxis_max] with realaxis_pts points
     * (kind 0: uniform grid of IntegrationPath.cpp:149-168, kind 1: Gauss-Legendre). */
    double realaxis_min, realaxis_max;
    int realaxis_pts, realaxis_kind;
    int precision;                 /* NEGF_PREC_FP64 or NEGF_PREC_MIXED */
    double mixed_fp64_band;        /* mixed mode: contour points with Im E below this [eV] and every
                                      real-axis point (see mixed_realaxis_fp32) stay FP64 (1e-3) */
    int flatband_dos_integration_pts; /* DOS path points at zero bias (NEGF_Common.H:416, 100) */
    /* Adaptive non-equilibrium limits (Read_AdaptiveIntegrationParams,
     * NEGF_Common.cpp:524-543; NEGF_Common.H:453-457). */
    int flag_adaptive_integration_limits;      /* 0 */
    int integrand_correction_interval;         /* 500 */
    double kT_window_around_singularity[2];    /* {1, 1} */
    int flag_noneq_integration_pts_density;    /* 1 when the densities below are given */
    double noneq_integration_pts_density[NEGF_MAX_NONEQ_PATHS]; /* points per kT of each path */
    /* Mixed mode, no counterpart in the reference: 1 also runs the real-axis
     * chains at least mixed_fp64_band above the axis (broadening
     * E_zPlus_imag >= band) in FP32 (0, default: real-axis chains stay FP64). */
    int mixed_realaxis_fp32;
} negf_tube_desc;

/* Fill `d` with the reference defaults. */
int negf_tube_desc_init(negf_tube_desc* d);

/* c_NEGF_Common::Initialize_NEGF_Params + Initialize_NEGF
 * (NEGF_Common.cpp:1256-1306): material parameters, sorted modes and
 * degeneracies (CNT.cpp:155-286), Hamiltonian (CNT.cpp:301-336), contact
 * info (CNT.cpp:338-352), energy limits and paths (NEGF_Common.cpp:1687-1816)
 * and Rho0 (NEGF_Common.cpp:3957-4092), on the current CUDA device. */
int negf_tube_create(const negf_tube_desc* d, negf_tube** out);
int negf_tube_destroy(negf_tube* t);

/* c_NEGF_Common::get_num_field_sites (NEGF_Common.H:555). */
int negf_tube_num_sites(const negf_tube* t, int* n_sites);
/* Modes kept: J index, degeneracy and beta_J = 2 gamma cos(pi J / m)
 * (CNT.cpp:227-292).  Arrays of length num_modes (may be NULL). */
int negf_tube_modes(const negf_tube* t, int* num_modes, int* J, int* degeneracy, double* beta);
/* Axial site positions [nm] (h_PTD_glo_vec, NEGF_Common.cpp:1074-1100, CNT.cpp:93-132). */
int negf_tube_site_positions(const negf_tube* t, double* y_nm);

/* Site potential U_n [eV] and the two contact potentials
 * (h_U_loc_data / U_contact; Nanostructure.cpp:494-504,
 * Add_PotentialToHamiltonian NEGF_Common.cpp:1656-1666).  Host pointer. */
int negf_tube_set_potential(negf_tube* t, const double* U, int n_sites, const double U_contact[2]);
/* Same with a device pointer; the copy is ordered on `stream`. */
int negf_tube_set_potential_device(negf_tube* t, const double* d_U, int n_sites, const double U_contact[2],
                                   void* stream);
/* Device pointer of the tube's potential buffer (writers must order their
 * writes before the next negf_compute_charge on the same stream). */
int negf_tube_potential_device_ptr(negf_tube* t, double** d_U);

/* set_Contact_Electrochemical_Potential (NEGF_Common.cpp:359-372): marks the
 * energy limits and paths for rebuilding at the next charge computation
 * (Solve_NEGF, NEGF_Common.cpp:1328-1337). */
int negf_tube_set_contact_mu(negf_tube* t, const double mu[2]);

/* Energy-point tables of the current paths (Define_EnergyLimits +
 * Update_IntegrationPaths).  kind: 0 Rho0, 1 RhoEq contour, 2 poles, 3 NonEq.
 * When buf != NULL writes (E.re, E.im, w.re, w.im, J.re, J.im) per point.
 * *count receives the number of points. */
int negf_tube_energy_points(negf_tube* t, int kind, double* buf, int* count);
/* Same tables computed from a descriptor alone (contact_mu of the
 * descriptor), without a device: host-side path logic only. */
int negf_desc_energy_points(const negf_tube_desc* d, int kind, double* buf, int* count);
/* Whether the non-equilibrium window is active (flag_noneq_exists). */
int negf_tube_noneq(negf_tube* t, int* noneq);
/* get_Total_Integration_Pts (NEGF_Common.cpp:1826-1841). */
int negf_tube_total_integration_pts(negf_tube* t, int* pts);

/* Restrict the energy points this process integrates to shard `rank` of
 * `world` (contiguous ranges of every tube's point list, Rho0 subtracted on
 * rank 0 only).  The partial charges of all ranks sum to the full charge. */
int negf_tube_set_energy_shard(negf_tube* t, int rank, int world);
/* The [lo, hi) range of point indices (RhoEq+poles first, then NonEq) that
 * shard `rank` of `world` integrates for a tube with `num_points` points. */
int negf_shard_range(int num_points, int rank, int world, int* lo, int* hi);

/* Solve_NEGF + Compute_InducedCharge (NEGF_Common.cpp:1309-1340, 2850-2900)
 * for a batch of tubes in one launch:
 *   Q[offset_t + n] = sum_modes [Im RhoEq_n + Re RhoNonEq_n - Im Rho0_n]
 * where offset_t is the running sum of the previous tubes' site counts
 * (num_field_sites_loc_NS_offset).  Q is a device pointer when
 * q_on_device != 0, else a host pointer (the call then synchronises `stream`). */
int negf_compute_charge(negf_tube* const* tubes, int num_tubes, double* Q, int q_on_device, void* stream);

/* Allocation-free variant of negf_compute_charge -- no counterpart in the
 * reference.  For callers that cannot allocate device memory when they need
 * the charge: applications whose device memory comes from their own pool
 * and that forbid the runtime allocator, and plugins that must not grow the
 * host program's footprint.  It runs the same kernels, but keeps the launch
 * tables, partial rows and checkpoints in one static device array of 32 MiB
 * that every GPU loading this library holds until exit; it calls no
 * cudaMalloc/cudaFree.  d_Q is a device pointer.  Problems that need more
 * than 32 MiB of scratch, or more than 64 tubes, are rejected with
 * NEGF_ERR_ARG, as are tubes that do not live on the current device.
 * NEGF_ERR_STATE marks a tube whose energy paths are stale; the public calls
 * that change paths (negf_tube_set_contact_mu,
 * negf_tube_correct_integration_limits) rebuild them before returning.  The
 * first call on a device looks up the array's address (set-up), so make it
 * before any stream capture.  All calls share the array: calls that overlap
 * on the GPU race and must be serialised by the caller. */
int negf_compute_charge_noalloc(negf_tube* const* tubes, int num_tubes, double* d_Q, void* stream);

/* Frees the device scratch (launch tables, partial rows, checkpoints) that
 * negf_compute_charge and negf_rs_compute_charge keep for the current device
 * and `stream`, after waiting for the last call made on it; the next call on
 * that stream allocates it again.  No counterpart in the reference, whose
 * device tables are members of each nanostructure object (Allocate_Arrays,
 * NEGF_Common.cpp:1421-1653, called from Initialize_NEGF; freed with the
 * object); here
 * the scratch belongs to the (device, stream) pair, not to a tube, is kept
 * between calls (a self-consistent loop reuses it every iteration), and this
 * call hands it back, e.g. before destroying `stream` or after the last
 * solve of a sweep.  A stream with no scratch is a no-op.
 * It waits on the host, so it is not for a stream that is being captured.
 * Charge plans and the allocation-free entry point are not affected. */
int negf_release_scratch(void* stream);

/* Per-call timing and work counters of the last negf_compute_charge
 * (kernel milliseconds measured with CUDA events on `stream`). */
typedef struct negf_stats {
    double rgf_kernel_ms;      /* both RGF passes */
    double pass1_kernel_ms;    /* pass 1: concurrent forward/backward sweeps */
    double pass2_kernel_ms;    /* pass 2: segment-parallel recompute + site contributions */
    double reduce_kernel_ms;   /* per-site reduction kernel */
    long long updates;         /* sum over chains of N (site*energy*mode updates) */
    long long updates_fp32;    /* of which computed in FP32 (mixed mode) */
    long long contour_updates; /* updates on contour/pole points */
    long long realaxis_updates;/* updates on real-axis points */
    int chains;                /* (tube, mode, energy) chains incl. padding */
    int warps;                 /* pass-1 warps launched */
    int units;                 /* pass-2 warps (segment groups) launched */
    int kernel_launches;       /* kernels launched by the call */
    int pieces;                /* pass-1 pieces per chain (parallel in length) */
    long long checkpoint_bytes;/* scratch bytes written+read by the kernel */
    int schedule;              /* NEGF_SCHEDULE_TWO_PASS or NEGF_SCHEDULE_FUSED */
} negf_stats;
int negf_last_stats(negf_stats* s);
/* Launch-shape knobs of negf_compute_charge.
 * NEGF_TUNE_PASS2_WARPS_PER_BLOCK: 1, 2 or 4 (default) warps per pass-2
 *   block; results are bitwise identical for every setting.
 * NEGF_TUNE_PASS1_PIECES: 0 (default, automatic) or P >= 1: the forward and
 *   backward sweeps of every chain run as P pieces of the tube in parallel
 *   ("parallel in length", for long tubes with few energies): 2 x 2 transfer
 *   matrices of each piece, a prefix over the pieces for their boundary
 *   states, then the pieces' sweeps.  Automatic: when the chains fill
 *   fewer than 4 warps per SM, enough pieces for about 8 warps per SM, each
 *   of >= 32 segments (256 sites), at most 128.  Results agree with P = 1 to
 *   rounding (relative 1e-10 in the tests, about 1e-12 measured).
 * NEGF_TUNE_SCHEDULE: 0 (default, automatic), NEGF_SCHEDULE_TWO_PASS or
 *   NEGF_SCHEDULE_FUSED.  Two-pass: pass 1 runs both sweeps of every chain
 *   and checkpoints them at every 8-site segment, pass 2 integrates the
 *   segments in parallel tiles (parallelism for few chains).  Fused: one
 *   kernel; the forward sweep crosses the first half of the tube and the
 *   backward sweep the second, each storing its own checkpoints, then each
 *   continues into the other half and integrates the segments it crosses
 *   (every site crossed twice instead of three times, half the checkpoint
 *   bytes; needs enough chains to fill the GPU).  Automatic: fused when the
 *   chains fill at least one warp per SM sub-partition and the sweeps run as
 *   one piece.  Results agree to rounding. */
#define NEGF_TUNE_PASS2_WARPS_PER_BLOCK 2
#define NEGF_TUNE_PASS1_PIECES 4
#define NEGF_TUNE_SCHEDULE 6
#define NEGF_TUNE_NN_GEMM 7
#define NEGF_SCHEDULE_TWO_PASS 1
#define NEGF_SCHEDULE_FUSED 2
/* NEGF_TUNE_NN_GEMM: the tensor-core path of negf_nn_gemm: 0 (default) or
 * NEGF_NN_GEMM_TCGEN05, the 5th-generation tensor cores (tcgen05.mma with
 * the accumulator in tensor memory) fed by the Tensor Memory Accelerator
 * where the operands allow it (16-byte aligned base and leading dimension,
 * non-overlapping batches), else by register-staged loads;
 * NEGF_NN_GEMM_TCGEN05_STAGED, the register-staged tcgen05 kernel only; or
 * NEGF_NN_GEMM_MMA_SYNC, warp-level mma.sync tiles.  All compute the same
 * BF16 x BF16 -> FP32 products; the summation order inside a K-16 step may
 * differ. */
#define NEGF_NN_GEMM_TCGEN05 1
#define NEGF_NN_GEMM_MMA_SYNC 2
#define NEGF_NN_GEMM_TCGEN05_STAGED 3
int negf_set_tuning(int key, int value);
/* Enable CUDA-event timing of negf_compute_charge (off by default). */
int negf_set_timing(int enable);

/* Real-space ring-block RGF (config shape "(13,0) with 26-atom ring
 * blocks"; the reference engine is mode space only, so this entry point has
 * no counterpart there).  Zigzag (m,0) tubes, m <= 16: blocks of two rings
 * (2m atoms) with the double bond inside a block and the single bond
 * between blocks, 2m x 2m complex FP64 blocks handled through Schur
 * complements on their m x m ring corners; the leads' ring corners from
 * the ring Fourier modes (a uniform lead decouples into the mode-space
 * chains: per-mode surface values by the analytic formula, or by the
 * decimation when the tube sets use_decimation, summed into a circulant).
 * Induced charge per ring into d_Q (device, N doubles): the tube's contour
 * and pole points with the mode-space coefficients, minus Rho0 at U = 0,
 * and for a biased tube the non-equilibrium real-axis term
 * (Compute_RhoNonEq, NEGF_Common.cpp:3115-3578): per real-axis point the
 * ring sums of the source and drain spectral functions
 * G_{n,c} Gamma_c G_{n,c}^dagger (Gamma_c = i (Sigma_c - Sigma_c^dagger) on
 * the contact ring's atoms) weighted by the mode-space coefficients, in
 * FP64.  d_Uatoms (device, [N][m]) gives per-atom potentials; null uses the
 * tube's ring potential on every atom, in which case the result equals the
 * mode-space charge with all m//2 + 1 distinct modes.  Tubes in mixed
 * precision run the contour and pole chains at least mixed_fp64_band above
 * the real axis in FP32 (m x m products on the tensor cores in TF32 with a
 * high/remainder split, the complex product in three real products); the
 * leads, the real-axis points, the Rho0 pass and the energy sum stay FP64.
 * The Rho0 pass (U = 0) does not depend on the potential: the first call for
 * a tube computes it and later calls reuse it.  Synchronous. */
int negf_rs_compute_charge(negf_tube* t, const double* d_Uatoms, double* d_Q, void* stream);

/* Surrogate-model kernels (no counterpart in the reference): the training
 * and inference kernels of the neural operator that starts the
 * self-consistent loop (electrostatic_b200/surrogate.py).  BF16 tensors are
 * passed as void* (bf16 storage), FP32 as float*; all pointers are device
 * pointers; launches are asynchronous on `stream`.
 * negf_nn_gemm: C[b] (M x N, FP32, leading dimension ldc, batch stride sC)
 * (+)= A[b] (M x K) B[b] (K x N) for b < batch; a_trans = 0: A[m][k] at
 * A + m lda + k, else at A + k lda + m; b_trans = 0: B[k][n] at B + k ldb + n,
 * else at B + n ldb + k; tensor-core mma (BF16 in, FP32 accumulate);
 * C_bf16 (optional) receives a BF16 copy of C.
 * negf_nn_gelu_fwd: pre = a + b + bias[col] (b, bias optional), out = GELU(pre)
 * (tanh form) or pre when activation = 0.  negf_nn_gelu_bwd: d = dy GELU'(pre).
 * negf_nn_colsum: column sums.  negf_nn_adam: Adam with bias correction on
 * FP32 master weights (+ BF16 copy).  negf_nn_rowdot: q[r] = h[r] . w + *b.
 * negf_nn_outer: dh[r][c] = dq[r] w[c].  negf_nn_mse: d = 2 (q - y) / n and
 * per-256-block partial sums of (q - y)^2. */
int negf_nn_gemm(int a_trans, int b_trans, int M, int N, int K, int batch, const void* A, int lda, long long sA,
                 const void* B, int ldb, long long sB, float* C, int ldc, long long sC, void* C_bf16, int accumulate,
                 void* stream);
int negf_nn_gelu_fwd(long long rows, int cols, const float* a, const float* b, const float* bias, float* pre,
                     float* out, void* out_bf16, int activation, void* stream);
int negf_nn_gelu_bwd(long long n, const float* dy, const float* pre, float* d, void* d_bf16, void* stream);
int negf_nn_colsum(long long rows, int cols, const float* x, float* out, int accumulate, void* stream);
int negf_nn_cast_bf16(long long n, const float* x, void* y, void* stream);
int negf_nn_adam(long long n, float* w, const float* g, float* m, float* v, void* w_bf16, float lr, float beta1,
                 float beta2, float eps, int step, float weight_decay, void* stream);
int negf_nn_rowdot(long long rows, int cols, const float* h, const float* w, const float* b, float* q, void* stream);
int negf_nn_outer(long long rows, int cols, const float* dq, const float* w, float* dh, void* dh_bf16, void* stream);
int negf_nn_mse(long long n, const float* q, const float* y, float* d, float* partials, void* stream);

/* Transport characteristics (c_NEGF_Common::Compute_DensityOfStates,
 * NEGF_Common.cpp:2390-2847, and Compute_Current, :4321-4816; called from
 * c_Nanostructure::PostProcess, Nanostructure.H:134-138).
 *
 * DOS path (Update_IntegrationPaths, NEGF_Common.cpp:2188-2250): the
 * non-equilibrium paths when the contacts are biased, else Gauss-Legendre on
 * [Re E_eta, E_rightmost] with flatband_dos_integration_pts points.
 * negf_compute_dos fills, per DOS energy (host arrays of
 * negf_tube_dos_points() entries): E (re, im interleaved), DOS per unit cell
 * (spin_degen * sum_sites sum_modes deg A_nn / 2pi / atoms per unit cell),
 * transmission sum_modes deg Gamma_0 Gamma_1 |G_0,N-1|^2, the conductance
 * integrand -T dF/dE (G_quantum = 1, Compute_Conductance :1873-1928) and its
 * total; ldos (optional, [E][N]) = sum_modes deg A_nn / 2pi per site.
 * negf_compute_current fills the terminal currents [A] of contacts 0 and 1
 * (2 q/h sum_E Re(w J (f_k - f_k')) T_k(E)) and optionally the integrand
 * probes [3][P] over the P = negf_tube_current_points() non-equilibrium
 * energies: 2q/h * sum_modes deg Re(Gn_nn) at n = N/2, 0, N-1 (:4684-4714).
 * Both run on the GPU and return when the host outputs are written; the
 * current is zero at zero bias. */
int negf_tube_dos_points(negf_tube* t, int* count);
int negf_tube_current_points(negf_tube* t, int* count);
int negf_compute_dos(negf_tube* t, double* E, double* dos, double* transmission, double* conductance,
                     double* total_conductance, double* ldos, void* stream);
int negf_compute_current(negf_tube* t, double* current, double* integrand, void* stream);
/* Adaptive non-equilibrium limits.  negf_tube_correct_integration_limits
 * is Update_IntegrationPaths with flag_correct_integration_limits
 * (NEGF_Common.cpp:2188-2215): the charge integrand on the current paths
 * (Compute_RhoNonEq's probe at site N/2, :3467-3542), its largest |value|
 * fixes E*, and Find_NonEq_Percent_Intercuts_Adaptively (:2062-2185) moves
 * the intercuts and point counts of 2 or 3 paths to a window of
 * kT_window_around_singularity around E*.  Solve_NEGF applies it when
 * flag_adaptive_integration_limits and iter % integrand_correction_interval
 * == 0 (:1316-1336); the caller owns that schedule.  No effect at zero bias
 * or with an explicit real-axis window.
 * negf_tube_noneq_integrand: the charge integrand probes [3][P]
 * (site N/2, N/4, 3N/4; Re(-spin/2pi sum_modes deg sum_k A^k_nn f_k)) over
 * the P current non-equilibrium energies.
 * negf_tube_noneq_layout: current path count, points per path, intercuts
 * [num_paths - 1] (percent) and E* [eV]. */
int negf_tube_correct_integration_limits(negf_tube* t, void* stream);
int negf_tube_noneq_integrand(negf_tube* t, double* integrand, void* stream);
int negf_tube_noneq_layout(negf_tube* t, int* num_paths, int* pts, double* intercuts, double* E_at_max);
/* Read_Table1D (NEGF_Common.cpp:237-285), used to initialise or restart the
 * charge from a `_Qout.dat` table (Initialize_ChargeAtFieldSites, :178-235;
 * file naming at :565-621): a header line, then `position value` per line;
 * the file must hold exactly n + 1 lines (else NEGF_ERR_IO with the
 * reference's message).  Host only. */
int negf_read_table1d(const char* filename, int n, double* values);
/* Writers with the reference's formats: transport_char.dat
 * (Write_Eql_Characteristics, NEGF_Common.cpp:1931-1975), the I.dat header
 * (Define_FileHeaderForCurrent, :69-84) and one appended I.dat line
 * (Write_Current, :4818-4840), and <step>_integrand.dat (Write_Integrand,
 * :1977-2015; integrand as returned by negf_compute_current). */
int negf_write_transport_char(negf_tube* t, const char* path, int count, const double* E, const double* dos,
                              const double* transmission, const double* conductance);
int negf_write_current_header(const char* path);
int negf_write_current(const char* path, int step, double Vds, double Vgs, const double* current,
                       double avg_intg_pts, int total_iterations, double total_conductance);
int negf_write_integrand(negf_tube* t, const char* path, int count, const double* E, const double* integrand);

/* Charge plans: the launch tables of a batch uploaded once, so that
 * negf_charge_plan_launch is kernel launches only (no allocation, no host
 * copy, no synchronisation) and can be captured in a CUDA graph.  A plan
 * with both FP64 and FP32 chains runs the FP32 ones beside the FP64 ones
 * on a side stream of the launch stream, made by the first launch (or
 * negf_compute_charge call) on that stream: make that first launch before
 * capturing the stream.  The
 * contact potentials are read on the device as U[0] and U[N-1] of each
 * tube's potential buffer (U_contact = U at the end sites,
 * Nanostructure.cpp:500-504).  d_Q: device output of sum N doubles (tube
 * order).  With NEGF_PLAN_AUTOTUNE the fused (warp per chain) schedule and
 * every two-pass (segment tile) schedule -- segments per unit 16/32/64 x
 * pass-2 warps per block 1/2/4, and, when the chains fill fewer than 4 warps
 * per SM, pass-1 pieces 1/2/4/8/automatic (parallel in length) -- are timed
 * on the batch and the fastest is kept (results agree to rounding; bitwise
 * within the two-pass shapes of one piece count).  Without it the schedule
 * and the pieces follow NEGF_TUNE_SCHEDULE's and NEGF_TUNE_PASS1_PIECES's
 * rules, as in negf_compute_charge.
 * negf_charge_plan_info's *pass2_warps_per_block is 0 when the fused
 * schedule was chosen.  A plan is stale (NEGF_ERR_STATE at
 * launch) once a tube's energy paths change (contact mu, adaptive limits);
 * d_skip (device int or null) skips the launch at kernel entry when set. */
#define NEGF_PLAN_AUTOTUNE 1
#define NEGF_PLAN_FP64 2     /* every chain in FP64 whatever the tubes' precision mode */
typedef struct negf_charge_plan negf_charge_plan;
int negf_charge_plan_create(negf_tube* const* tubes, int num_tubes, double* d_Q, int flags, negf_charge_plan** plan);
int negf_charge_plan_launch(negf_charge_plan* plan, const int* d_skip, void* stream);
int negf_charge_plan_info(const negf_charge_plan* plan, int* pass2_warps_per_block, int* segs_per_unit,
                          double* tuned_ms, long long* updates);
/* Pass-1 pieces of the plan's schedule (1 for the fused schedule). */
int negf_charge_plan_pieces(const negf_charge_plan* plan, int* pieces);
int negf_charge_plan_destroy(negf_charge_plan* plan);

/* Broyden modified-second mixing (Transport.H:203-208):
 * Set_Broyden_Parallel (Broyden_Parallel_General.cpp:68-248),
 * Execute_Broyden_Modified_Second_Algorithm_Parallel
 * (Broyden_Second_Parallel.cpp:213-486), Reset_Broyden_Parallel
 * (Broyden_Parallel_General.cpp:250-355).  All vectors live on the device. */
int negf_broyden_create(int num_sites, int max_step, double fraction, int norm_type, negf_broyden** out);
int negf_broyden_destroy(negf_broyden* b);
/* Initial input charge n_in (device or host pointer). */
int negf_broyden_set_input(negf_broyden* b, const double* n_in, int on_device, void* stream);
/* One mixing step with n_out (device pointer): updates the internal n_in and
 * copies it to d_n_in_out (device, may be NULL); *max_norm receives
 * Broyden_Norm (max over sites of the abs/rel residual of this step's input)
 * and d_norm (device, may be NULL) the per-site norm.  *status is 0, or 1 when
 * the step count would exceed max_step (the reference aborts there). */
int negf_broyden_step(negf_broyden* b, const double* d_n_out, double* d_n_in_out, double* d_norm,
                      double* max_norm, int* status, void* stream);
/* Reset for the next bias step; keep_charge mirrors
 * reset_with_previous_charge_distribution, otherwise n_in = init_value. */
int negf_broyden_reset(negf_broyden* b, int keep_charge, double init_value, void* stream);
/* Initial inverse Jacobian for the next solve (no counterpart in the
 * reference, whose loop starts from simple mixing G0 = fraction * I,
 * Broyden_Parallel_General.cpp:68-248): G0 = fraction * I + sum_j w_j v_j^T
 * for the k rows d_V[j][S], d_W[j][S] (device), so the first step gives
 * n_in - scalar * G0 F and later steps add their own rows after these.
 * Rows built from secant pairs (dn_j, dF_j) of a cheaper model, as the
 * method builds its own (v = dF/|dF|^2, w = -fraction dF + dn - sum_{i<j}
 * w_i (v_i . dF)), let a surrogate supply the starting Jacobian.  Call after
 * create or reset and before the first step; k <= max_step / 2, and the k
 * rows count against max_step.  A reset clears them.  The row count lives
 * in device memory, so launches captured earlier see it. */
int negf_broyden_set_initial_jacobian(negf_broyden* b, const double* d_V, const double* d_W, int k, void* stream);
/* Start the next solve keeping the secant rows of the solves so far as its
 * initial inverse Jacobian (no counterpart in the reference, whose
 * Reset_Broyden_Parallel clears them, Broyden_Parallel_General.cpp:250-355):
 * the next step is step 1 and G0 = fraction * I + sum_j w_j v_j^T over all
 * rows held, if there are at most min(keep_rows, max_step / 2) of them, else
 * over none (each row corrects the rows before it, so dropping the oldest
 * rows would leave no consistent inverse Jacobian).  Along a bias sweep the
 * Jacobian changes little from one bias point to the next, so the rows carry
 * over.  n_in stays (set a new start with negf_broyden_set_input); the kept
 * rows count against max_step.
 * Synchronises `stream` (it reads the step counters). */
int negf_broyden_restart(negf_broyden* b, int keep_rows, void* stream);
/* Per-segment secant updates (no counterpart in the reference, whose one
 * Broyden mixes the sites of all nanostructures with whole-vector dot
 * products, Broyden_Second_Parallel.cpp:213-486): the sites split into nseg
 * segments, offsets[0] = 0 < offsets[1] < ... < offsets[nseg] = num_sites
 * (host array), and every dot product of the update (V^T dF, V^T F and the
 * dF^T dF of a new row) runs over each segment's sites separately.  The
 * update is then block diagonal: nseg independent Broyden mixers in one
 * set of launches, which suits a batch of tubes whose potentials do not
 * couple (one segment per tube).  The norm and the stopping rule stay over
 * all sites.  nseg = 1 restores the whole-vector update.  Call after create
 * or reset, before seeding rows and before the first step; the setting
 * survives resets and restarts.  Synchronises the device. */
int negf_broyden_set_segments(negf_broyden* b, int nseg, const int* offsets, void* stream);
/* The secant rows held now (seeded rows first): device pointers of rows
 * 1 .. *rows of V and W ([rows][S] each, valid until the next step, reset or
 * restart), e.g. to seed another Broyden with negf_broyden_set_initial_jacobian
 * (no counterpart in the reference).  Synchronises `stream`. */
int negf_broyden_history(negf_broyden* b, double** d_V, double** d_W, int* rows, void* stream);
/* Broyden_Step (1-based). */
int negf_broyden_step_number(negf_broyden* b, int* step);
/* Device-resident Broyden step (no host synchronisation; capturable in a
 * CUDA graph).  d_flags: int[4] in device memory, zeroed by the caller at
 * the start of a solve: [0] converged (norm <= max_norm, the loop predicate
 * of Transport.cpp:385-505), [1] steps taken, [2] error (1: the step count
 * passed max_step, Transport.cpp:389-393; 2: non-finite norm), [3] skip
 * (= [0] or [2]).  Once [3] is set, this call and every *_masked / plan
 * launch given d_flags + 3 returns at kernel entry, so a captured sequence
 * of iterations stops itself.  The iteration index is read on the device. */
int negf_broyden_step_device(negf_broyden* b, const double* d_n_out, double max_norm, int* d_flags, void* stream);
/* Precision switching (no counterpart in the reference): d_flags int[8],
 * initialised by the caller to {0,0,0,0, 0,0,1,0}.  Until the first norm
 * below switch_norm the charge is taken to come from a low-precision plan
 * (launched with skip word d_flags + 5); from then on from an FP64 plan
 * (skip word d_flags + 6), and only an FP64 charge can satisfy max_norm.
 * [4] is set at the switch; [7] counts the steps taken on low-precision
 * charges. */
int negf_broyden_step_device_switch(negf_broyden* b, const double* d_n_out, double max_norm, double switch_norm,
                                    int* d_flags, void* stream);
/* Device pointer of the current input charge n_in. */
int negf_broyden_input_device_ptr(negf_broyden* b, double** d_n_in);

/* Device self-test of the kernels' numeric primitives (no counterpart in the
 * reference): which = 0 FP64 reciprocal, 1 FP32 reciprocal (n values in, n
 * out); real-space tile primitives on count m x m complex matrices (m = 4,
 * 13 or 16; in = [m, count, data], out = [m, count, results], complex values
 * re/im interleaved, row-major): 2 / 3 inverse in FP64 / FP32 (data: count
 * matrices; a NaN result marks a zero pivot), 4 / 5 product A B on the FP64
 * cores / FP32 tensor cores (data: count pairs A, B). */
int negf_device_selftest(int which, int n, const double* in, double* out);

/* Affine electrostatics stand-in used by the SCF harness:
 * d_U[i] = d_U0[i] + sum_j K[i*n + j] * d_Q[j]   (all device pointers). */
int negf_affine_potential_masked(const double* K, const double* U0, const double* Q, double* U, int n,
                                 const int* d_skip, void* stream);
int negf_affine_potential(const double* d_K, const double* d_U0, const double* d_Q, double* d_U, int n,
                          void* stream);
/* The same operator when K depends on the lattice distance only
 * (K[i][j] = tab[|idx[i] - idx[j]|], the sites on an integer lattice idx, as
 * the rings of a zigzag tube are): d_U[i] = d_U0[i] + sum_j tab[|idx[i] -
 * idx[j]|] d_Q[j], entries at distances >= ntab read as 0 (device pointers;
 * no n x n matrix is read). */
int negf_affine_potential_toeplitz(const double* d_tab, int ntab, const int* d_idx, const double* d_U0,
                                   const double* d_Q, double* d_U, int n, const int* d_skip, void* stream);
/* The lattice-distance update of a batch of tubes in one launch: tube t
 * writes d_U[t][i] = d_U0[t][i] + sum_j d_tab[t][|d_idx[t][i] - d_idx[t][j]|]
 * d_Q[t][j] for its n[t] sites (host arrays of device pointers, read once at
 * create; the launch reads the buffers they point to, so it can be captured
 * and replayed as the buffers change).  No counterpart in the reference. */
typedef struct negf_potential_batch negf_potential_batch;
int negf_potential_batch_create(int ntubes, const double* const* d_tab, const int* ntab, const int* const* d_idx,
                                const double* const* d_U0, const double* const* d_Q, double* const* d_U, const int* n,
                                negf_potential_batch** out);
int negf_potential_batch_launch(negf_potential_batch* b, const int* d_skip, void* stream);
int negf_potential_batch_destroy(negf_potential_batch* b);

/* Write_Data (NEGF_Common.cpp:1407-1418, 3043-3112, 4221-4254):
 * <prefix>_Qout.dat, <prefix>_norm.dat (axial position [nm], value; one
 * header line; precision 15) and <prefix>_U.dat (index, position, U).
 * Q and norm are host pointers of num_sites values (norm may be NULL). */
int negf_write_step(negf_tube* t, const char* prefix, const double* Q, const double* norm);

/* Message of the last failed call on this thread ("" if none). */
const char* negf_last_error(void);

#ifdef __cplusplus
}
#endif
#endif /* NEGF_B200_H_ */
