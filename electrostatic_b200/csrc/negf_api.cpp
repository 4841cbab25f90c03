// Host layer of the B200 NEGF engine: the C-ABI declared in include/negf_b200.h.
//
// Mirrors the charge-path interface of c_NEGF_Common<T> / c_CNT
// (Source/Solver/Transport/NEGF/NEGF_Common.H:518-606, CNT.H:13-103) and the
// Broyden interface of c_TransportSolver (Transport.H:203-208).  Physics set-up
// (modes, Hamiltonian constants, energy limits, integration paths, Fermi
// factors) runs here in FP64; every per-site, per-energy operation runs in the
// CUDA kernels of negf_rgf.cu / negf_broyden.cu.  There is no CPU compute path.

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstring>
#include <atomic>
#include <map>
#include <memory>
#include <mutex>
#include <numeric>
#include <string>
#include <vector>

#include "../../include/negf_b200.h"
#include "negf_internal.h"

using cplx = std::complex<double>;

namespace {

constexpr double kPi = 3.14159265358979323846;
constexpr double kKbEvPerK = 8.617333262e-5;  // Utils/SelectWarpXUtils/WarpXConst.H:61-62
constexpr double kSpinDegen = 2.0;            // NEGF_Common.H:351
constexpr double kQe = 1.602176634e-19;       // Utils/SelectWarpXUtils/WarpXConst.H
constexpr double kHeVperHz = 4.135667696e-15; // Utils/SelectWarpXUtils/WarpXConst.H:33

thread_local std::string g_err;

int fail(int code, const std::string& msg) {
    g_err = msg;
    return code;
}

#define NEGF_CUDA(call)                                                                             \
    do {                                                                                            \
        cudaError_t e_ = (call);                                                                    \
        if (e_ != cudaSuccess)                                                                      \
            return fail(NEGF_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));         \
    } while (0)

// ------------------------------------------------------------------ quadrature
// Gauss-Legendre nodes/weights on [-1, 1] by Newton iteration on P_n from the
// Chebyshev-like initial guess cos(pi (i - 1/4) / (n + 1/2)), stopping when the
// Newton step is below 3e-11 -- the published "gauleg" scheme that
// Utils/CodeUtils/CodeUtil.cpp:640-690 uses, so the energy grids coincide.
void gauss_legendre(int n, std::vector<double>& x, std::vector<double>& w) {
    x.assign(n, 0.0);
    w.assign(n, 0.0);
    for (int i = 1; i <= (n + 1) / 2; ++i) {
        double z = std::cos(kPi * (i - 0.25) / (n + 0.5)), step, dp;
        do {
            double p = 1.0, pm1 = 0.0;
            for (int j = 1; j <= n; ++j) {
                const double pm2 = pm1;
                pm1 = p;
                p = ((2.0 * j - 1.0) * z * pm1 - (j - 1.0) * pm2) / j;
            }
            dp = n * (z * p - pm1) / (z * z - 1.0);
            step = p / dp;
            z -= step;
        } while (std::fabs(step) > 3.0e-11);
        x[i - 1] = -z;
        x[n - i] = z;
        w[i - 1] = w[n - i] = 2.0 / ((1.0 - z * z) * dp * dp);
    }
}

struct Pt {
    cplx E, w, J;
};

// IntegrationPath.cpp:41-147: line (id 0) or circular arc through both end
// points with centre on Im = Im(max) (id 1), Gauss-Legendre in the parameter.
void gl_path(cplx a, cplx b, int n, int id, std::vector<Pt>& out) {
    if (n <= 0) return;
    std::vector<double> x, w;
    gauss_legendre(n, x, w);
    if (id == 0) {
        const cplx half = (b - a) * 0.5, mid = (b + a) * 0.5;
        for (int i = 0; i < n; ++i) out.push_back({half * x[i] + mid, w[i], half});
        return;
    }
    const double cr = (b.real() * b.real() - a.real() * a.real() - a.imag() * a.imag()) / (2 * (b.real() - a.real()));
    const double R = cr - b.real();
    double t1 = std::asin(std::fabs(a.imag()) / R);
    if (cr > a.real()) t1 = kPi - t1;
    const double t2 = kPi;
    for (int i = 0; i < n; ++i) {
        const double th = (t2 - t1) * 0.5 * x[i] + (t2 + t1) * 0.5;
        const cplx E(cr + R * std::cos(th), b.imag() + R * std::sin(th));
        const cplx J = (t2 - t1) * 0.5 * R * std::exp(cplx(0.0, th)) * cplx(0.0, 1.0);
        out.push_back({E, w[i], J});
    }
}

// IntegrationPath.cpp:149-168: uniform points, weight dE, factor 1.
void regular_path(cplx a, cplx b, int n, std::vector<Pt>& out) {
    if (n <= 0) return;
    if (n == 1) {
        out.push_back({a, b - a, 1.0});
        return;
    }
    const cplx dE = (b - a) / double(n - 1);
    for (int i = 0; i < n; ++i) out.push_back({a + double(i) * dE, dE, 1.0});
}

// NEGF_Common.cpp:1790-1795
cplx fermi(cplx EmMu, double kT) { return 1.0 / (std::exp(EmMu / kT) + 1.0); }

struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
    ~DevBuf() {
        if (p) cudaFree(p);
    }
    cudaError_t reserve(size_t b) {
        if (b <= bytes) return cudaSuccess;
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
        cudaError_t e = cudaMalloc(&p, b);
        if (e == cudaSuccess) bytes = b;
        return e;
    }
    template <typename T>
    T* as() const {
        return static_cast<T*>(p);
    }
};

struct ChainTable {
    std::vector<negf::ChainRec> chains;
    std::vector<negf::WarpRec> warps;
    std::vector<negf::ReduceTube> rts;
    std::vector<negf::SegUnit> units;
    std::vector<int> order;  // fused schedule: FP64 warps, then FP32 warps
    int n64 = 0, n32 = 0;
    long long partial_doubles = 0, scratch_doubles = 0;
    long long updates = 0, updates_fp32 = 0, contour_updates = 0, realaxis_updates = 0;
    int max_N = 0;
};

}  // namespace

struct negf_tube {
    negf_tube_desc d;
    int device = 0;
    // material (CNT.cpp:23-41, 155-292)
    double R = 0.0;
    int rings_per_uc = 4, atoms_per_ring = 17, N = 0;
    std::vector<int> modeJ, degen;
    std::vector<double> beta, gaps, y_nm;
    // potential
    double Uc[2] = {0.0, 0.0};
    double* d_U = nullptr;     // interior of d_U_pad: N sites
    double* d_zero = nullptr;  // interior of d_zero_pad
    double* d_U_pad = nullptr;  // kPadLo zeros, N sites, kPadHi zeros
    double* d_zero_pad = nullptr;
    double* d_rho0 = nullptr;
    double* d_rs_rho0 = nullptr;  // real-space Rho0 per ring (U = 0), made by the first real-space call
    // contacts / limits (NEGF_Common.cpp:1687-1787)
    double mu[2] = {0.0, 0.0}, kT[2] = {0.0, 0.0};
    double kT_min = 0, kT_max = 0, mu_min = 0, mu_max = 0;
    bool noneq = false, limits_dirty = true;
    cplx E_left, E_right, E_rightmost, E_zeta, E_eta;
    std::vector<Pt> eq_pts, noneq_pts, rho0_pts;
    std::vector<cplx> poles;
    int version = 0;
    long long serial = 0;  // unique per tube of the process (keys the cached launch tables)
    int shard_rank = 0, shard_world = 1;
    // adaptive non-equilibrium limits (NEGF_Common.H:453-457)
    double E_at_max_noneq_integrand = 0.0;
    ~negf_tube() {
        if (d_U_pad) cudaFree(d_U_pad);
        if (d_zero_pad) cudaFree(d_zero_pad);
        if (d_rho0) cudaFree(d_rho0);
        if (d_rs_rho0) cudaFree(d_rs_rho0);
    }
};

struct negf_broyden {
    negf::BroydenDev dev{};
    int step = 1;
    int device = 0;
    ~negf_broyden() {
        double* bufs[] = {dev.n_in, dev.n_prev, dev.F, dev.dF, dev.norm, dev.V, dev.W, dev.c, dev.sum, dev.scal, dev.part,
                          dev.dd};
        for (double* p : bufs)
            if (p) cudaFree(p);
        if (dev.step_dev) cudaFree(dev.step_dev);
        if (dev.seg_off) cudaFree(dev.seg_off);
        if (dev.seg_of) cudaFree(dev.seg_of);
    }
};

struct negf_charge_plan {
    std::vector<negf_tube*> tubes;
    std::vector<int> versions;
    DevBuf d_tubes, d_chains, d_warps, d_units, d_rts, d_partial, d_scratch, d_order, d_pieces;
    int num_warps = 0, num_units = 0, max_N = 0;
    int pieces = 1;  // pass-1 pieces of the two-pass schedule (parallel in length)
    int n64 = 0, n32 = 0;  // fused schedule: FP64 / FP32 warps in d_order
    cudaEvent_t fork = nullptr, join = nullptr;  // around the FP32 warps on the launch stream's side stream
    ~negf_charge_plan() {
        if (fork) cudaEventDestroy(fork);
        if (join) cudaEventDestroy(join);
    }
    int wpb = 4, spu = negf::kSegsPerUnit;
    int schedule = 0;  // negf::kScheduleTwoPass or kScheduleFused
    double* d_Q = nullptr;
    long long updates = 0;
    double tuned_ms = 0.0;
    bool force_fp64 = false;
};

namespace {

std::mutex g_mu;

// Device buffers and the cached launch table of the charge calls made on one
// (device, stream) pair.  Calls on the same stream are ordered by the stream;
// calls on different streams or devices get different workspaces, so their
// kernels never share scratch.  A workspace is reused only after the last
// kernel of its previous call (event `done`), which also orders a stream
// handle that the runtime hands out again after the caller destroyed the
// stream it first named.
struct Workspace {
    int device = 0;
    cudaStream_t stream = nullptr;
    DevBuf tubes, chains, warps, rts, units, partial, scratch, qbuf, pieces, order;
    cudaStream_t side = nullptr;                 // the FP32 warps of the fused schedule
    cudaEvent_t fork = nullptr, join = nullptr;  // around them
    // real-space pass (negf_rs_compute_charge)
    DevBuf rsE, rsFlags, rsU0, rsUa, rsCorners, rsGL, rsGLn, rsRows, rsStatus;
    // cached chain table
    std::vector<long long> key_serials;
    std::vector<int> key_versions;
    ChainTable table;
    bool table_valid = false;
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};  // timing of the last call
    cudaEvent_t done = nullptr;                                 // end of the last call's kernels
    bool used = false;
    ~Workspace() {
        // buffers belong to `device`; free them with it current
        int cur = -1;
        if (cudaGetDevice(&cur) == cudaSuccess && cur != device) cudaSetDevice(device);
        for (cudaEvent_t& e : ev)
            if (e) cudaEventDestroy(e);
        if (done) cudaEventDestroy(done);
        if (fork) cudaEventDestroy(fork);
        if (join) cudaEventDestroy(join);
        if (side) cudaStreamDestroy(side);
        DevBuf* bufs[] = {&tubes, &chains, &warps, &rts,  &units, &partial,   &scratch, &qbuf,   &pieces,
                          &order, &rsE,    &rsFlags, &rsU0, &rsUa, &rsCorners, &rsGL,    &rsGLn,  &rsRows,
                          &rsStatus};
        for (DevBuf* b : bufs) {
            if (b->p) cudaFree(b->p);
            b->p = nullptr;
        }
        if (cur >= 0 && cur != device) cudaSetDevice(cur);
    }
};

// Process-wide settings and the statistics of the last charge call.
struct Settings {
    bool timing = false;
    int warps_per_block = 4;
    int pass1_pieces = 0;  // 0: automatic
    int schedule = 0;      // 0: automatic, else NEGF_SCHEDULE_*
    int nn_gemm = 0;       // 0: default (tcgen05), else NEGF_NN_GEMM_*
    negf_stats stats{};
    Workspace* stats_ws = nullptr;  // workspace whose events time the last call (when timing)
};
Settings& settings() {
    static Settings s;
    return s;
}

struct WsKey {
    int device;
    cudaStream_t stream;
    bool operator<(const WsKey& o) const {
        return device != o.device ? device < o.device : std::less<cudaStream_t>()(stream, o.stream);
    }
};

std::map<WsKey, std::unique_ptr<Workspace>>& workspaces() {
    static std::map<WsKey, std::unique_ptr<Workspace>> all;
    return all;
}

// Workspace of the current device and `stream`, made on first use (callers
// hold g_mu).
int find_workspace(cudaStream_t stream, Workspace** out) {
    int dev = 0;
    NEGF_CUDA(cudaGetDevice(&dev));
    std::unique_ptr<Workspace>& w = workspaces()[WsKey{dev, stream}];
    if (!w) {
        w.reset(new Workspace());
        w->device = dev;
        w->stream = stream;
        NEGF_CUDA(cudaEventCreateWithFlags(&w->done, cudaEventDisableTiming));
        NEGF_CUDA(cudaEventCreateWithFlags(&w->fork, cudaEventDisableTiming));
        NEGF_CUDA(cudaEventCreateWithFlags(&w->join, cudaEventDisableTiming));
        NEGF_CUDA(cudaStreamCreateWithFlags(&w->side, cudaStreamNonBlocking));
    }
    *out = w.get();
    return NEGF_OK;
}

// The same, waiting on the stream for the previous call that used it.
int get_workspace(cudaStream_t stream, Workspace** out) {
    if (int rc = find_workspace(stream, out)) return rc;
    if ((*out)->used) NEGF_CUDA(cudaStreamWaitEvent(stream, (*out)->done, 0));
    return NEGF_OK;
}

// Side stream for the FP32 warps of a charge plan launched on `stream`: the
// one of that stream's workspace (callers hold g_mu).  One side stream per
// (device, launch stream), shared with negf_compute_charge on that stream,
// instead of one per plan: the block scheduler's interleaving of the two
// concurrent fused kernels came out differently for different side streams
// (config-4 batch with FP32 real axis: 1.59 or 1.80 ms per pass from one
// plan to the next); with the launch stream's side stream it was 1.59 ms
// in every run measured.
int plan_side_stream(cudaStream_t stream, cudaStream_t* side) {
    Workspace* w = nullptr;
    if (int rc = find_workspace(stream, &w)) return rc;
    *side = w->side;
    return NEGF_OK;
}

// Every tube of a batch must live on the current device (its buffers were
// allocated there by negf_tube_create).
int check_batch_device(negf_tube* const* tubes, int num_tubes) {
    int dev = 0;
    NEGF_CUDA(cudaGetDevice(&dev));
    for (int i = 0; i < num_tubes; ++i)
        if (tubes[i] && tubes[i]->device != dev)
            return fail(NEGF_ERR_ARG, "tube " + std::to_string(i) + " lives on device " +
                                          std::to_string(tubes[i]->device) + " but device " + std::to_string(dev) +
                                          " is current: every tube of a call must be on the current device");
    return NEGF_OK;
}

int require_device() {
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n == 0)
        return fail(NEGF_ERR_CUDA, std::string("no CUDA device available: ") +
                                       (e == cudaSuccess ? "device count is 0" : cudaGetErrorString(e)));
    return NEGF_OK;
}

// ------------------------------------------------------------------ material
double bandgap_of_mode(const negf_tube& t, int p) {  // CNT.cpp:155-176
    const int m = t.d.type_id[0], n = t.d.type_id[1];
    const double f = t.d.acc * t.d.gamma / t.R;
    const double c[6] = {std::fabs(3.0 * p - (2 * m + n)),  std::fabs(3.0 * p - (m + 2 * n)),
                         std::fabs(3.0 * p - (m - n)),       std::fabs(-3.0 * p + (2 * m + n)),
                         std::fabs(-3.0 * p + (m + 2 * n)),  std::fabs(3.0 * p - (m - n))};
    double best = f * c[0];
    for (int i = 1; i < 6; ++i) best = std::min(best, f * c[i]);
    return best;
}

// Sort of mode gaps.  The reference sorts with a last-element-pivot quicksort
// (CNT.cpp:178-225) whose tie order decides which J represents a degenerate
// pair; the same partition scheme is used so the representative J matches.
void sort_modes(std::vector<double>& v, std::vector<int>& id, int lo, int hi) {
    while (lo < hi) {
        const double pivot = v[hi];
        int j = lo;
        for (int i = lo; i <= hi; ++i)
            if (!(v[i] > pivot)) {
                std::swap(v[i], v[j]);
                std::swap(id[i], id[j]);
                ++j;
            }
        const int pos = j - 1;
        sort_modes(v, id, lo, pos - 1);
        lo = pos + 1;
    }
}

int setup_material(negf_tube& t) {
    const int m = t.d.type_id[0], n = t.d.type_id[1];
    if (m <= 0 || n < 0) return fail(NEGF_ERR_ARG, "type_id must be (m>0, n>=0)");
    if (t.d.num_unitcells <= 0) return fail(NEGF_ERR_ARG, "num_unitcells must be > 0");
    t.R = t.d.acc * std::sqrt(3.0 * (double(m) * m + double(n) * n + double(m) * n)) / (2.0 * kPi);
    if (n == 0) {
        t.rings_per_uc = 4;
        t.atoms_per_ring = m;
    } else {
        t.rings_per_uc = 2;
        t.atoms_per_ring = m - 1;
    }
    t.N = t.d.num_unitcells * t.rings_per_uc;
    std::vector<double> eg(t.atoms_per_ring);
    std::vector<int> idx(t.atoms_per_ring);
    for (int p = 1; p <= t.atoms_per_ring; ++p) {
        eg[p - 1] = bandgap_of_mode(t, p);
        idx[p - 1] = p;
    }
    sort_modes(eg, idx, 0, t.atoms_per_ring - 1);
    std::vector<int> J{idx[0]}, dg{1};
    std::vector<double> gp{eg[0]};
    for (int p = 1; p < t.atoms_per_ring; ++p) {  // distinct gaps, CNT.cpp:256-270
        if (eg[p] - gp.back() > 1e-6) {
            J.push_back(idx[p]);
            gp.push_back(eg[p]);
            dg.push_back(1);
        } else {
            dg.back() += 1;
        }
    }
    const int M = t.d.num_modes;
    if (M <= 0 || M > (int)J.size() || M > negf::kMaxModes)
        return fail(NEGF_ERR_ARG, "num_modes must be in [1, " + std::to_string(std::min<int>(J.size(), negf::kMaxModes)) +
                                      "] for this chirality");
    for (int j = 0; j < M; ++j) {
        t.modeJ.push_back(J[j]);
        t.degen.push_back(dg[j]);
        t.gaps.push_back(gp[j]);
        t.beta.push_back(2.0 * t.d.gamma * std::cos(kPi * J[j] / m));  // CNT.cpp:288-292
    }
    // axial ring positions, CNT.cpp:93-132 (atom 0 of each ring), in nm
    const double acc = t.d.acc;
    const double y0 = -(t.d.num_unitcells / 2.0) * 3.0 * acc - acc / 2.0;
    const double ring_y[4] = {acc, 1.5 * acc, 2.5 * acc, 3.0 * acc};
    t.y_nm.resize(t.N);
    for (int r = 0; r < t.N; ++r) {
        const int uc = r / t.rings_per_uc;
        const int k = r % t.rings_per_uc;
        const double y = (k < 4 ? ring_y[k] : 0.0) + 3 * acc * uc + y0;
        t.y_nm[r] = y / 1.e-9;
    }
    return NEGF_OK;
}

// ------------------------------------------------------------------ limits and paths
// Define_EnergyLimits, NEGF_Common.cpp:1687-1787.
void energy_limits(const negf_tube_desc& d, const double mu_in[2], double& kT_min, double& kT_max, double& mu_min,
                   double& mu_max, double kT[2], bool& noneq, cplx& E_left, cplx& E_right, cplx& E_rightmost,
                   cplx& E_zeta, cplx& E_eta, std::vector<cplx>& poles, bool window) {
    for (int c = 0; c < 2; ++c) kT[c] = kKbEvPerK * d.contact_T[c];
    mu_min = std::min(mu_in[0], mu_in[1]);
    mu_max = std::max(mu_in[0], mu_in[1]);
    kT_min = std::min(kT[0], kT[1]);
    kT_max = std::max(kT[0], kT[1]);
    noneq = std::fabs(mu_min - mu_max) > 1e-8 || std::fabs(kT_min - kT_max) > 0.01 || window;
    const cplx zp(0.0, d.E_zPlus_imag);
    E_left = d.E_valence_min + zp;
    E_rightmost = mu_max + d.Fermi_tail_factors[1] * kT_max + zp;
    const int num_poles = int((d.E_pole_max - kPi * kT_max) / (2.0 * kPi * kT_max) + 1);
    poles.clear();
    if (noneq) {
        E_right = mu_min - d.Fermi_tail_factors[0] * kT_max + zp;
        if (window) {
            E_right = cplx(d.realaxis_min, d.E_zPlus_imag);
            E_rightmost = cplx(d.realaxis_max, d.E_zPlus_imag);
        }
        E_zeta = cplx(E_right.real(), 2 * num_poles * kPi * kT_max);
        E_eta = cplx(E_right.real() - 14 * kT_max, E_zeta.imag());
    } else {
        E_right = E_rightmost;
        for (int p = 0; p < num_poles; ++p) poles.push_back(cplx(mu_min, kPi * kT_max * (2 * p + 1)));
        E_zeta = cplx(E_right.real(), 2 * num_poles * kPi * kT_max);
        const double tf = std::max(d.Fermi_tail_factors[0], d.Fermi_tail_factors[1]);
        E_eta = cplx(mu_min - tf * kT_max, E_zeta.imag());
    }
}

void update_paths(negf_tube& t) {
    if (!t.limits_dirty) return;
    const bool window = t.d.realaxis_pts > 0;
    energy_limits(t.d, t.mu, t.kT_min, t.kT_max, t.mu_min, t.mu_max, t.kT, t.noneq, t.E_left, t.E_right,
                  t.E_rightmost, t.E_zeta, t.E_eta, t.poles, window);
    // Update_IntegrationPaths, NEGF_Common.cpp:2188-2250
    t.eq_pts.clear();
    gl_path(t.E_right, t.E_zeta, t.d.eq_integration_pts[0], 0, t.eq_pts);
    gl_path(t.E_zeta, t.E_eta, t.d.eq_integration_pts[1], 0, t.eq_pts);
    gl_path(t.E_eta, t.E_left, t.d.eq_integration_pts[2], 1, t.eq_pts);
    t.noneq_pts.clear();
    if (t.noneq) {
        if (window) {
            if (t.d.realaxis_kind == 0)
                regular_path(t.E_right, t.E_rightmost, t.d.realaxis_pts, t.noneq_pts);
            else
                gl_path(t.E_right, t.E_rightmost, t.d.realaxis_pts, 0, t.noneq_pts);
        } else {  // Generate_NonEq_Paths, NEGF_Common.cpp:2018-2059
            const int np = std::max(1, t.d.num_noneq_paths);
            std::vector<cplx> mn(np), mx(np);
            mn[0] = t.E_right;
            mx[np - 1] = t.E_rightmost;
            const cplx len = t.E_rightmost - t.E_right;
            for (int p = 0; p < np - 1; ++p) {
                const double cut = t.d.noneq_percent_intercuts[0] < 0 ? (p + 1) * (100. / np)
                                                                       : t.d.noneq_percent_intercuts[p];
                mx[p] = t.E_right + (cut / 100.0) * len;
            }
            for (int p = 1; p < np; ++p) mn[p] = mx[p - 1];
            for (int p = 0; p < np; ++p) gl_path(mn[p], mx[p], t.d.noneq_integration_pts[p], 0, t.noneq_pts);
        }
    }
    t.limits_dirty = false;
    t.version++;
}

// Rho0 paths: Define_IntegrationPaths (NEGF_Common.cpp:1798-1806) with the
// limits of initialisation time (mu = 0, no window).
void rho0_paths(negf_tube& t) {
    const double mu0[2] = {0.0, 0.0};
    double kT[2], kTmin, kTmax, mumin, mumax;
    bool noneq;
    cplx L, Rr, Rm, Z, H;
    std::vector<cplx> poles;
    energy_limits(t.d, mu0, kTmin, kTmax, mumin, mumax, kT, noneq, L, Rr, Rm, Z, H, poles, false);
    t.rho0_pts.clear();
    const cplx zp(0.0, t.d.E_zPlus_imag);
    gl_path(zp, Z, 30, 0, t.rho0_pts);
    gl_path(Z, H, 30, 0, t.rho0_pts);
    gl_path(H, L, 30, 1, t.rho0_pts);
}

// ------------------------------------------------------------------ chain tables
struct TubePass {
    const negf_tube* t;
    int tube_index;    // index in the launch's TubeDev array
    long long q_off;   // offset of the tube's sites in Q
    bool rho0_pass;    // Rho0 (zero potential) instead of the charge pass
};

// Append-only output used by the chain-table builder: a growing std::vector
// (negf_compute_charge) or a fixed caller-provided array (the
// allocation-free entry point; overflow is reported, never allocated).
template <class T>
struct Out {
    std::vector<T>* vec = nullptr;
    T* arr = nullptr;
    size_t cap = 0, n = 0;
    bool overflow = false;
    void push(const T& v) {
        if (vec) {
            vec->push_back(v);
            ++n;
        } else if (n < cap) {
            arr[n++] = v;
        } else {
            overflow = true;
        }
    }
    T& at(size_t i) { return vec ? (*vec)[i] : arr[i]; }
    size_t size() const { return n; }
};

struct TableCounts {
    long long updates = 0, updates_fp32 = 0, contour_updates = 0, realaxis_updates = 0;
    long long partial_doubles = 0, scratch_doubles = 0;
    int max_N = 0;
};

// Energy point idx of a pass.  Contour chains: Im(c G) with
// c = (-2/pi) w J f_eq (RhoEq, NEGF_Common.cpp:3738-3754), (-2/pi) w J
// (Rho0, :4071-4084) or -4 i kT (poles, :3934-3948).  Real-axis chains:
// b_k = Re((-1/pi) w J f_k) (RhoNonEq, :3372-3466).  The degeneracy and
// Gamma_k are applied in the kernel.
struct Item {
    cplx E, c;
    double b0, b1;
    int kind;
};
int pass_items(const negf_tube& t, bool rho0_pass) {
    return rho0_pass ? (int)t.rho0_pts.size() : (int)(t.eq_pts.size() + t.poles.size() + t.noneq_pts.size());
}
Item pass_item(const negf_tube& t, bool rho0_pass, int idx) {
    if (rho0_pass) {
        const Pt& p = t.rho0_pts[idx];
        return {p.E, (-kSpinDegen / kPi) * p.w * p.J, 0, 0, negf::kContour};
    }
    const int ne = (int)t.eq_pts.size(), np = (int)t.poles.size();
    if (idx < ne) {
        const Pt& p = t.eq_pts[idx];
        return {p.E, (-kSpinDegen / kPi) * p.w * p.J * fermi(p.E - t.mu_min, t.kT_min), 0, 0, negf::kContour};
    }
    if (idx < ne + np) return {t.poles[idx - ne], cplx(0.0, -2 * t.kT_min * kSpinDegen), 0, 0, negf::kContour};
    const Pt& p = t.noneq_pts[idx - ne - np];
    const cplx base = (-kSpinDegen / (2 * kPi)) * p.w * p.J;
    return {p.E, 0.0, (base * fermi(p.E - t.mu[0], t.kT[0])).real(), (base * fermi(p.E - t.mu[1], t.kT[1])).real(),
            negf::kRealAxis};
}

// Whether Re E lies within `band` of a band edge of mode m in either lead.
// A lead of mode m is the chain with alternating hoppings beta_m and gamma at
// the contact potential U_c, whose bands are |E - U_c| in
// [| |beta_m| - gamma |, |beta_m| + gamma]; at the edges the surface Green's
// function has its square-root singularity and the group velocity vanishes,
// so mixed mode keeps real-axis chains there in FP64 (contour chains sit at
// least the band above the axis, hence at least that far from every edge).
// The contact potentials are the host values of the last
// negf_tube_set_potential[_device] (for a charge plan: at its creation).
bool near_lead_band_edge(const negf_tube& t, int m, cplx E, double band) {
    const double b = std::fabs(t.beta[m]), g = std::fabs(t.d.gamma);
    const double edges[4] = {std::fabs(b - g), b + g, -std::fabs(b - g), -(b + g)};
    for (int c = 0; c < 2; ++c)
        for (double e : edges)
            if (std::fabs(E.real() - t.Uc[c] - e) < band) return true;
    return false;
}

// Chains of one tube, grouped by (kind, precision) with each group padded
// to whole warps (padding lanes: mode -1, zero coefficients).
void build_tube_chains(Out<negf::ChainRec>& chains, Out<negf::WarpRec>& warps, TableCounts& cnt, const TubePass& tp) {
    const negf_tube& t = *tp.t;
    const int M = t.d.num_modes;
    const int total = pass_items(t, tp.rho0_pass);
    int lo = 0, hi = total;
    if (!tp.rho0_pass) negf_shard_range(total, t.shard_rank, t.shard_world, &lo, &hi);
    const bool mixed = t.d.precision == NEGF_PREC_MIXED && !tp.rho0_pass;
    const double band = t.d.mixed_fp64_band;
    for (int kind = 0; kind < 2; ++kind)
        for (int fp32 = 0; fp32 < 2; ++fp32) {
            if (fp32 && !mixed) continue;
            const size_t first = chains.size();
            for (int idx = lo; idx < hi; ++idx) {
                const Item it = pass_item(t, tp.rho0_pass, idx);
                if (it.kind != kind) continue;
                // FP32 recursions only for contour points at least `band` above the real
                // axis; real-axis chains (running products over the whole tube) stay FP64
                // unless mixed_realaxis_fp32 admits those at least `band` above it too
                const bool kind_ok = it.kind == negf::kContour || t.d.mixed_realaxis_fp32;
                const bool axis_ok = mixed && kind_ok && std::fabs(it.E.imag()) >= band;
                if (!axis_ok && fp32) continue;
                for (int m = 0; m < M; ++m) {
                    // real-axis chains also not within `band` of a band edge of the mode's leads
                    const bool edge = it.kind == negf::kRealAxis && near_lead_band_edge(t, m, it.E, band);
                    const int want32 = axis_ok && !edge ? 1 : 0;
                    if (want32 != fp32) continue;
                    negf::ChainRec c{};
                    c.Er = it.E.real();
                    c.Ei = it.E.imag();
                    c.cr = it.c.real();
                    c.ci = it.c.imag();
                    c.b0 = it.b0;
                    c.b1 = it.b1;
                    c.mode = m;
                    chains.push(c);
                    cnt.updates += t.N;
                    if (fp32) cnt.updates_fp32 += t.N;
                    if (kind == negf::kRealAxis)
                        cnt.realaxis_updates += t.N;
                    else
                        cnt.contour_updates += t.N;
                }
            }
            const size_t n = chains.size() - first;
            if (n == 0 || chains.overflow) continue;
            const negf::ChainRec proto = chains.at(first);
            for (size_t k = n; k % negf::kWarp; ++k) {
                negf::ChainRec p = proto;
                p.mode = -1;
                p.cr = p.ci = p.b0 = p.b1 = 0.0;
                chains.push(p);
            }
            for (size_t w = 0; w < (n + negf::kWarp - 1) / negf::kWarp; ++w) {
                negf::WarpRec wr{};
                wr.tube = tp.tube_index;
                wr.kind = kind;
                wr.fp32 = fp32;
                warps.push(wr);
            }
        }
}

// Streaming multiprocessors of the current device (cached per ordinal).
int device_sm_count() {
    static int cache[64] = {};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 148;
    if (!cache[dev]) {
        int v = 0;
        if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || v <= 0) v = 148;
        cache[dev] = v;
    }
    return cache[dev];
}

// RGF schedule of a launch of nw warps (NEGF_TUNE_SCHEDULE): fused when the
// sweeps run as one piece and the warps fill at least one per SM
// sub-partition (4 per SM), else two-pass (its segment tiles spread few
// chains over the whole GPU).
// Parallel in length when the chains alone cannot fill the GPU: about 8
// one-warp blocks per SM, pieces of >= 32 segments, at most 128 pieces (the
// prefix over the pieces is sequential per chain).
int auto_pieces(int nw, int max_N) {
    const int target = 8 * device_sm_count();
    const int maxp = std::min(128, std::max(1, ((max_N + negf::kSeg - 1) / negf::kSeg) / 32));
    return nw >= target / 2 ? 1 : std::min(maxp, (target + nw - 1) / std::max(nw, 1));
}

int choose_schedule(int setting, int nw, int pieces) {
    if (pieces > 1) return negf::kScheduleTwoPass;
    if (setting == NEGF_SCHEDULE_FUSED) return negf::kScheduleFused;
    if (setting == NEGF_SCHEDULE_TWO_PASS) return negf::kScheduleTwoPass;
    return nw >= 4 * device_sm_count() ? negf::kScheduleFused : negf::kScheduleTwoPass;
}

// Checkpoint bytes written + read by one launch: two-pass stores both sweeps'
// states at every segment (pass 1 writes, pass 2 reads); the fused schedule
// stores one record per segment ((Y, lambda) or (X, rho); (Y) or (X) on
// contour chains).
long long checkpoint_traffic(const std::vector<negf::WarpRec>& warps, const std::vector<negf::TubeDev>& tdev,
                             long long scratch_doubles, int schedule) {
    if (schedule != negf::kScheduleFused) return 2 * scratch_doubles * 8;
    long long b = 0;
    for (const negf::WarpRec& w : warps) {
        const long long nseg = (tdev[w.tube].N + negf::kSeg - 1) / negf::kSeg;
        b += nseg * (w.kind == negf::kRealAxis ? 3 : 2) * negf::kWarp * (w.fp32 ? 4 : 8);
    }
    return 2 * b;
}

// Launch tables of a set of tube passes.  Launch order: longest tubes first
// (order[] is caller scratch of passes.size() ints); rts[i] describes pass i.
void build_table_generic(const TubePass* passes, int num_passes, int* order, Out<negf::ChainRec>& chains,
                         Out<negf::WarpRec>& warps, Out<negf::SegUnit>& units, negf::ReduceTube* rts,
                         TableCounts& cnt, int segs_per_unit = negf::kSegsPerUnit) {
    cnt = TableCounts();
    for (int i = 0; i < num_passes; ++i) order[i] = i;
    for (int i = 1; i < num_passes; ++i) {  // stable insertion sort by descending N
        const int v = order[i];
        int j = i - 1;
        while (j >= 0 && passes[order[j]].t->N < passes[v].t->N) {
            order[j + 1] = order[j];
            --j;
        }
        order[j + 1] = v;
    }
    long long row = 0, ck = 0;
    for (int k = 0; k < num_passes; ++k) {
        const int oi = order[k];
        const TubePass& tp = passes[oi];
        const size_t w0 = warps.size();
        build_tube_chains(chains, warps, cnt, tp);
        const int N = tp.t->N;
        negf::ReduceTube rt{};
        rt.row_base = row;
        rt.q_off = tp.q_off;
        rt.N = N;
        rt.num_rows = int(warps.size() - w0);
        rt.rho0 = (!tp.rho0_pass && tp.t->shard_rank == 0) ? tp.t->d_rho0 : nullptr;
        const int nseg = (N + negf::kSeg - 1) / negf::kSeg;
        for (size_t w = w0; w < warps.size() && !warps.overflow; ++w) {
            warps.at(w).row_off = row;
            row += N;
            warps.at(w).ck_off = ck;
            ck += negf::rgf_scratch_doubles(N, warps.at(w).kind, warps.at(w).fp32);
            for (int s0 = 0; s0 < nseg; s0 += segs_per_unit)
                units.push({(int)w, s0, std::min(nseg, s0 + segs_per_unit), 0});
        }
        rts[oi] = rt;
        cnt.max_N = std::max(cnt.max_N, N);
    }
    cnt.partial_doubles = row;
    cnt.scratch_doubles = ck;
}

// Warp order of the fused schedule (FP64 warps first, then FP32 warps).
void fused_order(ChainTable& ct) {
    ct.order.clear();
    for (int pass = 0; pass < 2; ++pass)
        for (size_t w = 0; w < ct.warps.size(); ++w)
            if (ct.warps[w].fp32 == pass) ct.order.push_back((int)w);
    ct.n32 = 0;
    for (const negf::WarpRec& w : ct.warps) ct.n32 += w.fp32 ? 1 : 0;
    ct.n64 = (int)ct.warps.size() - ct.n32;
}

void build_table(ChainTable& ct, const std::vector<TubePass>& passes) {
    ct = ChainTable();
    Out<negf::ChainRec> oc;
    oc.vec = &ct.chains;
    Out<negf::WarpRec> ow;
    ow.vec = &ct.warps;
    Out<negf::SegUnit> ou;
    ou.vec = &ct.units;
    ct.rts.resize(passes.size());
    std::vector<int> order(passes.size());
    TableCounts cnt;
    build_table_generic(passes.data(), (int)passes.size(), order.data(), oc, ow, ou, ct.rts.data(), cnt);
    ct.updates = cnt.updates;
    ct.updates_fp32 = cnt.updates_fp32;
    ct.contour_updates = cnt.contour_updates;
    ct.realaxis_updates = cnt.realaxis_updates;
    ct.partial_doubles = cnt.partial_doubles;
    ct.scratch_doubles = cnt.scratch_doubles;
    ct.max_N = cnt.max_N;
    fused_order(ct);
}

int upload_and_launch(Workspace& W, const std::vector<TubePass>& passes, const std::vector<negf::TubeDev>& tdev,
                      bool rebuild, double* d_Q, cudaStream_t stream) {
    Settings& G = settings();
    ChainTable& ct = W.table;
    if (rebuild) {
        build_table(ct, passes);
        NEGF_CUDA(W.chains.reserve(std::max<size_t>(1, ct.chains.size()) * sizeof(negf::ChainRec)));
        NEGF_CUDA(W.warps.reserve(std::max<size_t>(1, ct.warps.size()) * sizeof(negf::WarpRec)));
        NEGF_CUDA(W.rts.reserve(std::max<size_t>(1, ct.rts.size()) * sizeof(negf::ReduceTube)));
        NEGF_CUDA(W.units.reserve(std::max<size_t>(1, ct.units.size()) * sizeof(negf::SegUnit)));
        NEGF_CUDA(W.partial.reserve(std::max<long long>(1, ct.partial_doubles) * sizeof(double)));
        NEGF_CUDA(W.scratch.reserve(std::max<long long>(1, ct.scratch_doubles) * sizeof(double)));
        if (!ct.chains.empty())
            NEGF_CUDA(cudaMemcpyAsync(W.chains.p, ct.chains.data(), ct.chains.size() * sizeof(negf::ChainRec),
                                      cudaMemcpyHostToDevice, stream));
        if (!ct.warps.empty())
            NEGF_CUDA(cudaMemcpyAsync(W.warps.p, ct.warps.data(), ct.warps.size() * sizeof(negf::WarpRec),
                                      cudaMemcpyHostToDevice, stream));
        if (!ct.units.empty())
            NEGF_CUDA(cudaMemcpyAsync(W.units.p, ct.units.data(), ct.units.size() * sizeof(negf::SegUnit),
                                      cudaMemcpyHostToDevice, stream));
        NEGF_CUDA(W.order.reserve(std::max<size_t>(1, ct.order.size()) * sizeof(int)));
        if (!ct.order.empty())
            NEGF_CUDA(cudaMemcpyAsync(W.order.p, ct.order.data(), ct.order.size() * sizeof(int),
                                      cudaMemcpyHostToDevice, stream));
    }
    // the reduce table carries device pointers that can change (rho0 of a rebuilt tube)
    for (size_t i = 0; i < passes.size(); ++i)
        ct.rts[i].rho0 = (!passes[i].rho0_pass && passes[i].t->shard_rank == 0) ? passes[i].t->d_rho0 : nullptr;
    NEGF_CUDA(cudaMemcpyAsync(W.rts.p, ct.rts.data(), ct.rts.size() * sizeof(negf::ReduceTube), cudaMemcpyHostToDevice,
                              stream));
    NEGF_CUDA(W.tubes.reserve(tdev.size() * sizeof(negf::TubeDev)));
    NEGF_CUDA(cudaMemcpyAsync(W.tubes.p, tdev.data(), tdev.size() * sizeof(negf::TubeDev), cudaMemcpyHostToDevice,
                              stream));
    const int nw = (int)ct.warps.size();
    if (G.timing) {
        for (auto& e : W.ev)
            if (!e) NEGF_CUDA(cudaEventCreate(&e));
        NEGF_CUDA(cudaEventRecord(W.ev[0], stream));
    }
    int pieces = G.pass1_pieces;
    if (pieces == 0 && G.schedule == NEGF_SCHEDULE_FUSED) pieces = 1;  // an explicit fused request wins
    if (pieces == 0) pieces = auto_pieces(nw, ct.max_N);
    pieces = std::max(1, pieces);
    const int schedule = choose_schedule(G.schedule, nw, pieces);
    if (schedule == negf::kScheduleFused) pieces = 1;
    if (pieces > 1) NEGF_CUDA(W.pieces.reserve(sizeof(double) * (size_t)nw * pieces * 24 * negf::kWarp));
    const negf::FusedOrder fo{W.order.as<int>(), ct.n64, ct.n32, W.side, W.fork, W.join};
    NEGF_CUDA(negf::launch_rgf(W.tubes.as<negf::TubeDev>(), W.chains.as<negf::ChainRec>(), W.warps.as<negf::WarpRec>(),
                               nw, W.units.as<negf::SegUnit>(), (int)ct.units.size(), W.partial.as<double>(),
                               W.scratch.p, G.warps_per_block, stream, G.timing ? W.ev[3] : nullptr, nullptr, pieces,
                               W.pieces.as<double>(), schedule, &fo));
    if (G.timing) NEGF_CUDA(cudaEventRecord(W.ev[1], stream));
    NEGF_CUDA(negf::launch_reduce(W.rts.as<negf::ReduceTube>(), (int)ct.rts.size(), ct.max_N, W.partial.as<double>(),
                                  d_Q, stream));
    if (G.timing) NEGF_CUDA(cudaEventRecord(W.ev[2], stream));
    NEGF_CUDA(cudaEventRecord(W.done, stream));
    W.used = true;
    negf_stats& st = G.stats;
    st = negf_stats{};
    st.updates = ct.updates;
    st.updates_fp32 = ct.updates_fp32;
    st.contour_updates = ct.contour_updates;
    st.realaxis_updates = ct.realaxis_updates;
    st.chains = (int)ct.chains.size();
    st.warps = nw;
    const bool fused = schedule == negf::kScheduleFused;
    const int fused_kernels = (ct.n64 > 0 ? 1 : 0) + (ct.n32 > 0 ? 1 : 0);
    st.kernel_launches =
        (nw > 0 ? (fused ? fused_kernels : pieces > 1 ? 4 : 2) : 0) + (ct.max_N > 0 && !ct.rts.empty() ? 1 : 0);
    st.pieces = pieces;
    st.units = fused ? 0 : (int)ct.units.size();
    st.checkpoint_bytes = checkpoint_traffic(ct.warps, tdev, ct.scratch_doubles, schedule);
    st.schedule = fused ? NEGF_SCHEDULE_FUSED : NEGF_SCHEDULE_TWO_PASS;
    G.stats_ws = G.timing ? &W : nullptr;
    return NEGF_OK;
}

negf::TubeDev make_tubedev(const negf_tube& t, bool rho0_pass) {
    negf::TubeDev d{};
    d.U = rho0_pass ? t.d_zero : t.d_U;
    d.N = t.N;
    d.num_modes = t.d.num_modes;
    d.gamma = t.d.gamma;
    d.Uc0 = rho0_pass ? 0.0 : t.Uc[0];
    d.Uc1 = rho0_pass ? 0.0 : t.Uc[1];
    d.use_decimation = t.d.use_decimation;
    d.dec_iters = t.d.decimation_max_iter + 2;
    d.dec_layers = t.d.decimation_layers;
    for (int m = 0; m < t.d.num_modes; ++m) {
        d.beta[m] = t.beta[m];
        d.degen[m] = t.degen[m];
    }
    return d;
}

// Contact potentials; in mixed precision the chain table depends on them
// (the band-edge rule), so a change marks it for rebuilding.
void set_contacts(negf_tube& t, const double Uc[2]) {
    if (t.d.precision == NEGF_PREC_MIXED && (t.Uc[0] != Uc[0] || t.Uc[1] != Uc[1])) t.version++;
    t.Uc[0] = Uc[0];
    t.Uc[1] = Uc[1];
}

int compute_rho0(negf_tube* t) {
    Workspace* W = nullptr;
    if (int rc = get_workspace(nullptr, &W)) return rc;
    rho0_paths(*t);
    std::vector<TubePass> passes{{t, 0, 0, true}};
    std::vector<negf::TubeDev> tdev{make_tubedev(*t, true)};
    W->table_valid = false;
    int rc = upload_and_launch(*W, passes, tdev, true, t->d_rho0, nullptr);
    W->table_valid = false;
    if (rc != NEGF_OK) return rc;
    NEGF_CUDA(cudaStreamSynchronize(nullptr));
    return NEGF_OK;
}

// ------------------------------------------------------------------ transport characteristics
// DOS energy path (NEGF_Common.cpp:2188-2250): the non-equilibrium paths when
// biased, else Gauss-Legendre on [Re E_eta, E_rightmost].
std::vector<Pt> dos_points(const negf_tube& t) {
    if (t.noneq) return t.noneq_pts;
    std::vector<Pt> v;
    gl_path(cplx(t.E_eta.real(), 0.0), t.E_rightmost, t.d.flatband_dos_integration_pts, 0, v);
    return v;
}

// One transport run of a tube over energies pts: red[e][8] (see
// negf::launch_transport) and, when ldos != null, LDOS [e][N].  Every buffer
// is local to the call (this runs once per bias step, not per SCF iteration).
int transport_run(negf_tube& t, const std::vector<Pt>& pts, std::vector<double>& red, double* ldos,
                  cudaStream_t s) {
    const int P = (int)pts.size(), M = t.d.num_modes, N = t.N;
    red.assign((size_t)P * 8, 0.0);
    if (P == 0) return NEGF_OK;
    std::vector<negf::ChainRec> chains;
    chains.reserve((size_t)P * M + negf::kWarp);
    for (int e = 0; e < P; ++e) {
        const double f0 = fermi(pts[e].E - t.mu[0], t.kT[0]).real();
        const double f1 = fermi(pts[e].E - t.mu[1], t.kT[1]).real();
        for (int m = 0; m < M; ++m) {
            negf::ChainRec c{};
            c.Er = pts[e].E.real();
            c.Ei = pts[e].E.imag();
            c.cr = f0;
            c.ci = f1;
            c.b0 = c.b1 = 1.0;
            c.mode = m;
            chains.push_back(c);
        }
    }
    while (chains.size() % negf::kWarp) {
        negf::ChainRec p = chains.back();
        p.mode = -1;
        p.cr = p.ci = p.b0 = p.b1 = 0.0;
        chains.push_back(p);
    }
    const int nw = (int)(chains.size() / negf::kWarp);
    const int nseg = (N + negf::kSeg - 1) / negf::kSeg;
    const int upw = (nseg + negf::kSegsPerUnit - 1) / negf::kSegsPerUnit;
    const long long per_warp = negf::rgf_scratch_doubles(N, negf::kRealAxis, 0);
    std::vector<negf::WarpRec> warps(nw);
    std::vector<negf::SegUnit> units;
    for (int w = 0; w < nw; ++w) {
        warps[w] = negf::WarpRec{};
        warps[w].tube = 0;
        warps[w].kind = negf::kRealAxis;
        warps[w].fp32 = 0;
        warps[w].ck_off = w * per_warp;
        for (int s0 = 0; s0 < nseg; s0 += negf::kSegsPerUnit)
            units.push_back({w, s0, std::min(nseg, s0 + negf::kSegsPerUnit), 0});
    }
    const negf::TubeDev td = make_tubedev(t, false);
    const size_t C = chains.size();
    DevBuf b_tube, b_chains, b_warps, b_units, b_scratch, b_part, b_cout, b_red, b_site, b_ldos;
    NEGF_CUDA(b_tube.reserve(sizeof(td)));
    NEGF_CUDA(b_chains.reserve(C * sizeof(negf::ChainRec)));
    NEGF_CUDA(b_warps.reserve(warps.size() * sizeof(negf::WarpRec)));
    NEGF_CUDA(b_units.reserve(units.size() * sizeof(negf::SegUnit)));
    NEGF_CUDA(b_scratch.reserve((size_t)nw * per_warp * sizeof(double)));
    NEGF_CUDA(b_part.reserve(units.size() * negf::kWarp * sizeof(double)));
    NEGF_CUDA(b_cout.reserve(C * 7 * sizeof(double)));
    NEGF_CUDA(b_red.reserve(red.size() * sizeof(double)));
    if (ldos) {
        NEGF_CUDA(b_site.reserve((size_t)N * C * sizeof(double)));
        NEGF_CUDA(b_ldos.reserve((size_t)P * N * sizeof(double)));
    }
    NEGF_CUDA(cudaMemcpyAsync(b_tube.p, &td, sizeof(td), cudaMemcpyHostToDevice, s));
    NEGF_CUDA(cudaMemcpyAsync(b_chains.p, chains.data(), C * sizeof(negf::ChainRec), cudaMemcpyHostToDevice, s));
    NEGF_CUDA(cudaMemcpyAsync(b_warps.p, warps.data(), warps.size() * sizeof(negf::WarpRec), cudaMemcpyHostToDevice,
                              s));
    NEGF_CUDA(cudaMemcpyAsync(b_units.p, units.data(), units.size() * sizeof(negf::SegUnit),
                              cudaMemcpyHostToDevice, s));
    // sites that a chain never reaches keep these zeros (N = 1, 2 probe rules)
    NEGF_CUDA(cudaMemsetAsync(b_cout.p, 0, C * 7 * sizeof(double), s));
    NEGF_CUDA(negf::launch_transport(b_tube.as<negf::TubeDev>(), b_chains.as<negf::ChainRec>(),
                                     b_warps.as<negf::WarpRec>(), nw, b_units.as<negf::SegUnit>(), (int)units.size(),
                                     b_scratch.p, b_part.as<double>(), b_cout.as<double>(),
                                     ldos ? b_site.as<double>() : nullptr, (long long)C, P, M, upw,
                                     b_red.as<double>(), ldos ? b_ldos.as<double>() : nullptr, N, s));
    NEGF_CUDA(cudaMemcpyAsync(red.data(), b_red.p, red.size() * sizeof(double), cudaMemcpyDeviceToHost, s));
    if (ldos)
        NEGF_CUDA(cudaMemcpyAsync(ldos, b_ldos.p, (size_t)P * N * sizeof(double), cudaMemcpyDeviceToHost, s));
    NEGF_CUDA(cudaStreamSynchronize(s));
    return NEGF_OK;
}

// Compute_Conductance (NEGF_Common.cpp:1873-1928): G_quantum = 1, dF/dE of
// contact 0 by finite differences with the first spacing deltaE = E_0 - E_1.
double conductance(const negf_tube& t, const std::vector<double>& E, const double* T, double* C) {
    const size_t P = E.size();
    for (size_t i = 0; i < P; ++i) C[i] = 0.0;
    if (P < 3) return 0.0;
    std::vector<double> dF(P);
    const double dE = E[0] - E[1], inv = 1. / (2 * dE);
    auto F = [&](size_t i) { return fermi(cplx(E[i], 0.0) - t.mu[0], t.kT[0]).real(); };
    dF[0] = (-3 * F(0) + 4 * F(1) - F(2)) * inv;
    const size_t n = P - 1;
    dF[n] = (3 * F(n) - 4 * F(n - 1) + F(n - 2)) * inv;
    for (size_t i = 1; i < n; ++i) dF[i] = (F(i + 1) - F(i - 1)) * inv;
    double sum = 0.0;
    for (size_t i = 0; i < P; ++i) {
        C[i] = -1.0 * T[i] * dF[i];
        sum += C[i] * dE;
    }
    return sum;
}

// Integrand of Compute_RhoNonEq at the probe sites (NEGF_Common.cpp:3467-3496):
// Re(-spin/2pi sum_modes deg sum_k A^k_nn f_k) at n = N/2, N/4, 3N/4 over the
// current non-equilibrium energies -> integrand [3][P].
int noneq_integrand(negf_tube& t, std::vector<double>& integrand, cudaStream_t s) {
    const std::vector<Pt>& pts = t.noneq_pts;
    std::vector<double> red;
    int rc = transport_run(t, pts, red, nullptr, s);
    if (rc) return rc;
    const int P = (int)pts.size();
    const double c = -1 * kSpinDegen / (2 * kPi);
    integrand.assign((size_t)3 * P, 0.0);
    for (int e = 0; e < P; ++e) {
        integrand[e] = c * red[8 * e + 3];
        integrand[(size_t)P + e] = c * red[8 * e + 6];
        integrand[(size_t)2 * P + e] = c * red[8 * e + 7];
    }
    return NEGF_OK;
}

// Find_NonEq_Percent_Intercuts_Adaptively (NEGF_Common.cpp:2062-2185): new
// intercuts and point counts of 2 or 3 non-equilibrium paths around E* (the
// energy of the largest |integrand|), in units of kT_0 from mu_0; the point
// densities per kT are fixed on first use.
void find_intercuts(negf_tube& t) {
    negf_tube_desc& d = t.d;
    const int np = d.num_noneq_paths;
    const double Es = (t.E_at_max_noneq_integrand - t.mu[0]) / t.kT[0];
    const double Emin = (t.E_right.real() - t.mu[0]) / t.kT[0];
    const double Emax = (t.E_rightmost.real() - t.mu[0]) / t.kT[0];
    double* cut = d.noneq_percent_intercuts;
    int* pts = d.noneq_integration_pts;
    double* den = d.noneq_integration_pts_density;
    if (cut[0] < 0)  // the uniform default, made explicit
        for (int p = 0; p < np - 1; ++p) cut[p] = (p + 1) * (100. / np);
    if (np == 3) {
        if (!d.flag_noneq_integration_pts_density) {
            den[0] = pts[0] / ((cut[0] / 100.) * (Emax - Emin));
            den[1] = pts[1] / (((cut[1] - cut[0]) / 100.) * (Emax - Emin));
            den[2] = pts[2] / (((100. - cut[1]) / 100.) * (Emax - Emin));
            d.flag_noneq_integration_pts_density = 1;
        }
        const double lo = std::max(Es - d.kT_window_around_singularity[0], Emin);
        const double hi = std::min(Es + d.kT_window_around_singularity[1], Emax);
        cut[0] = 100 * (lo - Emin) / (Emax - Emin);
        cut[1] = 100 * (hi - Emin) / (Emax - Emin);
        pts[0] = (int)(std::round(((lo - Emin) * den[0]) / 2) * 2);
        pts[1] = (int)(std::round(((hi - lo) * den[1]) / 2) * 2);
        pts[2] = (int)(std::round(((Emax - hi) * den[2]) / 2) * 2);
    } else if (np == 2) {
        if (!d.flag_noneq_integration_pts_density) {
            den[0] = pts[0] / ((cut[0] / 100.) * (Emax - Emin));
            den[1] = pts[1] / (((100 - cut[0]) / 100.) * (Emax - Emin));
            d.flag_noneq_integration_pts_density = 1;
        }
        const double hi = Es + d.kT_window_around_singularity[1];
        cut[0] = 100 * (hi - Emin) / (Emax - Emin);
        pts[0] = (int)(std::round(((hi - Emin) * den[0]) / 2) * 2);
        pts[1] = (int)(std::round(((Emax - hi) * den[1]) / 2) * 2);
    }
}

void write_table(FILE* f, const std::vector<double>& pos, const double* v, int n) {
    // Write_Table1D, NEGF_Common.cpp:4221-4254: setprecision(15), setw(35)
    for (int i = 0; i < n; ++i) std::fprintf(f, "%35.15g%35.15g\n", pos[i], v[i]);
}

}  // namespace

// ====================================================================== allocation-free planning
namespace negf {

int report(int code, const char* msg) { return fail(code, msg); }

// Plans one charge launch into caller-provided fixed arrays (no allocation).
// Requires every tube's energy paths to be current (they are rebuilt by
// negf_tube_create / negf_tube_set_contact_mu).
std::unique_lock<std::mutex> api_lock() { return std::unique_lock<std::mutex>(g_mu); }

int plan_charge_fixed(negf_tube* const* tubes, int num_tubes, FixedPlan& fp) {
    constexpr int kMaxPlanTubes = 64;
    if (!tubes || num_tubes <= 0) return fail(NEGF_ERR_ARG, "null or empty tube batch");
    for (int i = 0; i < num_tubes; ++i)
        if (!tubes[i]) return fail(NEGF_ERR_ARG, "null tube in batch");
    if (int rc = check_batch_device(tubes, num_tubes)) return rc;
    if (num_tubes > kMaxPlanTubes || num_tubes > fp.tube_cap)
        return fail(NEGF_ERR_ARG, "too many tubes for the allocation-free entry point (max " +
                                      std::to_string(std::min(kMaxPlanTubes, fp.tube_cap)) + ")");
    static TubePass passes[kMaxPlanTubes];  // calls of the allocation-free entry point never overlap (documented)
    static int order[kMaxPlanTubes];
    long long off = 0;
    for (int i = 0; i < num_tubes; ++i) {
        const negf_tube* t = tubes[i];
        if (t->limits_dirty) return fail(NEGF_ERR_STATE, "tube energy paths are not current");
        passes[i] = {t, i, off, false};
        fp.tubes[i] = make_tubedev(*t, false);
        off += t->N;
    }
    Out<ChainRec> oc;
    oc.arr = fp.chains;
    oc.cap = fp.chain_cap;
    Out<WarpRec> ow;
    ow.arr = fp.warps;
    ow.cap = fp.warp_cap;
    Out<SegUnit> ou;
    ou.arr = fp.units;
    ou.cap = fp.unit_cap;
    TableCounts cnt;
    build_table_generic(passes, num_tubes, order, oc, ow, ou, fp.rts, cnt);
    if (oc.overflow || ow.overflow || ou.overflow)
        return fail(NEGF_ERR_ARG, "problem exceeds the launch-table capacity of the allocation-free entry point (" +
                                      std::to_string(fp.chain_cap) + " chains, " + std::to_string(fp.warp_cap) +
                                      " warps)");
    fp.num_tubes = num_tubes;
    fp.num_chains = oc.size();
    fp.num_warps = ow.size();
    fp.num_units = ou.size();
    fp.partial_doubles = cnt.partial_doubles;
    fp.scratch_doubles = cnt.scratch_doubles;
    fp.max_N = cnt.max_N;
    fp.total_sites = off;
    return NEGF_OK;
}

}  // namespace negf

// ====================================================================== C-ABI
extern "C" {

const char* negf_last_error(void) { return g_err.c_str(); }

int negf_tube_desc_init(negf_tube_desc* d) {
    if (!d) return fail(NEGF_ERR_ARG, "null descriptor");
    std::memset(d, 0, sizeof(*d));
    d->type_id[0] = 17;
    d->type_id[1] = 0;
    d->num_unitcells = 100;
    d->num_modes = 1;
    d->acc = 1.42e-10;
    d->gamma = 2.5;
    d->contact_T[0] = d->contact_T[1] = 298.0;
    d->eq_integration_pts[0] = d->eq_integration_pts[1] = d->eq_integration_pts[2] = 30;
    d->num_noneq_paths = 1;
    d->noneq_integration_pts[0] = 100;
    d->noneq_percent_intercuts[0] = -1.0;
    d->E_valence_min = -14.0;
    d->E_pole_max = 10.0;
    d->E_zPlus_imag = 1e-8;
    d->Fermi_tail_factors[0] = d->Fermi_tail_factors[1] = 14.0;
    d->use_decimation = 0;
    d->decimation_max_iter = 30;
    d->decimation_layers = 10;
    d->precision = NEGF_PREC_FP64;
    d->mixed_fp64_band = 1e-3;
    d->mixed_realaxis_fp32 = 0;
    d->flatband_dos_integration_pts = 100;
    d->flag_adaptive_integration_limits = 0;
    d->integrand_correction_interval = 500;
    d->kT_window_around_singularity[0] = d->kT_window_around_singularity[1] = 1.0;
    d->flag_noneq_integration_pts_density = 0;
    return NEGF_OK;
}

int negf_tube_create(const negf_tube_desc* d, negf_tube** out) {
    if (!d || !out) return fail(NEGF_ERR_ARG, "null argument");
    *out = nullptr;
    if (d->num_noneq_paths < 1 || d->num_noneq_paths > NEGF_MAX_NONEQ_PATHS)
        return fail(NEGF_ERR_ARG, "num_noneq_paths out of range");
    for (int i = 0; i < 3; ++i)
        if (d->eq_integration_pts[i] < 0) return fail(NEGF_ERR_ARG, "eq_integration_pts must be >= 0");
    if (d->use_decimation && (d->decimation_layers < 2 || d->decimation_layers > 64))
        return fail(NEGF_ERR_ARG, "decimation_layers must be in [2, 64]");
    if (d->precision != NEGF_PREC_FP64 && d->precision != NEGF_PREC_MIXED)
        return fail(NEGF_ERR_ARG, "unknown precision mode");
    if (!(d->gamma > 0) || !(d->acc > 0)) return fail(NEGF_ERR_ARG, "gamma and acc must be > 0");
    if (!(d->contact_T[0] > 0) || !(d->contact_T[1] > 0)) return fail(NEGF_ERR_ARG, "contact_T must be > 0");
    if (d->realaxis_pts < 0 || (d->realaxis_pts > 0 && !(d->realaxis_max > d->realaxis_min)))
        return fail(NEGF_ERR_ARG, "real-axis window needs realaxis_max > realaxis_min");
    int rc = require_device();
    if (rc) return rc;
    std::unique_ptr<negf_tube> t(new negf_tube());
    t->d = *d;
    rc = setup_material(*t);
    if (rc) return rc;
    cudaGetDevice(&t->device);
    {
        static std::atomic<long long> next_serial{1};
        t->serial = next_serial++;
    }
    t->mu[0] = d->contact_mu[0];
    t->mu[1] = d->contact_mu[1];
    // zero padding on both sides lets the kernels load whole segments of U
    // without bounds checks
    const size_t padded = sizeof(double) * (negf::kPadLo + t->N + negf::kPadHi);
    NEGF_CUDA(cudaMalloc(&t->d_U_pad, padded));
    NEGF_CUDA(cudaMalloc(&t->d_zero_pad, padded));
    NEGF_CUDA(cudaMemset(t->d_U_pad, 0, padded));
    NEGF_CUDA(cudaMemset(t->d_zero_pad, 0, padded));
    t->d_U = t->d_U_pad + negf::kPadLo;
    t->d_zero = t->d_zero_pad + negf::kPadLo;
    NEGF_CUDA(cudaMalloc(&t->d_rho0, sizeof(double) * t->N));
    NEGF_CUDA(cudaMemset(t->d_rho0, 0, sizeof(double) * t->N));
    {
        std::lock_guard<std::mutex> lk(g_mu);
        rc = compute_rho0(t.get());
    }
    if (rc) return rc;
    update_paths(*t);
    *out = t.release();
    return NEGF_OK;
}

int negf_tube_destroy(negf_tube* t) {
    if (t) {
        std::lock_guard<std::mutex> lk(g_mu);
        delete t;  // cached launch tables are keyed by tube serials, never reused
    }
    return NEGF_OK;
}

int negf_tube_num_sites(const negf_tube* t, int* n) {
    if (!t || !n) return fail(NEGF_ERR_ARG, "null argument");
    *n = t->N;
    return NEGF_OK;
}

int negf_tube_modes(const negf_tube* t, int* num_modes, int* J, int* degeneracy, double* beta) {
    if (!t) return fail(NEGF_ERR_ARG, "null tube");
    const int M = t->d.num_modes;
    if (num_modes) *num_modes = M;
    for (int m = 0; m < M; ++m) {
        if (J) J[m] = t->modeJ[m];
        if (degeneracy) degeneracy[m] = t->degen[m];
        if (beta) beta[m] = t->beta[m];
    }
    return NEGF_OK;
}

int negf_tube_site_positions(const negf_tube* t, double* y) {
    if (!t || !y) return fail(NEGF_ERR_ARG, "null argument");
    std::copy(t->y_nm.begin(), t->y_nm.end(), y);
    return NEGF_OK;
}

int negf_tube_set_potential(negf_tube* t, const double* U, int n, const double Uc[2]) {
    if (!t || !U || !Uc) return fail(NEGF_ERR_ARG, "null argument");
    if (n != t->N) return fail(NEGF_ERR_ARG, "potential has " + std::to_string(n) + " sites, tube has " + std::to_string(t->N));
    for (int i = 0; i < n; ++i)
        if (!std::isfinite(U[i])) return fail(NEGF_ERR_NUMERIC, "non-finite potential at site " + std::to_string(i));
    if (!std::isfinite(Uc[0]) || !std::isfinite(Uc[1])) return fail(NEGF_ERR_NUMERIC, "non-finite contact potential");
    NEGF_CUDA(cudaMemcpy(t->d_U, U, sizeof(double) * n, cudaMemcpyHostToDevice));
    set_contacts(*t, Uc);
    return NEGF_OK;
}

int negf_tube_set_potential_device(negf_tube* t, const double* dU, int n, const double Uc[2], void* stream) {
    if (!t || !dU || !Uc) return fail(NEGF_ERR_ARG, "null argument");
    if (n != t->N) return fail(NEGF_ERR_ARG, "potential size mismatch");
    if (!std::isfinite(Uc[0]) || !std::isfinite(Uc[1])) return fail(NEGF_ERR_NUMERIC, "non-finite contact potential");
    if (dU != t->d_U)
        NEGF_CUDA(cudaMemcpyAsync(t->d_U, dU, sizeof(double) * n, cudaMemcpyDeviceToDevice, (cudaStream_t)stream));
    set_contacts(*t, Uc);
    return NEGF_OK;
}

int negf_tube_potential_device_ptr(negf_tube* t, double** dU) {
    if (!t || !dU) return fail(NEGF_ERR_ARG, "null argument");
    *dU = t->d_U;
    return NEGF_OK;
}

int negf_tube_set_contact_mu(negf_tube* t, const double mu[2]) {
    if (!t || !mu) return fail(NEGF_ERR_ARG, "null argument");
    if (!std::isfinite(mu[0]) || !std::isfinite(mu[1])) return fail(NEGF_ERR_NUMERIC, "non-finite contact mu");
    t->mu[0] = mu[0];
    t->mu[1] = mu[1];
    t->limits_dirty = true;
    update_paths(*t);  // host tables rebuilt here, not inside the charge calls
    return NEGF_OK;
}

int negf_tube_energy_points(negf_tube* t, int kind, double* buf, int* count) {
    if (!t || !count) return fail(NEGF_ERR_ARG, "null argument");
    update_paths(*t);
    if (kind == 0) rho0_paths(*t);
    if (kind == 2) {
        *count = (int)t->poles.size();
        if (buf)
            for (size_t i = 0; i < t->poles.size(); ++i) {
                double* b = buf + 6 * i;
                b[0] = t->poles[i].real();
                b[1] = t->poles[i].imag();
                b[2] = b[3] = b[4] = b[5] = 0.0;
            }
        return NEGF_OK;
    }
    const std::vector<Pt>* v = kind == 0 ? &t->rho0_pts : kind == 1 ? &t->eq_pts : kind == 3 ? &t->noneq_pts : nullptr;
    if (!v) return fail(NEGF_ERR_ARG, "kind must be 0..3");
    *count = (int)v->size();
    if (buf)
        for (size_t i = 0; i < v->size(); ++i) {
            double* b = buf + 6 * i;
            b[0] = (*v)[i].E.real();
            b[1] = (*v)[i].E.imag();
            b[2] = (*v)[i].w.real();
            b[3] = (*v)[i].w.imag();
            b[4] = (*v)[i].J.real();
            b[5] = (*v)[i].J.imag();
        }
    return NEGF_OK;
}

int negf_desc_energy_points(const negf_tube_desc* d, int kind, double* buf, int* count) {
    if (!d || !count) return fail(NEGF_ERR_ARG, "null argument");
    negf_tube t;  // host-only: no device buffers are allocated
    t.d = *d;
    t.mu[0] = d->contact_mu[0];
    t.mu[1] = d->contact_mu[1];
    return negf_tube_energy_points(&t, kind, buf, count);
}

int negf_tube_noneq(negf_tube* t, int* noneq) {
    if (!t || !noneq) return fail(NEGF_ERR_ARG, "null argument");
    update_paths(*t);
    *noneq = t->noneq ? 1 : 0;
    return NEGF_OK;
}

int negf_tube_total_integration_pts(negf_tube* t, int* pts) {
    if (!t || !pts) return fail(NEGF_ERR_ARG, "null argument");
    update_paths(*t);
    *pts = t->noneq ? (int)t->noneq_pts.size() : (int)t->eq_pts.size();
    return NEGF_OK;
}

int negf_shard_range(int num_points, int rank, int world, int* lo, int* hi) {
    if (!lo || !hi || world < 1 || rank < 0 || rank >= world || num_points < 0)
        return fail(NEGF_ERR_ARG, "bad shard arguments");
    *lo = (int)((long long)num_points * rank / world);
    *hi = (int)((long long)num_points * (rank + 1) / world);
    return NEGF_OK;
}

int negf_tube_set_energy_shard(negf_tube* t, int rank, int world) {
    if (!t || world < 1 || rank < 0 || rank >= world) return fail(NEGF_ERR_ARG, "bad shard arguments");
    t->shard_rank = rank;
    t->shard_world = world;
    t->version++;
    return NEGF_OK;
}

int negf_compute_charge(negf_tube* const* tubes, int num_tubes, double* Q, int q_on_device, void* stream) {
    if (!tubes || num_tubes <= 0 || !Q) return fail(NEGF_ERR_ARG, "null argument");
    cudaStream_t s = (cudaStream_t)stream;
    std::lock_guard<std::mutex> lk(g_mu);
    for (int i = 0; i < num_tubes; ++i)
        if (!tubes[i]) return fail(NEGF_ERR_ARG, "null tube in batch");
    if (int rc = check_batch_device(tubes, num_tubes)) return rc;
    Workspace* Wp = nullptr;
    if (int rc = get_workspace(s, &Wp)) return rc;
    Workspace& W = *Wp;
    std::vector<TubePass> passes;
    std::vector<negf::TubeDev> tdev;
    long long off = 0;
    bool same = W.table_valid && W.key_serials.size() == (size_t)num_tubes;
    for (int i = 0; i < num_tubes; ++i) {
        negf_tube* t = tubes[i];
        update_paths(*t);
        passes.push_back({t, i, off, false});
        tdev.push_back(make_tubedev(*t, false));
        off += t->N;
        if (same && (W.key_serials[i] != t->serial || W.key_versions[i] != t->version)) same = false;
    }
    double* dQ = Q;
    if (!q_on_device) {
        NEGF_CUDA(W.qbuf.reserve(sizeof(double) * off));
        dQ = W.qbuf.as<double>();
    }
    int rc = upload_and_launch(W, passes, tdev, !same, dQ, s);
    if (rc) {
        W.table_valid = false;
        return rc;
    }
    W.key_serials.clear();
    W.key_versions.clear();
    for (int i = 0; i < num_tubes; ++i) {
        W.key_serials.push_back(tubes[i]->serial);
        W.key_versions.push_back(tubes[i]->version);
    }
    W.table_valid = true;
    if (!q_on_device) {
        NEGF_CUDA(cudaMemcpyAsync(Q, dQ, sizeof(double) * off, cudaMemcpyDeviceToHost, s));
        NEGF_CUDA(cudaEventRecord(W.done, s));  // the next call may rewrite qbuf only after this copy
        NEGF_CUDA(cudaStreamSynchronize(s));
    }
    return NEGF_OK;
}

// ------------------------------------------------------------------ charge plans
namespace {
// Tables of a plan for a given number of segments per pass-2 unit.
int plan_tables(negf_charge_plan& p, int spu, bool upload_all) {
    const int n = (int)p.tubes.size();
    // an FP64 plan of mixed-precision tubes: their descriptors read as FP64 while the table is built
    std::vector<int> saved(n);
    for (int i = 0; i < n; ++i) {
        saved[i] = p.tubes[i]->d.precision;
        if (p.force_fp64) p.tubes[i]->d.precision = NEGF_PREC_FP64;
    }
    std::vector<TubePass> passes;
    std::vector<negf::TubeDev> tdev;
    long long off = 0;
    for (int i = 0; i < n; ++i) {
        passes.push_back({p.tubes[i], i, off, false});
        negf::TubeDev d = make_tubedev(*p.tubes[i], false);
        d.uc_from_U = 1;
        tdev.push_back(d);
        off += p.tubes[i]->N;
    }
    ChainTable ct;
    Out<negf::ChainRec> oc;
    oc.vec = &ct.chains;
    Out<negf::WarpRec> ow;
    ow.vec = &ct.warps;
    Out<negf::SegUnit> ou;
    ou.vec = &ct.units;
    ct.rts.resize(n);
    std::vector<int> order(n);
    TableCounts cnt;
    build_table_generic(passes.data(), n, order.data(), oc, ow, ou, ct.rts.data(), cnt, spu);
    for (int i = 0; i < n; ++i) p.tubes[i]->d.precision = saved[i];
    fused_order(ct);
    p.n64 = ct.n64;
    p.n32 = ct.n32;
    p.num_warps = (int)ct.warps.size();
    p.num_units = (int)ct.units.size();
    p.max_N = cnt.max_N;
    p.updates = cnt.updates;
    p.spu = spu;
    NEGF_CUDA(p.d_units.reserve(std::max<size_t>(1, ct.units.size()) * sizeof(negf::SegUnit)));
    if (!ct.units.empty())
        NEGF_CUDA(cudaMemcpy(p.d_units.p, ct.units.data(), ct.units.size() * sizeof(negf::SegUnit),
                             cudaMemcpyHostToDevice));
    if (!upload_all) return NEGF_OK;
    NEGF_CUDA(p.d_order.reserve(std::max<size_t>(1, ct.order.size()) * sizeof(int)));
    if (!ct.order.empty())
        NEGF_CUDA(cudaMemcpy(p.d_order.p, ct.order.data(), ct.order.size() * sizeof(int), cudaMemcpyHostToDevice));
    NEGF_CUDA(p.d_tubes.reserve(tdev.size() * sizeof(negf::TubeDev)));
    NEGF_CUDA(p.d_chains.reserve(std::max<size_t>(1, ct.chains.size()) * sizeof(negf::ChainRec)));
    NEGF_CUDA(p.d_warps.reserve(std::max<size_t>(1, ct.warps.size()) * sizeof(negf::WarpRec)));
    NEGF_CUDA(p.d_rts.reserve(ct.rts.size() * sizeof(negf::ReduceTube)));
    NEGF_CUDA(p.d_partial.reserve(std::max<long long>(1, cnt.partial_doubles) * sizeof(double)));
    NEGF_CUDA(p.d_scratch.reserve(std::max<long long>(1, cnt.scratch_doubles) * sizeof(double)));
    NEGF_CUDA(cudaMemcpy(p.d_tubes.p, tdev.data(), tdev.size() * sizeof(negf::TubeDev), cudaMemcpyHostToDevice));
    if (!ct.chains.empty())
        NEGF_CUDA(cudaMemcpy(p.d_chains.p, ct.chains.data(), ct.chains.size() * sizeof(negf::ChainRec),
                             cudaMemcpyHostToDevice));
    if (!ct.warps.empty())
        NEGF_CUDA(cudaMemcpy(p.d_warps.p, ct.warps.data(), ct.warps.size() * sizeof(negf::WarpRec),
                             cudaMemcpyHostToDevice));
    for (int i = 0; i < n; ++i) ct.rts[i].rho0 = p.tubes[i]->shard_rank == 0 ? p.tubes[i]->d_rho0 : nullptr;
    NEGF_CUDA(cudaMemcpy(p.d_rts.p, ct.rts.data(), ct.rts.size() * sizeof(negf::ReduceTube), cudaMemcpyHostToDevice));
    return NEGF_OK;
}

cudaError_t plan_launch(const negf_charge_plan& p, const int* skip, cudaStream_t s, cudaStream_t side) {
    const negf::FusedOrder fo{p.d_order.as<int>(), p.n64, p.n32, side, p.fork, p.join};
    cudaError_t e = negf::launch_rgf(p.d_tubes.as<negf::TubeDev>(), p.d_chains.as<negf::ChainRec>(),
                                     p.d_warps.as<negf::WarpRec>(), p.num_warps, p.d_units.as<negf::SegUnit>(),
                                     p.num_units, p.d_partial.as<double>(), p.d_scratch.p, p.wpb, s, nullptr, skip,
                                     p.schedule == negf::kScheduleFused ? 1 : p.pieces, p.d_pieces.as<double>(),
                                     p.schedule, &fo);
    if (e != cudaSuccess) return e;
    return negf::launch_reduce(p.d_rts.as<negf::ReduceTube>(), (int)p.tubes.size(), p.max_N,
                               p.d_partial.as<double>(), p.d_Q, s, skip);
}
}  // namespace

int negf_charge_plan_create(negf_tube* const* tubes, int num_tubes, double* d_Q, int flags, negf_charge_plan** out) {
    if (!tubes || num_tubes <= 0 || !d_Q || !out) return fail(NEGF_ERR_ARG, "null argument");
    *out = nullptr;
    int rc = require_device();
    if (rc) return rc;
    std::lock_guard<std::mutex> lk(g_mu);
    std::unique_ptr<negf_charge_plan> p(new negf_charge_plan());
    for (int i = 0; i < num_tubes; ++i)
        if (!tubes[i]) return fail(NEGF_ERR_ARG, "null tube in batch");
    if (int rc2 = check_batch_device(tubes, num_tubes)) return rc2;
    for (int i = 0; i < num_tubes; ++i) {
        update_paths(*tubes[i]);
        p->tubes.push_back(tubes[i]);
        p->versions.push_back(tubes[i]->version);
    }
    p->d_Q = d_Q;
    p->force_fp64 = (flags & NEGF_PLAN_FP64) != 0;
    NEGF_CUDA(cudaEventCreateWithFlags(&p->fork, cudaEventDisableTiming));
    NEGF_CUDA(cudaEventCreateWithFlags(&p->join, cudaEventDisableTiming));
    cudaStream_t side0 = nullptr;  // the autotuner's launches run on the legacy default stream
    if (int rc3 = plan_side_stream(0, &side0)) return rc3;
    p->wpb = settings().warps_per_block;
    rc = plan_tables(*p, negf::kSegsPerUnit, true);
    if (rc) return rc;
    {
        // pass-1 pieces as negf_compute_charge chooses them (the setting, else the automatic rule)
        int pc = settings().pass1_pieces;
        if (pc == 0 && settings().schedule == NEGF_SCHEDULE_FUSED) pc = 1;
        if (pc == 0) pc = auto_pieces(p->num_warps, p->max_N);
        p->pieces = std::max(1, pc);
    }
    p->schedule = choose_schedule(settings().schedule, p->num_warps, p->pieces);
    if (p->schedule == negf::kScheduleFused) p->pieces = 1;
    // piece candidates of the autotuner: only when the chains cannot fill the GPU
    std::vector<int> piece_cands = {1};
    if ((flags & NEGF_PLAN_AUTOTUNE) && p->num_warps < 4 * device_sm_count()) {
        const int maxp = std::min(128, std::max(1, ((p->max_N + negf::kSeg - 1) / negf::kSeg) / 32));
        for (int q : {2, 4, 8, auto_pieces(p->num_warps, p->max_N)})
            if (q > 1 && q <= maxp && std::find(piece_cands.begin(), piece_cands.end(), q) == piece_cands.end())
                piece_cands.push_back(q);
    }
    {
        int maxpc = p->pieces;
        for (int q : piece_cands) maxpc = std::max(maxpc, q);
        if (maxpc > 1)
            NEGF_CUDA(p->d_pieces.reserve(sizeof(double) * (size_t)std::max(1, p->num_warps) * maxpc * 24 *
                                          negf::kWarp));
    }
    if (flags & NEGF_PLAN_AUTOTUNE) {
        // time the fused schedule (wpb 0 below) and every two-pass shape
        // (segments per pass-2 unit x pass-2 warps per block x pass-1 pieces) on this batch
        cudaEvent_t e0, e1;
        NEGF_CUDA(cudaEventCreate(&e0));
        NEGF_CUDA(cudaEventCreate(&e1));
        double best = 1e300;
        int best_spu = negf::kSegsPerUnit, best_wpb = p->wpb, best_pc = 1;
        for (int spu : {16, 32, 64}) {
            rc = plan_tables(*p, spu, false);
            if (rc) break;
            for (int wpb : {0, 1, 2, 4}) {
                if (wpb == 0 && spu != 16) continue;  // the fused schedule has no segment units
                for (int pc : piece_cands) {
                    if (wpb == 0 && pc != 1) continue;  // the fused schedule runs whole chains
                    p->wpb = wpb == 0 ? 4 : wpb;
                    p->schedule = wpb == 0 ? negf::kScheduleFused : negf::kScheduleTwoPass;
                    p->pieces = pc;
                    cudaError_t e = plan_launch(*p, nullptr, 0, side0);
                    for (int r = 0; r < 3 && e == cudaSuccess; ++r) {
                        if (r == 1) e = cudaEventRecord(e0, 0);
                        if (e == cudaSuccess) e = plan_launch(*p, nullptr, 0, side0);
                    }
                    if (e == cudaSuccess) e = cudaEventRecord(e1, 0);
                    if (e == cudaSuccess) e = cudaEventSynchronize(e1);
                    float ms = 0.f;
                    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
                    if (e != cudaSuccess) {
                        cudaEventDestroy(e0);
                        cudaEventDestroy(e1);
                        return fail(NEGF_ERR_CUDA, cudaGetErrorString(e));
                    }
                    if (ms / 2 < best) {
                        best = ms / 2;
                        best_spu = spu;
                        best_wpb = wpb;
                        best_pc = pc;
                    }
                }
            }
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        if (rc) return rc;
        p->schedule = best_wpb == 0 ? negf::kScheduleFused : negf::kScheduleTwoPass;
        p->wpb = best_wpb == 0 ? 4 : best_wpb;
        p->pieces = best_pc;
        p->tuned_ms = best;
        rc = plan_tables(*p, best_spu, false);
        if (rc) return rc;
    }
    *out = p.release();
    return NEGF_OK;
}

int negf_charge_plan_launch(negf_charge_plan* p, const int* d_skip, void* stream) {
    if (!p) return fail(NEGF_ERR_ARG, "null plan");
    for (size_t i = 0; i < p->tubes.size(); ++i)
        if (p->tubes[i]->version != p->versions[i] || p->tubes[i]->limits_dirty)
            return fail(NEGF_ERR_STATE, "charge plan is stale: the energy paths of tube " + std::to_string(i) +
                                            " changed after the plan was made");
    cudaStream_t side = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_mu);
        if (int rc = plan_side_stream((cudaStream_t)stream, &side)) return rc;
    }
    NEGF_CUDA(plan_launch(*p, d_skip, (cudaStream_t)stream, side));
    return NEGF_OK;
}

int negf_charge_plan_pieces(const negf_charge_plan* p, int* pieces) {
    if (!p || !pieces) return fail(NEGF_ERR_ARG, "null argument");
    *pieces = p->schedule == negf::kScheduleFused ? 1 : p->pieces;
    return NEGF_OK;
}

int negf_charge_plan_info(const negf_charge_plan* p, int* pass2_warps_per_block, int* segs_per_unit,
                          double* tuned_ms, long long* updates) {
    if (!p) return fail(NEGF_ERR_ARG, "null plan");
    if (pass2_warps_per_block) *pass2_warps_per_block = p->schedule == negf::kScheduleFused ? 0 : p->wpb;
    if (segs_per_unit) *segs_per_unit = p->spu;
    if (tuned_ms) *tuned_ms = p->tuned_ms;
    if (updates) *updates = p->updates;
    return NEGF_OK;
}

int negf_charge_plan_destroy(negf_charge_plan* p) {
    delete p;
    return NEGF_OK;
}

int negf_set_tuning(int key, int value) {
    std::lock_guard<std::mutex> lk(g_mu);
    Settings& G = settings();
    switch (key) {
        case NEGF_TUNE_PASS2_WARPS_PER_BLOCK:
            if (value != 1 && value != 2 && value != 4) return fail(NEGF_ERR_ARG, "warps per block must be 1, 2 or 4");
            G.warps_per_block = value;
            return NEGF_OK;
        case NEGF_TUNE_PASS1_PIECES:
            if (value < 0 || value > 4096) return fail(NEGF_ERR_ARG, "pieces must be in [0, 4096] (0: automatic)");
            G.pass1_pieces = value;
            return NEGF_OK;
        case NEGF_TUNE_SCHEDULE:
            if (value != 0 && value != NEGF_SCHEDULE_TWO_PASS && value != NEGF_SCHEDULE_FUSED)
                return fail(NEGF_ERR_ARG, "schedule must be 0 (automatic), NEGF_SCHEDULE_TWO_PASS or NEGF_SCHEDULE_FUSED");
            G.schedule = value;
            return NEGF_OK;
        case NEGF_TUNE_NN_GEMM:
            if (value != 0 && value != NEGF_NN_GEMM_TCGEN05 && value != NEGF_NN_GEMM_MMA_SYNC &&
                value != NEGF_NN_GEMM_TCGEN05_STAGED)
                return fail(NEGF_ERR_ARG, "GEMM path must be 0 (default), NEGF_NN_GEMM_TCGEN05, "
                                          "NEGF_NN_GEMM_TCGEN05_STAGED or NEGF_NN_GEMM_MMA_SYNC");
            G.nn_gemm = value;
            return NEGF_OK;
        default:
            return fail(NEGF_ERR_ARG, "unknown tuning key");
    }
}

int negf_set_timing(int enable) {
    std::lock_guard<std::mutex> lk(g_mu);
    settings().timing = enable != 0;
    return NEGF_OK;
}

namespace {
// Kernel times of the last timed charge call, read from its workspace's
// events into the statistics (callers hold g_mu).
int collect_stats_times() {
    Settings& G = settings();
    if (Workspace* W = G.stats_ws) {
        NEGF_CUDA(cudaEventSynchronize(W->ev[2]));
        float a = 0, b = 0, p1 = 0;
        NEGF_CUDA(cudaEventElapsedTime(&a, W->ev[0], W->ev[1]));
        NEGF_CUDA(cudaEventElapsedTime(&b, W->ev[1], W->ev[2]));
        NEGF_CUDA(cudaEventElapsedTime(&p1, W->ev[0], W->ev[3]));
        G.stats.rgf_kernel_ms = a;
        G.stats.pass1_kernel_ms = p1;
        G.stats.pass2_kernel_ms = a - p1;
        G.stats.reduce_kernel_ms = b;
        G.stats_ws = nullptr;
    }
    return NEGF_OK;
}
}  // namespace

int negf_release_scratch(void* stream) {
    std::lock_guard<std::mutex> lk(g_mu);
    int dev = 0;
    NEGF_CUDA(cudaGetDevice(&dev));
    auto& all = workspaces();
    auto it = all.find(WsKey{dev, (cudaStream_t)stream});
    if (it == all.end()) return NEGF_OK;
    Workspace* w = it->second.get();
    // the last call's kernels (and the FP32 warps it ran on the side stream,
    // joined before `done`) must be finished before their buffers go
    if (w->used) NEGF_CUDA(cudaEventSynchronize(w->done));
    // the kernel times of a timed last call are read before its events go
    if (settings().stats_ws == w)
        if (int rc = collect_stats_times()) return rc;
    all.erase(it);
    return NEGF_OK;
}

int negf_last_stats(negf_stats* s) {
    if (!s) return fail(NEGF_ERR_ARG, "null argument");
    std::lock_guard<std::mutex> lk(g_mu);
    if (int rc = collect_stats_times()) return rc;
    *s = settings().stats;
    return NEGF_OK;
}


// ------------------------------------------------------------------ Broyden
int negf_broyden_create(int S, int max_step, double fraction, int norm_type, negf_broyden** out) {
    if (!out || S <= 0 || max_step < 2) return fail(NEGF_ERR_ARG, "bad Broyden arguments");
    if (norm_type != NEGF_NORM_ABSOLUTE && norm_type != NEGF_NORM_RELATIVE) return fail(NEGF_ERR_ARG, "bad norm type");
    int rc = require_device();
    if (rc) return rc;
    std::unique_ptr<negf_broyden> b(new negf_broyden());
    cudaGetDevice(&b->device);
    negf::BroydenDev& d = b->dev;
    d.S = S;
    d.max_step = max_step;
    d.norm_type = norm_type;
    d.fraction = fraction;
    d.scalar = 1.0;
    d.base = 0;
    d.nseg = 1;
    d.nblocks = std::min(1024, (S + 255) / 256);
    double** vec[] = {&d.n_in, &d.n_prev, &d.F, &d.dF, &d.norm, &d.sum};
    for (double** p : vec) {
        NEGF_CUDA(cudaMalloc(p, sizeof(double) * S));
        NEGF_CUDA(cudaMemset(*p, 0, sizeof(double) * S));
    }
    NEGF_CUDA(cudaMalloc(&d.V, sizeof(double) * (size_t)S * max_step));
    NEGF_CUDA(cudaMalloc(&d.W, sizeof(double) * (size_t)S * max_step));
    NEGF_CUDA(cudaMemset(d.V, 0, sizeof(double) * (size_t)S * max_step));
    NEGF_CUDA(cudaMemset(d.W, 0, sizeof(double) * (size_t)S * max_step));
    NEGF_CUDA(cudaMalloc(&d.c, sizeof(double) * max_step));
    NEGF_CUDA(cudaMemset(d.c, 0, sizeof(double) * max_step));
    NEGF_CUDA(cudaMalloc(&d.scal, sizeof(double) * 4));
    NEGF_CUDA(cudaMemset(d.scal, 0, sizeof(double) * 4));
    NEGF_CUDA(cudaMalloc(&d.part, sizeof(double) * 3 * d.nblocks));
    NEGF_CUDA(cudaMalloc(&d.step_dev, 2 * sizeof(int)));
    const int init[2] = {1, 0};
    NEGF_CUDA(cudaMemcpy(d.step_dev, init, 2 * sizeof(int), cudaMemcpyHostToDevice));
    *out = b.release();
    return NEGF_OK;
}

int negf_broyden_destroy(negf_broyden* b) {
    delete b;
    return NEGF_OK;
}

int negf_broyden_set_input(negf_broyden* b, const double* n_in, int on_device, void* stream) {
    if (!b || !n_in) return fail(NEGF_ERR_ARG, "null argument");
    NEGF_CUDA(cudaMemcpyAsync(b->dev.n_in, n_in, sizeof(double) * b->dev.S,
                              on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, (cudaStream_t)stream));
    if (!on_device) NEGF_CUDA(cudaStreamSynchronize((cudaStream_t)stream));
    return NEGF_OK;
}

int negf_broyden_step(negf_broyden* b, const double* d_n_out, double* d_n_in_out, double* d_norm, double* max_norm,
                      int* status, void* stream) {
    if (!b || !d_n_out) return fail(NEGF_ERR_ARG, "null argument");
    cudaStream_t s = (cudaStream_t)stream;
    if (status) *status = 0;
    if (b->step + b->dev.base > b->dev.max_step) {  // Transport.cpp:389-393 (seeded rows take capacity)
        if (status) *status = 1;
        return fail(NEGF_ERR_STATE, "Broyden_Step has exceeded the Broyden_Threshold_MaxStep");
    }
    NEGF_CUDA(negf::broyden_norm(b->dev, d_n_out, s));
    NEGF_CUDA(negf::broyden_update(b->dev, b->step - 1, s));
    b->step += 1;
    NEGF_CUDA(negf::set_int(b->dev.step_dev, b->step, s));
    if (d_n_in_out)
        NEGF_CUDA(cudaMemcpyAsync(d_n_in_out, b->dev.n_in, sizeof(double) * b->dev.S, cudaMemcpyDeviceToDevice, s));
    if (d_norm)
        NEGF_CUDA(cudaMemcpyAsync(d_norm, b->dev.norm, sizeof(double) * b->dev.S, cudaMemcpyDeviceToDevice, s));
    if (max_norm) {
        NEGF_CUDA(cudaMemcpyAsync(max_norm, b->dev.scal, sizeof(double), cudaMemcpyDeviceToHost, s));
        NEGF_CUDA(cudaStreamSynchronize(s));
        if (!std::isfinite(*max_norm)) return fail(NEGF_ERR_NUMERIC, "non-finite Broyden norm");
    }
    return NEGF_OK;
}

int negf_broyden_reset(negf_broyden* b, int keep_charge, double init_value, void* stream) {
    if (!b) return fail(NEGF_ERR_ARG, "null argument");
    cudaStream_t s = (cudaStream_t)stream;
    negf::BroydenDev& d = b->dev;
    if (!keep_charge) NEGF_CUDA(negf::broyden_set(d.n_in, init_value, d.S, s));
    double* vec[] = {d.n_prev, d.F, d.dF, d.norm, d.sum};
    for (double* p : vec) NEGF_CUDA(cudaMemsetAsync(p, 0, sizeof(double) * d.S, s));
    NEGF_CUDA(cudaMemsetAsync(d.V, 0, sizeof(double) * (size_t)d.S * d.max_step, s));
    NEGF_CUDA(cudaMemsetAsync(d.W, 0, sizeof(double) * (size_t)d.S * d.max_step, s));
    NEGF_CUDA(cudaMemsetAsync(d.c, 0, sizeof(double) * d.max_step * d.nseg, s));
    d.base = 0;
    b->step = 1;
    NEGF_CUDA(negf::set_int(d.step_dev, 1, s));
    NEGF_CUDA(negf::set_int(d.step_dev + 1, 0, s));
    return NEGF_OK;
}

int negf_broyden_set_initial_jacobian(negf_broyden* b, const double* d_V, const double* d_W, int k, void* stream) {
    if (!b || k < 0 || (k > 0 && (!d_V || !d_W))) return fail(NEGF_ERR_ARG, "bad initial-Jacobian arguments");
    negf::BroydenDev& d = b->dev;
    if (k > d.max_step / 2) return fail(NEGF_ERR_ARG, "at most max_step / 2 seeded rows");
    cudaStream_t s = (cudaStream_t)stream;
    int step = 0;
    NEGF_CUDA(cudaMemcpyAsync(&step, d.step_dev, sizeof(int), cudaMemcpyDeviceToHost, s));
    NEGF_CUDA(cudaStreamSynchronize(s));
    if (step != 1 || b->step != 1)
        return fail(NEGF_ERR_STATE, "the initial inverse Jacobian is set before the first step (after create or reset)");
    const size_t bytes = sizeof(double) * (size_t)d.S * k;
    if (k > 0) {
        NEGF_CUDA(cudaMemcpyAsync(d.V + d.S, d_V, bytes, cudaMemcpyDeviceToDevice, s));
        NEGF_CUDA(cudaMemcpyAsync(d.W + d.S, d_W, bytes, cudaMemcpyDeviceToDevice, s));
    }
    d.base = k;
    NEGF_CUDA(negf::set_int(d.step_dev + 1, k, s));
    return NEGF_OK;
}

int negf_broyden_set_segments(negf_broyden* b, int nseg, const int* offsets, void* stream) {
    if (!b || nseg < 1 || (nseg > 1 && !offsets)) return fail(NEGF_ERR_ARG, "bad segment arguments");
    negf::BroydenDev& d = b->dev;
    std::vector<int> off(nseg + 1), of;
    if (nseg > 1) {
        for (int g = 0; g <= nseg; ++g) off[g] = offsets[g];
        if (off[0] != 0 || off[nseg] != d.S) return fail(NEGF_ERR_ARG, "segment offsets must run from 0 to S");
        for (int g = 0; g < nseg; ++g)
            if (off[g + 1] <= off[g]) return fail(NEGF_ERR_ARG, "segment offsets must increase");
        of.resize(d.S);
        for (int g = 0; g < nseg; ++g)
            for (int i = off[g]; i < off[g + 1]; ++i) of[i] = g;
    }
    cudaStream_t s = (cudaStream_t)stream;
    int step = 0;
    NEGF_CUDA(cudaMemcpyAsync(&step, d.step_dev, sizeof(int), cudaMemcpyDeviceToHost, s));
    NEGF_CUDA(cudaStreamSynchronize(s));
    if (step != 1 || b->step != 1 || d.base != 0)
        return fail(NEGF_ERR_STATE, "segments are set before the first step and before seeding (after create or reset)");
    double* c = nullptr;
    double* dd = nullptr;
    int* seg_off = nullptr;
    int* seg_of = nullptr;
    NEGF_CUDA(cudaMalloc(&c, sizeof(double) * (size_t)d.max_step * nseg));
    NEGF_CUDA(cudaMemset(c, 0, sizeof(double) * (size_t)d.max_step * nseg));
    if (nseg > 1) {
        NEGF_CUDA(cudaMalloc(&dd, sizeof(double) * nseg));
        NEGF_CUDA(cudaMalloc(&seg_off, sizeof(int) * (nseg + 1)));
        NEGF_CUDA(cudaMalloc(&seg_of, sizeof(int) * d.S));
        NEGF_CUDA(cudaMemcpy(seg_off, off.data(), sizeof(int) * (nseg + 1), cudaMemcpyHostToDevice));
        NEGF_CUDA(cudaMemcpy(seg_of, of.data(), sizeof(int) * d.S, cudaMemcpyHostToDevice));
    }
    // the old buffers may still be read by work queued on other streams
    NEGF_CUDA(cudaDeviceSynchronize());
    cudaFree(d.c);
    if (d.dd) cudaFree(d.dd);
    if (d.seg_off) cudaFree(d.seg_off);
    if (d.seg_of) cudaFree(d.seg_of);
    d.c = c;
    d.dd = dd;
    d.seg_off = seg_off;
    d.seg_of = seg_of;
    d.nseg = nseg;
    return NEGF_OK;
}

int negf_broyden_restart(negf_broyden* b, int keep_rows, void* stream) {
    if (!b || keep_rows < 0) return fail(NEGF_ERR_ARG, "bad restart arguments");
    negf::BroydenDev& d = b->dev;
    cudaStream_t s = (cudaStream_t)stream;
    int st[2] = {1, 0};
    NEGF_CUDA(cudaMemcpyAsync(st, d.step_dev, 2 * sizeof(int), cudaMemcpyDeviceToHost, s));
    NEGF_CUDA(cudaStreamSynchronize(s));
    // rows 1 .. base are seeds, the solve added one row per step after its first.
    // Every row is a correction on top of the rows before it, so a subset that
    // drops the oldest rows is no consistent inverse Jacobian: keep all of them,
    // or none once they exceed the limit.
    const int rows = st[1] + std::max(0, st[0] - 2);
    const int keep = rows <= std::min(keep_rows, d.max_step / 2) ? rows : 0;
    d.base = keep;
    b->step = 1;
    NEGF_CUDA(negf::set_int(d.step_dev, 1, s));
    NEGF_CUDA(negf::set_int(d.step_dev + 1, keep, s));
    return NEGF_OK;
}

int negf_broyden_history(negf_broyden* b, double** d_V, double** d_W, int* rows, void* stream) {
    if (!b || !d_V || !d_W || !rows) return fail(NEGF_ERR_ARG, "null argument");
    negf::BroydenDev& d = b->dev;
    cudaStream_t s = (cudaStream_t)stream;
    int st[2] = {1, 0};
    NEGF_CUDA(cudaMemcpyAsync(st, d.step_dev, 2 * sizeof(int), cudaMemcpyDeviceToHost, s));
    NEGF_CUDA(cudaStreamSynchronize(s));
    *rows = st[1] + std::max(0, st[0] - 2);
    *d_V = d.V + d.S;  // row 1
    *d_W = d.W + d.S;
    return NEGF_OK;
}

int negf_broyden_step_number(negf_broyden* b, int* step) {
    if (!b || !step) return fail(NEGF_ERR_ARG, "null argument");
    // device-resident steps advance the device counter only
    NEGF_CUDA(cudaMemcpy(&b->step, b->dev.step_dev, sizeof(int), cudaMemcpyDeviceToHost));
    *step = b->step;
    return NEGF_OK;
}

int negf_broyden_step_device(negf_broyden* b, const double* d_n_out, double max_norm, int* d_flags, void* stream) {
    if (!b || !d_n_out || !d_flags) return fail(NEGF_ERR_ARG, "null argument");
    cudaStream_t s = (cudaStream_t)stream;
    NEGF_CUDA(negf::broyden_norm(b->dev, d_n_out, s, d_flags));
    NEGF_CUDA(negf::broyden_update(b->dev, 0, s, d_flags));
    NEGF_CUDA(negf::broyden_finish_step(b->dev, max_norm, 0.0, d_flags, s));
    return NEGF_OK;
}

int negf_broyden_step_device_switch(negf_broyden* b, const double* d_n_out, double max_norm, double switch_norm,
                                    int* d_flags, void* stream) {
    if (!b || !d_n_out || !d_flags || !(switch_norm > 0)) return fail(NEGF_ERR_ARG, "bad argument");
    cudaStream_t s = (cudaStream_t)stream;
    NEGF_CUDA(negf::broyden_norm(b->dev, d_n_out, s, d_flags));
    NEGF_CUDA(negf::broyden_update(b->dev, 0, s, d_flags));
    NEGF_CUDA(negf::broyden_finish_step(b->dev, max_norm, switch_norm, d_flags, s));
    return NEGF_OK;
}

int negf_broyden_input_device_ptr(negf_broyden* b, double** p) {
    if (!b || !p) return fail(NEGF_ERR_ARG, "null argument");
    *p = b->dev.n_in;
    return NEGF_OK;
}

int negf_device_selftest(int which, int n, const double* in, double* out) {
    if (!in || !out || n <= 0 || which < 0 || which > 5) return fail(NEGF_ERR_ARG, "bad self-test arguments");
    int rc = require_device();
    if (rc) return rc;
    DevBuf a, b;
    NEGF_CUDA(a.reserve(sizeof(double) * n));
    NEGF_CUDA(b.reserve(sizeof(double) * n));
    NEGF_CUDA(cudaMemcpy(a.p, in, sizeof(double) * n, cudaMemcpyHostToDevice));
    if (which <= 1) {
        NEGF_CUDA(negf::selftest(which, n, a.as<double>(), b.as<double>(), 0));
    } else {
        // in = [m, count, matrices...]; out = [m, count, results...]
        const int m = (int)in[0], count = (int)in[1];
        const long long per = (long long)(which >= 4 ? 4 : 2) * m * m;
        if (m != 4 && m != 13 && m != 16) return fail(NEGF_ERR_ARG, "self-test tiles: m must be 4, 13 or 16");
        if (count < 1 || 2 + per * count > n || 2 + 2LL * m * m * count > n)
            return fail(NEGF_ERR_ARG, "self-test tiles: n too small for count matrices");
        NEGF_CUDA(cudaMemset(b.p, 0, sizeof(double) * n));
        NEGF_CUDA(negf::rs_selftest(which, m, count, a.as<double>() + 2, b.as<double>() + 2, 0));
        NEGF_CUDA(cudaMemcpy(out, b.p, sizeof(double) * n, cudaMemcpyDeviceToHost));
        out[0] = m;
        out[1] = count;
        return NEGF_OK;
    }
    NEGF_CUDA(cudaMemcpy(out, b.p, sizeof(double) * n, cudaMemcpyDeviceToHost));
    return NEGF_OK;
}

int negf_affine_potential(const double* K, const double* U0, const double* Q, double* U, int n, void* stream) {
    if (!K || !U0 || !Q || !U || n <= 0) return fail(NEGF_ERR_ARG, "bad affine-potential arguments");
    NEGF_CUDA(negf::affine_potential(K, U0, Q, U, n, (cudaStream_t)stream));
    return NEGF_OK;
}

int negf_affine_potential_masked(const double* K, const double* U0, const double* Q, double* U, int n,
                                 const int* d_skip, void* stream) {
    if (!K || !U0 || !Q || !U || n <= 0) return fail(NEGF_ERR_ARG, "bad affine-potential arguments");
    NEGF_CUDA(negf::affine_potential(K, U0, Q, U, n, (cudaStream_t)stream, d_skip));
    return NEGF_OK;
}

int negf_affine_potential_toeplitz(const double* tab, int ntab, const int* idx, const double* U0, const double* Q,
                                   double* U, int n, const int* d_skip, void* stream) {
    if (!tab || ntab <= 0 || !idx || !U0 || !Q || !U || n <= 0)
        return fail(NEGF_ERR_ARG, "bad affine-potential arguments");
    NEGF_CUDA(negf::affine_toeplitz(tab, ntab, idx, U0, Q, U, n, (cudaStream_t)stream, d_skip));
    return NEGF_OK;
}

struct negf_potential_batch {
    negf::ToeplitzOp* d_ops = nullptr;
    int2* d_blocks = nullptr;
    int num_blocks = 0;
    ~negf_potential_batch() {
        if (d_ops) cudaFree(d_ops);
        if (d_blocks) cudaFree(d_blocks);
    }
};

int negf_potential_batch_create(int ntubes, const double* const* d_tab, const int* ntab, const int* const* d_idx,
                                const double* const* d_U0, const double* const* d_Q, double* const* d_U, const int* n,
                                negf_potential_batch** out) {
    if (!out || ntubes <= 0 || !d_tab || !ntab || !d_idx || !d_U0 || !d_Q || !d_U || !n)
        return fail(NEGF_ERR_ARG, "bad potential-batch arguments");
    std::vector<negf::ToeplitzOp> ops(ntubes);
    std::vector<int2> blocks;
    for (int t = 0; t < ntubes; ++t) {
        if (!d_tab[t] || ntab[t] <= 0 || !d_idx[t] || !d_U0[t] || !d_Q[t] || !d_U[t] || n[t] <= 0)
            return fail(NEGF_ERR_ARG, "bad potential-batch entry " + std::to_string(t));
        ops[t] = {d_tab[t], d_idx[t], d_U0[t], d_Q[t], d_U[t], ntab[t], n[t]};
        for (int r = 0; r < n[t]; r += 8) blocks.push_back(make_int2(t, r));
    }
    std::unique_ptr<negf_potential_batch> b(new negf_potential_batch());
    NEGF_CUDA(cudaMalloc(&b->d_ops, sizeof(negf::ToeplitzOp) * ops.size()));
    NEGF_CUDA(cudaMalloc(&b->d_blocks, sizeof(int2) * blocks.size()));
    NEGF_CUDA(cudaMemcpy(b->d_ops, ops.data(), sizeof(negf::ToeplitzOp) * ops.size(), cudaMemcpyHostToDevice));
    NEGF_CUDA(cudaMemcpy(b->d_blocks, blocks.data(), sizeof(int2) * blocks.size(), cudaMemcpyHostToDevice));
    b->num_blocks = (int)blocks.size();
    *out = b.release();
    return NEGF_OK;
}

int negf_potential_batch_launch(negf_potential_batch* b, const int* d_skip, void* stream) {
    if (!b) return fail(NEGF_ERR_ARG, "null potential batch");
    NEGF_CUDA(negf::affine_toeplitz_batch(b->d_ops, b->d_blocks, b->num_blocks, (cudaStream_t)stream, d_skip));
    return NEGF_OK;
}

int negf_potential_batch_destroy(negf_potential_batch* b) {
    delete b;
    return NEGF_OK;
}

// ------------------------------------------------------------------ surrogate-model kernels
int negf_nn_gemm(int a_trans, int b_trans, int M, int N, int K, int batch, const void* A, int lda, long long sA,
                 const void* B, int ldb, long long sB, float* C, int ldc, long long sC, void* C_bf16, int accumulate,
                 void* stream) {
    if (!A || !B || !C || M < 0 || N < 0 || K < 0 || batch < 0) return fail(NEGF_ERR_ARG, "bad GEMM arguments");
    int path;
    {
        std::lock_guard<std::mutex> lk(g_mu);
        const int v = settings().nn_gemm;
        path = v == NEGF_NN_GEMM_MMA_SYNC ? negf::kNnGemmMmaSync
               : v == NEGF_NN_GEMM_TCGEN05_STAGED ? negf::kNnGemmTcgen05Staged
                                                  : negf::kNnGemmTcgen05;
    }
    NEGF_CUDA(negf::nn_gemm(a_trans, b_trans, M, N, K, batch, A, lda, sA, B, ldb, sB, C, ldc, sC, C_bf16, accumulate,
                            (cudaStream_t)stream, path));
    return NEGF_OK;
}
int negf_nn_gelu_fwd(long long rows, int cols, const float* a, const float* b, const float* bias, float* pre,
                     float* out, void* out_bf16, int activation, void* stream) {
    if (!a) return fail(NEGF_ERR_ARG, "null input");
    NEGF_CUDA(negf::nn_gelu_fwd(rows, cols, a, b, bias, pre, out, out_bf16, activation, (cudaStream_t)stream));
    return NEGF_OK;
}
int negf_nn_gelu_bwd(long long n, const float* dy, const float* pre, float* d, void* d_bf16, void* stream) {
    if (!dy || !pre) return fail(NEGF_ERR_ARG, "null input");
    NEGF_CUDA(negf::nn_gelu_bwd(n, dy, pre, d, d_bf16, (cudaStream_t)stream));
    return NEGF_OK;
}
int negf_nn_colsum(long long rows, int cols, const float* x, float* out, int accumulate, void* stream) {
    if (!x || !out) return fail(NEGF_ERR_ARG, "null argument");
    NEGF_CUDA(negf::nn_colsum(rows, cols, x, out, accumulate, (cudaStream_t)stream));
    return NEGF_OK;
}
int negf_nn_cast_bf16(long long n, const float* x, void* y, void* stream) {
    if (!x || !y) return fail(NEGF_ERR_ARG, "null argument");
    NEGF_CUDA(negf::nn_cast_bf16(n, x, y, (cudaStream_t)stream));
    return NEGF_OK;
}
int negf_nn_adam(long long n, float* w, const float* g, float* m, float* v, void* w_bf16, float lr, float beta1,
                 float beta2, float eps, int step, float weight_decay, void* stream) {
    if (!w || !g || !m || !v || step < 1) return fail(NEGF_ERR_ARG, "bad Adam arguments");
    NEGF_CUDA(negf::nn_adam(n, w, g, m, v, w_bf16, lr, beta1, beta2, eps, step, weight_decay, (cudaStream_t)stream));
    return NEGF_OK;
}
int negf_nn_rowdot(long long rows, int cols, const float* h, const float* w, const float* b, float* q, void* stream) {
    if (!h || !w || !q) return fail(NEGF_ERR_ARG, "null argument");
    NEGF_CUDA(negf::nn_rowdot(rows, cols, h, w, b, q, (cudaStream_t)stream));
    return NEGF_OK;
}
int negf_nn_outer(long long rows, int cols, const float* dq, const float* w, float* dh, void* dh_bf16, void* stream) {
    if (!dq || !w) return fail(NEGF_ERR_ARG, "null argument");
    NEGF_CUDA(negf::nn_outer(rows, cols, dq, w, dh, dh_bf16, (cudaStream_t)stream));
    return NEGF_OK;
}
int negf_nn_mse(long long n, const float* q, const float* y, float* d, float* partials, void* stream) {
    if (!q || !y || !d || !partials) return fail(NEGF_ERR_ARG, "null argument");
    NEGF_CUDA(negf::nn_mse(n, q, y, d, partials, (cudaStream_t)stream));
    return NEGF_OK;
}

// ------------------------------------------------------------------ real-space ring blocks
int negf_rs_compute_charge(negf_tube* t, const double* d_Uatoms, double* d_Q, void* stream) {
    if (!t || !d_Q) return fail(NEGF_ERR_ARG, "null argument");
    std::lock_guard<std::mutex> lk(g_mu);
    update_paths(*t);
    const int m = t->d.type_id[0];
    if (t->d.type_id[1] != 0) return fail(NEGF_ERR_ARG, "real-space blocks are built for zigzag (m,0) tubes");
    if (2 * m > negf::rs_max_atoms_per_block())
        return fail(NEGF_ERR_ARG, "real-space blocks hold at most " + std::to_string(negf::rs_max_atoms_per_block()) +
                                      " atoms (m <= 16)");
    cudaStream_t s = (cudaStream_t)stream;
    const int N = t->N, K = N / 2;
    // energies: RhoEq contour and poles (coefficients as in the mode-space
    // pass) and, for a biased tube, the real-axis points of RhoNonEq
    // (Compute_RhoNonEq, NEGF_Common.cpp:3115-3578: b0 A^L + b1 A^R per ring,
    // FP64).  In mixed mode the contour and pole points at least
    // mixed_fp64_band above the real axis run in FP32; the FP64 chains go
    // first in the launch, the real-axis points last.  Rho0 (U = 0, FP64)
    // does not depend on the potential: like the mode-space Rho0 of
    // negf_tube_create (Compute_Rho0 once at initialisation,
    // NEGF_Common.cpp:1300) it is computed by the first real-space call for
    // the tube and kept.
    struct RsE {
        double Er, Ei, cr, ci;
        int flags;
    };
    std::vector<RsE> e64, e32, eneq, e0;
    const bool mixed = t->d.precision == NEGF_PREC_MIXED;
    const int neq = pass_items(*t, false);
    for (int idx = 0; idx < neq; ++idx) {
        const Item it = pass_item(*t, false, idx);
        if (it.kind == negf::kRealAxis) {
            eneq.push_back({it.E.real(), it.E.imag(), it.b0, it.b1, 0});
            continue;
        }
        const bool fp32 = mixed && std::fabs(it.E.imag()) >= t->d.mixed_fp64_band;
        (fp32 ? e32 : e64).push_back({it.E.real(), it.E.imag(), it.c.real(), it.c.imag(), fp32 ? 1 : 0});
    }
    if (!t->d_rs_rho0) {
        rho0_paths(*t);
        const int n0 = pass_items(*t, true);
        for (int idx = 0; idx < n0; ++idx) {
            const Item it = pass_item(*t, true, idx);
            e0.push_back({it.E.real(), it.E.imag(), it.c.real(), it.c.imag(), 2});
        }
    }
    std::vector<RsE> all(e64);
    all.insert(all.end(), e32.begin(), e32.end());
    all.insert(all.end(), eneq.begin(), eneq.end());
    const int P = (int)all.size(), P0 = (int)e0.size(), Pn = (int)eneq.size();
    const size_t mm = (size_t)m * m;
    const size_t pe = (size_t)std::max(std::max(P, P0), 1);
    // grow-only buffers of this (device, stream) kept across calls
    if (int rc = check_batch_device(&t, 1)) return rc;
    Workspace* Wp = nullptr;
    if (int rc = get_workspace(s, &Wp)) return rc;
    DevBuf &bE = Wp->rsE, &bFlags = Wp->rsFlags, &bU0 = Wp->rsU0, &bUa = Wp->rsUa, &bCorners = Wp->rsCorners,
           &bGL = Wp->rsGL, &bGLn = Wp->rsGLn, &bRows = Wp->rsRows, &bStatus = Wp->rsStatus;
    NEGF_CUDA(bE.reserve(sizeof(double) * 4 * pe));
    NEGF_CUDA(bFlags.reserve(sizeof(int) * pe));
    NEGF_CUDA(bUa.reserve(sizeof(double) * (size_t)N * m));
    NEGF_CUDA(bU0.reserve(sizeof(double) * (size_t)N * m));
    NEGF_CUDA(bCorners.reserve(16 * 2 * mm * pe));
    NEGF_CUDA(bGL.reserve(16 * mm * K * (size_t)std::max(std::max(P - Pn, P0), 1)));
    if (Pn > 0) NEGF_CUDA(bGLn.reserve(16 * mm * (2 * (size_t)K + 1) * Pn));
    NEGF_CUDA(bRows.reserve(sizeof(double) * (size_t)N * pe));
    NEGF_CUDA(bStatus.reserve(sizeof(int)));
    NEGF_CUDA(cudaMemsetAsync(bStatus.p, 0, sizeof(int), s));
    negf::RsLeads leads;
    leads.use_decimation = t->d.use_decimation;
    leads.dec_layers = t->d.decimation_layers;
    leads.dec_iters = t->d.decimation_max_iter + 2;
    double* dE = bE.as<double>();
    auto upload = [&](const std::vector<RsE>& v, std::vector<double>& host, std::vector<int>& hflags) -> int {
        const int n = (int)v.size();
        host.assign(4 * (size_t)std::max(n, 1), 0.0);
        hflags.assign((size_t)std::max(n, 1), 0);
        for (int i = 0; i < n; ++i) {
            host[i] = v[i].Er;
            host[n + i] = v[i].Ei;
            host[2 * n + i] = v[i].cr;
            host[3 * n + i] = v[i].ci;
            hflags[i] = v[i].flags;
        }
        NEGF_CUDA(cudaMemcpyAsync(dE, host.data(), sizeof(double) * 4 * n, cudaMemcpyHostToDevice, s));
        NEGF_CUDA(cudaMemcpyAsync(bFlags.p, hflags.data(), sizeof(int) * n, cudaMemcpyHostToDevice, s));
        return NEGF_OK;
    };
    std::vector<double> host0, host1;
    std::vector<int> hflags0, hflags1;
    if (!t->d_rs_rho0) {
        double* d_rho = nullptr;
        NEGF_CUDA(cudaMalloc(&d_rho, sizeof(double) * N));
        t->d_rs_rho0 = d_rho;
        NEGF_CUDA(cudaMemsetAsync(bU0.p, 0, sizeof(double) * (size_t)N * m, s));
        if (int rc = upload(e0, host0, hflags0)) return rc;
        NEGF_CUDA(negf::launch_realspace(m, K, t->d.gamma, dE, dE + P0, dE + 2 * P0, dE + 3 * P0, P0, 0,
                                         bFlags.as<int>(), bU0.as<double>(), bU0.as<double>(), 0.0, 0.0, leads,
                                         bCorners.p, bGL.p, nullptr, bRows.as<double>(), t->d_rs_rho0, nullptr,
                                         bStatus.as<int>(), s));
        NEGF_CUDA(cudaStreamSynchronize(s));  // the host energy tables are rewritten below
    }
    const double* Ua = d_Uatoms;
    if (!Ua) {
        NEGF_CUDA(negf::rs_expand(t->d_U, N, m, bUa.as<double>(), s));
        Ua = bUa.as<double>();
    }
    if (int rc = upload(all, host1, hflags1)) return rc;
    NEGF_CUDA(negf::launch_realspace(m, K, t->d.gamma, dE, dE + P, dE + 2 * P, dE + 3 * P, P, Pn, bFlags.as<int>(),
                                     Ua, bU0.as<double>(), t->Uc[0], t->Uc[1], leads, bCorners.p, bGL.p, bGLn.p,
                                     bRows.as<double>(), d_Q, t->d_rs_rho0, bStatus.as<int>(), s));
    int status = 0;
    NEGF_CUDA(cudaMemcpyAsync(&status, bStatus.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    NEGF_CUDA(cudaEventRecord(Wp->done, s));
    Wp->used = true;
    NEGF_CUDA(cudaStreamSynchronize(s));
    if (status) return fail(NEGF_ERR_NUMERIC, "zero pivot in a real-space block inversion");
    return NEGF_OK;
}

// ------------------------------------------------------------------ transport characteristics
int negf_tube_dos_points(negf_tube* t, int* count) {
    if (!t || !count) return fail(NEGF_ERR_ARG, "null argument");
    update_paths(*t);
    *count = (int)dos_points(*t).size();
    return NEGF_OK;
}

int negf_tube_current_points(negf_tube* t, int* count) {
    if (!t || !count) return fail(NEGF_ERR_ARG, "null argument");
    update_paths(*t);
    *count = t->noneq ? (int)t->noneq_pts.size() : 0;
    return NEGF_OK;
}

int negf_compute_dos(negf_tube* t, double* E, double* dos, double* transmission, double* conductance_out,
                     double* total_conductance, double* ldos, void* stream) {
    if (!t || !E || !dos || !transmission || !conductance_out) return fail(NEGF_ERR_ARG, "null argument");
    std::lock_guard<std::mutex> lk(g_mu);
    update_paths(*t);
    const std::vector<Pt> pts = dos_points(*t);
    std::vector<double> red;
    int rc = transport_run(*t, pts, red, ldos, (cudaStream_t)stream);
    if (rc) return rc;
    const int P = (int)pts.size();
    const int apuc = t->atoms_per_ring * t->rings_per_uc;  // CNT.H:52-55
    std::vector<double> Er(P);
    for (int e = 0; e < P; ++e) {
        E[2 * e] = pts[e].E.real();
        E[2 * e + 1] = pts[e].E.imag();
        Er[e] = pts[e].E.real();
        dos[e] = kSpinDegen * (red[8 * e] / (2. * kPi)) / apuc;  // NEGF_Common.cpp:2770-2773
        transmission[e] = red[8 * e + 1];
    }
    const double tot = conductance(*t, Er, transmission, conductance_out);
    if (total_conductance) *total_conductance = tot;
    return NEGF_OK;
}

int negf_compute_current(negf_tube* t, double* current, double* integrand, void* stream) {
    if (!t || !current) return fail(NEGF_ERR_ARG, "null argument");
    std::lock_guard<std::mutex> lk(g_mu);
    update_paths(*t);
    current[0] = current[1] = 0.0;
    if (!t->noneq) return NEGF_OK;
    const std::vector<Pt>& pts = t->noneq_pts;
    std::vector<double> red;
    int rc = transport_run(*t, pts, red, nullptr, (cudaStream_t)stream);
    if (rc) return rc;
    const int P = (int)pts.size();
    const double cm = kSpinDegen * kQe / kHeVperHz;  // NEGF_Common.cpp:4576-4577
    for (int e = 0; e < P; ++e) {
        // IF at contact k = Gamma_k (f_k - f_k') A^k'_nn (NEGF_Common.cpp:4662-4682)
        const cplx fk0 = fermi(pts[e].E - t->mu[0], t->kT[0]), fk1 = fermi(pts[e].E - t->mu[1], t->kT[1]);
        const cplx wJ = pts[e].w * pts[e].J;
        current[0] += (cm * (fk0 - fk1) * wJ).real() * red[8 * e + 1];
        current[1] += (cm * (fk1 - fk0) * wJ).real() * red[8 * e + 2];
        if (integrand)
            for (int k = 0; k < 3; ++k) integrand[(size_t)k * P + e] = cm * red[8 * e + 3 + k];
    }
    return NEGF_OK;
}

int negf_tube_noneq_integrand(negf_tube* t, double* integrand, void* stream) {
    if (!t || !integrand) return fail(NEGF_ERR_ARG, "null argument");
    std::lock_guard<std::mutex> lk(g_mu);
    update_paths(*t);
    if (!t->noneq) return NEGF_OK;
    std::vector<double> v;
    int rc = noneq_integrand(*t, v, (cudaStream_t)stream);
    if (rc) return rc;
    std::copy(v.begin(), v.end(), integrand);
    return NEGF_OK;
}

int negf_tube_correct_integration_limits(negf_tube* t, void* stream) {
    if (!t) return fail(NEGF_ERR_ARG, "null argument");
    std::lock_guard<std::mutex> lk(g_mu);
    update_paths(*t);  // Generate_NonEq_Paths with the current intercuts
    if (!t->noneq || t->d.realaxis_pts > 0) return NEGF_OK;
    std::vector<double> v;
    int rc = noneq_integrand(*t, v, (cudaStream_t)stream);
    if (rc) return rc;
    // the first energy of largest |integrand at N/2| (NEGF_Common.cpp:3527-3542)
    double mx = 0.0;
    for (size_t e = 0; e < t->noneq_pts.size(); ++e)
        if (mx < std::fabs(v[e])) {
            mx = std::fabs(v[e]);
            t->E_at_max_noneq_integrand = t->noneq_pts[e].E.real();
        }
    find_intercuts(*t);
    t->limits_dirty = true;  // Generate_NonEq_Paths with the new intercuts
    update_paths(*t);
    return NEGF_OK;
}

int negf_tube_noneq_layout(negf_tube* t, int* num_paths, int* pts, double* intercuts, double* E_at_max) {
    if (!t) return fail(NEGF_ERR_ARG, "null argument");
    update_paths(*t);
    const int np = t->d.num_noneq_paths;
    if (num_paths) *num_paths = np;
    for (int p = 0; p < np; ++p) {
        if (pts) pts[p] = t->d.noneq_integration_pts[p];
        if (intercuts && p < np - 1)
            intercuts[p] = t->d.noneq_percent_intercuts[0] < 0 ? (p + 1) * (100. / np) : t->d.noneq_percent_intercuts[p];
    }
    if (E_at_max) *E_at_max = t->E_at_max_noneq_integrand;
    return NEGF_OK;
}

int negf_write_transport_char(negf_tube* t, const char* path, int count, const double* E, const double* dos,
                              const double* transmission, const double* conductance_in) {
    if (!t || !path || count < 0 || (count > 0 && (!E || !dos || !transmission || !conductance_in)))
        return fail(NEGF_ERR_ARG, "null argument");
    update_paths(*t);
    FILE* f = std::fopen(path, "w");  // Write_Eql_Characteristics, NEGF_Common.cpp:1931-1975
    if (!f) return fail(NEGF_ERR_IO, std::string("cannot open ") + path);
    std::fprintf(f, " E_r, Fermi_Contact1, Fermi_Contact2, DOS_r, Transmission_r, Conductance_r \n");
    for (int i = 0; i < count; ++i) {
        const cplx Er(E[2 * i], 0.0);
        std::fprintf(f, "%20g%20g%20g%35g%35g%35g\n", E[2 * i], fermi(Er - t->mu[0], t->kT[0]).real(),
                     fermi(Er - t->mu[1], t->kT[1]).real(), dos[i], transmission[i], conductance_in[i]);
    }
    std::fclose(f);
    return NEGF_OK;
}

int negf_write_current_header(const char* path) {
    if (!path) return fail(NEGF_ERR_ARG, "null argument");
    FILE* f = std::fopen(path, "a");  // Define_FileHeaderForCurrent, NEGF_Common.cpp:69-84
    if (!f) return fail(NEGF_ERR_IO, std::string("cannot open ") + path);
    std::fprintf(f, "'step', 'Vds' , 'Vgs', ");
    for (int k = 0; k < 2; ++k) std::fprintf(f, ", 'I at contact_%d',", k + 1);
    // the reference's literal continues over a backslash-newline: one line with 22 spaces
    std::fprintf(f, "'Avg_intg_pts', 'Total_Iter', 'Broyden_Fraction', %22s'Broyden_Scalar', "
                    "'Conductance / (2q^2/h)'\n", "");
    std::fclose(f);
    return NEGF_OK;
}

int negf_write_current(const char* path, int step, double Vds, double Vgs, const double* current,
                       double avg_intg_pts, int total_iterations, double total_conductance) {
    if (!path || !current) return fail(NEGF_ERR_ARG, "null argument");
    FILE* f = std::fopen(path, "a");  // Write_Current, NEGF_Common.cpp:4818-4840
    if (!f) return fail(NEGF_ERR_IO, std::string("cannot open ") + path);
    std::fprintf(f, "%10d%15g%15g", step, Vds, Vgs);
    for (int k = 0; k < 2; ++k) std::fprintf(f, "%20g", current[k]);
    std::fprintf(f, "%10g%10d%20g\n", avg_intg_pts, total_iterations, total_conductance);
    std::fclose(f);
    return NEGF_OK;
}

int negf_write_integrand(negf_tube* t, const char* path, int count, const double* E, const double* integrand) {
    if (!t || !path || count < 0 || (count > 0 && (!E || !integrand))) return fail(NEGF_ERR_ARG, "null argument");
    update_paths(*t);
    FILE* f = std::fopen(path, "w");  // Write_Integrand, NEGF_Common.cpp:1977-2015
    if (!f) return fail(NEGF_ERR_IO, std::string("cannot open ") + path);
    std::fprintf(f, "(E_r-mu_0)/kT Intg_Channel Intg_Source Intg_Drain |F1-F2| E_r\n");
    for (int e = 0; e < count; ++e) {
        const cplx Er(E[2 * e], 0.0);
        const double fd = std::fabs(fermi(Er - t->mu[0], t->kT[0]).real() - fermi(Er - t->mu[1], t->kT[1]).real());
        std::fprintf(f, "%25.15g%25.15g%25.15g%25.15g%25.15g%25.15g\n", (E[2 * e] - t->mu[0]) / t->kT[0],
                     integrand[e], integrand[(size_t)count + e], integrand[2 * (size_t)count + e], fd, E[2 * e]);
    }
    std::fclose(f);
    return NEGF_OK;
}

int negf_read_table1d(const char* filename, int n, double* values) {
    if (!filename || n < 0 || (n > 0 && !values)) return fail(NEGF_ERR_ARG, "null argument");
    // Read_Table1D, NEGF_Common.cpp:237-285: header line, then `position value` per line
    FILE* f = std::fopen(filename, "r");
    if (!f) return fail(NEGF_ERR_IO, std::string("Failed to read file ") + filename);
    int lines = 0, c, last = '\n';
    while ((c = std::fgetc(f)) != EOF) {
        if (c == '\n') ++lines;
        last = c;
    }
    if (last != '\n') ++lines;  // a final line without a newline still counts
    if (lines - 1 != n) {
        std::fclose(f);
        return fail(NEGF_ERR_IO, "Assert size, " + std::to_string(n) + ", is not equal to the filesize-1, " +
                                     std::to_string(lines - 1) + " !");
    }
    std::rewind(f);
    while ((c = std::fgetc(f)) != EOF && c != '\n') {
    }
    for (int l = 0; l < n; ++l) {
        double pos, v;
        if (std::fscanf(f, "%lf %lf", &pos, &v) != 2) {
            std::fclose(f);
            return fail(NEGF_ERR_IO, std::string("malformed line ") + std::to_string(l + 2) + " in " + filename);
        }
        values[l] = v;
    }
    std::fclose(f);
    return NEGF_OK;
}

// ------------------------------------------------------------------ output
int negf_write_step(negf_tube* t, const char* prefix, const double* Q, const double* norm) {
    if (!t || !prefix || !Q) return fail(NEGF_ERR_ARG, "null argument");
    const std::string p(prefix);
    std::vector<double> U(t->N);
    NEGF_CUDA(cudaMemcpy(U.data(), t->d_U, sizeof(double) * t->N, cudaMemcpyDeviceToHost));
    {
        FILE* f = std::fopen((p + "_U.dat").c_str(), "w");  // Write_PotentialAtSites, NEGF_Common.cpp:3043-3078
        if (!f) return fail(NEGF_ERR_IO, "cannot open " + p + "_U.dat");
        for (int l = 0; l < t->N; ++l) std::fprintf(f, "%d%35.6g%35.6g\n", l, t->y_nm[l], U[l]);
        std::fclose(f);
    }
    {
        FILE* f = std::fopen((p + "_Qout.dat").c_str(), "w");  // Write_InducedCharge, :3094-3102
        if (!f) return fail(NEGF_ERR_IO, "cannot open " + p + "_Qout.dat");
        std::fprintf(f, "'axial location / (nm)', 'Induced charge per site / (e)'\n");
        write_table(f, t->y_nm, Q, t->N);
        std::fclose(f);
    }
    if (norm) {
        FILE* f = std::fopen((p + "_norm.dat").c_str(), "w");  // Write_ChargeNorm, :3104-3112
        if (!f) return fail(NEGF_ERR_IO, "cannot open " + p + "_norm.dat");
        std::fprintf(f, "'axial location / (nm)', 'norm\n");
        write_table(f, t->y_nm, norm, t->N);
        std::fclose(f);
    }
    return NEGF_OK;
}

}  // extern "C"
