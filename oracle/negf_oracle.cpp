// ORACLE — TEST INFRASTRUCTURE ONLY.
//
// CPU FP64 restatement of the ELEQTRONeX NEGF induced-charge path and its
// Broyden modified-second mixing.  Only the test suite, the smoke check and
// the CPU-baseline leg of the benchmark load this library; the product
// (libnegf_b200.so) never links or calls it.
//
// Every function cites the reference file:line it restates (paths relative
// to the reference project root, Source/Solver/Transport/ abbreviated "T/").
//
// Parity pins:
//   * scripts/negf_cpp/decimation_technique/Exec/output/{Sigma,DOS,Transmission}
//     (N=4, 10 energies on [-6,0], root (F-S)/D)  -> orc_fixture_sigma_dos_T
//   * scripts/negf_python/PointContact/cpp_results/1gpu/{Sigma,DOS,Transmission}
//     (N=4, 1000 energies on [-1,1], root (F+S)/D) -> orc_fixture_sigma_dos_T
//   Induced charge and Broyden outputs have no golden file in the reference;
//   they are pinned through the same recursion kernel that the fixtures pin.
//
// Complex division: Smith (1962), "Algorithm 116: Complex division",
// CACM 5(8):435.  The reference's AMReX GpuComplex operators are not part
// of the reference tree, so results can differ from it at the ulp level.

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <mutex>
#include <thread>
#include <vector>

using cplx = std::complex<double>;

namespace {

constexpr double kPi = 3.14159265358979323846;          // AMReX MathConst::pi
constexpr double kKbEvPerK = 8.617333262e-5;            // Utils/SelectWarpXUtils/WarpXConst.H:61-62
constexpr int kSpinDegen = 2;                           // NEGF/NEGF_Common.H:351
constexpr double kQe = 1.602176634e-19;                  // Utils/SelectWarpXUtils/WarpXConst.H
constexpr double kHeVperHz = 4.135667696e-15;            // Utils/SelectWarpXUtils/WarpXConst.H:33

// Smith (1962) complex division a / b.
inline cplx cdiv(cplx a, cplx b) {
    const double c = b.real(), d = b.imag();
    if (std::fabs(c) >= std::fabs(d)) {
        const double r = d / c, den = c + d * r;
        return cplx((a.real() + a.imag() * r) / den, (a.imag() - a.real() * r) / den);
    }
    const double r = c / d, den = c * r + d;
    return cplx((a.real() * r + a.imag()) / den, (a.imag() * r - a.real()) / den);
}
inline cplx cinv(cplx b) { return cdiv(cplx(1.0, 0.0), b); }
inline cplx cmul(cplx a, cplx b) {
    return cplx(a.real() * b.real() - a.imag() * b.imag(), a.real() * b.imag() + a.imag() * b.real());
}

// Utils/CodeUtils/CodeUtil.cpp:640-690 (Newton iteration on P_n, eps 3e-11).
void gauss_legendre(int n, std::vector<double>& x, std::vector<double>& w) {
    x.assign(n, 0.0);
    w.assign(n, 0.0);
    const double eps = 3.0e-11;
    const int m = (n + 1) / 2;
    for (int i = 1; i <= m; ++i) {
        double z = std::cos(kPi * (i - 0.25) / (n + 0.5));
        double z1, pp;
        do {
            double p1 = 1.0, p2 = 0.0;
            for (int j = 1; j <= n; ++j) {
                const double p3 = p2;
                p2 = p1;
                p1 = ((2.0 * j - 1.0) * z * p2 - (j - 1.0) * p3) / j;
            }
            pp = n * (z * p1 - p2) / (z * z - 1.0);
            z1 = z;
            z = z1 - p1 / pp;
        } while (std::fabs(z - z1) > eps);
        x[i - 1] = -z;
        x[n - i] = z;
        w[i - 1] = 2.0 / ((1.0 - z * z) * pp * pp);
        w[n - i] = w[i - 1];
    }
}

struct Path {
    std::vector<cplx> E, w, J;  // energy, weight, mul_factor (Jacobian)
};

// NEGF/IntegrationPath.cpp:41-147 (id 0 = line, id 1 = circular arc).
Path gl_path(cplx mn, cplx mx, int degree, int id) {
    Path p;
    std::vector<double> x, w;
    gauss_legendre(degree, x, w);
    p.E.resize(degree);
    p.w.resize(degree);
    p.J.resize(degree);
    if (id == 0) {
        for (int i = 0; i < degree; ++i) {
            p.E[i] = (mx - mn) * 0.5 * x[i] + (mx + mn) * 0.5;
            p.J[i] = (mx - mn) * 0.5;
            p.w[i] = w[i];
        }
    } else {
        const double cr = (mx.real() * mx.real() - mn.real() * mn.real() - mn.imag() * mn.imag()) /
                          (2 * (mx.real() - mn.real()));
        const double ci = mx.imag();
        const double R = cr - mx.real();
        double th1 = std::asin(std::fabs(mn.imag()) / R);
        if (cr > mn.real()) th1 = kPi - th1;
        const double th2 = kPi;
        for (int i = 0; i < degree; ++i) {
            const double th = (th2 - th1) * 0.5 * x[i] + (th2 + th1) * 0.5;
            p.E[i] = cplx(cr + R * std::cos(th), ci + R * std::sin(th));
            p.J[i] = (th2 - th1) * 0.5 * R * std::exp(cplx(0.0, th)) * cplx(0.0, 1.0);
            p.w[i] = w[i];
        }
    }
    return p;
}

// NEGF/IntegrationPath.cpp:149-168 (uniform points, weight dE, factor 1).
Path regular_path(cplx mn, cplx mx, int pts) {
    Path p;
    const cplx dE = (mx - mn) / static_cast<double>(pts - 1);
    p.E.resize(pts);
    p.w.resize(pts);
    p.J.resize(pts);
    for (int i = 0; i < pts; ++i) {
        p.E[i] = mn + static_cast<double>(i) * dE;
        p.w[i] = dE;
        p.J[i] = 1.0;
    }
    return p;
}

// NEGF/NEGF_Common.cpp:1790-1795.
cplx fermi(cplx EmMu, double kT) {
    const cplx one(1.0, 0.0);
    return cdiv(one, std::exp(EmMu / kT) + one);
}

struct Tube {
    // chirality and tight-binding (NEGF/CNT.cpp:11-41, CNT.H:16-18)
    int m = 17, n = 0, unitcells = 100, nmodes = 1;
    double acc = 1.42e-10, gamma = 2.5;
    double R = 0.0;
    int rings_per_uc = 4, atoms_per_ring = 17;
    int N = 0;  // Hsize_glo = num_field_sites
    std::vector<int> modeJ, degen;
    std::vector<double> beta, gap;
    // contacts / integration (NEGF/NEGF_Common.H:384-445)
    double T[2] = {298.0, 298.0}, mu[2] = {0.0, 0.0};
    int eq_pts[3] = {30, 30, 30};
    std::vector<int> noneq_pts = {100};
    std::vector<double> intercuts;
    double Evmin = -14.0, Epolemax = 10.0, zplus = 1e-8, tail_lo = 14.0, tail_hi = 14.0;
    int use_decimation = 0, dec_max_iter = 30, dec_layers = 10;
    int dec_tol_is_int = 1;  // NEGF/NEGF_Common.H:475 stores 1e-5 in an int
    double dec_rel_error = 1e-5;
    int sgf_mode = 0;  // 0 = reference root selection; 1 = (F-S)/D; 2 = (F+S)/D
    int flatband_dos_pts = 100;  // NEGF/NEGF_Common.H:416
    // adaptive non-equilibrium limits (NEGF/NEGF_Common.H:453-457)
    double kT_window[2] = {1.0, 1.0};
    bool has_density = false;
    std::vector<double> density;
    double E_at_max = 0.0;
    // explicit real-axis window (noneq always) when rt_pts > 0
    int rt_pts = 0, rt_kind = 0;  // 0 regular (IntegrationPath.cpp:149), 1 GL
    double rt_min = 0.0, rt_max = 0.0;
    // potential
    std::vector<double> U;
    double Uc[2] = {0.0, 0.0};
    // derived energy limits (NEGF_Common.cpp:1687-1787)
    double kT[2], kT_min, kT_max, mu_min, mu_max;
    bool noneq = false;
    cplx E_left, E_right, E_rightmost, E_zeta, E_eta;
    std::vector<cplx> poles;
    std::vector<Path> rho0_paths, eq_paths, noneq_paths;
    // results per site per mode
    std::vector<cplx> rho0, rhoeq, rhononeq;
    std::vector<double> rho0_im_sum;  // sum over modes of Im Rho0 (stored at init)
};

// NEGF/CNT.cpp:155-176
double bandgap_of_mode(const Tube& t, int p) {
    const int m = t.m, n = t.n;
    const double f = t.acc * t.gamma / t.R;
    double eg[6] = {f * std::fabs(3.0 * p - (2 * m + n)), f * std::fabs(3.0 * p - (m + 2 * n)),
                    f * std::fabs(3.0 * p - (m - n)),     f * std::fabs(-3.0 * p + (2 * m + n)),
                    f * std::fabs(-3.0 * p + (m + 2 * n)), f * std::fabs(3.0 * p - (m - n))};
    double mn = eg[0];
    for (int i = 1; i < 6; ++i)
        if (mn > eg[i]) mn = eg[i];
    return mn;
}

// NEGF/CNT.cpp:178-225 (quicksort with last-element pivot; ties keep its order)
int qs_partition(std::vector<double>& v, std::vector<int>& id, int lo, int hi, double pivot) {
    int i = lo, j = lo;
    while (i <= hi) {
        if (v[i] > pivot) {
            ++i;
        } else {
            std::swap(v[i], v[j]);
            std::swap(id[i], id[j]);
            ++i;
            ++j;
        }
    }
    return j - 1;
}
void qs(std::vector<double>& v, std::vector<int>& id, int lo, int hi) {
    if (lo < hi) {
        const double pivot = v[hi];
        const int pos = qs_partition(v, id, lo, hi, pivot);
        qs(v, id, lo, pos - 1);
        qs(v, id, pos + 1, hi);
    }
}

// NEGF/CNT.cpp:23-41, 227-292, 67-74
void set_material(Tube& t) {
    t.R = t.acc * std::sqrt(3.0 * (double(t.m) * t.m + double(t.n) * t.n + double(t.m) * t.n)) / (2.0 * kPi);
    if (t.n == 0) {
        t.rings_per_uc = 4;
        t.atoms_per_ring = t.m;
    } else {
        t.rings_per_uc = 2;
        t.atoms_per_ring = t.m - 1;
    }
    t.N = t.unitcells * t.rings_per_uc;
    std::vector<double> eg(t.atoms_per_ring);
    std::vector<int> idx(t.atoms_per_ring);
    for (int p = 1; p <= t.atoms_per_ring; ++p) {
        eg[p - 1] = bandgap_of_mode(t, p);
        idx[p - 1] = p;
    }
    qs(eg, idx, 0, t.atoms_per_ring - 1);
    std::vector<int> modes{idx[0]}, deg{1};
    std::vector<double> gaps{eg[0]};
    for (int p = 1; p < t.atoms_per_ring; ++p) {
        if (eg[p] - gaps.back() > 1e-6) {
            modes.push_back(idx[p]);
            gaps.push_back(eg[p]);
            deg.push_back(1);
        } else {
            deg.back() += 1;
        }
    }
    t.modeJ.clear();
    t.degen.clear();
    t.beta.clear();
    t.gap.clear();
    for (int j = 0; j < t.nmodes && j < (int)modes.size(); ++j) {
        t.modeJ.push_back(modes[j]);
        t.degen.push_back(deg[j]);
        t.gap.push_back(gaps[j]);
        t.beta.push_back(2.0 * t.gamma * std::cos(kPi * modes[j] / t.m));  // CNT.cpp:288-292
    }
    t.nmodes = (int)t.modeJ.size();
}

// NEGF/CNT.cpp:354-393 (analytic lead surface Green's function, one mode).
cplx surface_gf_analytic(double gamma, double beta, cplx EmU, int sgf_mode) {
    const cplx EmU_sq = EmU * EmU;
    const double g2 = gamma * gamma;
    const cplx F = EmU_sq + g2 - beta * beta;
    const cplx S = std::sqrt(F * F - 4.0 * EmU_sq * g2);
    const cplx D = 2.0 * g2 * EmU;
    const cplx v1 = cdiv(F + S, D);
    const cplx v2 = cdiv(F - S, D);
    if (sgf_mode == 1) return v2;  // decimation_technique/Source/main.cpp:66-91
    if (sgf_mode == 2) return v1;  // spectral_function_1D_pll/Source/main.cpp
    if (v1.imag() < 0.0) return v1;
    if (v2.imag() < 0.0) return v2;
    return cplx(0.0, 0.0);  // neither root has Im<0: gr keeps its zero initial value
}

// NEGF/NEGF_Common.cpp:1436-1508 (condensed lead) + 4095-4153 (decimation),
// specialised to the diagonal (mode-space) block: every block op is the
// element-wise scalar op on this mode.  Hb(0) = -beta, Hb(1) = -gamma.
cplx surface_gf_decimation(const Tube& t, double beta, cplx EmU, int* iters) {
    const int P = t.dec_layers;
    const cplx Hb[2] = {cplx(-beta, 0.0), cplx(-t.gamma, 0.0)};
    std::vector<cplx> Ht(P > 1 ? P : 2);
    Ht[P - 1] = cinv(EmU);
    cplx HtkP = Ht[P - 1];
    for (int k = P - 2; k >= 1; --k) {
        const int j = k % 2;
        const cplx temp1 = EmU - cmul(cmul(Hb[j], Ht[k + 1]), std::conj(Hb[j]));
        Ht[k] = cinv(temp1);
        HtkP = cmul(cmul(Ht[k], Hb[j]), HtkP);
    }
    cplx C = Ht[1];
    for (int k = 2; k < P; ++k) {
        const int j = (k - 1) % 2;
        C = Ht[k] + cmul(cmul(cmul(cmul(Ht[k], std::conj(Hb[j])), C), Hb[j]), Ht[k]);
    }
    const int id = (P - 1) % 2;
    const cplx Xi_s = cmul(cmul(Hb[0], Ht[1]), std::conj(Hb[0]));
    const cplx Xi = Xi_s + cmul(cmul(Hb[id], C), std::conj(Hb[id]));
    const cplx Pi = cmul(cmul(Hb[0], HtkP), Hb[id]);

    const cplx mu0 = EmU - Xi_s, nu0 = EmU - Xi, g0 = Pi;
    const cplx nu0i = cinv(nu0), g0d = std::conj(g0);
    const cplx t1 = cmul(g0, nu0i), t2 = cmul(t1, g0d), t3 = cmul(g0d, nu0i);
    cplx mu = mu0 - t2, nu = nu0 - t2 - cmul(t3, g0), ga = cmul(t1, g0), ze = cmul(t3, g0d);
    const double tol = t.dec_tol_is_int ? double(int(t.dec_rel_error)) : t.dec_rel_error;
    double err = 1.0;
    int i = 0;
    while (err > tol) {
        const cplx mu_old = mu;
        const cplx nui = cinv(nu);
        const cplx a = cmul(cmul(ze, nui), ga), b = cmul(cmul(ga, nui), ze);
        mu = mu - a;
        nu = nu - a - b;
        ga = cmul(cmul(ga, nui), ga);
        ze = cmul(cmul(ze, nui), ze);
        const cplx e = cdiv(mu - mu_old, mu + mu_old);
        err = std::sqrt(std::norm(std::sqrt(cmul(e, e))));  // Matrix_Block_Util.H:823-831
        if (i > t.dec_max_iter) break;
        ++i;
    }
    if (iters) *iters = i;
    return cinv(mu);
}

// NEGF/NEGF_Common.cpp:4165-4177: Sigma_c = tau g tau^dagger, tau = gamma (CNT.cpp:338-352).
void sigma_contacts(const Tube& t, cplx E, int mode, cplx out[2]) {
    for (int c = 0; c < 2; ++c) {
        const cplx EmU = E - t.Uc[c];
        const cplx g = t.use_decimation ? surface_gf_decimation(t, t.beta[mode], EmU, nullptr)
                                        : surface_gf_analytic(t.gamma, t.beta[mode], EmU, t.sgf_mode);
        const cplx tau(t.gamma, 0.0);
        out[c] = cmul(cmul(tau, g), std::conj(tau));
    }
}

// NEGF/NEGF_Common.cpp:1687-1787
void energy_limits(Tube& t) {
    for (int c = 0; c < 2; ++c) t.kT[c] = kKbEvPerK * t.T[c];
    t.mu_min = std::min(t.mu[0], t.mu[1]);
    t.mu_max = std::max(t.mu[0], t.mu[1]);
    t.kT_min = std::min(t.kT[0], t.kT[1]);
    t.kT_max = std::max(t.kT[0], t.kT[1]);
    t.noneq = false;
    if (std::fabs(t.mu_min - t.mu_max) > 1e-8) t.noneq = true;
    if (std::fabs(t.kT_min - t.kT_max) > 0.01) t.noneq = true;
    if (t.rt_pts > 0) t.noneq = true;
    const cplx zp(0.0, t.zplus);
    t.E_left = t.Evmin + zp;
    t.E_rightmost = t.mu_max + t.tail_hi * t.kT_max + zp;
    const int num_poles = int((t.Epolemax - kPi * t.kT_max) / (2.0 * kPi * t.kT_max) + 1);
    t.poles.clear();
    if (t.noneq) {
        t.E_right = t.mu_min - t.tail_lo * t.kT_max + zp;
        if (t.rt_pts > 0) {
            t.E_right = cplx(t.rt_min, t.zplus);
            t.E_rightmost = cplx(t.rt_max, t.zplus);
        }
        t.E_zeta = cplx(t.E_right.real(), 2 * num_poles * kPi * t.kT_max);
        t.E_eta = cplx(t.E_right.real() - 14 * t.kT_max, t.E_zeta.imag());
    } else {
        t.E_right = t.E_rightmost;
        for (int p = 0; p < num_poles; ++p) t.poles.push_back(cplx(t.mu_min, kPi * t.kT_max * (2 * p + 1)));
        t.E_zeta = cplx(t.E_right.real(), 2 * num_poles * kPi * t.kT_max);
        const double tf = std::max(t.tail_lo, t.tail_hi);
        t.E_eta = cplx(t.mu_min - tf * t.kT_max, t.E_zeta.imag());
    }
}

// NEGF/NEGF_Common.cpp:1798-1816 (Rho0), 2188-2250 (RhoEq), 2018-2059 (NonEq)
void build_paths(Tube& t) {
    const cplx zp(0.0, t.zplus);
    t.rho0_paths = {gl_path(zp, t.E_zeta, 30, 0), gl_path(t.E_zeta, t.E_eta, 30, 0),
                    gl_path(t.E_eta, t.E_left, 30, 1)};
}
void build_eq_noneq_paths(Tube& t) {
    t.eq_paths = {gl_path(t.E_right, t.E_zeta, t.eq_pts[0], 0), gl_path(t.E_zeta, t.E_eta, t.eq_pts[1], 0),
                  gl_path(t.E_eta, t.E_left, t.eq_pts[2], 1)};
    t.noneq_paths.clear();
    if (!t.noneq) return;
    if (t.rt_pts > 0) {
        t.noneq_paths.push_back(t.rt_kind == 0 ? regular_path(t.E_right, t.E_rightmost, t.rt_pts)
                                               : gl_path(t.E_right, t.E_rightmost, t.rt_pts, 0));
        return;
    }
    const int np = (int)t.noneq_pts.size();
    std::vector<cplx> mn(np), mx(np);
    mn[0] = t.E_right;
    mx[np - 1] = t.E_rightmost;
    const cplx len = t.E_rightmost - t.E_right;
    for (int p = 0; p < np - 1; ++p) mx[p] = t.E_right + (t.intercuts[p] / 100.0) * len;
    for (int p = 1; p < np; ++p) mn[p] = mx[p - 1];
    for (int p = 0; p < np; ++p) t.noneq_paths.push_back(gl_path(mn[p], mx[p], t.noneq_pts[p], 0));
}

// One energy point of the host recursion, NEGF/NEGF_Common.cpp:3238-3312.
struct Sweep {
    std::vector<cplx> alpha, X, Y, Xt, Yt, G;
    cplx sig[2];
};
void sweep(const Tube& t, const std::vector<double>& U, cplx E, int mode, Sweep& s) {
    const int N = t.N;
    s.alpha.resize(N);
    s.X.assign(N, 0.0);
    s.Y.assign(N, 0.0);
    s.Xt.assign(N, 0.0);
    s.Yt.assign(N, 0.0);
    s.G.resize(N);
    for (int n = 0; n < N; ++n) s.alpha[n] = E - U[n];  // h_minusHa = -U (NEGF_Common.cpp:1656-1666)
    sigma_contacts(t, E, mode, s.sig);
    s.alpha[0] -= s.sig[0];
    s.alpha[N - 1] -= s.sig[1];
    const cplx Hb[2] = {cplx(-t.beta[mode], 0.0), cplx(-t.gamma, 0.0)};  // CNT.cpp:322-335
    const cplx* Hc = Hb;
    s.Y[0] = 0.0;
    for (int n = 1; n < N; ++n) {
        const int p = (n - 1) % 2;
        s.Yt[n] = cdiv(Hc[p], s.alpha[n - 1] - s.Y[n - 1]);
        s.Y[n] = cmul(Hb[p], s.Yt[n]);
    }
    s.X[N - 1] = 0.0;
    for (int n = N - 2; n >= 0; --n) {
        const int p = n % 2;
        s.Xt[n] = cdiv(Hb[p], s.alpha[n + 1] - s.X[n + 1]);
        s.X[n] = cmul(Hc[p], s.Xt[n]);
    }
    for (int n = 0; n < N; ++n) s.G[n] = cinv(s.alpha[n] - s.X[n] - s.Y[n]);
}

// Work list over energies; each worker thread accumulates its own arrays and
// the partials are summed in worker order (deterministic for a fixed count).
struct EPoint {
    cplx E, w, J, f;  // f = equilibrium Fermi factor (RhoEq) or unused
    int kind;         // 0 Rho0, 1 RhoEq contour, 2 pole, 3 NonEq
};

void accumulate_point(const Tube& t, const std::vector<double>& U, const EPoint& ep, int faithful,
                      std::vector<cplx>& acc, Sweep& s) {
    const int N = t.N, M = t.nmodes;
    for (int m = 0; m < M; ++m) {
        sweep(t, U, ep.E, m, s);
        const double deg = t.degen[m];
        if (ep.kind == 0) {  // NEGF_Common.cpp:4071-4084
            const double c = -1 * kSpinDegen / (kPi);
            for (int n = 0; n < N; ++n) acc[n * M + m] += cmul(cmul(c * s.G[n], ep.w), ep.J) * deg;
        } else if (ep.kind == 1) {  // NEGF_Common.cpp:3738-3754
            const double c = -1. * kSpinDegen / kPi;
            for (int n = 0; n < N; ++n)
                acc[n * M + m] += cmul(cmul(cmul(c * s.G[n], ep.w), ep.J), ep.f) * deg;
        } else if (ep.kind == 2) {  // NEGF_Common.cpp:3934-3948
            const cplx pole_const(0.0, -2 * t.kT_min * kSpinDegen);
            for (int n = 0; n < N; ++n) acc[n * M + m] += cmul(pole_const, s.G[n]) * deg;
        } else {  // NEGF_Common.cpp:3372-3466
            const double c = -1 * kSpinDegen / (2 * kPi);
            cplx fk[2], Gam[2];
            for (int k = 0; k < 2; ++k) {
                fk[k] = fermi(ep.E - t.mu[k], t.kT[k]);
                Gam[k] = cmul(cplx(0.0, 1.0), s.sig[k] - std::conj(s.sig[k]));
            }
            const int kglo[2] = {0, N - 1};
            if (faithful) {
                // the reference's per-site walk from each contact: O(N) per site
                for (int n = 0; n < N; ++n) {
                    cplx AnF = 0.0;
                    for (int k = 0; k < 2; ++k) {
                        const int kg = kglo[k];
                        cplx tmp = cinv(s.alpha[kg] - s.X[kg] - s.Y[kg]);
                        for (int q = kg; q < n; ++q) tmp = cmul(-s.Xt[q], tmp);
                        for (int q = kg; q > n; --q) tmp = cmul(-s.Yt[q], tmp);
                        const cplx A = cmul(cmul(tmp, Gam[k]), std::conj(tmp));
                        AnF += cmul(A, fk[k]);
                    }
                    acc[n * M + m] += cmul(cmul(c * AnF, ep.w), ep.J) * deg;
                }
            } else {
                // same quantities as O(N) running products of the walk factors
                std::vector<cplx> g0(N), g1(N);
                g0[0] = cinv(s.alpha[0] - s.X[0] - s.Y[0]);
                for (int n = 1; n < N; ++n) g0[n] = cmul(-s.Xt[n - 1], g0[n - 1]);
                g1[N - 1] = cinv(s.alpha[N - 1] - s.X[N - 1] - s.Y[N - 1]);
                for (int n = N - 2; n >= 0; --n) g1[n] = cmul(-s.Yt[n + 1], g1[n + 1]);
                for (int n = 0; n < N; ++n) {
                    const cplx A0 = cmul(cmul(g0[n], Gam[0]), std::conj(g0[n]));
                    const cplx A1 = cmul(cmul(g1[n], Gam[1]), std::conj(g1[n]));
                    const cplx AnF = cmul(A0, fk[0]) + cmul(A1, fk[1]);
                    acc[n * M + m] += cmul(cmul(c * AnF, ep.w), ep.J) * deg;
                }
            }
        }
    }
}

void run_points(const Tube& t, const std::vector<double>& U, const std::vector<EPoint>& pts, int faithful,
                int nthreads, std::vector<cplx>& out) {
    const int N = t.N, M = t.nmodes;
    out.assign((size_t)N * M, 0.0);
    if (pts.empty()) return;
    nthreads = std::max(1, std::min<int>(nthreads, (int)pts.size()));
    std::vector<std::vector<cplx>> part(nthreads, std::vector<cplx>((size_t)N * M, 0.0));
    auto worker = [&](int tid) {
        Sweep s;
        // contiguous block of points per worker
        const size_t P = pts.size();
        const size_t lo = P * tid / nthreads, hi = P * (tid + 1) / nthreads;
        for (size_t i = lo; i < hi; ++i) accumulate_point(t, U, pts[i], faithful, part[tid], s);
    };
    if (nthreads == 1) {
        worker(0);
    } else {
        std::vector<std::thread> th;
        for (int i = 0; i < nthreads; ++i) th.emplace_back(worker, i);
        for (auto& x : th) x.join();
    }
    for (int i = 0; i < nthreads; ++i)
        for (size_t j = 0; j < out.size(); ++j) out[j] += part[i][j];
}

std::vector<EPoint> collect(const std::vector<Path>& paths, int kind, const Tube& t, size_t e_lo = 0,
                            size_t e_hi = SIZE_MAX) {
    std::vector<EPoint> v;
    size_t e = 0;
    for (const auto& p : paths)
        for (size_t i = 0; i < p.E.size(); ++i, ++e) {
            if (e < e_lo || e >= e_hi) continue;
            EPoint q{p.E[i], p.w[i], p.J[i], 0.0, kind};
            if (kind == 1) q.f = fermi(p.E[i] - t.mu_min, t.kT_min);
            v.push_back(q);
        }
    return v;
}

// ---------------------------------------------------------------- transport characteristics
// DOS energy path (NEGF_Common.cpp:2188-2250): the non-equilibrium paths when
// biased, else Gauss-Legendre on [Re E_eta, E_rightmost].
std::vector<Path> dos_paths(const Tube& t) {
    if (t.noneq) return t.noneq_paths;
    return {gl_path(cplx(t.E_eta.real(), 0.0), t.E_rightmost, t.flatband_dos_pts, 0)};
}

// G_{n,k} of contact k by the reference's walk from the contact site
// (NEGF_Common.cpp:2682-2694).
cplx contact_walk(const Sweep& s, int N, int kglo, int n) {
    cplx tmp = cinv(s.alpha[kglo] - s.X[kglo] - s.Y[kglo]);
    for (int q = kglo; q < n; ++q) tmp = cmul(-s.Xt[q], tmp);
    for (int q = kglo; q > n; --q) tmp = cmul(-s.Yt[q], tmp);
    return tmp;
}

// Compute_DensityOfStates, one energy (NEGF_Common.cpp:2654-2776): per site
// A_nn = sum_k G_nk Gamma_k G_nk^*, LDOS_n = sum_m deg A_nn / 2 pi; the
// transmission trace Gamma_0 A_tk[1] with A_tk[1] = G_kk Gamma_1 G_{0,k}^*
// walked from the drain to site 0 (CT_ID[1] = 0, CNT.cpp:343-344).
// faithful = 0 replaces the per-site walks by running products.
void dos_point(const Tube& t, const std::vector<double>& U, cplx E, int faithful, Sweep& s, double* ldos,
               double& trace0, double& trace1) {
    const int N = t.N, M = t.nmodes;
    for (int m = 0; m < M; ++m) {
        sweep(t, U, E, m, s);
        const double deg = t.degen[m];
        cplx Gam[2];
        for (int k = 0; k < 2; ++k) Gam[k] = cmul(cplx(0.0, 1.0), s.sig[k] - std::conj(s.sig[k]));
        const int kglo[2] = {0, N - 1};
        std::vector<cplx> g0, g1;
        if (!faithful) {
            g0.resize(N);
            g1.resize(N);
            g0[0] = cinv(s.alpha[0] - s.X[0] - s.Y[0]);
            for (int n = 1; n < N; ++n) g0[n] = cmul(-s.Xt[n - 1], g0[n - 1]);
            g1[N - 1] = cinv(s.alpha[N - 1] - s.X[N - 1] - s.Y[N - 1]);
            for (int n = N - 2; n >= 0; --n) g1[n] = cmul(-s.Yt[n + 1], g1[n + 1]);
        }
        for (int n = 0; n < N; ++n) {
            cplx A = 0.0;
            for (int k = 0; k < 2; ++k) {
                const cplx g = faithful ? contact_walk(s, N, kglo[k], n) : (k == 0 ? g0[n] : g1[n]);
                A += cmul(cmul(g, Gam[k]), std::conj(g));
            }
            const cplx val = A * deg / (2. * kPi);
            if (ldos) ldos[n] += val.real();
            trace0 += val.real();
        }
        // A_tk[1] at n = 0
        const cplx Gkk = cinv(s.alpha[N - 1] - s.X[N - 1] - s.Y[N - 1]);
        const cplx G0k = faithful ? contact_walk(s, N, N - 1, 0) : g1[0];
        cplx Akn = cmul(cmul(Gkk, Gam[1]), std::conj(G0k));
        for (int q = N - 2; q >= 0; --q) Akn = cmul(-s.Yt[q + 1], Akn);
        trace1 += (cmul(Gam[0], Akn) * deg).real();
    }
}

// Compute_Conductance (NEGF_Common.cpp:1873-1928): G_quantum = 1, dF/dE by
// finite differences with the first grid spacing deltaE = E_0 - E_1.
double conductance(const Tube& t, const std::vector<cplx>& E, const std::vector<double>& T, std::vector<double>& C) {
    const size_t P = E.size();
    C.assign(P, 0.0);
    if (P < 3) return 0.0;
    std::vector<double> dF(P, 0.0);
    const double dE = E[0].real() - E[1].real();
    const double inv = 1. / (2 * dE);
    auto F = [&](size_t i) { return fermi(E[i] - t.mu[0], t.kT[0]).real(); };
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

// Compute_Current, one energy of the non-equilibrium paths
// (NEGF_Common.cpp:4439-4722): at the contact sites IF = Gamma_k f_k A_nn -
// Gamma_k Gn_nn with Gn_nn = sum_k' A^k'_nn f_k'; integrand probes Gn_nn at
// n = N/2 (channel), 0 (source), N-1 (drain), as an if / else-if chain.
void current_point(const Tube& t, const std::vector<double>& U, const EPoint& ep, Sweep& s, double I[2],
                   double probe[3]) {
    const int N = t.N, M = t.nmodes;
    const double cm = kSpinDegen * kQe / kHeVperHz;
    cplx fk[2];
    for (int k = 0; k < 2; ++k) fk[k] = fermi(ep.E - t.mu[k], t.kT[k]);
    const int kglo[2] = {0, N - 1};
    const int sites[3] = {N / 2, 0, N - 1};
    for (int m = 0; m < M; ++m) {
        sweep(t, U, ep.E, m, s);
        const double deg = t.degen[m];
        cplx Gam[2];
        for (int k = 0; k < 2; ++k) Gam[k] = cmul(cplx(0.0, 1.0), s.sig[k] - std::conj(s.sig[k]));
        for (int i = 0; i < 3; ++i) {
            const int n = sites[i];
            if (i == 2 && n == sites[1]) continue;  // N = 1
            cplx A = 0.0, Gn = 0.0;
            for (int k = 0; k < 2; ++k) {
                const cplx g = contact_walk(s, N, kglo[k], n);
                const cplx Ak = cmul(cmul(g, Gam[k]), std::conj(g));
                A += Ak;
                Gn += cmul(Ak, fk[k]);
            }
            for (int k = 0; k < 2; ++k)
                if (n == kglo[k]) {
                    const cplx IF = cmul(cmul(Gam[k], fk[k]), A) - cmul(Gam[k], Gn);
                    I[k] += cmul(cmul(cm * IF * deg, ep.w), ep.J).real();
                }
            const cplx v = cm * Gn * deg;
            if (n == N / 2)
                probe[0] += v.real();
            else if (n == 0)
                probe[1] += v.real();
            else if (n == N - 1)
                probe[2] += v.real();
        }
    }
}

// ---------------------------------------------------------------- adaptive non-equilibrium limits
// Integrand probes of Compute_RhoNonEq (NEGF_Common.cpp:3467-3496):
// Re(c sum_modes deg sum_k A^k_nn f_k), c = -spin/2pi, at n = N/2, else N/4,
// else 3N/4, with the per-site contact walks.
void noneq_integrand_point(const Tube& t, const std::vector<double>& U, cplx E, Sweep& s, double out[3]) {
    const int N = t.N, M = t.nmodes;
    const double c = -1 * kSpinDegen / (2 * kPi);
    cplx fk[2];
    for (int k = 0; k < 2; ++k) fk[k] = fermi(E - t.mu[k], t.kT[k]);
    const int kglo[2] = {0, N - 1};
    cplx acc[3] = {0.0, 0.0, 0.0};
    for (int m = 0; m < M; ++m) {
        sweep(t, U, E, m, s);
        const double deg = t.degen[m];
        cplx Gam[2];
        for (int k = 0; k < 2; ++k) Gam[k] = cmul(cplx(0.0, 1.0), s.sig[k] - std::conj(s.sig[k]));
        for (int n = 0; n < N; ++n) {
            int slot = -1;
            if (n == N / 2)
                slot = 0;
            else if (n == N / 4)
                slot = 1;
            else if (n == N * 3 / 4)
                slot = 2;
            if (slot < 0) continue;
            cplx AnF = 0.0;
            for (int k = 0; k < 2; ++k) {
                const cplx g = contact_walk(s, N, kglo[k], n);
                AnF += cmul(cmul(cmul(g, Gam[k]), std::conj(g)), fk[k]);
            }
            acc[slot] += c * AnF * deg;
        }
    }
    for (int k = 0; k < 3; ++k) out[k] = acc[k].real();
}

// Find_NonEq_Percent_Intercuts_Adaptively (NEGF_Common.cpp:2062-2185).
void find_intercuts(Tube& t) {
    const int np = (int)t.noneq_pts.size();
    const double Es = (t.E_at_max - t.mu[0]) / t.kT[0];
    const double Emin = (t.E_right.real() - t.mu[0]) / t.kT[0];
    const double Emax = (t.E_rightmost.real() - t.mu[0]) / t.kT[0];
    std::vector<double>& cut = t.intercuts;
    std::vector<int>& pts = t.noneq_pts;
    if (np == 3) {
        if (!t.has_density) {
            t.density = {pts[0] / ((cut[0] / 100.) * (Emax - Emin)),
                         pts[1] / (((cut[1] - cut[0]) / 100.) * (Emax - Emin)),
                         pts[2] / (((100. - cut[1]) / 100.) * (Emax - Emin))};
            t.has_density = true;
        }
        const double lo = std::max(Es - t.kT_window[0], Emin);
        const double hi = std::min(Es + t.kT_window[1], Emax);
        cut[0] = 100 * (lo - Emin) / (Emax - Emin);
        cut[1] = 100 * (hi - Emin) / (Emax - Emin);
        pts[0] = (int)(std::round(((lo - Emin) * t.density[0]) / 2) * 2);
        pts[1] = (int)(std::round(((hi - lo) * t.density[1]) / 2) * 2);
        pts[2] = (int)(std::round(((Emax - hi) * t.density[2]) / 2) * 2);
    } else if (np == 2) {
        if (!t.has_density) {
            t.density = {pts[0] / ((cut[0] / 100.) * (Emax - Emin)),
                         pts[1] / (((100 - cut[0]) / 100.) * (Emax - Emin))};
            t.has_density = true;
        }
        const double hi = Es + t.kT_window[1];
        cut[0] = 100 * (hi - Emin) / (Emax - Emin);
        pts[0] = (int)(std::round(((hi - Emin) * t.density[0]) / 2) * 2);
        pts[1] = (int)(std::round(((Emax - hi) * t.density[1]) / 2) * 2);
    }
}

// ---------------------------------------------------------------- real-space ring blocks
// A zigzag (m,0) tube in real space: blocks of two rings (2m atoms); ring 2k
// and 2k+1 joined by the double bond (atom j to atoms j and j+1 mod m),
// ring 2k+1 to ring 2k+2 by the single bond (atom j to atom j); hopping
// gamma; on-site energy U per atom.  In mode space (Fourier over the ring)
// the double bond becomes 2 gamma cos(pi J / m) = beta_J and the single bond
// gamma (CNT.cpp:288-336), so with ring-uniform potentials the block RGF
// equals the sum over all m mode chains.  Leads: semi-infinite repetitions
// of one block at the contact potential, surface Green's functions by the
// Lopez Sancho-Sancho-Rubio decimation (J. Phys. F 15, 851 (1985)).
using CMat = std::vector<cplx>;  // row-major n x n

// Gauss-Jordan inverse with partial pivoting (returns false when singular).
bool cinvert(CMat& A, int n) {
    CMat I(n * n, 0.0);
    for (int i = 0; i < n; ++i) I[i * n + i] = 1.0;
    for (int p = 0; p < n; ++p) {
        int piv = p;
        double best = std::abs(A[p * n + p]);
        for (int r = p + 1; r < n; ++r)
            if (std::abs(A[r * n + p]) > best) {
                best = std::abs(A[r * n + p]);
                piv = r;
            }
        if (!(best > 0)) return false;
        if (piv != p)
            for (int c = 0; c < n; ++c) {
                std::swap(A[p * n + c], A[piv * n + c]);
                std::swap(I[p * n + c], I[piv * n + c]);
            }
        const cplx inv = cinv(A[p * n + p]);
        for (int c = 0; c < n; ++c) {
            A[p * n + c] = cmul(A[p * n + c], inv);
            I[p * n + c] = cmul(I[p * n + c], inv);
        }
        for (int r = 0; r < n; ++r) {
            if (r == p) continue;
            const cplx f = A[r * n + p];
            if (f == cplx(0.0, 0.0)) continue;
            for (int c = 0; c < n; ++c) {
                A[r * n + c] -= cmul(f, A[p * n + c]);
                I[r * n + c] -= cmul(f, I[p * n + c]);
            }
        }
    }
    A.swap(I);
    return true;
}
CMat cgemm(const CMat& A, const CMat& B, int n) {
    CMat C(n * n, 0.0);
    for (int i = 0; i < n; ++i)
        for (int k = 0; k < n; ++k) {
            const cplx a = A[i * n + k];
            if (a == cplx(0.0, 0.0)) continue;
            for (int j = 0; j < n; ++j) C[i * n + j] += cmul(a, B[k * n + j]);
        }
    return C;
}

// E - H of one block (2m atoms) with on-site potentials U[2m].
CMat rs_block(int m, double gamma, cplx E, const double* U) {
    const int n = 2 * m;
    CMat A(n * n, 0.0);
    for (int i = 0; i < n; ++i) A[i * n + i] = E - U[i];
    for (int j = 0; j < m; ++j) {
        const int a = j, b1 = m + j, b2 = m + (j + 1) % m;
        A[a * n + b1] -= gamma;
        A[b1 * n + a] -= gamma;
        A[a * n + b2] -= gamma;
        A[b2 * n + a] -= gamma;
    }
    return A;
}

// Surface Green's function of a semi-infinite lead of blocks at potential
// Uc.  left = true: the lead extends to the left and its surface block couples
// to the device through ring b (single bond to the device's ring a); the
// returned m x m corner is g[b][b].  left = false: lead to the right, corner
// g[a][a].  Decimation: eps_s += a g b, eps += a g b + b g a, a = a g a,
// b = b g b, with g = (E - eps)^-1, for `iters` iterations.
CMat rs_lead_corner(int m, double gamma, cplx E, double Uc, bool left, int iters) {
    const int n = 2 * m;
    std::vector<double> U(n, Uc);
    CMat eps = rs_block(m, gamma, E, U.data());  // holds E - eps
    CMat eps_s = eps;
    // tau = H_{i,i+1}: ring b of cell i to ring a of cell i+1, gamma I; in E - H: -gamma
    CMat tau(n * n, 0.0), taud(n * n, 0.0);
    for (int j = 0; j < m; ++j) {
        tau[(m + j) * n + j] = -gamma;
        taud[j * n + (m + j)] = -gamma;
    }
    // the surface that faces the device: left lead -> its last cell couples to the right (alpha = tau^dagger side)
    CMat al = left ? taud : tau, be = left ? tau : taud;
    for (int it = 0; it < iters; ++it) {
        CMat g = eps;
        cinvert(g, n);
        const CMat agb = cgemm(cgemm(al, g, n), be, n);
        const CMat bga = cgemm(cgemm(be, g, n), al, n);
        for (int i = 0; i < n * n; ++i) {
            eps_s[i] -= agb[i];
            eps[i] -= agb[i] + bga[i];
        }
        al = cgemm(cgemm(al, g, n), al, n);
        be = cgemm(cgemm(be, g, n), be, n);
    }
    CMat gs = eps_s;
    cinvert(gs, n);
    CMat corner(m * m);
    const int off = left ? m : 0;
    for (int i = 0; i < m; ++i)
        for (int j = 0; j < m; ++j) corner[i * m + j] = gs[(off + i) * n + (off + j)];
    return corner;
}

// Block RGF at one energy: the atom diagonal of G_kk for every block
// (out[k * 2m + i]).  Uatoms: [K][2m].
void rs_diag(int m, int K, double gamma, cplx E, const double* Uatoms, double Uc0, double Uc1, int iters,
             std::vector<cplx>& out) {
    const int n = 2 * m, mm = m * m;
    const double g2 = gamma * gamma;
    const CMat sL = rs_lead_corner(m, gamma, E, Uc0, true, iters);
    const CMat sR = rs_lead_corner(m, gamma, E, Uc1, false, iters);
    std::vector<CMat> gLbb(K, CMat(mm)), gRaa(K, CMat(mm));
    for (int k = 0; k < K; ++k) {  // forward: left-connected g_L, corner [b][b]
        CMat M = rs_block(m, gamma, E, Uatoms + (size_t)k * n);
        const CMat& c = k == 0 ? sL : gLbb[k - 1];
        for (int i = 0; i < m; ++i)
            for (int j = 0; j < m; ++j) M[i * n + j] -= g2 * c[i * m + j];
        cinvert(M, n);
        for (int i = 0; i < m; ++i)
            for (int j = 0; j < m; ++j) gLbb[k][i * m + j] = M[(m + i) * n + (m + j)];
    }
    for (int k = K - 1; k >= 0; --k) {  // backward: right-connected g_R, corner [a][a]
        CMat M = rs_block(m, gamma, E, Uatoms + (size_t)k * n);
        const CMat& c = k == K - 1 ? sR : gRaa[k + 1];
        for (int i = 0; i < m; ++i)
            for (int j = 0; j < m; ++j) M[(m + i) * n + (m + j)] -= g2 * c[i * m + j];
        cinvert(M, n);
        for (int i = 0; i < m; ++i)
            for (int j = 0; j < m; ++j) gRaa[k][i * m + j] = M[i * n + j];
    }
    out.assign((size_t)K * n, 0.0);
    for (int k = 0; k < K; ++k) {  // G_kk = (E - H_kk - Sigma_L - Sigma_R)^-1
        CMat M = rs_block(m, gamma, E, Uatoms + (size_t)k * n);
        const CMat& cl = k == 0 ? sL : gLbb[k - 1];
        const CMat& cr = k == K - 1 ? sR : gRaa[k + 1];
        for (int i = 0; i < m; ++i)
            for (int j = 0; j < m; ++j) {
                M[i * n + j] -= g2 * cl[i * m + j];
                M[(m + i) * n + (m + j)] -= g2 * cr[i * m + j];
            }
        cinvert(M, n);
        for (int i = 0; i < n; ++i) out[(size_t)k * n + i] = M[i * n + i];
    }
}

// Non-equilibrium ring sums at one real-axis energy: for every ring the sum
// over its atoms of the contact spectral functions A^c_nn = [G_{n,c} Gamma_c
// G_{n,c}^dagger]_nn (Compute_RhoNonEq, NEGF_Common.cpp:3372-3466, on the
// atom basis: Gamma_c = i (Sigma_c - Sigma_c^dagger), Sigma_L = gamma^2 sL on
// ring a of block 0, Sigma_R = gamma^2 sR on ring b of block K-1).  Dense
// 2m x 2m blocks: left-connected g_L for the source column (G_{k,0} =
// gamma G_kk[:, a] g_L[k-1]_{b,0}), right-connected g_R for the drain column
// (G_{k,K-1} = gamma G_kk[:, b] g_R[k+1]_{a,K-1}), G_kk from both sides.
// outL / outR: [2K] ring sums.
void rs_noneq(int m, int K, double gamma, cplx E, const double* Uatoms, double Uc0, double Uc1, int iters,
              std::vector<double>& outL, std::vector<double>& outR) {
    const int n = 2 * m, mm = m * m;
    const double g2 = gamma * gamma;
    const CMat sL = rs_lead_corner(m, gamma, E, Uc0, true, iters);
    const CMat sR = rs_lead_corner(m, gamma, E, Uc1, false, iters);
    std::vector<CMat> gL(K), gR(K);
    for (int k = 0; k < K; ++k) {
        CMat M = rs_block(m, gamma, E, Uatoms + (size_t)k * n);
        for (int i = 0; i < m; ++i)
            for (int j = 0; j < m; ++j)
                M[i * n + j] -= g2 * (k == 0 ? sL[i * m + j] : gL[k - 1][(m + i) * n + (m + j)]);
        cinvert(M, n);
        gL[k] = M;
    }
    for (int k = K - 1; k >= 0; --k) {
        CMat M = rs_block(m, gamma, E, Uatoms + (size_t)k * n);
        for (int i = 0; i < m; ++i)
            for (int j = 0; j < m; ++j)
                M[(m + i) * n + (m + j)] -= g2 * (k == K - 1 ? sR[i * m + j] : gR[k + 1][i * n + j]);
        cinvert(M, n);
        gR[k] = M;
    }
    // Gamma of each contact (m x m)
    CMat GamL(mm), GamR(mm);
    for (int i = 0; i < m; ++i)
        for (int j = 0; j < m; ++j) {
            const cplx a = g2 * sL[i * m + j], at = std::conj(g2 * sL[j * m + i]);
            const cplx b = g2 * sR[i * m + j], bt = std::conj(g2 * sR[j * m + i]);
            GamL[i * m + j] = cplx(0.0, 1.0) * (a - at);
            GamR[i * m + j] = cplx(0.0, 1.0) * (b - bt);
        }
    // PL[k] = g_L[k]_{b_k, a_0} (m x m), PR[k] = g_R[k]_{a_k, b_{K-1}}
    std::vector<CMat> PL(K, CMat(mm)), PR(K, CMat(mm));
    for (int k = 0; k < K; ++k)
        for (int i = 0; i < m; ++i)
            for (int j = 0; j < m; ++j) {
                cplx v = 0.0;
                if (k == 0) {
                    v = gL[0][(m + i) * n + j];
                } else {
                    for (int l = 0; l < m; ++l) v += gL[k][(m + i) * n + l] * PL[k - 1][l * m + j];
                    v *= gamma;
                }
                PL[k][i * m + j] = v;
            }
    for (int k = K - 1; k >= 0; --k)
        for (int i = 0; i < m; ++i)
            for (int j = 0; j < m; ++j) {
                cplx v = 0.0;
                if (k == K - 1) {
                    v = gR[k][i * n + (m + j)];
                } else {
                    for (int l = 0; l < m; ++l) v += gR[k][i * n + (m + l)] * PR[k + 1][l * m + j];
                    v *= gamma;
                }
                PR[k][i * m + j] = v;
            }
    outL.assign(2 * (size_t)K, 0.0);
    outR.assign(2 * (size_t)K, 0.0);
    std::vector<cplx> col(n * m);
    for (int k = 0; k < K; ++k) {
        CMat M = rs_block(m, gamma, E, Uatoms + (size_t)k * n);
        for (int i = 0; i < m; ++i)
            for (int j = 0; j < m; ++j) {
                M[i * n + j] -= g2 * (k == 0 ? sL[i * m + j] : gL[k - 1][(m + i) * n + (m + j)]);
                M[(m + i) * n + (m + j)] -= g2 * (k == K - 1 ? sR[i * m + j] : gR[k + 1][i * n + j]);
            }
        cinvert(M, n);  // G_kk
        for (int side = 0; side < 2; ++side) {
            // col = G_{k,c} restricted to the contact ring's atoms (2m x m)
            const int off = side == 0 ? 0 : m;  // G_kk column block touching the neighbour towards the contact
            const bool at_contact = side == 0 ? k == 0 : k == K - 1;
            for (int r = 0; r < n; ++r)
                for (int j = 0; j < m; ++j) {
                    cplx v = 0.0;
                    if (at_contact) {
                        v = M[r * n + off + j];
                    } else {
                        const CMat& Pn = side == 0 ? PL[k - 1] : PR[k + 1];
                        for (int l = 0; l < m; ++l) v += M[r * n + off + l] * Pn[l * m + j];
                        v *= gamma;
                    }
                    col[r * m + j] = v;
                }
            const CMat& Gam = side == 0 ? GamL : GamR;
            std::vector<double>& out = side == 0 ? outL : outR;
            for (int r = 0; r < n; ++r) {
                cplx a = 0.0;
                for (int i = 0; i < m; ++i)
                    for (int j = 0; j < m; ++j) a += col[r * m + i] * Gam[i * m + j] * std::conj(col[r * m + j]);
                out[2 * k + r / m] += a.real();
            }
        }
    }
}

// ---------------------------------------------------------------- Broyden
// T/Broyden_Second_Parallel.cpp:9-211 (CPU branch) and
// T/Broyden_Parallel_General.cpp:68-355 (set-up and reset).
struct Broyden {
    int S = 0, maxstep = 200, norm_type = 0;  // 0 absolute, 1 relative
    int step = 1;
    double fraction = 0.1, scalar = 1.0, norm = 1.0, normsum_prev = 1e10, normsum = 1e10;
    std::vector<double> n_in, n_prev, F, dF, Nrm, V, W, c, sum;  // V: [S][maxstep], W: [maxstep][S]
};

}  // namespace

extern "C" {

// ------------------------------------------------------------- quadrature
void orc_gauss_legendre(int n, double* x, double* w) {
    std::vector<double> xv, wv;
    gauss_legendre(n, xv, wv);
    std::memcpy(x, xv.data(), sizeof(double) * n);
    std::memcpy(w, wv.data(), sizeof(double) * n);
}

// ------------------------------------------------------------- fixtures
// scripts/negf_cpp/decimation_technique/Source/main.cpp:540-790 (the RGF +
// spectral-function kernel) with Sigma = gamma^2 g (main.cpp:184-201).
// root: 1 -> (F-S)/D, 2 -> (F+S)/D.  Output per energy: Sigma (re,im) of both
// contacts, DOS (re,im) = trace(A)/2pi, T (re,im) = Gamma_0 * A_{0,0} from contact 1.
void orc_fixture_sigma_dos_T(int N, double beta, double gamma, int nE, const double* E_re, double eta,
                             int root, double* sigma, double* dos, double* T) {
    for (int e = 0; e < nE; ++e) {
        const cplx E(E_re[e], eta);
        const cplx g = surface_gf_analytic(gamma, beta, E, root);
        const cplx Sig = gamma * gamma * g;  // pow(gamma,2.) * gr
        const cplx Sg[2] = {Sig, Sig};
        std::vector<cplx> alpha(N, E), X(N, 0.0), Y(N, 0.0), Xt(N, 0.0), Yt(N, 0.0);
        alpha[0] -= Sg[0];
        alpha[N - 1] -= Sg[1];
        const cplx B[2] = {-beta, -gamma}, C[2] = {-beta, -gamma};
        for (int n = 1; n < N; ++n) {
            const int p = (n - 1) % 2;
            Yt[n] = cdiv(C[p], alpha[n - 1] - Y[n - 1]);
            Y[n] = cmul(B[p], Yt[n]);
        }
        for (int n = N - 2; n >= 0; --n) {
            const int p = n % 2;
            Xt[n] = cdiv(B[p], alpha[n + 1] - X[n + 1]);
            X[n] = cmul(C[p], Xt[n]);
        }
        const int kglo[2] = {0, N - 1};
        cplx trace(0.0), T12(0.0);
        for (int n = 0; n < N; ++n) {
            cplx Atk1(0.0), Adiag(0.0);
            for (int k = 0; k < 2; ++k) {
                const int kg = kglo[k];
                const cplx Gkk = cinv(alpha[kg] - X[kg] - Y[kg]);
                cplx tmp = Gkk;
                for (int q = kg; q < n; ++q) tmp = cmul(-Xt[q], tmp);
                for (int q = kg; q > n; --q) tmp = cmul(-Yt[q], tmp);
                const cplx Gam(-2.0 * Sg[k].imag(), 0.0);
                cplx Akn = cmul(cmul(Gkk, Gam), std::conj(tmp));
                if (n == kg) Adiag += Akn;
                for (int q = kg + 1; q < N; ++q) {
                    Akn = cmul(-Xt[q - 1], Akn);
                    if (q == n) Adiag += Akn;
                }
                for (int q = kg - 1; q >= 0; --q) {
                    Akn = cmul(-Yt[q + 1], Akn);
                    if (q == n) Adiag += Akn;
                }
                if (k == 1 && n == 0) Atk1 = Akn;  // contact_transmission_index[1] = 0
            }
            trace += Adiag;
            if (n == 0) T12 = cmul(cplx(-2.0 * Sg[0].imag(), 0.0), Atk1);
        }
        const cplx d = trace / (2.0 * kPi);
        sigma[4 * e + 0] = Sg[0].real();
        sigma[4 * e + 1] = Sg[0].imag();
        sigma[4 * e + 2] = Sg[1].real();
        sigma[4 * e + 3] = Sg[1].imag();
        dos[2 * e] = d.real();
        dos[2 * e + 1] = d.imag();
        T[2 * e] = T12.real();
        T[2 * e + 1] = T12.imag();
    }
}

// ------------------------------------------------------------- tube
void* orc_tube_new(int m, int n, int unitcells, int nmodes, double acc, double gamma) {
    Tube* t = new Tube();
    t->m = m;
    t->n = n;
    t->unitcells = unitcells;
    t->nmodes = nmodes;
    t->acc = acc;
    t->gamma = gamma;
    set_material(*t);
    t->U.assign(t->N, 0.0);
    return t;
}
void orc_tube_free(void* h) { delete static_cast<Tube*>(h); }
int orc_tube_num_sites(void* h) { return static_cast<Tube*>(h)->N; }
int orc_tube_num_modes(void* h) { return static_cast<Tube*>(h)->nmodes; }
double orc_tube_radius(void* h) { return static_cast<Tube*>(h)->R; }
void orc_tube_modes(void* h, int* J, int* degen, double* beta, double* gap) {
    Tube* t = static_cast<Tube*>(h);
    for (int i = 0; i < t->nmodes; ++i) {
        J[i] = t->modeJ[i];
        degen[i] = t->degen[i];
        beta[i] = t->beta[i];
        gap[i] = t->gap[i];
    }
}
void orc_tube_set_contacts(void* h, double T0, double T1, double mu0, double mu1) {
    Tube* t = static_cast<Tube*>(h);
    t->T[0] = T0;
    t->T[1] = T1;
    t->mu[0] = mu0;
    t->mu[1] = mu1;
}
void orc_tube_set_integration(void* h, const int* eq_pts, int n_noneq, const int* noneq_pts,
                              const double* intercuts, double Evmin, double Epolemax, double zplus,
                              double tail_lo, double tail_hi) {
    Tube* t = static_cast<Tube*>(h);
    for (int i = 0; i < 3; ++i) t->eq_pts[i] = eq_pts[i];
    t->noneq_pts.assign(noneq_pts, noneq_pts + n_noneq);
    t->intercuts.clear();
    if (n_noneq > 1) {
        if (intercuts) {
            t->intercuts.assign(intercuts, intercuts + n_noneq - 1);
        } else {  // NEGF_Common.cpp:483-491
            for (int c = 0; c < n_noneq - 1; ++c) t->intercuts.push_back((c + 1) * (100. / n_noneq));
        }
    }
    t->Evmin = Evmin;
    t->Epolemax = Epolemax;
    t->zplus = zplus;
    t->tail_lo = tail_lo;
    t->tail_hi = tail_hi;
}
void orc_tube_set_realaxis_window(void* h, double rt_min, double rt_max, int pts, int kind) {
    Tube* t = static_cast<Tube*>(h);
    t->rt_min = rt_min;
    t->rt_max = rt_max;
    t->rt_pts = pts;
    t->rt_kind = kind;
}
void orc_tube_set_decimation(void* h, int use, int max_iter, int layers, double rel_error, int tol_is_int) {
    Tube* t = static_cast<Tube*>(h);
    t->use_decimation = use;
    t->dec_max_iter = max_iter;
    t->dec_layers = layers;
    t->dec_rel_error = rel_error;
    t->dec_tol_is_int = tol_is_int;
}
void orc_tube_set_sgf_mode(void* h, int mode) { static_cast<Tube*>(h)->sgf_mode = mode; }
void orc_tube_set_potential(void* h, const double* U, double Uc0, double Uc1) {
    Tube* t = static_cast<Tube*>(h);
    t->U.assign(U, U + t->N);
    t->Uc[0] = Uc0;
    t->Uc[1] = Uc1;
}

// Surface GF / self-energy of one mode at one energy (test access).
void orc_tube_sigma(void* h, int mode, double E_re, double E_im, double Uc, double* out) {
    Tube* t = static_cast<Tube*>(h);
    const cplx E(E_re, E_im);
    const cplx EmU = E - Uc;
    const cplx g = t->use_decimation ? surface_gf_decimation(*t, t->beta[mode], EmU, nullptr)
                                     : surface_gf_analytic(t->gamma, t->beta[mode], EmU, t->sgf_mode);
    const cplx s = cmul(cmul(cplx(t->gamma, 0), g), cplx(t->gamma, -0.0));
    out[0] = s.real();
    out[1] = s.imag();
}

// Energy limits + path tables.  kinds: 0 Rho0, 1 RhoEq, 2 poles, 3 NonEq.
// Returns the number of points of that kind; when buf != null writes
// (E.re, E.im, w.re, w.im, J.re, J.im) per point.
int orc_tube_paths(void* h, int kind, double* buf) {
    Tube* t = static_cast<Tube*>(h);
    energy_limits(*t);
    build_eq_noneq_paths(*t);
    std::vector<Path> paths;
    if (kind == 0) {
        // Rho0 is defined at initialisation with mu = 0 (NEGF_Common.cpp:1275-1300)
        Tube t0 = *t;
        t0.mu[0] = t0.mu[1] = 0.0;
        t0.rt_pts = 0;
        energy_limits(t0);
        build_paths(t0);
        paths = t0.rho0_paths;
    } else if (kind == 1) {
        paths = t->eq_paths;
    } else if (kind == 3) {
        paths = t->noneq_paths;
    } else {
        if (buf)
            for (size_t i = 0; i < t->poles.size(); ++i) {
                buf[6 * i] = t->poles[i].real();
                buf[6 * i + 1] = t->poles[i].imag();
                for (int j = 2; j < 6; ++j) buf[6 * i + j] = 0.0;
            }
        return (int)t->poles.size();
    }
    int k = 0;
    for (auto& p : paths)
        for (size_t i = 0; i < p.E.size(); ++i, ++k)
            if (buf) {
                buf[6 * k] = p.E[i].real();
                buf[6 * k + 1] = p.E[i].imag();
                buf[6 * k + 2] = p.w[i].real();
                buf[6 * k + 3] = p.w[i].imag();
                buf[6 * k + 4] = p.J[i].real();
                buf[6 * k + 5] = p.J[i].imag();
            }
    return k;
}

int orc_tube_noneq(void* h) {
    Tube* t = static_cast<Tube*>(h);
    energy_limits(*t);
    return t->noneq ? 1 : 0;
}

// NEGF_Common.cpp:3957-4092, computed at initialisation with U = 0, U_contact = 0, mu = 0.
void orc_tube_rho0(void* h, int nthreads) {
    Tube* t = static_cast<Tube*>(h);
    Tube t0 = *t;
    t0.mu[0] = t0.mu[1] = 0.0;
    t0.Uc[0] = t0.Uc[1] = 0.0;
    t0.rt_pts = 0;
    energy_limits(t0);
    build_paths(t0);
    std::vector<double> U0(t->N, 0.0);
    run_points(t0, U0, collect(t0.rho0_paths, 0, t0), 0, nthreads, t->rho0);
    t->rho0_im_sum.assign(t->N, 0.0);
    for (int n = 0; n < t->N; ++n)
        for (int m = 0; m < t->nmodes; ++m) t->rho0_im_sum[n] += t->rho0[(size_t)n * t->nmodes + m].imag();
}

// Compute_InducedCharge (NEGF_Common.cpp:2850-2900): Q_n = sum_m [Im RhoEq + Re RhoNonEq - Im Rho0].
// faithful=1 uses the reference's O(N)-per-site contact walk.
// Optional per-component outputs (sum over modes): eq_im, noneq_re, rho0_im.
void orc_tube_charge(void* h, int faithful, int nthreads, double* Q, double* eq_im, double* noneq_re,
                     double* rho0_im) {
    Tube* t = static_cast<Tube*>(h);
    if (t->rho0_im_sum.size() != (size_t)t->N) orc_tube_rho0(h, nthreads);
    energy_limits(*t);
    build_eq_noneq_paths(*t);
    auto pts = collect(t->eq_paths, 1, *t);
    if (!t->noneq)
        for (auto& p : t->poles) pts.push_back(EPoint{p, 1.0, 1.0, 0.0, 2});
    run_points(*t, t->U, pts, faithful, nthreads, t->rhoeq);
    if (t->noneq)
        run_points(*t, t->U, collect(t->noneq_paths, 3, *t), faithful, nthreads, t->rhononeq);
    else
        t->rhononeq.assign((size_t)t->N * t->nmodes, 0.0);
    const int M = t->nmodes;
    for (int n = 0; n < t->N; ++n) {
        double a = 0, b = 0;
        for (int m = 0; m < M; ++m) {
            a += t->rhoeq[(size_t)n * M + m].imag();
            b += t->rhononeq[(size_t)n * M + m].real();
        }
        Q[n] = a + b - t->rho0_im_sum[n];
        if (eq_im) eq_im[n] = a;
        if (noneq_re) noneq_re[n] = b;
        if (rho0_im) rho0_im[n] = t->rho0_im_sum[n];
    }
}

// Charge contribution of an explicit subset of energy points (multi-rank
// sharding checks): kind 1 = RhoEq contour points [e_lo, e_hi), kind 3 = NonEq.
void orc_tube_partial(void* h, int kind, int e_lo, int e_hi, int nthreads, double* out) {
    Tube* t = static_cast<Tube*>(h);
    energy_limits(*t);
    build_eq_noneq_paths(*t);
    std::vector<cplx> acc;
    const auto& paths = (kind == 1) ? t->eq_paths : t->noneq_paths;
    run_points(*t, t->U, collect(paths, kind, *t, e_lo, e_hi), 0, nthreads, acc);
    for (int n = 0; n < t->N; ++n) {
        double s = 0;
        for (int m = 0; m < t->nmodes; ++m)
            s += kind == 1 ? acc[(size_t)n * t->nmodes + m].imag() : acc[(size_t)n * t->nmodes + m].real();
        out[n] = s;
    }
}

// Bounded CPU-baseline sample: the points whose index in the concatenated
// list [RhoEq contour + poles, NonEq] is congruent to `offset` modulo
// `stride`, integrated exactly as in orc_tube_charge (faithful walk when
// faithful=1).  Writes the per-site partial sum and returns the number of
// (site, mode, energy) updates processed.
long long orc_tube_sample(void* h, int faithful, int nthreads, int stride, int offset, double* out) {
    Tube* t = static_cast<Tube*>(h);
    energy_limits(*t);
    build_eq_noneq_paths(*t);
    auto eq = collect(t->eq_paths, 1, *t);
    if (!t->noneq)
        for (auto& p : t->poles) eq.push_back(EPoint{p, 1.0, 1.0, 0.0, 2});
    auto ne = t->noneq ? collect(t->noneq_paths, 3, *t) : std::vector<EPoint>{};
    std::vector<EPoint> se, sn;
    for (size_t i = 0; i < eq.size(); ++i)
        if ((long long)i % stride == offset) se.push_back(eq[i]);
    for (size_t i = 0; i < ne.size(); ++i)
        if ((long long)(i + eq.size()) % stride == offset) sn.push_back(ne[i]);
    std::vector<cplx> a, b;
    run_points(*t, t->U, se, faithful, nthreads, a);
    run_points(*t, t->U, sn, faithful, nthreads, b);
    const int M = t->nmodes;
    for (int n = 0; n < t->N; ++n) {
        double s = 0;
        for (int m = 0; m < M; ++m) {
            if (!a.empty()) s += a[(size_t)n * M + m].imag();
            if (!b.empty()) s += b[(size_t)n * M + m].real();
        }
        out[n] = s;
    }
    return (long long)(se.size() + sn.size()) * M * t->N;
}

// ------------------------------------------------------------- Broyden
// DOS / transmission / conductance over the tube's DOS path.  Returns the
// number of energies; with E != null writes E (re, im), dos, T, conductance
// per energy, the total conductance, and optionally LDOS [e][n].
int orc_tube_dos(void* h, int faithful, int nthreads, double* E, double* dos, double* T, double* cond,
                 double* total_cond, double* ldos) {
    Tube* t = static_cast<Tube*>(h);
    energy_limits(*t);
    build_eq_noneq_paths(*t);
    const auto paths = dos_paths(*t);
    std::vector<cplx> Ev;
    for (const auto& p : paths)
        for (auto e : p.E) Ev.push_back(e);
    const int P = (int)Ev.size();
    if (!E) return P;
    const int N = t->N;
    std::vector<double> tr0(P, 0.0), tr1(P, 0.0);
    nthreads = std::max(1, std::min(nthreads, P));
    auto worker = [&](int tid) {
        Sweep s;
        for (int e = P * tid / nthreads; e < P * (tid + 1) / nthreads; ++e)
            dos_point(*t, t->U, Ev[e], faithful, s, ldos ? ldos + (size_t)e * N : nullptr, tr0[e], tr1[e]);
    };
    if (ldos) std::fill(ldos, ldos + (size_t)P * N, 0.0);
    std::vector<std::thread> th;
    for (int i = 0; i < nthreads; ++i) th.emplace_back(worker, i);
    for (auto& x : th) x.join();
    const int apuc = t->atoms_per_ring * t->rings_per_uc;  // CNT.H:52-55
    std::vector<double> Tv(P), C;
    for (int e = 0; e < P; ++e) {
        E[2 * e] = Ev[e].real();
        E[2 * e + 1] = Ev[e].imag();
        dos[e] = kSpinDegen * tr0[e] / apuc;
        T[e] = Tv[e] = tr1[e];
    }
    // Compute_Conductance takes the energies as complex numbers with the real part only
    std::vector<cplx> Er(P);
    for (int e = 0; e < P; ++e) Er[e] = cplx(Ev[e].real(), 0.0);
    const double tot = conductance(*t, Er, Tv, C);
    for (int e = 0; e < P; ++e) cond[e] = C[e];
    if (total_cond) *total_cond = tot;
    return P;
}
void orc_tube_set_flatband_dos_pts(void* h, int pts) { static_cast<Tube*>(h)->flatband_dos_pts = pts; }

// Terminal currents over the non-equilibrium paths; integrand probes
// (channel, source, drain) per energy when probes != null ([3][P]).
int orc_tube_current(void* h, int nthreads, double* I, double* probes) {
    Tube* t = static_cast<Tube*>(h);
    energy_limits(*t);
    build_eq_noneq_paths(*t);
    const auto pts = collect(t->noneq_paths, 3, *t);
    const int P = (int)pts.size();
    I[0] = I[1] = 0.0;
    if (P == 0) return 0;
    std::vector<double> Ie(2 * P, 0.0), pr(3 * P, 0.0);
    nthreads = std::max(1, std::min(nthreads, P));
    auto worker = [&](int tid) {
        Sweep s;
        for (int e = P * tid / nthreads; e < P * (tid + 1) / nthreads; ++e)
            current_point(*t, t->U, pts[e], s, &Ie[2 * e], &pr[3 * e]);
    };
    std::vector<std::thread> th;
    for (int i = 0; i < nthreads; ++i) th.emplace_back(worker, i);
    for (auto& x : th) x.join();
    for (int e = 0; e < P; ++e) {
        I[0] += Ie[2 * e];
        I[1] += Ie[2 * e + 1];
        if (probes)
            for (int k = 0; k < 3; ++k) probes[(size_t)k * P + e] = pr[3 * e + k];
    }
    return P;
}

// Integrand probes [3][P] of Compute_RhoNonEq over the current non-equilibrium energies.
int orc_tube_noneq_integrand(void* h, int nthreads, double* out) {
    Tube* t = static_cast<Tube*>(h);
    energy_limits(*t);
    build_eq_noneq_paths(*t);
    std::vector<cplx> Ev;
    for (const auto& p : t->noneq_paths)
        for (auto e : p.E) Ev.push_back(e);
    const int P = (int)Ev.size();
    if (!out || P == 0) return P;
    std::vector<double> v(3 * (size_t)P);
    nthreads = std::max(1, std::min(nthreads, P));
    auto worker = [&](int tid) {
        Sweep s;
        for (int e = P * tid / nthreads; e < P * (tid + 1) / nthreads; ++e)
            noneq_integrand_point(*t, t->U, Ev[e], s, &v[3 * (size_t)e]);
    };
    std::vector<std::thread> th;
    for (int i = 0; i < nthreads; ++i) th.emplace_back(worker, i);
    for (auto& x : th) x.join();
    for (int e = 0; e < P; ++e)
        for (int k = 0; k < 3; ++k) out[(size_t)k * P + e] = v[3 * (size_t)e + k];
    return P;
}

// Update_IntegrationPaths with flag_correct_integration_limits (NEGF_Common.cpp:2200-2211).
void orc_tube_set_adaptive(void* h, double win_lo, double win_hi, int n_density, const double* density) {
    Tube* t = static_cast<Tube*>(h);
    t->kT_window[0] = win_lo;
    t->kT_window[1] = win_hi;
    t->has_density = n_density > 0;
    t->density.assign(density, density + std::max(0, n_density));
}
void orc_tube_correct_limits(void* h, int nthreads) {
    Tube* t = static_cast<Tube*>(h);
    energy_limits(*t);
    build_eq_noneq_paths(*t);
    if (!t->noneq || t->rt_pts > 0) return;
    const int P = orc_tube_noneq_integrand(h, 1, nullptr);
    std::vector<double> v(3 * (size_t)std::max(P, 1));
    orc_tube_noneq_integrand(h, nthreads, v.data());
    std::vector<cplx> Ev;
    for (const auto& p : t->noneq_paths)
        for (auto e : p.E) Ev.push_back(e);
    double mx = 0.0;
    for (int e = 0; e < P; ++e)
        if (mx < std::fabs(v[e])) {
            mx = std::fabs(v[e]);
            t->E_at_max = Ev[e].real();
        }
    find_intercuts(*t);
    build_eq_noneq_paths(*t);
}
int orc_tube_noneq_layout(void* h, int* pts, double* cuts, double* E_at_max) {
    Tube* t = static_cast<Tube*>(h);
    const int np = (int)t->noneq_pts.size();
    for (int p = 0; p < np; ++p) pts[p] = t->noneq_pts[p];
    for (int p = 0; p + 1 < np; ++p) cuts[p] = t->intercuts[p];
    *E_at_max = t->E_at_max;
    return np;
}

// Real-space charge per ring of a zigzag tube over the tube's contour + poles
// (and Rho0 at U = 0) and, when biased, its non-equilibrium paths:
// Q_ring = sum_atoms [Im(RhoEq - Rho0) + Re RhoNonEq] with the same
// coefficients as the mode-space pass.  Uatoms: [N][m] per-atom potentials
// (null: ring-uniform from the tube's U).  Returns -1 for a chiral tube.
int orc_tube_rs_charge(void* h, const double* Uatoms, int iters, int nthreads, double* Q) {
    Tube* t = static_cast<Tube*>(h);
    energy_limits(*t);
    build_eq_noneq_paths(*t);
    if (t->n != 0) return -1;
    const int m = t->m, N = t->N, K = N / 2, n = 2 * m;
    std::vector<double> Ua((size_t)N * m), U0((size_t)N * m, 0.0);
    for (int r = 0; r < N; ++r)
        for (int j = 0; j < m; ++j) Ua[(size_t)r * m + j] = Uatoms ? Uatoms[(size_t)r * m + j] : t->U[r];
    // ring r = 2k + (0 | 1) -> block k atoms [0, m) | [m, 2m): same layout as [N][m]
    auto pts = collect(t->eq_paths, 1, *t);
    for (auto& p : t->poles) pts.push_back(EPoint{p, 1.0, 1.0, 0.0, 2});
    Tube t0 = *t;
    t0.mu[0] = t0.mu[1] = 0.0;
    t0.rt_pts = 0;
    energy_limits(t0);
    build_paths(t0);
    auto pts0 = collect(t0.rho0_paths, 0, t0);
    auto run = [&](const std::vector<EPoint>& P, const std::vector<double>& Uv, double Uc0, double Uc1,
                   std::vector<double>& acc) {
        acc.assign(N, 0.0);
        const int T = std::max(1, std::min<int>(nthreads, (int)P.size()));
        std::vector<std::vector<double>> part(T, std::vector<double>(N, 0.0));
        auto worker = [&](int tid) {
            std::vector<cplx> d;
            for (size_t i = P.size() * tid / T; i < P.size() * (tid + 1) / T; ++i) {
                const EPoint& ep = P[i];
                rs_diag(m, K, t->gamma, ep.E, Uv.data(), Uc0, Uc1, iters, d);
                cplx c;
                if (ep.kind == 0)
                    c = cmul((-1 * kSpinDegen / kPi) * ep.w, ep.J);
                else if (ep.kind == 1)
                    c = cmul(cmul((-1. * kSpinDegen / kPi) * ep.w, ep.J), ep.f);
                else
                    c = cplx(0.0, -2 * t->kT_min * kSpinDegen);
                for (int r = 0; r < N; ++r) {
                    cplx s = 0.0;
                    for (int j = 0; j < m; ++j) s += d[(size_t)(r / 2) * n + (r % 2) * m + j];
                    part[tid][r] += cmul(c, s).imag();
                }
            }
        };
        std::vector<std::thread> th;
        for (int i = 0; i < T; ++i) th.emplace_back(worker, i);
        for (auto& x : th) x.join();
        for (int i = 0; i < T; ++i)
            for (int r = 0; r < N; ++r) acc[r] += part[i][r];
    };
    std::vector<double> eq, r0, ne(N, 0.0);
    run(pts, Ua, t->Uc[0], t->Uc[1], eq);
    run(pts0, U0, 0.0, 0.0, r0);
    if (t->noneq) {
        // Re RhoNonEq: sum_c Re(-spin/2pi w J f_c) A^c per ring
        auto pn = collect(t->noneq_paths, 3, *t);
        const int T = std::max(1, std::min<int>(nthreads, (int)pn.size()));
        std::vector<std::vector<double>> part(T, std::vector<double>(N, 0.0));
        auto worker = [&](int tid) {
            std::vector<double> aL, aR;
            for (size_t i = pn.size() * tid / T; i < pn.size() * (tid + 1) / T; ++i) {
                const EPoint& ep = pn[i];
                rs_noneq(m, K, t->gamma, ep.E, Ua.data(), t->Uc[0], t->Uc[1], iters, aL, aR);
                const cplx base = cmul((-1. * kSpinDegen / (2 * kPi)) * ep.w, ep.J);
                const double b0 = cmul(base, fermi(ep.E - t->mu[0], t->kT[0])).real();
                const double b1 = cmul(base, fermi(ep.E - t->mu[1], t->kT[1])).real();
                for (int r = 0; r < N; ++r) part[tid][r] += b0 * aL[r] + b1 * aR[r];
            }
        };
        std::vector<std::thread> th;
        for (int i = 0; i < T; ++i) th.emplace_back(worker, i);
        for (auto& x : th) x.join();
        for (int i = 0; i < T; ++i)
            for (int r = 0; r < N; ++r) ne[r] += part[i][r];
    }
    for (int r = 0; r < N; ++r) Q[r] = eq[r] + ne[r] - r0[r];
    return 0;
}

void* orc_broyden_new(int S, int maxstep, double fraction, int norm_type, const double* n_in) {
    Broyden* b = new Broyden();
    b->S = S;
    b->maxstep = maxstep;
    b->fraction = fraction;
    b->norm_type = norm_type;
    b->n_in.assign(n_in, n_in + S);
    b->n_prev.assign(S, 0.0);
    b->F.assign(S, 0.0);
    b->dF.assign(S, 0.0);
    b->Nrm.assign(S, 0.0);
    b->V.assign((size_t)S * maxstep, 0.0);
    b->W.assign((size_t)S * maxstep, 0.0);
    b->c.assign(maxstep, 0.0);
    b->sum.assign(S, 0.0);
    return b;
}
void orc_broyden_free(void* h) { delete static_cast<Broyden*>(h); }

// T/Broyden_Second_Parallel.cpp:18-211.  Returns the max norm (Broyden_Norm).
double orc_broyden_step(void* h, const double* n_out, double* n_in_out, double* norm_out) {
    Broyden* b = static_cast<Broyden*>(h);
    const int S = b->S, MS = b->maxstep;
    auto Vt = [&](int site, int it) -> double& { return b->V[(size_t)site * MS + it]; };
    auto Wm = [&](int it, int site) -> double& { return b->W[(size_t)it * S + site]; };
    std::fill(b->Nrm.begin(), b->Nrm.end(), 0.0);
    std::fill(b->sum.begin(), b->sum.end(), 0.0);
    std::fill(b->c.begin(), b->c.end(), 0.0);
    double nsum = 0.0;
    for (int s = 0; s < S; ++s) {
        const double Fc = b->n_in[s] - n_out[s];
        if (b->norm_type == 0) {
            b->Nrm[s] = std::fabs(Fc);
            nsum += Fc * Fc;
        } else {
            b->Nrm[s] = std::fabs(Fc / (b->n_in[s] + n_out[s]));
            nsum += b->Nrm[s] * b->Nrm[s];
        }
    }
    double mx = S > 0 ? b->Nrm[0] : 0.0;
    for (int s = 1; s < S; ++s)
        if (mx < b->Nrm[s]) mx = b->Nrm[s];
    b->norm = mx;
    b->normsum = std::sqrt(nsum);
    double denom = 0.0;
    for (int s = 0; s < S; ++s) {
        const double Fc = b->n_in[s] - n_out[s];
        b->dF[s] = Fc - b->F[s];
        b->F[s] = Fc;
        denom += b->dF[s] * b->dF[s];
    }
    b->normsum_prev = b->normsum;
    const int m = b->step - 1;
    if (m > 0) {
        for (int it = 1; it <= m - 1; ++it) {
            double s_ = 0.0;
            for (int s = 0; s < S; ++s) s_ += Vt(s, it) * b->dF[s];
            b->c[it] = s_;
        }
        for (int s = 0; s < S; ++s) {
            double s_ = 0.0;
            for (int it = 1; it <= m - 1; ++it) s_ += Wm(it, s) * b->c[it];
            b->sum[s] = s_;
        }
        for (int s = 0; s < S; ++s) {
            const double dn = b->n_in[s] - b->n_prev[s];
            Vt(s, m) = b->dF[s] / denom;
            Wm(m, s) = -b->fraction * b->dF[s] + dn - b->sum[s];
        }
        std::fill(b->c.begin(), b->c.end(), 0.0);
        for (int it = 1; it <= m; ++it) {
            double s_ = 0.0;
            for (int s = 0; s < S; ++s) s_ += Vt(s, it) * b->F[s];
            b->c[it] = s_;
        }
        for (int s = 0; s < S; ++s) {
            double s_ = 0.0;
            for (int it = 1; it <= m; ++it) s_ += Wm(it, s) * b->c[it];
            b->sum[s] = s_;
        }
    }
    for (int s = 0; s < S; ++s) {
        b->n_prev[s] = b->n_in[s];
        b->n_in[s] = b->n_prev[s] - b->scalar * b->fraction * b->F[s] - b->scalar * b->sum[s];
    }
    b->step += 1;
    if (n_in_out) std::memcpy(n_in_out, b->n_in.data(), sizeof(double) * S);
    if (norm_out) std::memcpy(norm_out, b->Nrm.data(), sizeof(double) * S);
    return mx;
}
int orc_broyden_stepno(void* h) { return static_cast<Broyden*>(h)->step; }

// T/Broyden_Parallel_General.cpp:250-347
void orc_broyden_reset(void* h, int keep_charge, double init_value) {
    Broyden* b = static_cast<Broyden*>(h);
    if (!keep_charge) std::fill(b->n_in.begin(), b->n_in.end(), init_value);
    std::fill(b->n_prev.begin(), b->n_prev.end(), 0.0);
    std::fill(b->F.begin(), b->F.end(), 0.0);
    std::fill(b->dF.begin(), b->dF.end(), 0.0);
    std::fill(b->Nrm.begin(), b->Nrm.end(), 0.0);
    std::fill(b->V.begin(), b->V.end(), 0.0);
    std::fill(b->W.begin(), b->W.end(), 0.0);
    std::fill(b->sum.begin(), b->sum.end(), 0.0);
    std::fill(b->c.begin(), b->c.end(), 0.0);
    b->step = 1;
    b->norm = 1.0;
    b->scalar = 1.0;
    b->normsum = b->normsum_prev = 1e10;
}

}  // extern "C"
