"""The oracle against the reference's own known-answer files.

tests/golden/*.txt are the committed outputs of the reference's standalone RGF
programs (tests/golden/make_golden.py lists their origin).  The files print 6
significant digits, so the bound is 1e-5 relative.
"""
import os

import numpy as np
import pytest

BETA = 2 * 2.5 * np.cos(np.pi * 6 / 17)  # get_beta(2.5, 17, 6), decimation_technique/Source/main.cpp:976-979
GOLDEN = {
    # tag: (surface-GF root, E range)
    "decimation": (1, (-6.0, 0.0)),
    "pointcontact_1gpu": (2, (-1.0, 1.0)),
}


def _load(tag, name):
    p = os.path.join(os.path.dirname(__file__), "golden", f"{tag}_{name}.txt")
    return np.loadtxt(p, skiprows=1)


@pytest.mark.parametrize("tag", sorted(GOLDEN))
def test_fixture_sigma_dos_transmission(oracle, tag):
    root, (lo, hi) = GOLDEN[tag]
    S, D, T = _load(tag, "Sigma"), _load(tag, "DOS"), _load(tag, "Transmission")
    n = len(S)
    E = lo + np.arange(n) * ((hi - lo) / (n - 1))
    assert np.allclose(E, S[:, 0], rtol=0, atol=5e-6)
    sig, dos, tr = oracle.fixture_sigma_dos_T(4, BETA, 2.5, E, 1e-8, root)
    # Sigma of both contacts (real, imag); 6 printed digits
    for col, gold in ((0, S[:, 1]), (1, S[:, 2]), (2, S[:, 3]), (3, S[:, 4])):
        np.testing.assert_allclose(sig[:, col], gold, rtol=1e-5, atol=1e-12)
    np.testing.assert_allclose(dos[:, 0], D[:, 1], rtol=1e-5, atol=1e-30)
    np.testing.assert_allclose(tr[:, 0], T[:, 1], rtol=1e-5, atol=1e-30)


def test_gauss_legendre_exactness(oracle):
    # CodeUtil.cpp:640-690 stops Newton at a 3e-11 step and evaluates the
    # weight derivative at the previous iterate: moments are exact to ~1e-10.
    for n in (1, 2, 3, 7, 30, 64):
        x, w = oracle.gauss_legendre(n)
        assert np.all(np.diff(x) > 0)
        for k in range(2 * n):
            exact = 0.0 if k % 2 else 2.0 / (k + 1)
            assert abs(np.sum(w * x ** k) - exact) < 1e-9


def test_modes_17_0(oracle):
    t = oracle.OracleTube(type_id=(17, 0), num_unitcells=10, num_modes=3)
    J, deg, beta, gap = t.modes()
    assert t.N == 40
    assert abs(t.radius - 0.6655e-9) < 1e-12
    assert list(deg) == [2, 2, 2]
    assert np.all(np.diff(gap) > 0)
    np.testing.assert_allclose(np.abs(beta), 2 * 2.5 * np.abs(np.cos(np.pi * J / 17)))


def _dense_G(E, U, beta, gamma, sig0, sig1):
    """Dense (E - H - Sigma)^-1 of the mode-space chain, numpy inverse."""
    N = len(U)
    A = np.zeros((N, N), complex)
    for n in range(N):
        A[n, n] = E - U[n]
    A[0, 0] -= sig0
    A[N - 1, N - 1] -= sig1
    for n in range(N - 1):
        h = -beta if n % 2 == 0 else -gamma
        A[n, n + 1] = A[n + 1, n] = h
    return np.linalg.inv(A)


def test_fixture_against_dense_inverse(oracle):
    """DOS/T of the fixture kernel equal trace/|G_0,N-1|^2 of the dense inverse."""
    N, gamma = 6, 2.5
    E = np.array([-2.0, -0.3, 0.4, 1.7])
    sig, dos, tr = oracle.fixture_sigma_dos_T(N, BETA, gamma, E, 1e-3, 2)
    for i, e in enumerate(E):
        s0 = complex(sig[i, 0], sig[i, 1])
        G = _dense_G(e + 1e-3j, np.zeros(N), BETA, gamma, s0, s0)
        g0 = -2 * s0.imag
        A = G[:, [0]] * g0 @ G[:, [0]].conj().T + G[:, [N - 1]] * g0 @ G[:, [N - 1]].conj().T
        np.testing.assert_allclose(dos[i, 0], np.trace(A).real / (2 * np.pi), rtol=1e-10)
        np.testing.assert_allclose(tr[i, 0], g0 * g0 * abs(G[0, N - 1]) ** 2, rtol=1e-10)


def _small_tube(oracle, **kw):
    base = dict(type_id=(17, 0), num_unitcells=6, num_modes=2, eq_integration_pts=(20, 20, 24),
                noneq_integration_pts=(40,), E_zPlus_imag=1e-3)
    base.update(kw)
    return oracle.OracleTube(**base)


def test_faithful_walk_equals_running_products(oracle):
    """The reference's O(N)-per-site contact walk equals the O(N) running products."""
    t = _small_tube(oracle, contact_mu=(0.0, -0.3))
    rng = np.random.default_rng(1)
    t.set_potential(rng.uniform(-0.2, 0.2, t.N), (0.05, -0.25))
    a = t.charge(faithful=True)
    b = t.charge(faithful=False)
    np.testing.assert_allclose(a, b, rtol=1e-11, atol=1e-14 * np.abs(a).max())


def test_flat_band_zero_charge(oracle):
    """U = 0, mu = 0 equilibrium: RhoEq equals Rho0 up to the pole/contour split."""
    t = _small_tube(oracle, eq_integration_pts=(60, 60, 60), E_zPlus_imag=1e-8)
    t.set_potential(np.zeros(t.N), (0.0, 0.0))
    Q, eq, ne, r0 = t.charge(components=True)
    assert np.max(np.abs(Q)) < 2e-3 * np.max(np.abs(r0))


def test_charge_components_against_dense_inverse(oracle):
    """RhoEq of a few contour points, recomputed from the dense inverse."""
    t = _small_tube(oracle, num_unitcells=3, eq_integration_pts=(4, 4, 6))
    N = t.N
    rng = np.random.default_rng(7)
    U = rng.uniform(-0.3, 0.3, N)
    Uc = (0.1, -0.1)
    t.set_potential(U, Uc)
    E, w, J = t.paths(1)
    J_, deg, beta, _ = t.modes()
    kT = 8.617333262e-5 * 298.0
    # RhoEq = sum (-2/pi) w J f(E - mu_min) G_nn deg  + poles(-4i kT G_nn deg)
    acc = np.zeros(N)
    for m in range(t.M):
        for e, ww, jj in zip(E, w, J):
            s0, s1 = t.sigma(m, e, Uc[0]), t.sigma(m, e, Uc[1])
            G = _dense_G(e, U, beta[m], 2.5, s0, s1)
            f = 1.0 / (np.exp(e / kT) + 1.0)
            acc += ((-2 / np.pi) * ww * jj * f * np.diag(G) * deg[m]).imag
        Ep, _, _ = t.paths(2)
        for e in Ep:
            s0, s1 = t.sigma(m, e, Uc[0]), t.sigma(m, e, Uc[1])
            G = _dense_G(e, U, beta[m], 2.5, s0, s1)
            acc += (-4j * kT * np.diag(G) * deg[m]).imag
    Q, eq, ne, r0 = t.charge(components=True)
    np.testing.assert_allclose(eq, acc, rtol=1e-9, atol=1e-12)


def test_broyden_oracle_linear_problem(oracle):
    """Broyden modified-second converges on a contractive linear map n_out = A n + b."""
    rng = np.random.default_rng(3)
    S = 30
    A = rng.normal(0, 0.5 / np.sqrt(S), (S, S))
    b = rng.normal(0, 1, S)
    n = np.zeros(S)
    br = oracle.OracleBroyden(n, max_step=100, fraction=0.1, norm_type="absolute")
    nrm = 1.0
    it = 0
    while nrm > 1e-10 and it < 90:
        nrm, n, _ = br.step(A @ n + b)
        it += 1
    fixed = np.linalg.solve(np.eye(S) - A, b)
    assert it < 2 * S + 5  # Broyden terminates in <= 2S steps on linear maps (exact arithmetic)
    np.testing.assert_allclose(n, fixed, atol=1e-8)


def _dos_compare_tube(oracle, faithful):
    t = oracle.OracleTube(type_id=(17, 0), num_unitcells=1, num_modes=2, contact_mu=(0.0, -1e-4),
                          realaxis_window=(-1.0, 1.0, 200, 0), E_zPlus_imag=1e-8)
    t.set_potential(np.zeros(t.N), (0.0, 0.0))
    return t.dos(faithful=faithful, nthreads=4)


@pytest.mark.parametrize("faithful", [True, False])
def test_dos_transmission_against_reference_output(oracle, faithful):
    """Compute_DensityOfStates restated (NEGF_Common.cpp:2390-2847) against the
    reference engine's committed DOS_Compare output: (17,0), N=4, 2 modes,
    200 uniform energies on [-1, 1] + 1e-8 i (6 printed digits; the gap values
    near 1e-15 pin the broadening and the lead self-energies)."""
    here = os.path.join(os.path.dirname(__file__), "golden")
    gT = np.loadtxt(os.path.join(here, "dos_compare_gpu_Transmission.txt"), skiprows=1)
    gD = np.loadtxt(os.path.join(here, "dos_compare_gpu_LDOS.txt"), skiprows=1)
    d = _dos_compare_tube(oracle, faithful)
    assert np.allclose(d["E"].real, gT[:, 0], rtol=0, atol=1e-6)
    assert np.max(np.abs(d["T"] - gT[:, 1]) / np.abs(gT[:, 1])) < 1e-5
    assert np.max(np.abs(d["dos"] - gD[:, 1]) / np.abs(gD[:, 1])) < 1e-5


def test_current_against_dense_inverse(oracle):
    """Terminal current (NEGF_Common.cpp:4321-4816) against a dense-inverse
    Landauer sum over the same non-equilibrium energy grid."""
    t = oracle.OracleTube(type_id=(17, 0), num_unitcells=3, num_modes=2, contact_mu=(-0.2, -0.6),
                          contact_T=(300.0, 300.0), noneq_integration_pts=(40, 30), E_zPlus_imag=1e-6)
    rng = np.random.default_rng(5)
    U = 0.1 * rng.standard_normal(t.N)
    t.set_potential(U, (U[0], U[-1]))
    I, probes = t.current(nthreads=4, probes=True)
    E, w, J = t.paths(3)
    J_, deg, beta, _ = t.modes()
    kB, q, h = 8.617333262e-5, 1.602176634e-19, 4.135667696e-15
    kT = kB * 300.0
    f = lambda x, mu: 1.0 / (np.exp((x - mu) / kT) + 1.0)
    N, g = t.N, 2.5
    Iref = 0.0
    for e in range(len(E)):
        Te = 0.0
        for m in range(len(beta)):
            S = [t.sigma(m, E[e], U[0]), t.sigma(m, E[e], U[-1])]
            A = np.zeros((N, N), complex)
            for n in range(N):
                A[n, n] = E[e] - U[n]
            for n in range(N - 1):
                hop = -beta[m] if n % 2 == 0 else -g
                A[n, n + 1] = A[n + 1, n] = -hop
            A[0, 0] -= S[0]
            A[-1, -1] -= S[1]
            G = np.linalg.inv(A)
            G0 = [1j * (S[k] - np.conj(S[k])) for k in range(2)]
            Te += deg[m] * (G0[0] * G0[1] * abs(G[0, N - 1]) ** 2).real
        Iref += (2 * q / h * (f(E[e], -0.2) - f(E[e], -0.6)) * w[e] * J[e]).real * Te
    assert abs(I[0] - Iref) / abs(Iref) < 1e-8
    assert abs(I[1] + Iref) / abs(Iref) < 1e-8
    assert probes.shape == (3, len(E)) and np.all(np.isfinite(probes))


@pytest.mark.parametrize("m,cells,mu", [(7, 3, (0.0, -0.3)), (13, 2, (-0.2, -0.5)), (4, 2, (0.1, -0.2))])
def test_oracle_realspace_noneq_equals_mode_space(oracle, m, cells, mu):
    """The oracle's dense-block real-space charge of a biased tube (contour,
    poles and the source/drain spectral functions at the real-axis points)
    equals its mode-space charge over all m // 2 + 1 distinct modes for a
    ring-uniform potential."""
    kw = dict(type_id=(m, 0), num_unitcells=cells, num_modes=m // 2 + 1, contact_mu=mu, contact_T=(300.0, 320.0),
              eq_integration_pts=(16, 16, 24), noneq_integration_pts=(40,), E_pole_max=3.0, E_zPlus_imag=1e-3)
    o = oracle.OracleTube(noneq_percent_intercuts=None, **kw)
    assert o.noneq()
    rng = np.random.default_rng(1)
    U = 0.1 * rng.standard_normal(o.N)
    o.set_potential(U, (U[0], U[-1]))
    Qm = o.charge(nthreads=4)
    Qr = o.rs_charge(nthreads=4)
    assert np.abs(Qm - Qr).max() <= 1e-12 * np.abs(Qm).max()


def _dense_rs_sums(m, K, g, E, Ua, Uc0, Uc1, iters=40):
    """Numpy dense twin of the real-space energy point: lead corners by
    Sancho-Rubio decimation of the 2m-atom cell, the whole device inverted at
    once; returns (tr G per ring, A^L per ring, A^R per ring)."""
    n = 2 * m

    def block(E, u):
        A = np.diag(E - u).astype(complex)
        for j in range(m):
            for b in (m + j, m + (j + 1) % m):
                A[j, b] -= g
                A[b, j] -= g
        return A

    def lead(u, left):
        eps = block(E, np.full(n, u))
        eps_s = eps.copy()
        tau = np.zeros((n, n))
        for j in range(m):
            tau[m + j, j] = -g
        al, be = (tau.T, tau) if left else (tau, tau.T)
        for _ in range(iters):
            G = np.linalg.inv(eps)
            agb, bga = al @ G @ be, be @ G @ al
            eps_s, eps = eps_s - agb, eps - agb - bga
            al, be = al @ G @ al, be @ G @ be
        gs = np.linalg.inv(eps_s)
        o = m if left else 0
        return gs[o:o + m, o:o + m]

    sL, sR = lead(Uc0, True), lead(Uc1, False)
    N = n * K
    M = np.zeros((N, N), complex)
    for k in range(K):
        M[k * n:(k + 1) * n, k * n:(k + 1) * n] = block(E, np.concatenate([Ua[2 * k], Ua[2 * k + 1]]))
        if k + 1 < K:
            for j in range(m):
                M[k * n + m + j, (k + 1) * n + j] = M[(k + 1) * n + j, k * n + m + j] = -g
    SL, SR = g * g * sL, g * g * sR
    M[:m, :m] -= SL
    M[N - m:, N - m:] -= SR
    G = np.linalg.inv(M)
    GL, GR = 1j * (SL - SL.conj().T), 1j * (SR - SR.conj().T)
    AL = np.einsum("ni,ij,nj->n", G[:, :m], GL, G[:, :m].conj()).real
    AR = np.einsum("ni,ij,nj->n", G[:, N - m:], GR, G[:, N - m:].conj()).real
    ring = lambda v: v.reshape(2 * K, m).sum(1)
    return ring(np.diag(G)), ring(AL), ring(AR)


def test_oracle_realspace_noneq_per_atom_against_dense(oracle):
    """Per-atom potentials (no mode decoupling): the oracle's biased
    real-space charge difference between two potentials equals a dense numpy
    evaluation over the same energy points (contour: Im(c tr G); real axis:
    b0 A^L + b1 A^R); the U = 0 Rho0 term cancels in the difference."""
    m, cells, g = 4, 2, 2.5
    kw = dict(type_id=(m, 0), num_unitcells=cells, num_modes=1, contact_mu=(0.0, -0.3), contact_T=(300.0, 320.0),
              eq_integration_pts=(12, 12, 16), noneq_integration_pts=(24,), E_pole_max=3.0, E_zPlus_imag=1e-2)
    o = oracle.OracleTube(noneq_percent_intercuts=None, **kw)
    N, K = o.N, o.N // 2
    rng = np.random.default_rng(11)
    kT = 8.617333262e-5 * np.array(kw["contact_T"])
    mu = np.array(kw["contact_mu"])
    fermi = lambda E, mu_, kT_: 1.0 / (1.0 + np.exp((E - mu_) / kT_))
    Ee, we, Je = o.paths(1)
    En, wn, Jn = o.paths(3)
    assert len(o.paths(2)[0]) == 0  # biased: no poles
    qs, dense = [], []
    for _ in range(2):
        U = 0.1 * rng.standard_normal(N)
        Ua = U[:, None] + 0.05 * rng.standard_normal((N, m))
        o.set_potential(U, (U[0], U[-1]))
        qs.append(o.rs_charge(Uatoms=Ua, nthreads=4))
        q = np.zeros(N)
        for E, w, J in zip(Ee, we, Je):
            c = (-2.0 / np.pi) * w * J * fermi(E, mu.min(), kT.min())
            q += (c * _dense_rs_sums(m, K, g, E, Ua, U[0], U[-1])[0]).imag
        for E, w, J in zip(En, wn, Jn):
            base = (-2.0 / (2 * np.pi)) * w * J
            _, aL, aR = _dense_rs_sums(m, K, g, E, Ua, U[0], U[-1])
            q += (base * fermi(E, mu[0], kT[0])).real * aL + (base * fermi(E, mu[1], kT[1])).real * aR
        dense.append(q)
    d_or, d_np = qs[0] - qs[1], dense[0] - dense[1]
    assert np.abs(d_or - d_np).max() <= 1e-9 * np.abs(d_np).max(), np.abs(d_or - d_np).max() / np.abs(d_np).max()
