// Complex FP64 scalars and the surface Green's function of one lead mode
// chain (alternating hoppings beta and gamma, the surface site's first bond
// beta).  Included inside namespace negf's anonymous namespace by the mode-space
// kernels (negf_rgf.cu) and by the real-space leads (negf_realspace.cu),
// which assemble a ring corner from these per-mode values; it holds no
// #include and no namespace of its own.
#pragma once

struct cd {
    double x, y;
};
__device__ __forceinline__ cd cadd(cd a, cd b) { return {a.x + b.x, a.y + b.y}; }
__device__ __forceinline__ cd csub(cd a, cd b) { return {a.x - b.x, a.y - b.y}; }
__device__ __forceinline__ cd cmul(cd a, cd b) { return {a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x}; }
__device__ __forceinline__ cd cscale(double s, cd a) { return {s * a.x, s * a.y}; }
__device__ __forceinline__ cd cconj(cd a) { return {a.x, -a.y}; }
__device__ __forceinline__ cd cinv(cd a) {
    const double r = 1.0 / (a.x * a.x + a.y * a.y);
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
