// cooling.cuh -- device functions of the implicit cooling solve, shared by
// the exact solver (cooling.cu) and the surrogate's fallback (mlp.cu).
//
// Same structure as DoCooling (GPU_sph/With_cooling/Model_C/
// myPhotoLibsGPU.h:615-686): solve  u - u_old - ratefact * Lambda_net(u) * dt = 0
// with ratefact = nH^2/rho, by bracketing (factors of 1.1) and bisection to
// |du/u| <= tol, in FP64 and with every loop bounded.  Lambda_net is the
// synthetic cooling function of the cooling-cloud workload: a log-log table of
// Lambda(T) (n_bins power-law pieces between T0 and T1) and a constant heating
// per H atom; T = (gamma-1) mu m_H u / k_B.
#pragma once
#include "sph_internal.cuh"

#define KB_CGS 1.380649e-16
#define MH_CGS 1.6726e-24

struct CoolDev {
    const double *logL;
    const double *lamT;  // Lambda(T_e) / T_e at the bin edges T_e (host-computed)
    int nb;
    double logT0, logT1, mu, gamma, XH, gheat, tol;
    int max_iter;
};

__device__ __forceinline__ double cool_lambda(const CoolDev &c, double T, double *slope) {
    const double lt = log10(T);
    const double dl = (c.logT1 - c.logT0) / c.nb;
    int k = (int)floor((lt - c.logT0) / dl);
    k = k < 0 ? 0 : (k > c.nb - 1 ? c.nb - 1 : k);
    const double s = (c.logL[k + 1] - c.logL[k]) / dl;
    const double ll = c.logL[k] + s * (lt - (c.logT0 + k * dl));
    if (slope) *slope = s;
    return exp10(ll);
}

__device__ __forceinline__ double cool_net(const CoolDev &c, double u, double nH) {
    const double T = (c.gamma - 1.0) * c.mu * MH_CGS / KB_CGS * u;
    return c.gheat / nH - cool_lambda(c, T, nullptr);
}

// returns the bisection count, -1 if the tolerance was not reached
__device__ __forceinline__ int cool_solve(const CoolDev &c, double rho, double u_old, double dt, double *u_new) {
    const double nH = c.XH * rho / MH_CGS;
    const double ratefact = nH * nH / rho;
    double u = u_old, up = u, lo = u;
    const double r0 = u - u_old - ratefact * cool_net(c, u, nH) * dt;
    int guard = 0;
    if (r0 > 0.0) {
        while (up - u_old - ratefact * cool_net(c, up, nH) * dt > 0.0 && guard++ < 2000) up /= 1.1;
        lo = up;
        up = lo * 1.1;
    } else if (r0 < 0.0) {
        while (up - u_old - ratefact * cool_net(c, up, nH) * dt < 0.0 && guard++ < 2000) up *= 1.1;
        lo = up / 1.1;
    } else {
        *u_new = u;
        return 0;
    }
    double du = u;
    int it = 1;
    while (fabs(du / u) > c.tol && it < c.max_iter) {
        u = 0.5 * (lo + up);
        const double r = u - u_old - ratefact * cool_net(c, u, nH) * dt;
        if (r > 0.0) up = u; else lo = u;
        du = fabs(up - lo);
        it++;
    }
    *u_new = u;
    return fabs(du / u) > c.tol ? -1 : it;
}


// Newton-step estimate of the error of an approximate solution u of
// u - u_old - ratefact * net(u) * dt = 0:  delta = r(u) / r'(u), with
// r'(u) = 1 + ratefact * dt * s * Lambda(T) / u (Lambda ~ T^s inside a bin,
// T ~ u).  Returns |delta|/u, or +inf where r' <= 0 (the estimate is void).
__device__ __forceinline__ double cool_error_estimate(const CoolDev &c, double rho, double u_old,
                                                      double dt, double u) {
    const double nH = c.XH * rho / MH_CGS;
    const double ratefact = nH * nH / rho;
    const double T = (c.gamma - 1.0) * c.mu * MH_CGS / KB_CGS * u;
    double s;
    const double lam = cool_lambda(c, T, &s);
    const double r = u - u_old - ratefact * (c.gheat / nH - lam) * dt;
    const double rp = 1.0 + ratefact * dt * s * lam / u;
    if (!(rp > 0.0) || !(u > 0.0)) return INFINITY;
    return fabs(r / rp) / u;
}

// Newton steps of the implicit equation from an approximate solution *u (the
// surrogate's prediction): at each iterate r(u) and r'(u) give the error
// estimate |r/r'|/u; the iterate is kept as soon as that estimate is within
// tol / 4, else u <- u - r/r' (when r' > 0 and the step keeps u positive),
// at most four steps.  *est <- the estimate of the returned *u (+inf when it
// is void).  One cooling-function evaluation per iterate.
__device__ __forceinline__ void cool_newton_polish(const CoolDev &c, double rho, double u_old,
                                                   double dt, double *u, double *est, double tol) {
    const double nH = c.XH * rho / MH_CGS;
    const double ratefact = nH * nH / rho;
    const double kT = (c.gamma - 1.0) * c.mu * MH_CGS / KB_CGS;
    double uu = *u;
    *est = INFINITY;
    for (int it = 0; it < 5; it++) {
        double s;
        const double lam = cool_lambda(c, kT * uu, &s);
        const double r = uu - u_old - ratefact * (c.gheat / nH - lam) * dt;
        const double rp = 1.0 + ratefact * dt * s * lam / uu;
        if (!(rp > 0.0) || !(uu > 0.0)) break;  // the estimate is void here
        const double e = fabs(r / rp) / uu;
        *u = uu;
        *est = e;
        if (e <= 0.25 * tol || it == 4) break;
        const double u1 = uu - r / rp;
        if (!(u1 > 0.0)) break;
        uu = u1;
    }
}

// True when r(u) = u - u_old - ratefact*net(u)*dt is strictly increasing on
// [u_lo, u_hi]: r'(u) = 1 + ratefact*dt*s*Lambda(T)/u.  Inside a table bin
// Lambda ~ T^s, so Lambda/u ~ T^(s-1): r' > 1 where s >= 0, and where s < 0 r'
// grows with T, so its smallest value in a bin is at the bin's lower end.  The
// interval is monotone iff r' > 0 at T(u_lo) (when its bin has s < 0) and at
// the lower edge of every bin with s < 0 that starts inside the interval;
// Lambda/T at the edges is tabulated, so only T(u_lo) needs a transcendental.
__device__ __forceinline__ bool cool_monotone(const CoolDev &c, double rho, double dt, double u_lo,
                                              double u_hi) {
    const double nH = c.XH * rho / MH_CGS;
    const double A = nH * nH / rho * dt;
    const double kT = (c.gamma - 1.0) * c.mu * MH_CGS / KB_CGS;
    const double dl = (c.logT1 - c.logT0) / c.nb;
    const double T0 = kT * u_lo, T1 = kT * u_hi;
    if (!(T0 > 0.0) || !(T1 >= T0)) return false;
    const double l0 = log10(T0), l1 = log10(T1);
    int k = (int)floor((l0 - c.logT0) / dl);
    k = k < 0 ? 0 : (k > c.nb - 1 ? c.nb - 1 : k);
    double s = (c.logL[k + 1] - c.logL[k]) / dl;
    if (s < 0.0) {
        const double lam = exp10(c.logL[k] + s * (l0 - (c.logT0 + k * dl)));
        if (!(1.0 + A * s * lam * kT / T0 > 0.0)) return false;
    }
    // lower edges of the bins after T0's bin, up to T1 (edge k at logT0 + k dl;
    // below bin 0 and above bin nb-1 the end slopes continue, no edges)
    int kend = (int)floor((l1 - c.logT0) / dl);
    kend = kend > c.nb - 1 ? c.nb - 1 : kend;
    for (int e = k + 1; e <= kend; e++) {
        s = (c.logL[e + 1] - c.logL[e]) / dl;
        if (s < 0.0) {
            if (!(1.0 + A * s * c.lamT[e] * kT > 0.0)) return false;
        }
    }
    return true;
}

// accept a surrogate solution un (after cool_newton_polish, estimate est)?
__device__ __forceinline__ bool cool_accept(const CoolDev &c, double rho, double u_old, double dt,
                                            double un, double est, double tol) {
    if (!(est <= tol) || !(un > 0.0)) return false;
    const double lo = fmin(u_old, un / 1.1), hi = fmax(u_old, un * 1.1);
    return cool_monotone(c, rho, dt, lo, hi);
}

// ---- the surrogate's side in FP32 -------------------------------------------
// The surrogate is accepted to a relative error of mlp_err_tol (1e-3 by
// default), far above FP32 rounding, so its Newton polish, error estimate and
// monotonicity test run in FP32, where the logarithm and exponential are
// single SFU instructions (the FP64 ones are long FMA-pipe sequences and made
// the FP64 polish as slow as the exact bisection it should replace).  The
// residual u - u_old - ratefact * net * dt is formed in FP32 from FP32 u and
// u_old: its rounding (~1e-7 u) is four orders below the tolerance.  The
// products are ordered so that no intermediate leaves the FP32 range:
// ratefact = nH^2 / rho reaches 1e29 and ratefact * dt 1e42, but ratefact *
// Lambda stays below 1e10 and its product with dt below 1e25.  The exact
// solver and the fallback stay in FP64.
__device__ __forceinline__ float cool_lambda_f(const CoolDev &c, float T, float *slope) {
    const float lt = __log10f(T);
    const float lT0 = (float)c.logT0;
    const float dl = (float)((c.logT1 - c.logT0) / c.nb);
    int k = (int)floorf((lt - lT0) / dl);
    k = k < 0 ? 0 : (k > c.nb - 1 ? c.nb - 1 : k);
    const float L0 = (float)c.logL[k], L1 = (float)c.logL[k + 1];
    const float s = (L1 - L0) / dl;
    if (slope) *slope = s;
    return __exp10f(L0 + s * (lt - (lT0 + k * dl)));
}

__device__ __forceinline__ void cool_newton_polish_f(const CoolDev &c, double rho, double u_old,
                                                     double dt, double *u, double *est, double tol) {
    const double nHd = c.XH * rho / MH_CGS;
    const float ratefact = (float)(nHd * nHd / rho);
    const float kT = (float)((c.gamma - 1.0) * c.mu * MH_CGS / KB_CGS);
    const float gn = (float)(c.gheat / nHd);
    const float uo = (float)u_old, fdt = (float)dt, ftol = (float)tol;
    float uu = (float)*u;
    *est = INFINITY;
    for (int it = 0; it < 5; it++) {
        float s;
        const float lam = cool_lambda_f(c, kT * uu, &s);
        const float r = uu - uo - (ratefact * (gn - lam)) * fdt;
        const float rp = 1.f + (ratefact * lam) * fdt * s / uu;
        if (!(rp > 0.f) || !(uu > 0.f)) break;  // the estimate is void here
        const float e = fabsf(r / rp) / uu;
        *u = (double)uu;
        *est = (double)e;
        if (e <= 0.25f * ftol || it == 4) break;
        const float u1 = uu - r / rp;
        if (!(u1 > 0.f)) break;
        uu = u1;
    }
}

__device__ __forceinline__ bool cool_monotone_f(const CoolDev &c, double rho, double dt, double u_lo,
                                                double u_hi) {
    // A = ratefact * dt can pass the FP32 range: it is applied in FP64 to
    // the Lambda / T values (two multiplies, no transcendental)
    const double A = (c.XH * rho / MH_CGS) * (c.XH * rho / MH_CGS) / rho * dt;
    const float kT = (float)((c.gamma - 1.0) * c.mu * MH_CGS / KB_CGS);
    const float lT0 = (float)c.logT0;
    const float dl = (float)((c.logT1 - c.logT0) / c.nb);
    const float T0 = kT * (float)u_lo, T1 = kT * (float)u_hi;
    if (!(T0 > 0.f) || !(T1 >= T0)) return false;
    const float l0 = __log10f(T0), l1 = __log10f(T1);
    int k = (int)floorf((l0 - lT0) / dl);
    k = k < 0 ? 0 : (k > c.nb - 1 ? c.nb - 1 : k);
    float s = (float)(c.logL[k + 1] - c.logL[k]) / dl;
    if (s < 0.f) {
        const float lam = __exp10f((float)c.logL[k] + s * (l0 - (lT0 + k * dl)));
        if (!(1.0 + A * (double)(s * (lam / T0) * kT) > 0.0)) return false;
    }
    int kend = (int)floorf((l1 - lT0) / dl);
    kend = kend > c.nb - 1 ? c.nb - 1 : kend;
    for (int e = k + 1; e <= kend; e++) {
        s = (float)(c.logL[e + 1] - c.logL[e]) / dl;
        if (s < 0.f) {
            if (!(1.0 + A * (double)s * c.lamT[e] * (double)kT > 0.0)) return false;
        }
    }
    return true;
}

__device__ __forceinline__ bool cool_accept_f(const CoolDev &c, double rho, double u_old, double dt,
                                              double un, double est, double tol) {
    if (!(est <= tol) || !(un > 0.0)) return false;
    const double lo = fmin(u_old, un / 1.1), hi = fmax(u_old, un * 1.1);
    return cool_monotone_f(c, rho, dt, lo, hi);
}

static inline CoolDev cool_dev_of(const sph_ctx *ctx) {
    const sph_cooling_params &p = ctx->cool;
    CoolDev c;
    c.logL = ctx->cool_table;
    c.lamT = ctx->cool_table + 4097;
    c.nb = p.n_bins;
    c.logT0 = p.logT0;
    c.logT1 = p.logT1;
    c.mu = p.mu;
    c.gamma = p.gamma;
    c.XH = p.XH;
    c.gheat = p.gamma_heat;
    c.tol = p.tol;
    c.max_iter = p.max_iter;
    return c;
}
