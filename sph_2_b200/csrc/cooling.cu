// cooling.cu -- implicit per-particle cooling solve.
//
// Same structure as DoCooling (GPU_sph/With_cooling/Model_C/
// myPhotoLibsGPU.h:615-686): solve  u - u_old - ratefact * Lambda_net(u) * dt = 0
// with ratefact = nH^2/rho, by bracketing (factors of 1.1) and bisection to
// |du/u| <= tol, in FP64 and with every loop bounded.  Lambda_net is the
// synthetic cooling function of the cooling-cloud workload: a log-log table of
// Lambda(T) (n_bins power-law pieces between T0 and T1) and a constant heating
// per H atom; T = (gamma-1) mu m_H u / k_B.  The reference's table path
// (hcoolingx, hfvCLibs_v7_hfv_v2.h:1240-1418) is replaced by this solve.
#include "sph_internal.cuh"

#define KB_CGS 1.380649e-16
#define MH_CGS 1.6726e-24

struct CoolDev {
    const double *logL;
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
__device__ int cool_solve(const CoolDev &c, double rho, double u_old, double dt, double *u_new) {
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

__global__ void k_cool_arrays(CoolDev c, int n, const double *__restrict__ rho,
                              const double *__restrict__ u_old, const double *__restrict__ dt,
                              double *__restrict__ u_new, int *__restrict__ iters,
                              long long *status) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double un;
    int it = cool_solve(c, rho[i], u_old[i], dt[i], &un);
    u_new[i] = un;
    if (iters) iters[i] = it;
    if (it < 0) status_add(status, SPH_S_COOL_NOCONV, 1);
}

// in-step form: code units -> cgs -> code units, dt per cloud
__global__ void k_cool_state(CoolDev c, int n, const double *__restrict__ rho,
                             double *__restrict__ u, const int *__restrict__ cloud,
                             const double *__restrict__ dt, double ur, double uu, double ut,
                             long long *status) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double un;
    int it = cool_solve(c, rho[i] * ur, u[i] * uu, dt[cloud[i]] * ut, &un);
    u[i] = un / uu;
    if (it < 0) status_add(status, SPH_S_COOL_NOCONV, 1);
}

static CoolDev cool_dev(sph_ctx *ctx) {
    const sph_cooling_params &p = ctx->cool;
    CoolDev c;
    c.logL = ctx->cool_table;
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

int launch_cool_solve(sph_ctx *ctx, int n, const double *rho, const double *u_old, const double *dt,
                      double *u_new, int *iters) {
    if (n <= 0) return SPH_OK;
    k_cool_arrays<<<div_up(n, 128), 128, 0, ctx->stream>>>(cool_dev(ctx), n, rho, u_old, dt, u_new,
                                                           iters, ctx->status);
    return ctx_check_launch(ctx, "cool_solve");
}

int launch_cooling_exact(sph_ctx *ctx) {
    if (!ctx->cool_ok) return SPH_ERR_STATE;
    const int n = ctx->n, c = ctx->cur;
    if (n <= 0) return SPH_OK;
    k_cool_state<<<div_up(n, 128), 128, 0, ctx->stream>>>(
        cool_dev(ctx), n, ctx->rho, ctx->st[c][ST_U], ctx->cloud[c], ctx->dt, ctx->cool.unit_rho,
        ctx->cool.unit_u, ctx->cool.unit_t, ctx->status);
    return ctx_check_launch(ctx, "cooling_exact");
}

// the surrogate path needs the exact solver as a device function
__device__ int cool_solve_ext(const CoolDev &c, double rho, double u_old, double dt,
                              double *u_new) {
    return cool_solve(c, rho, u_old, dt, u_new);
}

extern "C" {

int sph_cooling_setup(sph_ctx *ctx, const sph_cooling_params *p, const double *log_lambda) {
    if (!ctx || !p || !log_lambda) return SPH_ERR_ARG;
    if (p->n_bins < 1 || p->n_bins > 4096 || !(p->logT1 > p->logT0) || p->max_iter < 1 ||
        !(p->tol > 0.0) || !(p->unit_rho > 0) || !(p->unit_u > 0) || !(p->unit_t > 0))
        return SPH_ERR_ARG;
    cudaSetDevice(ctx->device);
    if (!ctx->cool_table) {
        void *q = nullptr;
        CK(cudaMalloc(&q, sizeof(double) * 4097));
        ctx->allocs.push_back(q);
        ctx->dev_bytes += sizeof(double) * 4097;
        ctx->cool_table = (double *)q;
    }
    CK(cudaMemcpy(ctx->cool_table, log_lambda, sizeof(double) * (p->n_bins + 1),
                  cudaMemcpyHostToDevice));
    ctx->cool = *p;
    ctx->cool_ok = true;
    return SPH_OK;
}

int sph_cooling_exact(sph_ctx *ctx) {
    if (!ctx) return SPH_ERR_ARG;
    cudaSetDevice(ctx->device);
    return launch_cooling_exact(ctx);
}

int sph_cooling_mlp(sph_ctx *ctx) {
    if (!ctx) return SPH_ERR_ARG;
    cudaSetDevice(ctx->device);
    return launch_cooling_mlp(ctx);
}

int sph_cool_solve(sph_ctx *ctx, int32_t n, const double *rho, const double *u_old,
                   const double *dt, double *u_new, int32_t *iters, int32_t host) {
    if (!ctx || n < 0) return SPH_ERR_ARG;
    if (!ctx->cool_ok) return SPH_ERR_STATE;
    if (n == 0) return SPH_OK;
    if (!rho || !u_old || !dt || !u_new) return SPH_ERR_ARG;
    cudaSetDevice(ctx->device);
    if (!host) return launch_cool_solve(ctx, n, rho, u_old, dt, u_new, iters);
    double *d = nullptr;
    int *di = nullptr;
    CK(cudaMalloc(&d, sizeof(double) * 4 * n));
    if (iters) CK(cudaMalloc(&di, sizeof(int) * n));
    CK(cudaMemcpy(d, rho, sizeof(double) * n, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(d + n, u_old, sizeof(double) * n, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(d + 2 * (size_t)n, dt, sizeof(double) * n, cudaMemcpyHostToDevice));
    int rc = launch_cool_solve(ctx, n, d, d + n, d + 2 * (size_t)n, d + 3 * (size_t)n, di);
    if (!rc) {
        CK(cudaStreamSynchronize(ctx->stream));
        CK(cudaMemcpy(u_new, d + 3 * (size_t)n, sizeof(double) * n, cudaMemcpyDeviceToHost));
        if (iters) CK(cudaMemcpy(iters, di, sizeof(int) * n, cudaMemcpyDeviceToHost));
    }
    cudaFree(d);
    if (di) cudaFree(di);
    return rc;
}

}  // extern "C"
