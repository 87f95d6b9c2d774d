// cooling.cu -- implicit per-particle cooling solve.
//
// The solver itself is in cooling.cuh.  The reference's table path
// (hcoolingx, hfvCLibs_v7_hfv_v2.h:1240-1418) is replaced by this solve.
#include <math.h>

#include <vector>

#include "cooling.cuh"

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

static CoolDev cool_dev(sph_ctx *ctx) { return cool_dev_of(ctx); }

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

extern "C" {

int sph_cooling_setup(sph_ctx *ctx, const sph_cooling_params *p, const double *log_lambda) {
    if (!ctx || !p || !log_lambda) return SPH_ERR_ARG;
    if (p->n_bins < 1 || p->n_bins > 4096 || !(p->logT1 > p->logT0) || p->max_iter < 1 ||
        !(p->tol > 0.0) || !(p->unit_rho > 0) || !(p->unit_u > 0) || !(p->unit_t > 0))
        return SPH_ERR_ARG;
    cudaSetDevice(ctx->device);
    if (!ctx->cool_table) {
        void *q = nullptr;
        CK(cudaMalloc(&q, sizeof(double) * 2 * 4097));
        ctx->allocs.push_back(q);
        ctx->dev_bytes += sizeof(double) * 2 * 4097;
        ctx->cool_table = (double *)q;
    }
    CK(cudaMemcpyAsync(ctx->cool_table, log_lambda, sizeof(double) * (p->n_bins + 1),
                       cudaMemcpyHostToDevice, ctx->stream));
    {
        // Lambda(T_e) / T_e at the bin edges, for the surrogate's monotonicity test
        const double dl = (p->logT1 - p->logT0) / p->n_bins;
        std::vector<double> lamT(p->n_bins + 1);
        for (int e = 0; e <= p->n_bins; e++) lamT[e] = pow(10.0, log_lambda[e] - (p->logT0 + e * dl));
        CK(cudaMemcpyAsync(ctx->cool_table + 4097, lamT.data(), sizeof(double) * (p->n_bins + 1),
                           cudaMemcpyHostToDevice, ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
    }
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
    // stream-ordered before the solve on the context's non-blocking stream
    CK(cudaMemcpyAsync(d, rho, sizeof(double) * n, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(d + n, u_old, sizeof(double) * n, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(d + 2 * (size_t)n, dt, sizeof(double) * n, cudaMemcpyHostToDevice, ctx->stream));
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
