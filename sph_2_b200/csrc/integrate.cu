// integrate.cu -- kick-drift-kick leapfrog in FP64, the trapezoidal u update,
// the Courant time step and the FP64 energy / momentum reductions.
//
// Replaces v_evolve, r_evolveT, u_updater, acc_g_sph (hfvCLibs_v7_hfv_v2.h:
// 806-994), the host-side updates of MPI_sph/sph_code/sph_mpi4_v4.py:284-424,
// dt_array_indiv_dt (hfvCLibs:999-1078; O(N) signal-velocity loop per
// particle, disabled in the Evrard driver) and getKE/getPE (libsx.py:571-620).
// The time step of every cloud is a per-cloud device scalar so a captured
// step graph needs no host round trip.
#include "sph_internal.cuh"

namespace {

// Courant estimate of particle i: C min(h / v_sig, sqrt(h / |a|)), or 0 if
// it is not a finite positive number
__device__ __forceinline__ double courant_dt(double hi, double vs, double ax, double ay, double az,
                                             double courant) {
    const double amag = sqrt(ax * ax + ay * ay + az * az);
    double t = hi / fmax(vs, 1e-300);
    if (amag > 0.0) t = fmin(t, sqrt(hi / amag));
    t *= courant;
    return (t > 0.0 && isfinite(t)) ? t : 0.0;
}

template <class R>
__global__ void k_kick(int n, double *__restrict__ vx, double *__restrict__ vy,
                       double *__restrict__ vz, const double *__restrict__ asph,
                       const double *__restrict__ agrav, const int *__restrict__ cloud,
                       const double *__restrict__ dt, double fac, typename R4<R>::T *__restrict__ p1,
                       int cfl, const double *__restrict__ h, const double *__restrict__ vsig,
                       double courant, unsigned long long *__restrict__ dt_bits) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = i < n;
    int c = 0;
    double t = 0.0;
    if (valid) {
        c = cloud[i];
        const double d = dt[c] * fac;
        const double ax = asph[i] + agrav[i], ay = asph[(size_t)n + i] + agrav[(size_t)n + i],
                     az = asph[2 * (size_t)n + i] + agrav[2 * (size_t)n + i];
        const double nx = vx[i] + ax * d, ny = vy[i] + ay * d, nz = vz[i] + az * d;
        vx[i] = nx;
        vy[i] = ny;
        vz[i] = nz;
        typename R4<R>::T q = p1[i];
        q.x = (R)nx; q.y = (R)ny; q.z = (R)nz;
        p1[i] = q;
        if (cfl) t = courant_dt(h[i], vsig[i], ax, ay, az, courant);
    }
    if (cfl) cloud_min(dt_bits, valid, c, t);
}

// the Courant estimate alone (prologue), from a = a_sph + a_grav
__global__ void k_cfl(int n, const double *__restrict__ asph, const double *__restrict__ agrav,
                      const int *__restrict__ cloud, const double *__restrict__ h,
                      const double *__restrict__ vsig, double courant,
                      unsigned long long *__restrict__ dt_bits) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = i < n;
    int c = 0;
    double t = 0.0;
    if (valid) {
        const double ax = asph[i] + agrav[i], ay = asph[(size_t)n + i] + agrav[(size_t)n + i],
                     az = asph[2 * (size_t)n + i] + agrav[2 * (size_t)n + i];
        c = cloud[i];
        t = courant_dt(h[i], vsig[i], ax, ay, az, courant);
    }
    cloud_min(dt_bits, valid, c, t);
}

// dt[c] <- min(Courant estimate, dt_max) (or the fixed step); reset the bits
__global__ void k_dt_commit(int ncloud, unsigned long long *dt_bits, double *dt, double dt_max,
                            double dt_fixed) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= ncloud) return;
    if (dt_fixed > 0.0) {
        dt[c] = dt_fixed;
    } else {
        unsigned long long b = dt_bits[c];
        if (b != ~0ULL) {
            double v = ord_to_dbl(b);
            if (dt_max > 0.0) v = fmin(v, dt_max);
            dt[c] = v;
        }
    }
    dt_bits[c] = ~0ULL;
}

template <class R>
__global__ void k_kick_drift(int n, double *__restrict__ x, double *__restrict__ y,
                             double *__restrict__ z, double *__restrict__ vx,
                             double *__restrict__ vy, double *__restrict__ vz,
                             const double *__restrict__ asph, const double *__restrict__ agrav,
                             const int *__restrict__ cloud, const double *__restrict__ dt,
                             int do_kick) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double d = dt[cloud[i]];
    double nx = vx[i], ny = vy[i], nz = vz[i];
    if (do_kick) {
        const double h = 0.5 * d;
        nx += (asph[i] + agrav[i]) * h;
        ny += (asph[(size_t)n + i] + agrav[(size_t)n + i]) * h;
        nz += (asph[2 * (size_t)n + i] + agrav[2 * (size_t)n + i]) * h;
        vx[i] = nx;
        vy[i] = ny;
        vz[i] = nz;
    }
    x[i] += nx * d;
    y[i] += ny * d;
    z[i] += nz * d;
}

// u <- u + dt/2 (du/dt + du/dt_prev) (u_updater, hfvCLibs_v7_hfv_v2.h:921-931).
// keep > 0: with cooling on, the cooled u can be far below the u that
// du/dt_prev was computed from, and the trapezoid can then overshoot below
// zero (negative pressure, NaN sound speed); there the step may at most halve
// u, the limiter of Gadget-2's entropy update.  keep = 0 is the reference's
// update unchanged.
__global__ void k_update_u(int n, double *__restrict__ u, double *__restrict__ dudt_prev,
                           const double *__restrict__ dudt, const int *__restrict__ cloud,
                           const double *__restrict__ dt, int first, double keep) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double d = dt[cloud[i]];
    const double du = dudt[i];
    const double u0 = u[i];
    double un = first ? u0 + du * d : u0 + 0.5 * d * (du + dudt_prev[i]);
    if (keep > 0.0 && un < keep * u0) un = keep * u0;
    u[i] = un;
    dudt_prev[i] = du;
}

// block partials of [KE, U, PE, px, py, pz, Lx, Ly, Lz, M]
constexpr int NE = 10;
__global__ void __launch_bounds__(256)
    k_energy_partial(int n, const double *__restrict__ x, const double *__restrict__ y,
                     const double *__restrict__ z, const double *__restrict__ vx,
                     const double *__restrict__ vy, const double *__restrict__ vz,
                     const double *__restrict__ m, const double *__restrict__ u,
                     const double *__restrict__ pot, int have_pot, double *__restrict__ part) {
    __shared__ double sh[NE][256];
    const int t = threadIdx.x;
    double e[NE] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
    for (int i = blockIdx.x * blockDim.x + t; i < n; i += gridDim.x * blockDim.x) {
        const double mi = m[i], X = x[i], Y = y[i], Z = z[i], VX = vx[i], VY = vy[i], VZ = vz[i];
        e[0] += 0.5 * mi * (VX * VX + VY * VY + VZ * VZ);
        e[1] += mi * u[i];
        if (have_pot) e[2] += 0.5 * mi * pot[i];
        e[3] += mi * VX;
        e[4] += mi * VY;
        e[5] += mi * VZ;
        e[6] += mi * (Y * VZ - Z * VY);
        e[7] += mi * (Z * VX - X * VZ);
        e[8] += mi * (X * VY - Y * VX);
        e[9] += mi;
    }
    for (int k = 0; k < NE; k++) sh[k][t] = e[k];
    __syncthreads();
    for (int s = 128; s > 0; s >>= 1) {
        if (t < s)
            for (int k = 0; k < NE; k++) sh[k][t] += sh[k][t + s];
        __syncthreads();
    }
    if (t < NE) part[blockIdx.x * NE + t] = sh[t][0];
}

__global__ void k_energy_final(int nb, const double *__restrict__ part, double *__restrict__ out) {
    int k = threadIdx.x;
    if (k >= NE) return;
    double s = 0.0;
    for (int b = 0; b < nb; b++) s += part[b * NE + k];
    out[k] = s;
}

}  // namespace

int launch_kick(sph_ctx *ctx, double fac, bool cfl) {
    const int n = ctx->n, c = ctx->cur;
    if (n <= 0) return SPH_OK;
    double *const *st = ctx->st[c];
    if (ctx->cfg.precision == SPH_PREC_MIXED)
        k_kick<float><<<div_up(n, 256), 256, 0, ctx->stream>>>(
            n, st[ST_VX], st[ST_VY], st[ST_VZ], ctx->asph, ctx->agrav, ctx->cloud[c], ctx->dt, fac,
            (float4 *)ctx->p1, cfl ? 1 : 0, st[ST_H], ctx->vsig, ctx->cfg.courant, ctx->dt_bits);
    else
        k_kick<double><<<div_up(n, 256), 256, 0, ctx->stream>>>(
            n, st[ST_VX], st[ST_VY], st[ST_VZ], ctx->asph, ctx->agrav, ctx->cloud[c], ctx->dt, fac,
            (double4 *)ctx->p1, cfl ? 1 : 0, st[ST_H], ctx->vsig, ctx->cfg.courant, ctx->dt_bits);
    return ctx_check_launch(ctx, "kick");
}

int launch_kick_drift(sph_ctx *ctx) {
    const int n = ctx->n, c = ctx->cur;
    if (n <= 0) return SPH_OK;
    double *const *st = ctx->st[c];
    k_kick_drift<double><<<div_up(n, 256), 256, 0, ctx->stream>>>(
        n, st[ST_X], st[ST_Y], st[ST_Z], st[ST_VX], st[ST_VY], st[ST_VZ], ctx->asph, ctx->agrav,
        ctx->cloud[c], ctx->dt, 1);
    return ctx_check_launch(ctx, "kick_drift");
}

int launch_drift(sph_ctx *ctx) {
    const int n = ctx->n, c = ctx->cur;
    if (n <= 0) return SPH_OK;
    double *const *st = ctx->st[c];
    k_kick_drift<double><<<div_up(n, 256), 256, 0, ctx->stream>>>(
        n, st[ST_X], st[ST_Y], st[ST_Z], st[ST_VX], st[ST_VY], st[ST_VZ], ctx->asph, ctx->agrav,
        ctx->cloud[c], ctx->dt, 0);
    return ctx_check_launch(ctx, "drift");
}

int launch_update_u(sph_ctx *ctx, bool first) {
    const int n = ctx->n, c = ctx->cur;
    if (n <= 0) return SPH_OK;
    k_update_u<<<div_up(n, 256), 256, 0, ctx->stream>>>(n, ctx->st[c][ST_U],
                                                        ctx->st[c][ST_DUDT_PREV], ctx->dudt,
                                                        ctx->cloud[c], ctx->dt, first ? 1 : 0,
                                                        (ctx->cfg.flags & SPH_FLAG_COOLING) ? 0.5 : 0.0);
    return ctx_check_launch(ctx, "update_u");
}

// Courant estimate from the current accelerations (no kick) + commit
int launch_cfl(sph_ctx *ctx) {
    const int n = ctx->n, c = ctx->cur;
    if (n > 0 && ctx->cfg.dt_fixed <= 0.0)
        k_cfl<<<div_up(n, 256), 256, 0, ctx->stream>>>(n, ctx->asph, ctx->agrav, ctx->cloud[c],
                                                       ctx->st[c][ST_H], ctx->vsig,
                                                       ctx->cfg.courant, ctx->dt_bits);
    k_dt_commit<<<div_up(ctx->ncloud, 128), 128, 0, ctx->stream>>>(
        ctx->ncloud, ctx->dt_bits, ctx->dt, ctx->cfg.dt_max, ctx->cfg.dt_fixed);
    return ctx_check_launch(ctx, "cfl");
}

int launch_dt_commit(sph_ctx *ctx) {
    k_dt_commit<<<div_up(ctx->ncloud, 128), 128, 0, ctx->stream>>>(
        ctx->ncloud, ctx->dt_bits, ctx->dt, ctx->cfg.dt_max, ctx->cfg.dt_fixed);
    return ctx_check_launch(ctx, "dt_commit");
}

int launch_energies(sph_ctx *ctx, double *out10) {
    const int n = ctx->n, c = ctx->cur;
    double *const *st = ctx->st[c];
    const int nb = 296;
    double *part = ctx->red;
    double *fin = ctx->red + (size_t)nb * NE;
    k_energy_partial<<<nb, 256, 0, ctx->stream>>>(n, st[ST_X], st[ST_Y], st[ST_Z], st[ST_VX],
                                                  st[ST_VY], st[ST_VZ], st[ST_M], st[ST_U],
                                                  ctx->pot, 1, part);
    k_energy_final<<<1, 32, 0, ctx->stream>>>(nb, part, fin);
    CK(cudaMemcpyAsync(out10, fin, NE * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return ctx_check_launch(ctx, "energies");
}
