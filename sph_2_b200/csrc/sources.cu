// sources.cu -- mass sources and external fields of the AGN runs: outflow
// particle injection and the isothermal galaxy potential.
//
// Replaces outflow_injector2 (Particles_in_BH_Tree_II/Evrard_test/
// hfvCLibs_v7_hfv_v2.h:1094-1210) and galaxy_isothermal_potential
// (:1215-1235), both written for Richings et al. (2018)'s set-up.
//
// Injection: the mass M_dot dt (plus what the last call left over) is spawned
// as pairs of particles of mass m placed at +r and -r, r uniform in radius up
// to r_max and isotropic in direction (azimuth 2 pi u, polar angle
// acos(2u - 1)), moving radially outward at v_in, with u and the
// smoothing length (and softening) of the last particle injected before.  The
// reference runs this serially in one thread with one cuRAND state per pair;
// here one thread builds one pair, the new particles are appended after the
// last stored particle (their original ids continue the count), and each
// pair's three uniforms come from a counter-based generator keyed by (seed,
// pair number): the SplitMix64 output function (Steele, Lea and Flood 2014)
// of seed + golden-ratio increments, so a pair is the same whatever the launch
// shape.  The numbers differ from cuRAND's, the distribution does not.
//
// Isothermal potential: a = -G M(r) r_vec / r^3 with M(r) = 2 sigma^2 r / G,
// i.e. a = -2 sigma^2 r_vec / r^2, added to the gravitational acceleration
// of every particle after the walk (a particle at r = 0 gets none; the
// reference divides by zero there).
#include "sph_internal.cuh"

namespace {

__host__ __device__ __forceinline__ unsigned long long splitmix64(unsigned long long z) {
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}

// uniform in (0, 1] from the k-th draw of pair j
__device__ __forceinline__ double pair_uniform(unsigned long long seed, long long j, int k) {
    const unsigned long long z = splitmix64(seed + 0x9e3779b97f4a7c15ULL * (unsigned long long)(3 * j + k + 1));
    return (double)((z >> 11) + 1) * 0x1.0p-53;
}

__global__ void k_inject_pairs(int npairs, unsigned long long seed, int n0, int id0, int cloud,
                               double r_max, double v_in, double m,
                               double u, const double *__restrict__ h_src, double *const *st,
                               int *__restrict__ id, int *__restrict__ cl,
                               double *__restrict__ dudt) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= npairs) return;
    const long long j = p;
    const double rt = pair_uniform(seed, j, 0) * r_max;
    const double th = pair_uniform(seed, j, 1) * 2.0 * SPH_PI;
    const double ph = acos(2.0 * pair_uniform(seed, j, 2) - 1.0);
    const double sp = sin(ph);
    const double xt = rt * sp * cos(th), yt = rt * sp * sin(th), zt = rt * cos(ph);
    const double rr = sqrt(xt * xt + yt * yt + zt * zt);
    const double s = rr > 0.0 ? v_in / rr : 0.0;
    const double h = *h_src;
    // the pair: +r / +v and -r / -v
    for (int side = 0; side < 2; side++) {
        const int i = n0 + 2 * p + side;
        const double sg = side ? -1.0 : 1.0;
        st[ST_X][i] = sg * xt;
        st[ST_Y][i] = sg * yt;
        st[ST_Z][i] = sg * zt;
        st[ST_VX][i] = sg * xt * s;
        st[ST_VY][i] = sg * yt * s;
        st[ST_VZ][i] = sg * zt * s;
        st[ST_M][i] = m;
        st[ST_H][i] = h;
        st[ST_U][i] = u;
        st[ST_DUDT_PREV][i] = 0.0;
        st[ST_HNB][i] = 0.0;
        id[i] = id0 + 2 * p + side;
        cl[i] = cloud;
        dudt[i] = 0.0;
    }
}

// h of the particle whose original id is `want` (storage slot found by scan;
// ids are unique, so one thread at most writes)
__global__ void k_h_of_id(int n, const int *__restrict__ id, const double *__restrict__ h, int want,
                          double *__restrict__ out) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s < n && id[s] == want) *out = h[s];
}

__global__ void k_isothermal(int n, const double *__restrict__ x, const double *__restrict__ y,
                             const double *__restrict__ z, double two_sigma2,
                             double *__restrict__ agrav, int stride) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double X = x[i], Y = y[i], Z = z[i];
    const double r2 = X * X + Y * Y + Z * Z;
    if (!(r2 > 0.0)) return;
    const double f = two_sigma2 / r2;
    agrav[i] -= f * X;
    agrav[(size_t)stride + i] -= f * Y;
    agrav[2 * (size_t)stride + i] -= f * Z;
}

}  // namespace

// the external isothermal field of sigma = cfg.ext_sigma, added to agrav
int launch_external_potential(sph_ctx *ctx, cudaStream_t s) {
    const int n = ctx->n, c = ctx->cur;
    if (n <= 0 || !(ctx->cfg.ext_sigma > 0.0)) return SPH_OK;
    const double sg = ctx->cfg.ext_sigma;
    // agrav holds three blocks of n (x block, y block, z block)
    k_isothermal<<<div_up(n, 256), 256, 0, s>>>(n, ctx->st[c][ST_X], ctx->st[c][ST_Y],
                                                ctx->st[c][ST_Z], 2.0 * sg * sg, ctx->agrav, n);
    return ctx_check_launch(ctx, "external_potential");
}

// Append npairs pairs after the n stored particles (the caller checked the
// capacity and that `cloud` is the last cloud, so clouds stay contiguous).
// The three-block acceleration arrays (stride n) are laid out again at the
// new stride, the new particles' entries zero.
int launch_inject_pairs(sph_ctx *ctx, int npairs, unsigned long long seed, int cloud,
                        double r_max, double v_in, double m, double u, int h_id, double h_first) {
    const int n0 = ctx->n, c = ctx->cur, n1 = n0 + 2 * npairs;
    cudaStream_t s = ctx->stream;
    double *hbuf = ctx->red;
    CK(cudaMemcpyAsync(hbuf, &h_first, sizeof(double), cudaMemcpyHostToDevice, s));
    if (h_id >= 0)
        k_h_of_id<<<div_up(max(n0, 1), 256), 256, 0, s>>>(n0, ctx->id[c], ctx->st[c][ST_H], h_id,
                                                          hbuf);
    CK(cudaMemcpyAsync(ctx->st_table, ctx->st[c], sizeof(double *) * ST_N, cudaMemcpyHostToDevice, s));
    k_inject_pairs<<<div_up(npairs, 128), 128, 0, s>>>(npairs, seed, n0, n0, cloud, r_max, v_in, m,
                                                       u, hbuf, ctx->st_table, ctx->id[c],
                                                       ctx->cloud[c], ctx->dudt);
    // relayout of a_sph and a_grav through the scratch buffer (2 N doubles)
    double *tmp = ctx->red + 8;
    for (double *a : {ctx->asph, ctx->agrav}) {
        if (n0 > 0)
            CK(cudaMemcpyAsync(tmp, a + n0, sizeof(double) * 2 * n0, cudaMemcpyDeviceToDevice, s));
        CK(cudaMemsetAsync(a + n0, 0, sizeof(double) * (3 * (size_t)n1 - n0), s));
        if (n0 > 0) {
            CK(cudaMemcpyAsync(a + n1, tmp, sizeof(double) * n0, cudaMemcpyDeviceToDevice, s));
            CK(cudaMemcpyAsync(a + 2 * (size_t)n1, tmp + n0, sizeof(double) * n0,
                               cudaMemcpyDeviceToDevice, s));
        }
    }
    for (double *a : {ctx->vsig, ctx->pot, ctx->rho, ctx->P, ctx->c, ctx->divV, ctx->curlV})
        CK(cudaMemsetAsync(a + n0, 0, sizeof(double) * 2 * npairs, s));
    return ctx_check_launch(ctx, "inject_pairs");
}
