/*
 * sph_oracle.c -- CPU ORACLE (test infrastructure only).
 *
 * This file is the checker, never the product.  Only tests/, the smoke()
 * entry point and the cpu_baseline / reference arm of bench.py load it.  The
 * GPU library under sph_2_b200/csrc never links or calls it.
 *
 * Two groups of functions live here, all in IEEE FP64, compiled with
 * -ffp-contract=off so that every product and sum is rounded exactly as
 * written (the GPU FP64 kernels spell out the same roundings with __dmul_rn /
 * __dadd_rn, which is what makes keys, neighbour lists and tree nodes
 * bit-exact between the two):
 *
 *  (A) restatements of the reference's own CPU step (hassanfv/SPH_2,
 *      11_Dec_2022/MPI_sph/sph_code/libsx.py and shear.py).  They keep the
 *      reference's row-range signature (nbeg, nend) and its all-pairs loops.
 *      They are pinned against golden vectors produced by running the numba
 *      reference itself (tests/golden/make_golden.py), and they are the
 *      timed CPU baseline (OpenMP over row ranges = the reference's MPI
 *      row split, sph_mpi4_v4.py:57-65).
 *
 *  (B) the project method the CUDA path implements: Morton keys, exact
 *      neighbour predicate, Newton smoothing length, list-based SPH sums with
 *      Monaghan-Gingold (1983) or Gadget/Balsara viscosity, Karras radix
 *      tree with FP64 monopole+quadrupole moments, the group Barnes-Hut walk
 *      with the same acceptance test, Plummer direct summation, and the
 *      implicit cooling solve.  Where the reference has no counterpart
 *      (Morton keys, Newton h, quadrupole tree, synthetic cooling table) the
 *      parity is pinned only by this restatement and by FP64 direct sums.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORC_PI 3.14159265358979323846
#define SIG (1.0 / ORC_PI)

/* ------------------------------------------------------------------------ */
/* M4 cubic spline, sigma = 1/pi, support 2h (libsx.py:69-80, shear.py:109-121) */
static inline double w_m4(double rr, double hij)
{
    double q = rr / hij;
    double h3 = hij * hij * hij;
    if (q <= 1.0) return SIG / h3 * (1.0 - (3.0 / 2.0) * q * q + (3.0 / 4.0) * q * q * q);
    if (q <= 2.0) { double t = 2.0 - q; return SIG / h3 * (1.0 / 4.0) * t * t * t; }
    return 0.0;
}

/* scalar nW such that gradW = nW * (dx,dy,dz)  (shear.py:109-121, incl. q+1e-20) */
static inline double gradw_m4(double rr, double hij)
{
    double q = rr / hij;
    double h5 = hij * hij * hij * hij * hij;
    if (q <= 1.0) return SIG / h5 * (-3.0 + 9.0 / 4.0 * q);
    if (q <= 2.0) { double t = 2.0 - q; return -3.0 * SIG / 4.0 / h5 * t * t / (q + 1e-20); }
    return 0.0;
}

/* ======================================================================== */
/* (A) restatements of the reference CPU step                               */
/* ======================================================================== */

/* getDensity_mpi, libsx.py:52-86 */
void ref_density(int N, const double *pos, const double *m, const double *h,
                 int nbeg, int nend, double *rho)
{
#pragma omp parallel for schedule(dynamic, 16)
    for (int i = nbeg; i < nend; i++) {
        double s = 0.0;
        for (int j = 0; j < N; j++) {
            double dx = pos[3 * i] - pos[3 * j], dy = pos[3 * i + 1] - pos[3 * j + 1], dz = pos[3 * i + 2] - pos[3 * j + 2];
            double rr = sqrt(dx * dx + dy * dy + dz * dz);
            double hij = 0.5 * (h[i] + h[j]);
            s += m[j] * w_m4(rr, hij);
        }
        rho[i - nbeg] = s;
    }
}

/* div_curlVel_mpi, shear.py:78-142 */
void ref_div_curl(int N, const double *pos, const double *v, const double *rho, const double *m,
                  const double *h, int nbeg, int nend, double *divV, double *curlV)
{
#pragma omp parallel for schedule(dynamic, 16)
    for (int i = nbeg; i < nend; i++) {
        double s = 0.0, cx = 0.0, cy = 0.0, cz = 0.0;
        for (int j = 0; j < N; j++) {
            double dx = pos[3 * i] - pos[3 * j], dy = pos[3 * i + 1] - pos[3 * j + 1], dz = pos[3 * i + 2] - pos[3 * j + 2];
            double rr = sqrt(dx * dx + dy * dy + dz * dz);
            double hij = 0.5 * (h[i] + h[j]);
            double nW = gradw_m4(rr, hij);
            double gx = nW * dx, gy = nW * dy, gz = nW * dz;
            double vx = v[3 * i] - v[3 * j], vy = v[3 * i + 1] - v[3 * j + 1], vz = v[3 * i + 2] - v[3 * j + 2];
            double f = m[j] / rho[i];
            s += f * (-vx * gx - vy * gy - vz * gz);
            cx += f * (vy * gz - vz * gy);
            cy += f * (vz * gx - vx * gz);
            cz += f * (vx * gy - vy * gx);
        }
        divV[i - nbeg] = fabs(s);
        curlV[i - nbeg] = sqrt(cx * cx + cy * cy + cz * cz);
    }
}

/* Pair viscosity.  mode 0: Monaghan & Gingold 1983 (libsx.py:236-245);
 * mode 1: Gadget signal velocity (shear.py:291-306).  Balsara factor f_ij
 * (shear.py:309-313) applied when balsara != 0. */
static inline double pi_ij(int mode, int balsara, double vr, double rr, double hij,
                           double ci, double cj, double rhoi, double rhoj,
                           double fi, double fj, double alpha, double beta, double eta)
{
    double PI = 0.0;
    if (vr <= 0.0) {
        double rhoij = 0.5 * (rhoi + rhoj);
        if (mode == 0) {
            double cij = 0.5 * (ci + cj);
            double mu = hij * vr / (rr * rr + hij * hij * eta * eta);
            PI = (-alpha * cij * mu + beta * mu * mu) / rhoij;
        } else {
            double w = vr / (rr + 1e-5);
            double vsig = ci + cj - 3.0 * w;
            PI = -0.5 * alpha * vsig * w / rhoij;
        }
    }
    if (balsara) PI = 0.5 * (fi + fj) * PI;
    return PI;
}

static inline double balsara_f(double divV, double curlV, double c, double h)
{
    return divV / (divV + curlV + 0.0001 * c / h);
}

/* getAcc_sph_shear_mpi (shear.py:243-330, mode 1 + Balsara) and
 * getAcc_sph_mpiXXX (libsx.py:185-262, mode 0, no Balsara). */
void ref_acc_sph(int N, const double *pos, const double *v, const double *rho, const double *P,
                 const double *c, const double *h, const double *m, const double *divV,
                 const double *curlV, double alpha, double beta, double eta, int mode, int balsara,
                 int nbeg, int nend, double *acc)
{
#pragma omp parallel for schedule(dynamic, 16)
    for (int i = nbeg; i < nend; i++) {
        double ax = 0.0, ay = 0.0, az = 0.0;
        double fi = balsara ? balsara_f(divV[i], curlV[i], c[i], h[i]) : 0.0;
        for (int j = 0; j < N; j++) {
            double dx = pos[3 * i] - pos[3 * j], dy = pos[3 * i + 1] - pos[3 * j + 1], dz = pos[3 * i + 2] - pos[3 * j + 2];
            double rr = sqrt(dx * dx + dy * dy + dz * dz);
            double hij = 0.5 * (h[i] + h[j]);
            double nW = gradw_m4(rr, hij);
            double gx = nW * dx, gy = nW * dy, gz = nW * dz;
            double vx = v[3 * i] - v[3 * j], vy = v[3 * i + 1] - v[3 * j + 1], vz = v[3 * i + 2] - v[3 * j + 2];
            double vr = vx * dx + vy * dy + vz * dz;
            double fj = balsara ? balsara_f(divV[j], curlV[j], c[j], h[j]) : 0.0;
            double PI = pi_ij(mode, balsara, vr, rr, hij, c[i], c[j], rho[i], rho[j], fi, fj, alpha, beta, eta);
            double t = m[j] * (P[i] / (rho[i] * rho[i]) + P[j] / (rho[j] * rho[j]) + PI);
            ax -= t * gx; ay -= t * gy; az -= t * gz;
        }
        acc[3 * (i - nbeg)] = ax; acc[3 * (i - nbeg) + 1] = ay; acc[3 * (i - nbeg) + 2] = az;
    }
}

/* get_dU_shear_mpi (shear.py:413-485) / get_dU_mpiXXXX (libsx.py:427-497) */
void ref_dudt(int N, const double *pos, const double *v, const double *rho, const double *P,
              const double *c, const double *h, const double *m, const double *divV,
              const double *curlV, double alpha, double beta, double eta, int mode, int balsara,
              int nbeg, int nend, double *dudt)
{
#pragma omp parallel for schedule(dynamic, 16)
    for (int i = nbeg; i < nend; i++) {
        double du = 0.0;
        double fi = balsara ? balsara_f(divV[i], curlV[i], c[i], h[i]) : 0.0;
        for (int j = 0; j < N; j++) {
            double dx = pos[3 * i] - pos[3 * j], dy = pos[3 * i + 1] - pos[3 * j + 1], dz = pos[3 * i + 2] - pos[3 * j + 2];
            double rr = sqrt(dx * dx + dy * dy + dz * dz);
            double hij = 0.5 * (h[i] + h[j]);
            double nW = gradw_m4(rr, hij);
            double gx = nW * dx, gy = nW * dy, gz = nW * dz;
            double vx = v[3 * i] - v[3 * j], vy = v[3 * i + 1] - v[3 * j + 1], vz = v[3 * i + 2] - v[3 * j + 2];
            double vg = vx * gx + vy * gy + vz * gz;
            double vr = vx * dx + vy * dy + vz * dz;
            double fj = balsara ? balsara_f(divV[j], curlV[j], c[j], h[j]) : 0.0;
            double PI = pi_ij(mode, balsara, vr, rr, hij, c[i], c[j], rho[i], rho[j], fi, fj, alpha, beta, eta);
            du += m[j] * (P[i] / (rho[i] * rho[i]) + PI / 2.0) * vg;
        }
        dudt[i - nbeg] = du;
    }
}

/* spline-softened gravity kernel factor of libsx.py:924-934 */
static inline double fk_spline(double rr, double epsij)
{
    double q = rr / epsij;
    double inv_r3 = 1.0 / (rr * rr * rr);
    if (q <= 1.0) return (1.0 / (epsij * epsij * epsij)) * ((4.0 / 3.0) - (6.0 / 5.0) * q * q + (1.0 / 2.0) * q * q * q);
    if (q <= 2.0) {
        double q3 = q * q * q;
        return inv_r3 * ((-1.0 / 15.0) + (8.0 / 3.0) * q3 - 3.0 * q3 * q + (6.0 / 5.0) * q3 * q * q - (1.0 / 6.0) * q3 * q3);
    }
    return inv_r3;
}

/* getAcc_g_smth_mimj_mpi, libsx.py:910-947: pairwise over i in [nbeg,nend),
 * j > i, scattering to both i and j.  field is N x 3 and is a PARTIAL sum
 * (the reference sums the ranks' fields, sph_mpi4_v4.py:326-337).  The
 * OpenMP version keeps one partial field per thread and sums them, which is
 * the same decomposition. */
void ref_acc_g_smth(int N, const double *pos, const double *mass, double G, const double *eps,
                    int nbeg, int nend, double *field)
{
    memset(field, 0, sizeof(double) * 3 * (size_t)N);
#pragma omp parallel
    {
        double *loc = (double *)calloc((size_t)3 * N, sizeof(double));
#pragma omp for schedule(dynamic, 8)
        for (int i = nbeg; i < nend; i++) {
            for (int j = i + 1; j < N; j++) {
                double dx = pos[3 * j] - pos[3 * i], dy = pos[3 * j + 1] - pos[3 * i + 1], dz = pos[3 * j + 2] - pos[3 * i + 2];
                double rr = sqrt(dx * dx + dy * dy + dz * dz);
                double epsij = 0.5 * (eps[i] + eps[j]);
                double fk = fk_spline(rr, epsij);
                loc[3 * i] += G * fk * dx * mass[j]; loc[3 * j] -= G * fk * dx * mass[i];
                loc[3 * i + 1] += G * fk * dy * mass[j]; loc[3 * j + 1] -= G * fk * dy * mass[i];
                loc[3 * i + 2] += G * fk * dz * mass[j]; loc[3 * j + 2] -= G * fk * dz * mass[i];
            }
        }
#pragma omp critical
        for (size_t k = 0; k < (size_t)3 * N; k++) field[k] += loc[k];
        free(loc);
    }
}

/* h_smooth_fast_mpi, libsx.py:854-902 (Nngb in [45,55], +-0.3 % steps).
 * The reference loop has no exit on non-convergence (it only prints); the
 * restatement stops after max_iter and counts such rows in the return value. */
int ref_h_smooth_fast(int N, const double *pos, const double *h, int nbeg, int nend,
                      int max_iter, double *hres)
{
    int bad = 0;
#pragma omp parallel reduction(+ : bad)
    {
        double *dist = (double *)malloc(sizeof(double) * (size_t)N);
#pragma omp for schedule(dynamic, 16)
        for (int i = nbeg; i < nend; i++) {
            double hi = h[i];
            for (int j = 0; j < N; j++) {
                double dx = pos[3 * j] - pos[3 * i], dy = pos[3 * j + 1] - pos[3 * i + 1], dz = pos[3 * j + 2] - pos[3 * i + 2];
                dist[j] = sqrt(dx * dx + dy * dy + dz * dz);
            }
            int n = 0;
            for (int j = 0; j < N; j++) n += dist[j] < 2.0 * hi;
            int it = 0;
            while (n > 55 || n < 45) {
                if (n > 55) hi -= 0.003 * hi;
                if (n < 45) hi += 0.003 * hi;
                n = 0;
                for (int j = 0; j < N; j++) n += dist[j] < 2.0 * hi;
                if (++it > max_iter) { bad++; break; }
            }
            hres[i - nbeg] = hi;
        }
        free(dist);
    }
    return bad;
}

static double kth_smallest(double *a, int n, int k)
{
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        double piv = a[(lo + hi) / 2];
        int i = lo, j = hi;
        while (i <= j) {
            while (a[i] < piv) i++;
            while (a[j] > piv) j--;
            if (i <= j) { double t = a[i]; a[i] = a[j]; a[j] = t; i++; j--; }
        }
        if (k <= j) hi = j; else if (k >= i) lo = i; else return a[k];
    }
    return a[k];
}

/* smoothing_length_mpi, libsx.py:781-802: half the distance to the 51st
 * nearest particle (sorted index 50, the particle itself at index 0). */
void ref_smoothing_length(int N, const double *pos, int nbeg, int nend, double *hres)
{
#pragma omp parallel
    {
        double *dist = (double *)malloc(sizeof(double) * (size_t)N);
#pragma omp for schedule(dynamic, 16)
        for (int i = nbeg; i < nend; i++) {
            for (int j = 0; j < N; j++) {
                double dx = pos[3 * j] - pos[3 * i], dy = pos[3 * j + 1] - pos[3 * i + 1], dz = pos[3 * j + 2] - pos[3 * i + 2];
                dist[j] = sqrt(dx * dx + dy * dy + dz * dz);
            }
            hres[i - nbeg] = kth_smallest(dist, N, 50) * 0.5;
        }
        free(dist);
    }
}

/* getKE, libsx.py:571-580 */
double ref_ke(int N, const double *v, const double *m)
{
    double ke = 0.0;
    for (int i = 0; i < N; i++) ke += 0.5 * m[i] * (v[3 * i] * v[3 * i] + v[3 * i + 1] * v[3 * i + 1] + v[3 * i + 2] * v[3 * i + 2]);
    return ke;
}

/* getPE, libsx.py:585-620 (spline-softened, epsilon_ij = mean) */
double ref_pe(int N, const double *pos, const double *m, double G, const double *eps)
{
    double pe = 0.0;
#pragma omp parallel for reduction(+ : pe) schedule(dynamic, 16)
    for (int i = 0; i < N; i++) {
        for (int j = i + 1; j < N; j++) {
            double dx = pos[3 * i] - pos[3 * j], dy = pos[3 * i + 1] - pos[3 * j + 1], dz = pos[3 * i + 2] - pos[3 * j + 2];
            double rr = sqrt(dx * dx + dy * dy + dz * dz);
            double fk = 0.0, inv_r = rr != 0.0 ? 1.0 / rr : 0.0;
            double e = 0.5 * (eps[i] + eps[j]);
            double q = rr / e;
            if (q <= 1.0 && q != 0.0)
                fk = m[j] * ((-2.0 / e) * ((1.0 / 3.0) * q * q - (3.0 / 20.0) * q * q * q * q + (1.0 / 20.0) * q * q * q * q * q) + 7.0 / 5.0 / e);
            if (q > 1.0 && q <= 2.0)
                fk = m[j] * ((-1.0 / 15.0) * inv_r - (1.0 / e) * ((4.0 / 3.0) * q * q - q * q * q + (3.0 / 10.0) * q * q * q * q - (1.0 / 30.0) * q * q * q * q * q) + 8.0 / 5.0 / e);
            if (q > 2.0) fk = m[j] * inv_r;
            pe -= G * m[i] * fk;
        }
    }
    return pe;
}

/* ======================================================================== */
/* (B) the project method                                                   */
/* ======================================================================== */

/* --- Morton keys ------------------------------------------------------- */
static inline uint64_t spread3(uint64_t v)
{
    v &= 0x1fffffULL;
    v = (v | v << 32) & 0x1f00000000ffffULL;
    v = (v | v << 16) & 0x1f0000ff0000ffULL;
    v = (v | v << 8) & 0x100f00f00f00f00fULL;
    v = (v | v << 4) & 0x10c30c30c30c30c3ULL;
    v = (v | v << 2) & 0x1249249249249249ULL;
    return v;
}

static inline uint64_t cell_coord(double x, double lo, double ext, int bits)
{
    double t = (x - lo) / ext;
    double s = t * (double)(1ULL << bits);
    uint64_t c = s <= 0.0 ? 0 : (uint64_t)s;
    uint64_t cmax = (1ULL << bits) - 1;
    return c > cmax ? cmax : c;
}

/* Per-cloud axis-aligned box: box[6*k..] = xmin,ymin,zmin,xmax,ymax,zmax.
 * cloud_start has ncloud+1 entries; particles of cloud k are the index
 * range [cloud_start[k], cloud_start[k+1]). */
void orc_cloud_boxes(int ncloud, const int *cloud_start, const double *x, const double *y,
                     const double *z, double *box)
{
    for (int k = 0; k < ncloud; k++) {
        double b[6] = {INFINITY, INFINITY, INFINITY, -INFINITY, -INFINITY, -INFINITY};
        for (int i = cloud_start[k]; i < cloud_start[k + 1]; i++) {
            b[0] = fmin(b[0], x[i]); b[1] = fmin(b[1], y[i]); b[2] = fmin(b[2], z[i]);
            b[3] = fmax(b[3], x[i]); b[4] = fmax(b[4], y[i]); b[5] = fmax(b[5], z[i]);
        }
        memcpy(box + 6 * k, b, sizeof b);
    }
}

/* key = (cloud << 3*bits) | interleave(ix, iy, iz); x takes the highest bit
 * of each triple.  ext = largest side of the cloud's box (cubic cells). */
void orc_morton_keys(int N, const double *x, const double *y, const double *z, const int *cloud,
                     const double *box, int bits, uint64_t *key)
{
    for (int i = 0; i < N; i++) {
        const double *b = box + 6 * cloud[i];
        double ex = b[3] - b[0], ey = b[4] - b[1], ez = b[5] - b[2];
        double ext = fmax(ex, fmax(ey, ez));
        if (!(ext > 0.0)) ext = 1.0;
        uint64_t ix = cell_coord(x[i], b[0], ext, bits);
        uint64_t iy = cell_coord(y[i], b[1], ext, bits);
        uint64_t iz = cell_coord(z[i], b[2], ext, bits);
        key[i] = ((uint64_t)cloud[i] << (3 * bits)) | (spread3(ix) << 2) | (spread3(iy) << 1) | spread3(iz);
    }
}

/* --- exact neighbour predicate ----------------------------------------- */
static inline int is_ngb(double xi, double yi, double zi, double hi, double xj, double yj, double zj, double hj)
{
    double dx = xi - xj, dy = yi - yj, dz = zi - zj;
    double r2 = dx * dx + dy * dy;
    r2 = r2 + dz * dz;
    double s = hi + hj;
    return r2 <= s * s;
}

/* Uniform grid over [lo, lo+n*cs) per axis, particles binned by cell. */
typedef struct { double lo[3]; double cs; int n[3]; int *start; int *idx; } grid_t;

static void grid_build(grid_t *g, int N, const double *x, const double *y, const double *z, double cs)
{
    double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    const double *p[3] = {x, y, z};
    for (int i = 0; i < N; i++)
        for (int d = 0; d < 3; d++) { lo[d] = fmin(lo[d], p[d][i]); hi[d] = fmax(hi[d], p[d][i]); }
    long ncell = 1;
    for (int d = 0; d < 3; d++) {
        int n = (int)((hi[d] - lo[d]) / cs) + 1;
        if (n > 256) n = 256;
        if (n < 1) n = 1;
        g->n[d] = n; g->lo[d] = lo[d]; ncell *= n;
    }
    double ext = 0.0;
    for (int d = 0; d < 3; d++) ext = fmax(ext, (hi[d] - lo[d]) / g->n[d]);
    g->cs = ext > cs ? ext : cs;
    if (!(g->cs > 0.0)) g->cs = 1.0;
    g->start = (int *)calloc((size_t)ncell + 1, sizeof(int));
    g->idx = (int *)malloc(sizeof(int) * (size_t)(N > 0 ? N : 1));
    int *cell = (int *)malloc(sizeof(int) * (size_t)(N > 0 ? N : 1));
    for (int i = 0; i < N; i++) {
        int c[3];
        for (int d = 0; d < 3; d++) {
            int k = (int)((p[d][i] - g->lo[d]) / g->cs);
            c[d] = k < 0 ? 0 : (k >= g->n[d] ? g->n[d] - 1 : k);
        }
        cell[i] = (c[2] * g->n[1] + c[1]) * g->n[0] + c[0];
        g->start[cell[i] + 1]++;
    }
    for (long k = 0; k < ncell; k++) g->start[k + 1] += g->start[k];
    int *fill = (int *)malloc(sizeof(int) * (size_t)ncell);
    memcpy(fill, g->start, sizeof(int) * (size_t)ncell);
    for (int i = 0; i < N; i++) g->idx[fill[cell[i]]++] = i;
    free(fill); free(cell);
}

static void grid_free(grid_t *g) { free(g->start); free(g->idx); }

static int cmp_int(const void *a, const void *b) { int x = *(const int *)a, y = *(const int *)b; return (x > y) - (x < y); }

/* Neighbour lists: j is a neighbour of i iff |r_ij|^2 <= (h_i+h_j)^2 with
 * the rounding of is_ngb().  Rows sorted ascending by index.  Two-pass CSR:
 * with lists == NULL only counts are written (counts[i]); otherwise offsets
 * (N+1, prefix of counts) must be given and lists filled. */
void orc_neighbours(int N, const double *x, const double *y, const double *z, const double *h,
                    const int *cloud, int *counts, const int64_t *offsets, int *lists)
{
    if (N <= 0) return;
    double hmax = 0.0, hsum = 0.0;
    for (int i = 0; i < N; i++) { hmax = fmax(hmax, h[i]); hsum += h[i]; }
    double cs = 2.0 * hsum / N;
    if (!(cs > 0.0)) cs = 1.0;
    grid_t g;
    grid_build(&g, N, x, y, z, cs);
#pragma omp parallel for schedule(dynamic, 64)
    for (int i = 0; i < N; i++) {
        double R = h[i] + hmax;
        int lo[3], hi[3];
        const double pi[3] = {x[i], y[i], z[i]};
        for (int d = 0; d < 3; d++) {
            lo[d] = (int)floor((pi[d] - R - g.lo[d]) / g.cs) - 1;
            hi[d] = (int)floor((pi[d] + R - g.lo[d]) / g.cs) + 1;
            if (lo[d] < 0) lo[d] = 0;
            if (hi[d] > g.n[d] - 1) hi[d] = g.n[d] - 1;
        }
        int n = 0;
        int64_t o = lists ? offsets[i] : 0;
        for (int cz = lo[2]; cz <= hi[2]; cz++)
            for (int cy = lo[1]; cy <= hi[1]; cy++)
                for (int cx = lo[0]; cx <= hi[0]; cx++) {
                    int c = (cz * g.n[1] + cy) * g.n[0] + cx;
                    for (int k = g.start[c]; k < g.start[c + 1]; k++) {
                        int j = g.idx[k];
                        if (cloud && cloud[j] != cloud[i]) continue;
                        if (is_ngb(x[i], y[i], z[i], h[i], x[j], y[j], z[j], h[j])) {
                            if (lists) lists[o + n] = j;
                            n++;
                        }
                    }
                }
        if (lists) qsort(lists + o, (size_t)n, sizeof(int), cmp_int);
        else counts[i] = n;
    }
    grid_free(&g);
}

/* --- Newton smoothing length ------------------------------------------
 * Solve f(h) = (4pi/3)(2h)^3 rho_i(h) - n_ngb m_i = 0 with the gather
 * density rho_i(h) = sum_j m_j W(r_ij, h).  f is non-decreasing in h; the
 * iteration is Newton safeguarded by a bracket (bisection when the Newton
 * step leaves it), converged when |dh| < tol*h (FP64 test).  Replaces the
 * count-based iteration of libsx.py:854-902 / hfvCLibs_v7_hfv_v2.h:367-455. */
static void density_h_and_dh(int N, int i, const double *x, const double *y, const double *z,
                             const double *m, const int *cloud, double h, const grid_t *g,
                             double *rho, double *drho)
{
    double R = 2.0 * h, s = 0.0, ds = 0.0;
    int lo[3], hi[3];
    const double pi[3] = {x[i], y[i], z[i]};
    for (int d = 0; d < 3; d++) {
        lo[d] = (int)floor((pi[d] - R - g->lo[d]) / g->cs) - 1;
        hi[d] = (int)floor((pi[d] + R - g->lo[d]) / g->cs) + 1;
        if (lo[d] < 0) lo[d] = 0;
        if (hi[d] > g->n[d] - 1) hi[d] = g->n[d] - 1;
    }
    double h3 = h * h * h, h4 = h3 * h;
    for (int cz = lo[2]; cz <= hi[2]; cz++)
        for (int cy = lo[1]; cy <= hi[1]; cy++)
            for (int cx = lo[0]; cx <= hi[0]; cx++) {
                int c = (cz * g->n[1] + cy) * g->n[0] + cx;
                for (int k = g->start[c]; k < g->start[c + 1]; k++) {
                    int j = g->idx[k];
                    if (cloud && cloud[j] != cloud[i]) continue;
                    double dx = x[i] - x[j], dy = y[i] - y[j], dz = z[i] - z[j];
                    double r = sqrt(dx * dx + dy * dy + dz * dz);
                    double q = r / h;
                    if (q >= 2.0) continue;
                    double w, dw;
                    if (q <= 1.0) { w = 1.0 - 1.5 * q * q + 0.75 * q * q * q; dw = 3.0 - 7.5 * q * q + 4.5 * q * q * q; }
                    else { double t = 2.0 - q; w = 0.25 * t * t * t; dw = 1.5 * t * t * (1.0 - q); }
                    s += m[j] * w;
                    ds += m[j] * dw;
                }
            }
    *rho = SIG / h3 * s;
    *drho = -SIG / h4 * ds;
}

int orc_newton_h(int N, const double *x, const double *y, const double *z, const double *m,
                 const int *cloud, const double *h_in, double n_ngb, double tol, int max_iter,
                 double *h_out, int *iters)
{
    if (N <= 0) return 0;
    double hsum = 0.0;
    for (int i = 0; i < N; i++) hsum += h_in[i];
    grid_t g;
    grid_build(&g, N, x, y, z, 2.0 * hsum / N);
    int bad = 0;
#pragma omp parallel for schedule(dynamic, 32) reduction(+ : bad)
    for (int i = 0; i < N; i++) {
        double h = h_in[i], lo = 0.0, hi = INFINITY;
        int it = 0, ok = 0;
        const double c = 4.0 * ORC_PI / 3.0 * 8.0;
        for (it = 1; it <= max_iter; it++) {
            double rho, drho;
            density_h_and_dh(N, i, x, y, z, m, cloud, h, &g, &rho, &drho);
            double f = c * h * h * h * rho - n_ngb * m[i];
            double fp = c * h * h * (3.0 * rho + h * drho);
            if (f < 0.0) lo = h; else hi = h;
            double hn;
            if (fp > 0.0) hn = h - f / fp; else hn = -1.0;
            /* a Newton step below the tolerance is accepted before any bracket
             * test: in FP64 it can round to exactly h (= a bracket end) */
            if (fp > 0.0 && fabs(f / fp) < tol * h) { h = hn; ok = 1; break; }
            /* at most a factor 1.25 per iteration */
            if (hn > 1.25 * h) hn = 1.25 * h;
            if (hn > 0.0 && hn < h / 1.25) hn = h / 1.25;
            if (!(hn > lo && hn < hi)) {
                if (hi == INFINITY) hn = 1.25 * h;
                else if (lo == 0.0) hn = h / 1.25;
                else hn = 0.5 * (lo + hi);
            }
            double dh = hn - h;
            h = hn;
            if (fabs(dh) < tol * fabs(h - dh)) { ok = 1; break; }
        }
        h_out[i] = h;
        if (iters) iters[i] = it;
        if (!ok) bad++;
    }
    grid_free(&g);
    return bad;
}

/* --- list-based SPH sums (same formulas as section A) ------------------ */
void orc_density_list(int N, const double *x, const double *y, const double *z, const double *m,
                      const double *h, const int64_t *off, const int *lst, double *rho)
{
#pragma omp parallel for schedule(static)
    for (int i = 0; i < N; i++) {
        double s = 0.0;
        for (int64_t k = off[i]; k < off[i + 1]; k++) {
            int j = lst[k];
            double dx = x[i] - x[j], dy = y[i] - y[j], dz = z[i] - z[j];
            double rr = sqrt(dx * dx + dy * dy + dz * dz);
            s += m[j] * w_m4(rr, 0.5 * (h[i] + h[j]));
        }
        rho[i] = s;
    }
}

void orc_divcurl_list(int N, const double *x, const double *y, const double *z, const double *vx,
                      const double *vy, const double *vz, const double *rho, const double *m,
                      const double *h, const int64_t *off, const int *lst, double *divV, double *curlV)
{
#pragma omp parallel for schedule(static)
    for (int i = 0; i < N; i++) {
        double s = 0.0, cx = 0.0, cy = 0.0, cz = 0.0;
        for (int64_t k = off[i]; k < off[i + 1]; k++) {
            int j = lst[k];
            double dx = x[i] - x[j], dy = y[i] - y[j], dz = z[i] - z[j];
            double rr = sqrt(dx * dx + dy * dy + dz * dz);
            double nW = gradw_m4(rr, 0.5 * (h[i] + h[j]));
            double gx = nW * dx, gy = nW * dy, gz = nW * dz;
            double ux = vx[i] - vx[j], uy = vy[i] - vy[j], uz = vz[i] - vz[j];
            double f = m[j] / rho[i];
            s += f * (-ux * gx - uy * gy - uz * gz);
            cx += f * (uy * gz - uz * gy);
            cy += f * (uz * gx - ux * gz);
            cz += f * (ux * gy - uy * gx);
        }
        divV[i] = fabs(s);
        curlV[i] = sqrt(cx * cx + cy * cy + cz * cz);
    }
}

/* acceleration (want_acc) and/or du/dt (want_du) plus the signal velocity
 * max_j (c_i + c_j - 3 w_ij) used by the Courant limit
 * (hfvCLibs_v7_hfv_v2.h:1021-1050, restricted to neighbours). */
void orc_force_list(int N, const double *x, const double *y, const double *z, const double *vx,
                    const double *vy, const double *vz, const double *rho, const double *P,
                    const double *c, const double *h, const double *m, const double *divV,
                    const double *curlV, double alpha, double beta, double eta, int mode, int balsara,
                    const int64_t *off, const int *lst, double *ax, double *ay, double *az,
                    double *dudt, double *vsig)
{
#pragma omp parallel for schedule(static)
    for (int i = 0; i < N; i++) {
        double sx = 0.0, sy = 0.0, sz = 0.0, du = 0.0, vs = 0.0;
        double fi = balsara ? balsara_f(divV[i], curlV[i], c[i], h[i]) : 0.0;
        for (int64_t k = off[i]; k < off[i + 1]; k++) {
            int j = lst[k];
            double dx = x[i] - x[j], dy = y[i] - y[j], dz = z[i] - z[j];
            double rr = sqrt(dx * dx + dy * dy + dz * dz);
            double hij = 0.5 * (h[i] + h[j]);
            double nW = gradw_m4(rr, hij);
            double gx = nW * dx, gy = nW * dy, gz = nW * dz;
            double ux = vx[i] - vx[j], uy = vy[i] - vy[j], uz = vz[i] - vz[j];
            double vr = ux * dx + uy * dy + uz * dz;
            double fj = balsara ? balsara_f(divV[j], curlV[j], c[j], h[j]) : 0.0;
            double PI = pi_ij(mode, balsara, vr, rr, hij, c[i], c[j], rho[i], rho[j], fi, fj, alpha, beta, eta);
            double t = m[j] * (P[i] / (rho[i] * rho[i]) + P[j] / (rho[j] * rho[j]) + PI);
            sx -= t * gx; sy -= t * gy; sz -= t * gz;
            du += m[j] * (P[i] / (rho[i] * rho[i]) + PI / 2.0) * (ux * gx + uy * gy + uz * gz);
            double w = vr / (rr + 1e-5);
            double v = c[i] + c[j] - 3.0 * w;
            if (v > vs) vs = v;
        }
        if (ax) { ax[i] = sx; ay[i] = sy; az[i] = sz; }
        if (dudt) dudt[i] = du;
        if (vsig) vsig[i] = vs;
    }
}

/* Individual time steps: dt_array_indiv_dt (Particles_in_BH_Tree_II/
 * Evrard_test/hfvCLibs_v7_hfv_v2.h:999-1078) restated in FP64 with its
 * signal-velocity maximum (from 0, self included) over the neighbour list
 * instead of all N particles; the six estimates
 *   C h / vsig_max, C h / (h |div| + max(c, |v|)(1 + 0.6 alpha)),
 *   0.4 sqrt(eps / |a|), 0.4 eps / |v|, sqrt(h / |a_grav|), sqrt(h / |a|)
 * and dh/dt = h div / 3 (:1071-1076) with the signed divergence
 * div = -(1/rho_i) sum_j m_j v_ij . gradW_ij over the same list. */
void orc_dt_individual(int N, const double *x, const double *y, const double *z, const double *vx,
                       const double *vy, const double *vz, const double *m, const double *h,
                       const double *rho, const double *c, const double *asph,
                       const double *agrav, double eps, double C, double alpha,
                       const int64_t *off, const int *lst, double *dt, double *dhdt)
{
#pragma omp parallel for schedule(static)
    for (int i = 0; i < N; i++) {
        double vs = 0.0, s = 0.0;
        for (int64_t k = off[i]; k < off[i + 1]; k++) {
            int j = lst[k];
            double dx = x[i] - x[j], dy = y[i] - y[j], dz = z[i] - z[j];
            double rr = sqrt(dx * dx + dy * dy + dz * dz);
            double ux = vx[i] - vx[j], uy = vy[i] - vy[j], uz = vz[i] - vz[j];
            double vr = ux * dx + uy * dy + uz * dz;
            double w = vr / (rr + 1e-5);
            double v = c[i] + c[j] - 3.0 * w;
            if (v > vs) vs = v;
            s -= m[j] * gradw_m4(rr, 0.5 * (h[i] + h[j])) * vr;
        }
        double div = s / rho[i];
        double gx = agrav[i], gy = agrav[N + i], gz = agrav[2 * (size_t)N + i];
        double tx = asph[i] + gx, ty = asph[N + i] + gy, tz = asph[2 * (size_t)N + i] + gz;
        double ag = sqrt(gx * gx + gy * gy + gz * gz), at = sqrt(tx * tx + ty * ty + tz * tz);
        double va = sqrt(vx[i] * vx[i] + vy[i] * vy[i] + vz[i] * vz[i]);
        double e[6];
        e[0] = C * h[i] / vs;
        e[1] = C * h[i] / (h[i] * fabs(div) + fmax(c[i], va) * (1.0 + 0.6 * alpha));
        e[2] = 0.4 * sqrt(eps / at);
        e[3] = 0.4 * eps / va;
        e[4] = sqrt(h[i] / ag);
        e[5] = sqrt(h[i] / at);
        double d = e[0];
        for (int q = 1; q < 6; q++)
            if (e[q] <= d) d = e[q];
        dt[i] = d;
        dhdt[i] = h[i] * div / 3.0;
    }
}

/* Outflow pairs of outflow_injector2 (hfvCLibs_v7_hfv_v2.h:1094-1210) with
 * the project's counter-based uniforms in place of cuRAND: pair j draws
 * u_k = ((splitmix64(seed + G (3j + k + 1)) >> 11) + 1) 2^-53, k = 0, 1, 2
 * (G the 64-bit golden-ratio increment, SplitMix64's output function of
 * Steele, Lea and Flood 2014), then r = u_0 r_max, azimuth 2 pi u_1, polar
 * angle acos(2 u_2 - 1), velocity v_in along +r; the pair is (+r, +v),
 * (-r, -v).  Outputs 2 npairs rows. */
static uint64_t splitmix64(uint64_t z)
{
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}

void orc_outflow_pairs(uint64_t seed, int npairs, double r_max, double v_in, double *x, double *y,
                       double *z, double *vx, double *vy, double *vz)
{
    for (int j = 0; j < npairs; j++) {
        double u[3];
        for (int k = 0; k < 3; k++) {
            uint64_t w = splitmix64(seed + 0x9e3779b97f4a7c15ULL * (uint64_t)(3 * (int64_t)j + k + 1));
            u[k] = (double)((w >> 11) + 1) * 0x1.0p-53;
        }
        double rt = u[0] * r_max, th = u[1] * 2.0 * ORC_PI, ph = acos(2.0 * u[2] - 1.0);
        double sp = sin(ph);
        double xt = rt * sp * cos(th), yt = rt * sp * sin(th), zt = rt * cos(ph);
        double rr = sqrt(xt * xt + yt * yt + zt * zt);
        double s = rr > 0.0 ? v_in / rr : 0.0;
        for (int side = 0; side < 2; side++) {
            double sg = side ? -1.0 : 1.0;
            int i = 2 * j + side;
            x[i] = sg * xt; y[i] = sg * yt; z[i] = sg * zt;
            vx[i] = sg * xt * s; vy[i] = sg * yt * s; vz[i] = sg * zt * s;
        }
    }
}

/* galaxy_isothermal_potential (hfvCLibs_v7_hfv_v2.h:1215-1235): M(r) =
 * 2 sigma^2 r / G, a = -G M(r) x / r^3 = -2 sigma^2 x / r^2 (0 at r = 0) */
void orc_isothermal(int N, const double *x, const double *y, const double *z, double sigma,
                    double *ax, double *ay, double *az)
{
    for (int i = 0; i < N; i++) {
        double r2 = x[i] * x[i] + y[i] * y[i] + z[i] * z[i];
        double f = r2 > 0.0 ? 2.0 * sigma * sigma / r2 : 0.0;
        ax[i] = -f * x[i]; ay[i] = -f * y[i]; az[i] = -f * z[i];
    }
}

/* Table heating/cooling of hcoolingx (hfvCLibs_v7_hfv_v2.h:1240-1418) in FP64
 * on the FP32 grid: nearest radius (kpc) and n_H entries (the first grid value
 * at or above, or the one below when nearer; the last above the grid), the
 * metallicity row z_row, the first u row at or above u of the column
 * u_evol[kpc][.][nH][z][0] (the last above it), the first time at or above
 * dt; u_new linear in u between that row and the one below (the row itself at
 * the bottom), and the N_M ion fractions of the cell.  dims = N_kpc, N_nH,
 * N_Z, N_T, N_M, N_Time; grid = kpc, nH, Z, T, time concatenated. */
static int tab_nearest(const float *g, int n, double v)
{
    int k = -1;
    for (int j = 0; j < n; j++)
        if (v <= (double)g[j]) { k = j; break; }
    if (k > 0 && fabs((double)g[k - 1] - v) < fabs((double)g[k] - v)) k -= 1;
    return k < 0 ? n - 1 : k;
}

void orc_cool_table(const int *dims, const float *grid, const float *uev, const float *frac,
                    int z_row, int N, const double *x, const double *y, const double *z,
                    const double *rho, const double *u, const double *dt, double unit_rho,
                    double unit_u, double unit_t, double unit_len, double kpc_cm, double XH,
                    double mH, double *u_new, float *ion)
{
    const int nk = dims[0], nh = dims[1], nz = dims[2], nt = dims[3], nm = dims[4], ntime = dims[5];
    const float *gk = grid, *gh = grid + nk, *gtime = grid + nk + nh + nz + nt;
    const size_t s_kpc = (size_t)nt * nh * nz * ntime, s_T = (size_t)nh * nz * ntime,
                 s_nH = (size_t)nz * ntime;
    for (int i = 0; i < N; i++) {
        double r = sqrt(x[i] * x[i] + y[i] * y[i] + z[i] * z[i]);
        int ik = tab_nearest(gk, nk, r * unit_len / kpc_cm);
        int ih = tab_nearest(gh, nh, rho[i] * unit_rho * XH / mH);
        size_t base = ik * s_kpc + ih * s_nH + (size_t)z_row * ntime;
        double ui = u[i] * unit_u;
        int iu = -1;
        for (int j = 0; j < nt; j++)
            if (ui <= (double)uev[base + j * s_T]) { iu = j; break; }
        if (iu < 0) iu = nt - 1;
        double dts = dt[i] * unit_t;
        int it = -1;
        for (int j = 0; j < ntime; j++)
            if (dts <= (double)gtime[j]) { it = j; break; }
        if (it < 0) it = ntime - 1;
        double un;
        if (iu > 0) {
            double U1 = uev[base + (iu - 1) * s_T], U2 = uev[base + iu * s_T];
            double e1 = uev[base + (iu - 1) * s_T + it], e2 = uev[base + iu * s_T + it];
            double fhi = (ui - U1) / (U2 - U1), flo = 1.0 - fhi;
            un = flo * e1 + fhi * e2;
        } else {
            un = uev[base + it];
        }
        u_new[i] = un / unit_u;
        size_t mb = ik * s_kpc * nm + iu * s_T * nm + ih * s_nH * nm + (size_t)z_row * nm * ntime + it;
        for (int k = 0; k < nm; k++) ion[(size_t)i * nm + k] = frac[mb + (size_t)k * ntime];
    }
}

/* --- Plummer direct summation (FP64) ----------------------------------- */
void orc_grav_direct(int N, const double *x, const double *y, const double *z, const double *m,
                     const int *cloud, double G, double eps, int ntarget, const int *targets,
                     double *ax, double *ay, double *az, double *pot)
{
    double e2 = eps * eps;
#pragma omp parallel for schedule(dynamic, 4)
    for (int t = 0; t < ntarget; t++) {
        int i = targets[t];
        double sx = 0.0, sy = 0.0, sz = 0.0, sp = 0.0;
        for (int j = 0; j < N; j++) {
            if (j == i) continue;
            if (cloud && cloud[j] != cloud[i]) continue;
            double dx = x[i] - x[j], dy = y[i] - y[j], dz = z[i] - z[j];
            double r2 = dx * dx + dy * dy + dz * dz + e2;
            double rinv = 1.0 / sqrt(r2);
            double g = m[j] * rinv * rinv * rinv;
            sx -= g * dx; sy -= g * dy; sz -= g * dz;
            sp -= m[j] * rinv;
        }
        ax[t] = G * sx; ay[t] = G * sy; az[t] = G * sz;
        if (pot) pot[t] = G * sp;
    }
}

/* --- Karras (2012) binary radix tree over sorted keys ------------------
 * Internal nodes 0..N-2, leaf of particle p at node N-1+p.  child[2*n],
 * child[2*n+1] and the particle range [first[n], last[n]] per node. */
static inline int delta_pref(const uint64_t *k, int N, int i, int j)
{
    if (j < 0 || j > N - 1) return -1;
    uint64_t a = k[i], b = k[j];
    if (a == b) return 64 + __builtin_clz((uint32_t)i ^ (uint32_t)j);
    return __builtin_clzll(a ^ b);
}

void orc_build_radix_tree(int N, const uint64_t *key, int *child, int *parent, int *first, int *last)
{
    int nn = 2 * N - 1;
    for (int n = 0; n < nn; n++) parent[n] = -1;
    for (int p = 0; p < N; p++) { first[N - 1 + p] = p; last[N - 1 + p] = p; child[2 * (N - 1 + p)] = -1; child[2 * (N - 1 + p) + 1] = -1; }
    for (int i = 0; i < N - 1; i++) {
        int d = (delta_pref(key, N, i, i + 1) - delta_pref(key, N, i, i - 1)) > 0 ? 1 : -1;
        int dmin = delta_pref(key, N, i, i - d);
        int lmax = 2;
        while (delta_pref(key, N, i, i + lmax * d) > dmin) lmax *= 2;
        int l = 0;
        for (int t = lmax / 2; t >= 1; t /= 2)
            if (delta_pref(key, N, i, i + (l + t) * d) > dmin) l += t;
        int j = i + l * d;
        int dnode = delta_pref(key, N, i, j);
        int s = 0;
        for (int t = (l + 1) / 2;; t = (t + 1) / 2) {
            if (delta_pref(key, N, i, i + (s + t) * d) > dnode) s += t;
            if (t == 1) break;
        }
        int gam = i + s * d + (d < 0 ? -1 : 0);
        int lo = i < j ? i : j, hi = i < j ? j : i;
        int L = (lo == gam) ? N - 1 + gam : gam;
        int R = (hi == gam + 1) ? N - 1 + gam + 1 : gam + 1;
        child[2 * i] = L; child[2 * i + 1] = R;
        parent[L] = i; parent[R] = i;
        first[i] = lo; last[i] = hi;
    }
}

/* Node moments in FP64, children combined in the fixed order (left, right).
 * node_f64 layout per node (16 doubles):
 *  0..2 com, 3 mass, 4..9 Qxx Qyy Qzz Qxy Qxz Qyz (second moments about the
 *  com), 10..12 box min, 13..15 box max.  hmax[n] = max smoothing length. */
#define NREC 16
static void combine(double *o, const double *a, const double *b)
{
    double M = a[3] + b[3];
    double c[3];
    for (int d = 0; d < 3; d++) c[d] = (a[3] * a[d] + b[3] * b[d]) / M;
    double da[3] = {a[0] - c[0], a[1] - c[1], a[2] - c[2]};
    double db[3] = {b[0] - c[0], b[1] - c[1], b[2] - c[2]};
    const int ia[6] = {0, 1, 2, 0, 0, 1}, ib[6] = {0, 1, 2, 1, 2, 2};
    for (int q = 0; q < 6; q++) {
        double ta = a[4 + q] + a[3] * da[ia[q]] * da[ib[q]];
        double tb = b[4 + q] + b[3] * db[ia[q]] * db[ib[q]];
        o[4 + q] = ta + tb;
    }
    o[0] = c[0]; o[1] = c[1]; o[2] = c[2]; o[3] = M;
    for (int d = 0; d < 3; d++) { o[10 + d] = fmin(a[10 + d], b[10 + d]); o[13 + d] = fmax(a[13 + d], b[13 + d]); }
}

/* Moments of a node of at most GROUP_DIRECT particles of one cloud (a node
 * inside a walk group) summed directly over its particle range f..l in
 * index order: mass, com = sum(m x) / M, second moments sum((m d_a) d_b)
 * about the com, box.  Larger nodes combine their children. */
#define GROUP_DIRECT 32
static void direct_moments(double *o, int f, int l, const double *x, const double *y,
                           const double *z, const double *m)
{
    double M = 0.0, sx = 0.0, sy = 0.0, sz = 0.0;
    double lo[3] = {x[f], y[f], z[f]}, hi[3] = {x[f], y[f], z[f]};
    for (int p = f; p <= l; p++) {
        M = M + m[p];
        sx = sx + m[p] * x[p]; sy = sy + m[p] * y[p]; sz = sz + m[p] * z[p];
        lo[0] = fmin(lo[0], x[p]); lo[1] = fmin(lo[1], y[p]); lo[2] = fmin(lo[2], z[p]);
        hi[0] = fmax(hi[0], x[p]); hi[1] = fmax(hi[1], y[p]); hi[2] = fmax(hi[2], z[p]);
    }
    const double cx = sx / M, cy = sy / M, cz = sz / M;
    double qxx = 0.0, qyy = 0.0, qzz = 0.0, qxy = 0.0, qxz = 0.0, qyz = 0.0;
    for (int p = f; p <= l; p++) {
        const double dx = x[p] - cx, dy = y[p] - cy, dz = z[p] - cz;
        const double tx = m[p] * dx, ty = m[p] * dy, tz = m[p] * dz;
        qxx = qxx + tx * dx; qxy = qxy + tx * dy; qxz = qxz + tx * dz;
        qyy = qyy + ty * dy; qyz = qyz + ty * dz; qzz = qzz + tz * dz;
    }
    o[0] = cx; o[1] = cy; o[2] = cz; o[3] = M;
    o[4] = qxx; o[5] = qyy; o[6] = qzz; o[7] = qxy; o[8] = qxz; o[9] = qyz;
    for (int d = 0; d < 3; d++) { o[10 + d] = lo[d]; o[13 + d] = hi[d]; }
}

void orc_tree_moments(int N, const int *child, const int *first, const int *last, const int *cloud,
                      const double *x, const double *y, const double *z,
                      const double *m, const double *h, double *node, double *hmax)
{
    int nn = 2 * N - 1;
    for (int p = 0; p < N; p++) {
        double *o = node + (size_t)NREC * (N - 1 + p);
        memset(o, 0, sizeof(double) * NREC);
        o[0] = x[p]; o[1] = y[p]; o[2] = z[p]; o[3] = m[p];
        o[10] = x[p]; o[11] = y[p]; o[12] = z[p]; o[13] = x[p]; o[14] = y[p]; o[15] = z[p];
        hmax[N - 1 + p] = h[p];
    }
    /* post-order by explicit stack */
    if (N < 2) return;
    int *stack = (int *)malloc(sizeof(int) * (size_t)nn * 2);
    char *done = (char *)calloc((size_t)nn, 1);
    int sp = 0;
    stack[sp++] = 0;
    while (sp) {
        int n = stack[sp - 1];
        int L = child[2 * n], R = child[2 * n + 1];
        int lpend = (L < N - 1) && !done[L], rpend = (R < N - 1) && !done[R];
        if (lpend || rpend) {
            if (rpend) stack[sp++] = R;
            if (lpend) stack[sp++] = L;
            continue;
        }
        if (last[n] - first[n] + 1 <= GROUP_DIRECT && (!cloud || cloud[first[n]] == cloud[last[n]]))
            direct_moments(node + (size_t)NREC * n, first[n], last[n], x, y, z, m);
        else
            combine(node + (size_t)NREC * n, node + (size_t)NREC * L, node + (size_t)NREC * R);
        hmax[n] = fmax(hmax[L], hmax[R]);
        done[n] = 1;
        sp--;
    }
    free(stack); free(done);
    (void)nn;
}

/* Opening radius of a node: r_open = l/theta + delta with l the largest side
 * of the particle box and delta the distance of the com from the box centre
 * (the Bonsai form of the Barnes-Hut criterion).  Returns r_open^2. */
static inline double open_r2(const double *o, double theta)
{
    double l = fmax(o[13] - o[10], fmax(o[14] - o[11], o[15] - o[12]));
    double cx = (o[10] + o[13]) * 0.5, cy = (o[11] + o[14]) * 0.5, cz = (o[12] + o[15]) * 0.5;
    double ex = o[0] - cx, ey = o[1] - cy, ez = o[2] - cz;
    double d2 = ex * ex + ey * ey;
    d2 = d2 + ez * ez;
    double r = l / theta + sqrt(d2);
    return r * r;
}

void orc_open_r2(int nn, const double *node, double theta, double *r2)
{
    for (int n = 0; n < nn; n++) r2[n] = open_r2(node + (size_t)NREC * n, theta);
}

/* squared distance from point c to the box [bmin, bmax] (0 inside) */
static inline double box_dist2(const double *bmin, const double *bmax, const double *c)
{
    double t[3];
    for (int d = 0; d < 3; d++) {
        double a = bmin[d] - c[d], b = c[d] - bmax[d];
        double v = a > b ? a : b;
        t[d] = v > 0.0 ? v : 0.0;
    }
    double s = t[0] * t[0] + t[1] * t[1];
    return s + t[2] * t[2];
}

/* Group Barnes-Hut walk.  Groups are index ranges [gstart[g], gstart[g]+gcount[g])
 * of one cloud; groot[g] is the tree node of that cloud.  A node is accepted
 * (multipole) when the squared distance from its com to the group's box is
 * >= r_open^2, otherwise it is opened; nodes with at most leaf_size particles
 * that are opened are summed particle by particle (Plummer).  acc/pot are
 * FP64; ncell/npart count the interactions per particle. */
void orc_walk(int N, const double *x, const double *y, const double *z, const double *m,
              const int *child, const int *first, const int *last, const double *node,
              const double *ropen2, int ngroup, const int *gstart, const int *gcount,
              const int *groot, int leaf_size, double G, double eps, double *ax, double *ay,
              double *az, double *pot, int64_t *ncell, int64_t *npart)
{
    double e2 = eps * eps;
#pragma omp parallel
    {
        int *stack = (int *)malloc(sizeof(int) * (size_t)(4 * N + 64));
#pragma omp for schedule(dynamic, 4)
        for (int g = 0; g < ngroup; g++) {
            int s0 = gstart[g], nc = gcount[g];
            double bmin[3] = {INFINITY, INFINITY, INFINITY}, bmax[3] = {-INFINITY, -INFINITY, -INFINITY};
            for (int i = s0; i < s0 + nc; i++) {
                bmin[0] = fmin(bmin[0], x[i]); bmin[1] = fmin(bmin[1], y[i]); bmin[2] = fmin(bmin[2], z[i]);
                bmax[0] = fmax(bmax[0], x[i]); bmax[1] = fmax(bmax[1], y[i]); bmax[2] = fmax(bmax[2], z[i]);
            }
            for (int i = s0; i < s0 + nc; i++) { ax[i] = ay[i] = az[i] = 0.0; if (pot) pot[i] = 0.0; }
            int64_t nC = 0, nP = 0;
            int sp = 0;
            stack[sp++] = groot[g];
            while (sp) {
                int n = stack[--sp];
                const double *o = node + (size_t)NREC * n;
                int cnt = last[n] - first[n] + 1;
                double d2 = box_dist2(bmin, bmax, o);
                if (d2 >= ropen2[n] && cnt > 1) {
                    nC++;
                    for (int i = s0; i < s0 + nc; i++) {
                        double dx = x[i] - o[0], dy = y[i] - o[1], dz = z[i] - o[2];
                        double r2 = dx * dx + dy * dy + dz * dz + e2;
                        double rinv = 1.0 / sqrt(r2), ri2 = rinv * rinv;
                        double g3 = rinv * ri2, g5 = g3 * ri2, g7 = g5 * ri2;
                        double qx = o[4] * dx + o[7] * dy + o[8] * dz;
                        double qy = o[7] * dx + o[5] * dy + o[9] * dz;
                        double qz = o[8] * dx + o[9] * dy + o[6] * dz;
                        double dqd = dx * qx + dy * qy + dz * qz;
                        double tr = o[4] + o[5] + o[6];
                        double s = -o[3] * g3 + 1.5 * tr * g5 - 7.5 * dqd * g7;
                        ax[i] += G * (s * dx + 3.0 * g5 * qx);
                        ay[i] += G * (s * dy + 3.0 * g5 * qy);
                        az[i] += G * (s * dz + 3.0 * g5 * qz);
                        if (pot) pot[i] -= G * (o[3] * rinv + 0.5 * (3.0 * dqd * g5 - tr * g3));
                    }
                } else if (cnt <= leaf_size) {
                    nP += cnt;
                    for (int i = s0; i < s0 + nc; i++) {
                        for (int j = first[n]; j <= last[n]; j++) {
                            double dx = x[i] - x[j], dy = y[i] - y[j], dz = z[i] - z[j];
                            double r2 = dx * dx + dy * dy + dz * dz + e2;
                            double rinv = 1.0 / sqrt(r2);
                            double gg = m[j] * rinv * rinv * rinv;
                            ax[i] -= G * gg * dx; ay[i] -= G * gg * dy; az[i] -= G * gg * dz;
                            if (pot && j != i) pot[i] -= G * m[j] * rinv;
                        }
                    }
                } else {
                    stack[sp++] = child[2 * n + 1];
                    stack[sp++] = child[2 * n];
                }
            }
            for (int i = s0; i < s0 + nc; i++) { if (ncell) ncell[i] = nC; if (npart) npart[i] = nP; }
        }
        free(stack);
    }
}

/* --- cooling ------------------------------------------------------------
 * Synthetic cooling function: Lambda(T) given at nb+1 log-spaced edges
 * between T0 and T1 and interpolated as a power law inside each bin; below
 * T0 / above T1 the end slopes continue.  Net rate per nH^2 is
 * Gamma/nH - Lambda(T) with a constant heating Gamma (erg/s per H).
 * T = (gamma-1) mu m_H u / k_B (fixed mu). */
typedef struct {
    const double *logL; int nb; double logT0, logT1;
    double mu, gamma, XH, gamma_heat;
} cool_t;

#define KB_CGS 1.380649e-16
#define MH_CGS 1.6726e-24

static double lambda_T(const cool_t *c, double T, double *slope)
{
    double lt = log10(T);
    double dl = (c->logT1 - c->logT0) / c->nb;
    double f = (lt - c->logT0) / dl;
    int k = (int)floor(f);
    if (k < 0) k = 0;
    if (k > c->nb - 1) k = c->nb - 1;
    double s = (c->logL[k + 1] - c->logL[k]) / dl;
    double ll = c->logL[k] + s * (lt - (c->logT0 + k * dl));
    if (slope) *slope = s;
    return pow(10.0, ll);
}

static double net_rate(const cool_t *c, double u, double nH)
{
    double T = (c->gamma - 1.0) * c->mu * MH_CGS / KB_CGS * u;
    return c->gamma_heat / nH - lambda_T(c, T, NULL);
}

/* Implicit solve of u - u_old - ratefact * net(u) * dt = 0 with the
 * bracketing (factor 1.1) and bisection of myPhotoLibsGPU.h:615-686.
 * Returns the number of bisection iterations (or -1 when not converged). */
int orc_do_cooling(const double *logL, int nb, double logT0, double logT1, double mu, double gamma,
                   double XH, double gamma_heat, double rho, double u_old, double dt, double tol,
                   int max_iter, double *u_new)
{
    cool_t c = {logL, nb, logT0, logT1, mu, gamma, XH, gamma_heat};
    double nH = XH * rho / MH_CGS;
    double ratefact = nH * nH / rho;
    double u = u_old, up = u, lo = u;
    double r0 = u - u_old - ratefact * net_rate(&c, u, nH) * dt;
    int nb_it = 0;
    if (r0 > 0.0) {
        while (up - u_old - ratefact * net_rate(&c, up, nH) * dt > 0.0 && nb_it++ < 2000) up /= 1.1;
        lo = up; up = lo * 1.1;
    } else if (r0 < 0.0) {
        while (up - u_old - ratefact * net_rate(&c, up, nH) * dt < 0.0 && nb_it++ < 2000) up *= 1.1;
        lo = up / 1.1;
    } else { *u_new = u; return 0; }
    double du = u;
    int it = 1;
    while (fabs(du / u) > tol && it < max_iter) {
        u = 0.5 * (lo + up);
        double r = u - u_old - ratefact * net_rate(&c, u, nH) * dt;
        if (r > 0.0) up = u; else lo = u;
        du = fabs(up - lo);
        it++;
    }
    *u_new = u;
    return fabs(du / u) > tol ? -1 : it;
}

void orc_do_cooling_batch(const double *logL, int nb, double logT0, double logT1, double mu,
                          double gamma, double XH, double gamma_heat, int n, const double *rho,
                          const double *u_old, const double *dt, double tol, int max_iter,
                          double *u_new, int *iters)
{
#pragma omp parallel for schedule(dynamic, 256)
    for (int i = 0; i < n; i++) {
        int it = orc_do_cooling(logL, nb, logT0, logT1, mu, gamma, XH, gamma_heat, rho[i], u_old[i],
                                dt[i], tol, max_iter, u_new + i);
        if (iters) iters[i] = it;
    }
}

/* FP32 restatement of the bracket + bisection of myPhotoLibsGPU.h:615-686
 * over an arbitrary rate callback, used to pin the structure bit-exactly
 * against the reference's compiled DoCooling (oracle/_ref). */
typedef float (*rate_fn_f32)(float u, float nH, float XH);

float orc_do_cooling_f32(rate_fn_f32 rate, float rho, float u_old, float dt, float XH)
{
    int niter = 1;
    float mH = (float)1.6726e-24;
    float nH = XH * rho / mH;
    float ratefact = nH * nH / rho;
    float u = u_old, up = u, lo = 0.0f;
    float net = rate(u, nH, XH);
    if (u - u_old - ratefact * net * dt > 0.0f) {
        while (up - u_old - ratefact * rate(up, nH, XH) * dt > 0.0f) up /= 1.1f;
        lo = up;
        up = lo * 1.1f;
    }
    if (u - u_old - ratefact * net * dt < 0.0f) {
        while (up - u_old - ratefact * rate(up, nH, XH) * dt < 0.0f) up *= 1.1f;
        lo = up / 1.1f;
    }
    float du = u;
    while ((fabsf(du / u) > 0.0001f) && (niter < 100)) {
        u = 0.5f * (lo + up);
        net = rate(u, nH, XH);
        if (u - u_old - ratefact * net * dt > 0.0f) up = u; else lo = u;
        du = fabsf(up - lo);
        niter++;
    }
    return u;
}

int orc_num_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
