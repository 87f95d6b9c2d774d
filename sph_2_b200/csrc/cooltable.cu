// cooltable.cu -- table-based heating and cooling with ion fractions.
//
// Replaces hcoolingx (Particles_in_BH_Tree_II/Evrard_test/hfvCLibs_v7_hfv_v2.h:
// 1240-1418) and the reading of its grid file coolHeatGridNew.bin
// (Evrard_test/hfvGpuSphBHtree_v3_check_v1_cooling_t3_Evrard.cu:137-179).
//
// File layout (native-endian):
//   int32 N_kpc, N_nH, N_Z, N_T, N_M, N_Time;
//   float32 kpc[N_kpc], nH[N_nH], Z[N_Z], T[N_T], time_s[N_Time];
//   float32 u_evol[N_kpc][N_T][N_nH][N_Z][N_Time]   (u after a time time_s, cgs)
//   float32 mu[N_kpc][N_T][N_nH][N_Z][N_Time]
//   float32 frac[N_kpc][N_T][N_nH][N_Z][N_M][N_Time] (ion fractions of N_M species)
//
// Per particle (one thread each): r in kpc and n_H = rho X_H / m_H pick the
// nearest grid entry (the first entry at or above the value, or the one below
// it when that is nearer; the last entry above the grid); the metallicity row
// is fixed (the reference assumes [Z/H] = -1, row 1); the u column of the
// initial states U[t] = u_evol[kpc][t][nH][Z][0] gives the first row with
// u <= U[t] (the last row above it), dt the first time at or above dt (the
// last above it); u_new interpolates linearly in u between that row and the
// one below (the reference extrapolates above the column's top and takes the
// row itself at the bottom), and the N_M ion fractions of the chosen cell are
// copied.  The reference stages the U column in one global array that every
// thread overwrites (a race between particles of different cells); here each
// thread reads its own column.  The arithmetic is FP64 on the FP32 tables,
// rounded as written, so the oracle's restatement gives the same bits.
#include <cstdio>
#include <vector>

#include "sph_internal.cuh"

namespace {

struct TabDev {
    const float *kpc, *nH, *T, *time_s, *uev, *frac;
    int n_kpc, n_nH, n_Z, n_T, n_M, n_time, z_row;
    double unit_rho, unit_u, unit_t, unit_len, kpc_cm, XH, mH;
};

// first j with v <= g[j]; the nearer of j and j-1 when j > 0; the last entry
// when v is above the grid (hcoolingx's kpc and n_H rule)
__device__ __forceinline__ int nearest_index(const float *g, int n, double v) {
    int k = -1;
    for (int j = 0; j < n; j++)
        if (v <= (double)g[j]) {
            k = j;
            break;
        }
    if (k > 0) {
        const double d1 = fabs(xsub((double)g[k], v)), d2 = fabs(xsub((double)g[k - 1], v));
        if (d2 < d1) k -= 1;
    }
    return k < 0 ? n - 1 : k;
}

__global__ void k_cool_table(TabDev t, int n, const double *__restrict__ x,
                             const double *__restrict__ y, const double *__restrict__ z,
                             const double *__restrict__ rho, double *__restrict__ u,
                             const int *__restrict__ cloud, const double *__restrict__ dt,
                             float *__restrict__ ion) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double r = __dsqrt_rn(xadd(xadd(xmul(x[i], x[i]), xmul(y[i], y[i])), xmul(z[i], z[i])));
    const double r_kpc = xdiv(xmul(r, t.unit_len), t.kpc_cm);
    const int ik = nearest_index(t.kpc, t.n_kpc, r_kpc);
    const double nh = xdiv(xmul(xmul(rho[i], t.unit_rho), t.XH), t.mH);
    const int ih = nearest_index(t.nH, t.n_nH, nh);
    const size_t s_kpc = (size_t)t.n_T * t.n_nH * t.n_Z * t.n_time;
    const size_t s_T = (size_t)t.n_nH * t.n_Z * t.n_time;
    const size_t s_nH = (size_t)t.n_Z * t.n_time;
    const size_t base = ik * s_kpc + ih * s_nH + (size_t)t.z_row * t.n_time;
    const double ui = xmul(u[i], t.unit_u);
    int iu = -1;
    for (int j = 0; j < t.n_T; j++)
        if (ui <= (double)t.uev[base + j * s_T]) {
            iu = j;
            break;
        }
    if (iu < 0) iu = t.n_T - 1;
    const double dts = xmul(dt[cloud[i]], t.unit_t);
    int it = -1;
    for (int j = 0; j < t.n_time; j++)
        if (dts <= (double)t.time_s[j]) {
            it = j;
            break;
        }
    if (it < 0) it = t.n_time - 1;
    double uev;
    if (iu > 0) {
        const double U1 = t.uev[base + (iu - 1) * s_T], U2 = t.uev[base + iu * s_T];
        const double e1 = t.uev[base + (iu - 1) * s_T + it], e2 = t.uev[base + iu * s_T + it];
        const double fhi = xdiv(xsub(ui, U1), xsub(U2, U1));
        const double flo = xsub(1.0, fhi);
        uev = xadd(xmul(flo, e1), xmul(fhi, e2));
    } else {
        uev = t.uev[base + it];
    }
    u[i] = xdiv(uev, t.unit_u);
    if (ion) {
        const size_t m_kpc = s_kpc * t.n_M, m_T = s_T * t.n_M, m_nH = s_nH * t.n_M;
        const size_t mb = ik * m_kpc + iu * m_T + ih * m_nH + (size_t)t.z_row * t.n_M * t.n_time + it;
        for (int k = 0; k < t.n_M; k++) ion[(size_t)i * t.n_M + k] = t.frac[mb + (size_t)k * t.n_time];
    }
}

__global__ void k_scatter_rows_by_id(int n, int w, const int *__restrict__ id,
                                     const float *__restrict__ src, float *__restrict__ dst) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)n * w) return;
    const int s = (int)(t / w), k = (int)(t % w);
    dst[(size_t)id[s] * w + k] = src[t];
}

struct HostFile {
    FILE *f;
    explicit HostFile(const char *path) : f(fopen(path, "rb")) {}
    ~HostFile() {
        if (f) fclose(f);
    }
    bool read(void *p, size_t bytes) { return bytes == 0 || fread(p, 1, bytes, f) == bytes; }
};

// header and size check; dims = N_kpc, N_nH, N_Z, N_T, N_M, N_Time
int table_header(HostFile &F, int32_t dims[6], long long *cells) {
    if (!F.f) return SPH_ERR_IO;
    if (fseek(F.f, 0, SEEK_END) != 0) return SPH_ERR_IO;
    const long long sz = ftell(F.f);
    if (fseek(F.f, 0, SEEK_SET) != 0) return SPH_ERR_IO;
    if (!F.read(dims, 6 * sizeof(int32_t))) return SPH_ERR_IO;
    long long c5 = 1;
    for (int k = 0; k < 6; k++) {
        if (dims[k] < 1 || dims[k] > (1 << 20)) return SPH_ERR_IO;
        if (k != 4) c5 *= dims[k];
    }
    const long long grids = (long long)dims[0] + dims[1] + dims[2] + dims[3] + dims[5];
    const long long want = 24 + 4 * (grids + 2 * c5 + c5 * dims[4]);
    if (c5 > (1LL << 34) || sz != want) return SPH_ERR_IO;
    *cells = c5;
    return SPH_OK;
}

}  // namespace

int launch_cooling_table(sph_ctx *ctx) {
    if (!ctx->tab_ok) return SPH_ERR_STATE;
    const int n = ctx->n, c = ctx->cur;
    if (n <= 0) return SPH_OK;
    const sph_cool_table_params &p = ctx->tab;
    TabDev t;
    const int *d = ctx->tab_dims;
    t.n_kpc = d[0]; t.n_nH = d[1]; t.n_Z = d[2]; t.n_T = d[3]; t.n_M = d[4]; t.n_time = d[5];
    t.kpc = ctx->tab_grid;
    t.nH = t.kpc + d[0];
    t.T = t.nH + d[1] + d[2];
    t.time_s = t.T + d[3];
    t.uev = ctx->tab_uev;
    t.frac = ctx->tab_frac;
    t.z_row = p.z_row;
    t.unit_rho = p.unit_rho; t.unit_u = p.unit_u; t.unit_t = p.unit_t; t.unit_len = p.unit_length;
    t.kpc_cm = p.kpc_cm; t.XH = p.XH; t.mH = p.mH;
    double *const *st = ctx->st[c];
    k_cool_table<<<div_up(n, 128), 128, 0, ctx->stream>>>(t, n, st[ST_X], st[ST_Y], st[ST_Z],
                                                          ctx->rho, st[ST_U], ctx->cloud[c],
                                                          ctx->dt, ctx->ion);
    return ctx_check_launch(ctx, "cooling_table");
}

extern "C" {

int sph_cooling_table_dims(const char *path, int32_t *dims6) {
    if (!path || !dims6) return SPH_ERR_ARG;
    HostFile F(path);
    long long cells = 0;
    return table_header(F, dims6, &cells);
}

int sph_cooling_table_load(sph_ctx *ctx, const char *path, const sph_cool_table_params *p) {
    if (!ctx || !path || !p) return SPH_ERR_ARG;
    if (!(p->unit_rho > 0) || !(p->unit_u > 0) || !(p->unit_t > 0) || !(p->unit_length > 0) ||
        !(p->kpc_cm > 0) || !(p->XH > 0) || !(p->mH > 0))
        return SPH_ERR_ARG;
    HostFile F(path);
    int32_t d[6];
    long long cells = 0;
    int rc = table_header(F, d, &cells);
    if (rc) return rc;
    if (p->z_row < 0 || p->z_row >= d[2]) return SPH_ERR_ARG;
    const size_t ng = (size_t)d[0] + d[1] + d[2] + d[3] + d[5];
    std::vector<float> grid(ng), uev((size_t)cells), mu((size_t)cells), frac((size_t)cells * d[4]);
    if (!F.read(grid.data(), 4 * ng) || !F.read(uev.data(), 4 * (size_t)cells) ||
        !F.read(mu.data(), 4 * (size_t)cells) || !F.read(frac.data(), 4 * frac.size()))
        return SPH_ERR_IO;
    cudaSetDevice(ctx->device);
    // the tables are replaced, never grown in place: free the old ones
    for (void *q : {(void *)ctx->tab_grid, (void *)ctx->tab_uev, (void *)ctx->tab_frac,
                    (void *)ctx->ion}) {
        if (!q) continue;
        cudaFree(q);
        for (auto &a : ctx->allocs)
            if (a == q) a = nullptr;
    }
    ctx->tab_grid = ctx->tab_uev = ctx->tab_frac = ctx->ion = nullptr;
    ctx->tab_ok = false;
    auto dal = [&](float **out, size_t count) -> int {
        void *q = nullptr;
        cudaError_t e = cudaMalloc(&q, std::max<size_t>(count, 64) * sizeof(float));
        if (e != cudaSuccess) return ctx_fail(ctx, e, "cudaMalloc", __LINE__);
        ctx->allocs.push_back(q);
        *out = (float *)q;
        return SPH_OK;
    };
    if ((rc = dal(&ctx->tab_grid, ng)) || (rc = dal(&ctx->tab_uev, uev.size())) ||
        (rc = dal(&ctx->tab_frac, frac.size())) || (rc = dal(&ctx->ion, (size_t)ctx->cfg.n_max * d[4])))
        return rc;
    CK(cudaMemcpy(ctx->tab_grid, grid.data(), 4 * ng, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(ctx->tab_uev, uev.data(), 4 * uev.size(), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(ctx->tab_frac, frac.data(), 4 * frac.size(), cudaMemcpyHostToDevice));
    CK(cudaMemset(ctx->ion, 0, 4 * (size_t)ctx->cfg.n_max * d[4]));
    for (int k = 0; k < 6; k++) ctx->tab_dims[k] = d[k];
    ctx->tab = *p;
    ctx->tab_ok = true;
    return SPH_OK;
}

int sph_cooling_table(sph_ctx *ctx) {
    if (!ctx) return SPH_ERR_ARG;
    cudaSetDevice(ctx->device);
    return launch_cooling_table(ctx);
}

int sph_get_ion_frac(sph_ctx *ctx, float *out, int32_t host) {
    if (!ctx || !out) return SPH_ERR_ARG;
    if (!ctx->tab_ok) return SPH_ERR_STATE;
    cudaSetDevice(ctx->device);
    const int n = ctx->n, w = ctx->tab_dims[4];
    if (n <= 0) return SPH_OK;
    float *buf = (float *)ctx->red;  // 2 N doubles hold N w floats for w <= 4
    float *tmp = nullptr;
    if (w > 4) CK(cudaMalloc(&tmp, sizeof(float) * (size_t)n * w));
    float *dst = tmp ? tmp : buf;
    const long long tot = (long long)n * w;
    k_scatter_rows_by_id<<<div_up(tot, 256), 256, 0, ctx->stream>>>(n, w, ctx->id[ctx->cur],
                                                                   ctx->ion, dst);
    cudaError_t e = cudaMemcpyAsync(out, dst, sizeof(float) * tot,
                                    host ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice,
                                    ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (tmp) cudaFree(tmp);
    if (e != cudaSuccess) return ctx_fail(ctx, e, "get_ion_frac", __LINE__);
    return ctx_check_launch(ctx, "get_ion_frac");
}

}  // extern "C"
