// snapio.cu -- the reference's binary initial-condition and snapshot files,
// read and written on the host so that reference-made ICs drive this path and
// its analysis scripts read this path's output.
//
// IC file (written by Particles_in_BH_Tree_II/Evrard_test/IC_evrard4.cu:245-260,
// read by hfvCLibs_v7_hfv_v2.h:59-101), native-endian:
//     int32 N; int32 Typ[N]; float32 x, y, z, vx, vy, vz, u, h, eps, mass [N each]
// Snapshot (hfvCLibs_v7_hfv_v2.h:107-143, read by Evrard_test/
// singlex_gpu_data.py:55-72):
//     int32 N; int32 N_ionFrac; int32 Typ[N];
//     float32 x, y, z, vx, vy, vz, rho, h, u, mass [N each];
//     float32 ionFrac[N_ionFrac]; int32 ngbDebug[N]
// The path here is gas only (Typ 0); the reference's black-hole (-1) and
// outflow particle types are outside it, so an IC holding them is rejected.
// The snapshot's per-particle int32 debug slot carries the neighbour count.
#include <cstdio>
#include <cstring>
#include <vector>

#include "sph_internal.cuh"

namespace {

struct HostFile {
    FILE *f;
    HostFile(const char *path, const char *mode) : f(fopen(path, mode)) {}
    ~HostFile() {
        if (f) fclose(f);
    }
    bool read(void *p, size_t bytes) { return bytes == 0 || fread(p, 1, bytes, f) == bytes; }
    bool write(const void *p, size_t bytes) { return bytes == 0 || fwrite(p, 1, bytes, f) == bytes; }
};

long long file_bytes(FILE *f) {
    if (fseek(f, 0, SEEK_END) != 0) return -1;
    long long sz = ftell(f);
    if (fseek(f, 0, SEEK_SET) != 0) return -1;
    return sz;
}

constexpr int IC_FLOAT_FIELDS = 10;

int ic_header(HostFile &F, int32_t *n) {
    if (!F.f) return SPH_ERR_IO;
    const long long sz = file_bytes(F.f);
    int32_t N = -1;
    if (sz < 4 || !F.read(&N, 4)) return SPH_ERR_IO;
    if (N < 0 || sz != 4 + (long long)N * 4 * (1 + IC_FLOAT_FIELDS)) return SPH_ERR_IO;
    *n = N;
    return SPH_OK;
}

}  // namespace

int sph_ic_count(const char *path, int32_t *n) {
    if (!path || !n) return SPH_ERR_ARG;
    HostFile F(path, "rb");
    return ic_header(F, n);
}

int sph_load_ic(sph_ctx *ctx, const char *path, double *eps_out) {
    if (!ctx || !path) return SPH_ERR_ARG;
    HostFile F(path, "rb");
    int32_t n = 0;
    int rc = ic_header(F, &n);
    if (rc) return rc;
    if (n > ctx->cfg.n_max) return SPH_ERR_CAPACITY;
    std::vector<int32_t> typ(n);
    if (!F.read(typ.data(), sizeof(int32_t) * n)) return SPH_ERR_IO;
    for (int i = 0; i < n; i++)
        if (typ[i] != 0) return SPH_ERR_ARG;  // gas particles only
    // x y z vx vy vz u h eps mass, widened to FP64
    std::vector<float> buf(n);
    std::vector<std::vector<double>> f(IC_FLOAT_FIELDS, std::vector<double>(n));
    for (int k = 0; k < IC_FLOAT_FIELDS; k++) {
        if (!F.read(buf.data(), sizeof(float) * n)) return SPH_ERR_IO;
        for (int i = 0; i < n; i++) f[k][i] = (double)buf[i];
    }
    if (eps_out)
        for (int i = 0; i < n; i++) eps_out[i] = f[8][i];
    return sph_load(ctx, n, nullptr, f[0].data(), f[1].data(), f[2].data(), f[3].data(),
                    f[4].data(), f[5].data(), f[9].data(), f[7].data(), f[6].data(), 1);
}

int sph_write_ic(sph_ctx *ctx, const char *path, const double *eps) {
    if (!ctx || !path) return SPH_ERR_ARG;
    const int n = sph_count(ctx);
    if (n < 0) return n;
    // IC_evrard4.cu writes eps = h when no softening is given (:224-229)
    const int fields[IC_FLOAT_FIELDS] = {SPH_F_X,  SPH_F_Y, SPH_F_Z, SPH_F_VX, SPH_F_VY,
                                         SPH_F_VZ, SPH_F_U, SPH_F_H, -1,       SPH_F_M};
    std::vector<double> tmp(n);
    std::vector<std::vector<float>> out(IC_FLOAT_FIELDS, std::vector<float>(n));
    for (int k = 0; k < IC_FLOAT_FIELDS; k++) {
        const double *src = tmp.data();
        if (fields[k] >= 0) {
            int rc = sph_get_field(ctx, fields[k], tmp.data(), 1, 0);
            if (rc) return rc;
        } else if (eps) {
            src = eps;
        } else {
            int rc = sph_get_field(ctx, SPH_F_H, tmp.data(), 1, 0);
            if (rc) return rc;
        }
        for (int i = 0; i < n; i++) out[k][i] = (float)src[i];
    }
    HostFile F(path, "wb");
    if (!F.f) return SPH_ERR_IO;
    const int32_t N = n;
    std::vector<int32_t> typ(n, 0);
    bool ok = F.write(&N, 4) && F.write(typ.data(), sizeof(int32_t) * n);
    for (int k = 0; k < IC_FLOAT_FIELDS && ok; k++) ok = F.write(out[k].data(), sizeof(float) * n);
    return ok ? SPH_OK : SPH_ERR_IO;
}

int sph_write_snapshot(sph_ctx *ctx, const char *path, const float *ion_frac, int32_t n_ion_frac) {
    if (!ctx || !path || n_ion_frac < 0 || (n_ion_frac > 0 && !ion_frac)) return SPH_ERR_ARG;
    const int n = sph_count(ctx);
    if (n < 0) return n;
    const int fields[10] = {SPH_F_X,  SPH_F_Y,   SPH_F_Z, SPH_F_VX, SPH_F_VY,
                            SPH_F_VZ, SPH_F_RHO, SPH_F_H, SPH_F_U,  SPH_F_M};
    std::vector<double> tmp(n);
    std::vector<std::vector<float>> out(10, std::vector<float>(n));
    for (int k = 0; k < 10; k++) {
        int rc = sph_get_field(ctx, fields[k], tmp.data(), 1, 0);
        if (rc) return rc;
        for (int i = 0; i < n; i++) out[k][i] = (float)tmp[i];
    }
    // neighbour count per particle (original order) in the int32 debug slot;
    // -1 (the reference's fill value) while no list has been built
    std::vector<int32_t> ngb(n, -1);
    if (n > 0 && ctx->lists_ok) {
        std::vector<int32_t> cnt(n), ids(n);
        CK(cudaStreamSynchronize(ctx->stream));
        CK(cudaMemcpy(cnt.data(), ctx->ngb_cnt, sizeof(int32_t) * n, cudaMemcpyDeviceToHost));
        int rc = sph_get_ids(ctx, ids.data(), 1);
        if (rc) return rc;
        for (int s = 0; s < n; s++) ngb[ids[s]] = cnt[s];
    }
    HostFile F(path, "wb");
    if (!F.f) return SPH_ERR_IO;
    const int32_t hdr[2] = {n, n_ion_frac};
    std::vector<int32_t> typ(n, 0);
    bool ok = F.write(hdr, sizeof(hdr)) && F.write(typ.data(), sizeof(int32_t) * n);
    for (int k = 0; k < 10 && ok; k++) ok = F.write(out[k].data(), sizeof(float) * n);
    ok = ok && F.write(ion_frac, sizeof(float) * n_ion_frac) &&
         F.write(ngb.data(), sizeof(int32_t) * n);
    return ok ? SPH_OK : SPH_ERR_IO;
}

// ---- FP64 restart -----------------------------------------------------------
// The reference restarts from text dumps of its float arrays
// (GPU_sph/With_metal_cooling/Check_Restart_version/hfv_sph_gpu_v5.cu); a run
// resumed from those differs from the run that continued.  The restart file
// here holds what the next step reads, in FP64 and in storage order: the
// state fields (x y z vx vy vz m h u du/dt_prev and the largest neighbour h,
// which sets the next candidate radius), the original ids and clouds, the
// accelerations of the last step (the next step's first kick uses them) and
// every cloud's time step.  Reading it restores the storage order as well, so
// the next sort sees the same input order and the resumed run repeats the
// continuing one bit for bit.  Cooling tables and MLP parameters are set up
// separately.
//   char magic[8] "SPHB200R"; int32 version (1), n, ncloud, prologue_done,
//   last_injected_id, pad; int64 step_count;
//   int32 cloud_start[ncloud + 1]; double dt[ncloud];
//   int32 id[n], cloud[n]; double state[ST_N][n]; double a_sph[3n], a_grav[3n]
namespace {
const char RESTART_MAGIC[8] = {'S', 'P', 'H', 'B', '2', '0', '0', 'R'};
struct RestartHeader {
    char magic[8];
    int32_t version, n, ncloud, prologue_done, last_injected_id, pad;
    int64_t step_count;
};
}  // namespace

int sph_write_restart(sph_ctx *ctx, const char *path) {
    if (!ctx || !path) return SPH_ERR_ARG;
    CK(cudaSetDevice(ctx->device));
    CK(cudaStreamSynchronize(ctx->stream_g));
    CK(cudaStreamSynchronize(ctx->stream));
    const int n = ctx->n, nc = ctx->ncloud, c = ctx->cur;
    RestartHeader h{};
    memcpy(h.magic, RESTART_MAGIC, 8);
    h.version = 1;
    h.n = n;
    h.ncloud = nc;
    h.prologue_done = ctx->prologue_done ? 1 : 0;
    h.last_injected_id = ctx->last_injected_id;
    h.step_count = ctx->step_count;
    std::vector<double> dt(nc > 0 ? nc : 1);
    std::vector<int32_t> ids(n > 0 ? n : 1), cl(n > 0 ? n : 1);
    std::vector<double> buf((size_t)(n > 0 ? n : 1) * 3);
    if (nc > 0) CK(cudaMemcpy(dt.data(), ctx->dt, sizeof(double) * nc, cudaMemcpyDeviceToHost));
    if (n > 0) {
        CK(cudaMemcpy(ids.data(), ctx->id[c], sizeof(int32_t) * n, cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(cl.data(), ctx->cloud[c], sizeof(int32_t) * n, cudaMemcpyDeviceToHost));
    }
    HostFile F(path, "wb");
    if (!F.f) return SPH_ERR_IO;
    bool ok = F.write(&h, sizeof h) &&
              F.write(ctx->cloud_start_h.data(), sizeof(int32_t) * (nc + 1)) &&
              F.write(dt.data(), sizeof(double) * nc) && F.write(ids.data(), sizeof(int32_t) * n) &&
              F.write(cl.data(), sizeof(int32_t) * n);
    for (int k = 0; k < ST_N && ok; k++) {
        if (n > 0) CK(cudaMemcpy(buf.data(), ctx->st[c][k], sizeof(double) * n, cudaMemcpyDeviceToHost));
        ok = F.write(buf.data(), sizeof(double) * n);
    }
    for (double *a : {ctx->asph, ctx->agrav}) {
        if (!ok) break;
        if (n > 0) CK(cudaMemcpy(buf.data(), a, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost));
        ok = F.write(buf.data(), sizeof(double) * 3 * n);
    }
    // a context resumed from this file starts with a full rebuild; so does
    // this one, so that both continue alike
    ctx->topo_ok = false;
    return ok ? SPH_OK : SPH_ERR_IO;
}

int sph_read_restart(sph_ctx *ctx, const char *path) {
    if (!ctx || !path) return SPH_ERR_ARG;
    HostFile F(path, "rb");
    if (!F.f) return SPH_ERR_IO;
    const long long sz = file_bytes(F.f);
    RestartHeader h{};
    if (sz < (long long)sizeof h || !F.read(&h, sizeof h) || memcmp(h.magic, RESTART_MAGIC, 8) != 0 ||
        h.version != 1 || h.n < 0 || h.ncloud < 1)
        return SPH_ERR_IO;
    const long long n = h.n, nc = h.ncloud;
    const long long want = (long long)sizeof h + 4 * (nc + 1) + 8 * nc + 8 * n + 8 * n * (ST_N + 6);
    if (sz != want) return SPH_ERR_IO;
    if (n > ctx->cfg.n_max || nc > ctx->cfg.n_cloud_max) return SPH_ERR_CAPACITY;
    std::vector<int32_t> cs(nc + 1), ids(n > 0 ? n : 1), cl(n > 0 ? n : 1);
    std::vector<double> dt(nc), buf((size_t)(n > 0 ? n : 1) * 3);
    if (!F.read(cs.data(), 4 * (nc + 1)) || !F.read(dt.data(), 8 * nc) || !F.read(ids.data(), 4 * n) ||
        !F.read(cl.data(), 4 * n))
        return SPH_ERR_IO;
    if (cs[0] != 0 || cs[nc] != n) return SPH_ERR_IO;
    CK(cudaSetDevice(ctx->device));
    drop_graphs(ctx);
    CK(cudaStreamSynchronize(ctx->stream_g));
    CK(cudaStreamSynchronize(ctx->stream));
    cudaStream_t s = ctx->stream;
    ctx->cur = 0;
    for (int k = 0; k < ST_N; k++) {
        if (!F.read(buf.data(), 8 * n)) return SPH_ERR_IO;
        if (n > 0) CK(cudaMemcpy(ctx->st[0][k], buf.data(), 8 * n, cudaMemcpyHostToDevice));
    }
    for (double *a : {ctx->asph, ctx->agrav}) {
        if (!F.read(buf.data(), 8 * 3 * n)) return SPH_ERR_IO;
        if (n > 0) CK(cudaMemcpy(a, buf.data(), 8 * 3 * n, cudaMemcpyHostToDevice));
    }
    if (n > 0) {
        CK(cudaMemcpy(ctx->id[0], ids.data(), 4 * n, cudaMemcpyHostToDevice));
        CK(cudaMemcpy(ctx->cloud[0], cl.data(), 4 * n, cudaMemcpyHostToDevice));
        CK(cudaMemset(ctx->divV, 0, 8 * n));
        CK(cudaMemset(ctx->curlV, 0, 8 * n));
        CK(cudaMemset(ctx->pot, 0, 8 * n));
    }
    ctx->n = (int)n;
    ctx->ncloud = (int)nc;
    ctx->ngroup = (int)(n + nc);
    ctx->cloud_start_h.assign(cs.begin(), cs.end());
    CK(cudaMemcpy(ctx->cloud_start, cs.data(), 4 * (nc + 1), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(ctx->dt, dt.data(), 8 * nc, cudaMemcpyHostToDevice));
    CK(cudaMemset(ctx->dt_bits, 0xff, 8 * nc));
    CK(cudaMemset(ctx->d_ngroup, 0, sizeof(int)));
    int rc = launch_pack_p1(ctx);
    if (rc) return rc;
    CK(cudaStreamSynchronize(s));
    ctx->tree_ok = ctx->lists_ok = ctx->rho_ok = ctx->divcurl_ok = ctx->cand_ok = false;
    ctx->p2_dirty = true;
    ctx->prologue_done = h.prologue_done != 0;
    ctx->step_count = h.step_count;
    ctx->topo_ok = false;  // the topology is not in the file: the next step rebuilds
    ctx->last_injected_id = h.last_injected_id;
    return ctx_check_launch(ctx, "read_restart");
}
