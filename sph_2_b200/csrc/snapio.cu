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
