// capi.cu -- the extern "C" boundary of libsphb200.so (include/sph_b200.h):
// context lifetime, device memory (allocated once at context creation; the
// reference allocates and frees the neighbour list and tree every step,
// EVR.cu:1148, 1417-1446), field transfer in original particle order, the
// phase entry points, the prologue and the CUDA-graph step.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <numeric>

#include "sph_internal.cuh"

int ctx_fail(sph_ctx *ctx, cudaError_t e, const char *what, int line) {
    char buf[512];
    snprintf(buf, sizeof buf, "%s failed (%s) at capi line %d", what, cudaGetErrorString(e), line);
    if (ctx) ctx->err = buf;
    return e == cudaErrorMemoryAllocation ? SPH_ERR_NOMEM : SPH_ERR_CUDA;
}

int ctx_check_launch(sph_ctx *ctx, const char *what) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return ctx_fail(ctx, e, what, 0);
    return SPH_OK;
}

int launch_dt_commit(sph_ctx *ctx);

// blocks for a persistent kernel: every SM filled to its occupancy limit
// (looked up once per kernel and block size)
int persistent_grid(sph_ctx *ctx, const void *kernel, int block, size_t smem) {
    const auto key = std::make_pair(kernel, block);
    auto it = ctx->occupancy.find(key);
    if (it != ctx->occupancy.end()) return ctx->num_sms * it->second;
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, block, smem) != cudaSuccess ||
        per_sm < 1)
        per_sm = 1;
    ctx->occupancy[key] = per_sm;
    return ctx->num_sms * per_sm;
}

void drop_graphs(sph_ctx *ctx) {
    for (int k = 0; k < 2; k++)
        for (int r = 0; r < 2; r++)
            if (ctx->graph[k][r]) {
                cudaGraphExecDestroy(ctx->graph[k][r]);
                ctx->graph[k][r] = nullptr;
            }
    ctx->graph_valid = false;
}

int queue_launch(sph_ctx *ctx, cudaStream_t s, int slot, const void *kernel, int block,
                 int static_grid, int *grid, unsigned **queue) {
    if (ctx->cfg.flags & SPH_FLAG_STATIC_GRID) {
        *grid = static_grid;
        *queue = nullptr;
        return SPH_OK;
    }
    *grid = std::min(static_grid, persistent_grid(ctx, kernel, block, 0));
    *queue = ctx->work + slot;
    CK(cudaMemsetAsync(*queue, 0, sizeof(unsigned), s));
    return SPH_OK;
}

namespace {

template <class T>
int dalloc(sph_ctx *ctx, T **p, size_t count) {
    size_t bytes = std::max<size_t>(count * sizeof(T), 256);
    void *q = nullptr;
    cudaError_t e = cudaMalloc(&q, bytes);
    if (e != cudaSuccess) return ctx_fail(ctx, e, "cudaMalloc", __LINE__);
    ctx->allocs.push_back(q);
    ctx->dev_bytes += (int64_t)bytes;
    *p = (T *)q;
    return SPH_OK;
}

#define DA(ptr, count)                          \
    do {                                        \
        int r_ = dalloc(ctx, &(ptr), (count));  \
        if (r_) return r_;                      \
    } while (0)

__global__ void k_iota(int n, int *a) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) a[i] = i;
}
__global__ void k_scatter_by_id(int n, const int *__restrict__ id, const double *__restrict__ src,
                                double *__restrict__ dst) {
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s < n) dst[id[s]] = src[s];
}
__global__ void k_scatter_int_by_id(int n, const int *__restrict__ id, const int *__restrict__ src,
                                    int *__restrict__ dst) {
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s < n) dst[id[s]] = src[s];
}
__global__ void k_gather_by_id(int n, const int *__restrict__ id, const double *__restrict__ src,
                               double *__restrict__ dst) {
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s < n) dst[s] = src[id[s]];
}

bool valid_lanes(int l) { return l == 1 || l == 2 || l == 4 || l == 8 || l == 16 || l == 32; }

int check_cfg(const sph_config *c) {
    if (c->n_max < 1 || c->n_cloud_max < 1) return SPH_ERR_ARG;
    if (c->n_cloud_max > (1 << 20)) return SPH_ERR_ARG;
    if (c->precision != SPH_PREC_FP64 && c->precision != SPH_PREC_MIXED) return SPH_ERR_ARG;
    if (c->av_mode != SPH_AV_MG83 && c->av_mode != SPH_AV_GADGET) return SPH_ERR_ARG;
    if (c->leaf_size < 1 || c->leaf_size > 64) return SPH_ERR_ARG;
    if (!valid_lanes(c->ngb_lanes)) return SPH_ERR_ARG;
    // the neighbour-sum kernels are compiled for at most 256 threads per block
    if (c->block_size < 64 || c->block_size > 256 || c->block_size % 32) return SPH_ERR_ARG;
    if (c->max_ngb < 32 || c->max_ngb > 512) return SPH_ERR_ARG;
    if (c->walk_blocks < 0 || c->walk_blocks > 64) return SPH_ERR_ARG;
    if (c->h_max_iter < 1 || c->h_max_iter > 1000) return SPH_ERR_ARG;
    if (!(c->theta > 0.0 && c->theta <= 1.0)) return SPH_ERR_ARG;
    if (!(c->theta_local >= 0.0 && c->theta_local < 1.0)) return SPH_ERR_ARG;
    if (!(c->theta_small >= 0.0 && c->theta_small < 1.0) || c->small_cell < 0) return SPH_ERR_ARG;
    if (!(c->eps > 0.0) || !(c->n_ngb > 1.0) || !(c->h_tol > 0.0)) return SPH_ERR_ARG;
    if (!(c->courant > 0.0)) return SPH_ERR_ARG;
    if (c->dt_mode != SPH_DT_COURANT && c->dt_mode != SPH_DT_INDIVIDUAL) return SPH_ERR_ARG;
    if (!(c->ext_sigma >= 0.0)) return SPH_ERR_ARG;
    if (c->rebuild_every < 0 || c->rebuild_every > 1000) return SPH_ERR_ARG;
    return SPH_OK;
}

double *field_ptr(sph_ctx *ctx, int f) {
    const int c = ctx->cur;
    const size_t n = ctx->n;
    switch (f) {
        case SPH_F_X: return ctx->st[c][ST_X];
        case SPH_F_Y: return ctx->st[c][ST_Y];
        case SPH_F_Z: return ctx->st[c][ST_Z];
        case SPH_F_VX: return ctx->st[c][ST_VX];
        case SPH_F_VY: return ctx->st[c][ST_VY];
        case SPH_F_VZ: return ctx->st[c][ST_VZ];
        case SPH_F_M: return ctx->st[c][ST_M];
        case SPH_F_H: return ctx->st[c][ST_H];
        case SPH_F_U: return ctx->st[c][ST_U];
        case SPH_F_U_PREV: return ctx->st[c][ST_U];
        case SPH_F_DUDT_PREV: return ctx->st[c][ST_DUDT_PREV];
        case SPH_F_RHO: return ctx->rho;
        case SPH_F_P: return ctx->P;
        case SPH_F_C: return ctx->c;
        case SPH_F_DIVV: return ctx->divV;
        case SPH_F_CURLV: return ctx->curlV;
        case SPH_F_AX_SPH: return ctx->asph;
        case SPH_F_AY_SPH: return ctx->asph + n;
        case SPH_F_AZ_SPH: return ctx->asph + 2 * n;
        case SPH_F_AX_GRAV: return ctx->agrav;
        case SPH_F_AY_GRAV: return ctx->agrav + n;
        case SPH_F_AZ_GRAV: return ctx->agrav + 2 * n;
        case SPH_F_DUDT: return ctx->dudt;
        case SPH_F_VSIG: return ctx->vsig;
        case SPH_F_POT: return ctx->pot;
        default: return nullptr;
    }
}


int enter(sph_ctx *ctx) {
    if (!ctx) return SPH_ERR_ARG;
    cudaError_t e = cudaSetDevice(ctx->device);
    if (e != cudaSuccess) return ctx_fail(ctx, e, "cudaSetDevice", __LINE__);
    return SPH_OK;
}

int ensure_timing(sph_ctx *ctx) {
    if (ctx->tev_ok) return SPH_OK;
    for (int k = 0; k < 16; k++) CK(cudaEventCreate(&ctx->tev[k]));
    ctx->tev_ok = true;
    return SPH_OK;
}

// an event visible outside the step: an external event node while the
// step is captured into a graph, a plain record when it runs eagerly (the
// external flag is refused outside a capture)
cudaError_t record_ext(cudaEvent_t e, cudaStream_t s) {
    cudaStreamCaptureStatus st = cudaStreamCaptureStatusNone;
    cudaError_t r = cudaStreamIsCapturing(s, &st);
    if (r != cudaSuccess) return r;
    return st == cudaStreamCaptureStatusActive ? cudaEventRecordWithFlags(e, s, cudaEventRecordExternal)
                                               : cudaEventRecord(e, s);
}

#define MARK(k, strm)                                         \
    do {                                                      \
        if (timing) CK(record_ext(ctx->tev[k], (strm)));      \
    } while (0)

// the body of one step, queued on ctx->stream; refit: keep the storage order
// and the tree topology of the last full rebuild and refit the tree to the
// drifted particles (no sort, no Karras split, no group tables)
int step_body(sph_ctx *ctx, bool refit) {
    int rc;
    const bool fused = ctx->cfg.flags & SPH_FLAG_DUDT_FUSED;
    const bool pot = ctx->cfg.flags & SPH_FLAG_POTENTIAL;
    const bool timing = ctx->cfg.flags & SPH_FLAG_TIMING;
    if (timing && (rc = ensure_timing(ctx))) return rc;
    MARK(0, ctx->stream);
    if ((rc = launch_kick_drift(ctx))) return rc;
    MARK(1, ctx->stream);
    if ((rc = refit ? launch_sort_refit(ctx) : launch_sort(ctx))) return rc;
    MARK(2, ctx->stream);
    CK(record_ext(ctx->ev_io[0], ctx->stream));
    if ((rc = refit ? launch_tree_refit(ctx, false) : launch_tree(ctx, false))) return rc;
    MARK(3, ctx->stream);
    // gravity depends only on the tree: run it beside the SPH passes
    CK(cudaEventRecord(ctx->ev_fork, ctx->stream));
    CK(cudaStreamWaitEvent(ctx->stream_g, ctx->ev_fork, 0));
    MARK(13, ctx->stream_g);
    ctx->in_step = true;
    rc = launch_gravity(ctx, ctx->stream_g, pot);
    ctx->in_step = false;
    if (rc) return rc;
    MARK(14, ctx->stream_g);
    CK(cudaEventRecord(ctx->ev_join, ctx->stream_g));
    if ((rc = launch_smoothing_h(ctx))) return rc;
    MARK(4, ctx->stream);
    // lists and density in one pass over the candidate rows of the h iteration
    MARK(5, ctx->stream);
    if ((rc = launch_lists_density(ctx))) return rc;
    MARK(6, ctx->stream);
    CK(record_ext(ctx->ev_io[1], ctx->stream));
    MARK(7, ctx->stream);
    if ((rc = launch_forces(ctx, true, fused, false))) return rc;
    MARK(8, ctx->stream);
    CK(cudaStreamWaitEvent(ctx->stream, ctx->ev_join, 0));
    const bool courant = ctx->cfg.dt_fixed <= 0.0 && ctx->cfg.dt_mode == SPH_DT_COURANT;
    if ((rc = launch_kick(ctx, 0.5, courant))) return rc;
    MARK(9, ctx->stream);
    CK(record_ext(ctx->ev_io[2], ctx->stream));
    if (!fused)
        if ((rc = launch_forces(ctx, false, true, false))) return rc;
    MARK(10, ctx->stream);
    if ((rc = launch_update_u(ctx, false))) return rc;
    if (ctx->cfg.flags & SPH_FLAG_COOLING) {
        if (ctx->cfg.flags & SPH_FLAG_COOLING_TABLE) rc = launch_cooling_table(ctx);
        else if (ctx->cfg.flags & SPH_FLAG_COOLING_MLP) rc = launch_cooling_mlp(ctx);
        else rc = launch_cooling_exact(ctx);
        if (rc) return rc;
    }
    if (ctx->cfg.dt_fixed <= 0.0 && ctx->cfg.dt_mode == SPH_DT_INDIVIDUAL)
        if ((rc = launch_dt_individual(ctx))) return rc;
    rc = launch_dt_commit(ctx);
    MARK(11, ctx->stream);
    if (!rc) CK(record_ext(ctx->ev_io[3], ctx->stream));
    return rc;
}

__global__ void k_fma_peak(float *out, int iters, float a, float b) {
    float x0 = threadIdx.x * 1e-3f, x1 = x0 + 1.f, x2 = x0 + 2.f, x3 = x0 + 3.f;
    float x4 = x0 + 4.f, x5 = x0 + 5.f, x6 = x0 + 6.f, x7 = x0 + 7.f;
    for (int i = 0; i < iters; i++) {
#pragma unroll
        for (int k = 0; k < 16; k++) {
            x0 = fmaf(x0, a, b); x1 = fmaf(x1, a, b); x2 = fmaf(x2, a, b); x3 = fmaf(x3, a, b);
            x4 = fmaf(x4, a, b); x5 = fmaf(x5, a, b); x6 = fmaf(x6, a, b); x7 = fmaf(x7, a, b);
        }
    }
    float s = x0 + x1 + x2 + x3 + x4 + x5 + x6 + x7;
    if (s == 1234.5f) out[0] = s;
}

// the same chains as packed f32x2 FMAs (two per instruction; measured at the
// scalar rate within 3 % on B200: the FP32 pipe, not the issue slot, bounds it)
__global__ void k_fma2_peak(float *out, int iters, float a, float b) {
    const float2 A = make_float2(a, a), B = make_float2(b, b);
    float2 x[8];
#pragma unroll
    for (int q = 0; q < 8; q++) x[q] = make_float2(threadIdx.x * 1e-3f + q, q + 0.5f);
    for (int i = 0; i < iters; i++) {
#pragma unroll
        for (int k = 0; k < 16; k++) {
#pragma unroll
            for (int q = 0; q < 8; q++) x[q] = __ffma2_rn(x[q], A, B);
        }
    }
    float s = 0.f;
#pragma unroll
    for (int q = 0; q < 8; q++) s += x[q].x + x[q].y;
    if (s == 1234.5f) out[0] = s;
}

}  // namespace

extern "C" {

int sph_default_config(sph_config *c) {
    if (!c) return SPH_ERR_ARG;
    memset(c, 0, sizeof *c);
    c->n_max = 1 << 20;
    c->n_cloud_max = 1;
    c->precision = SPH_PREC_MIXED;
    c->av_mode = SPH_AV_MG83;
    c->balsara = 0;
    c->leaf_size = 8;
    c->ngb_lanes = 4;
    c->block_size = 128;
    c->max_ngb = 256;
    c->h_max_iter = 64;
    c->flags = 0;
    c->walk_blocks = 0;
    c->n_ngb = 64.0;
    c->h_tol = 1e-3;
    c->gamma = 5.0 / 3.0;
    c->alpha = 1.0;
    c->beta = 2.0;
    c->eta = 0.1;
    c->G = 1.0;
    c->eps = 1e-2;
    c->theta = 0.5;
    c->courant = 0.25;
    c->dt_max = 0.0;
    c->dt_fixed = 0.0;
    c->rebuild_every = 1;
    return SPH_OK;
}

int sph_ctx_create(const sph_config *cfg, sph_ctx **out) {
    if (!cfg || !out) return SPH_ERR_ARG;
    *out = nullptr;
    int rc = check_cfg(cfg);
    if (rc) return rc;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1) return SPH_ERR_CUDA;
    sph_ctx *ctx = new sph_ctx();
    ctx->cfg = *cfg;
    cudaGetDevice(&ctx->device);
    cudaDeviceGetAttribute(&ctx->num_sms, cudaDevAttrMultiProcessorCount, ctx->device);
    auto fail = [&](int r) {
        sph_ctx_destroy(ctx);
        return r;
    };
    const size_t N = cfg->n_max, NN = 2 * N, K = cfg->max_ngb, C = cfg->n_cloud_max;
    const size_t rs = cfg->precision == SPH_PREC_MIXED ? 16 : 32;  // Real4 bytes
    // the SPH passes (latency/memory bound) get the high-priority stream, the
    // compute-bound gravity walk the low-priority one, so the block scheduler
    // feeds the SPH passes first and fills the rest of each SM with the walk
    int prio_low = 0, prio_high = 0;
    cudaDeviceGetStreamPriorityRange(&prio_low, &prio_high);
    if (cudaStreamCreateWithPriority(&ctx->stream, cudaStreamNonBlocking, prio_high) != cudaSuccess)
        return fail(SPH_ERR_CUDA);
    ctx->own_stream = true;
    if (cudaStreamCreateWithPriority(&ctx->stream_g, cudaStreamNonBlocking, prio_low) != cudaSuccess)
        return fail(SPH_ERR_CUDA);
    cudaEventCreateWithFlags(&ctx->ev_fork, cudaEventDisableTiming);
    cudaEventCreateWithFlags(&ctx->ev_join, cudaEventDisableTiming);
    for (int k = 0; k < 4; k++)
        if (cudaEventCreateWithFlags(&ctx->ev_io[k], cudaEventDisableTiming) != cudaSuccess)
            return fail(SPH_ERR_CUDA);
#define DAF(ptr, count)                            \
    do {                                           \
        int r_ = dalloc(ctx, &(ptr), (count));     \
        if (r_) return fail(r_);                   \
    } while (0)
    for (int b = 0; b < 2; b++) {
        for (int k = 0; k < ST_N; k++) DAF(ctx->st[b][k], N);
        DAF(ctx->id[b], N);
        DAF(ctx->cloud[b], N);
    }
    DAF(ctx->rho, N); DAF(ctx->P, N); DAF(ctx->c, N); DAF(ctx->divV, N); DAF(ctx->curlV, N);
    DAF(ctx->asph, 3 * N); DAF(ctx->agrav, 3 * N);
    DAF(ctx->dudt, N); DAF(ctx->vsig, N); DAF(ctx->pot, N);
    DAF(ctx->p0, N);
    unsigned char *tmpb;
    DAF(tmpb, rs * N); ctx->p1 = tmpb;
    DAF(tmpb, rs * N); ctx->p2 = tmpb;
    DAF(tmpb, rs * N); ctx->pw = tmpb;
    DAF(ctx->key[0], N); DAF(ctx->key[1], N); DAF(ctx->key_in, N);
    DAF(ctx->val[0], N); DAF(ctx->val[1], N);
    ctx->sort_blocks = div_up(N, 2048);
    DAF(ctx->hist, 256 * (size_t)ctx->sort_blocks + 256);
    DAF(ctx->box, 6 * C);
    DAF(ctx->corg, 3 * C);
    DAF(ctx->cloud_start, C + 1);
    DAF(ctx->child, 2 * NN); DAF(ctx->parent, NN); DAF(ctx->first, NN); DAF(ctx->last, NN);
    DAF(ctx->flag, NN);
    DAF(ctx->node, 16 * NN); DAF(ctx->hmax, NN); DAF(ctx->ropen2, NN);
    float4 *nb4;
    DAF(nb4, 2 * NN); ctx->node_box = nb4;
    DAF(tmpb, rs * NN); ctx->wA = tmpb;
    DAF(tmpb, rs * NN); ctx->wB = tmpb;
    DAF(tmpb, rs * NN); ctx->wC = tmpb;
    DAF(ctx->wL, NN);
    DAF(ctx->croot, C);
    const size_t G = N + C + 1;
    DAF(ctx->gstart, G); DAF(ctx->gcount, G); DAF(ctx->groot_g, G); DAF(ctx->gnode, G);
    DAF(ctx->gmark, N); DAF(ctx->gpos, N); DAF(ctx->gnode_at, N);
    DAF(ctx->scan_tmp, N / 1024 + 64);
    DAF(ctx->d_ngroup, 1);
    DAF(ctx->ngb, K * N); DAF(ctx->ngb_cnt, N);
    DAF(ctx->cand_idx, K * N);
    DAF(ctx->cand_cnt, N);
    DAF(ctx->lflag, N + 3);
    DAF(ctx->mlist, N);
    DAF(ctx->retry, N); DAF(ctx->hcand, N); DAF(ctx->hiter, N); DAF(ctx->hover, N);
    DAF(ctx->hsr, N); DAF(ctx->dmv, N); DAF(ctx->gdm, N);
    DAF(ctx->dmv_max, C + 1);
    ctx->rows_ok = (int *)(ctx->dmv_max + C);
    DAF(ctx->kept_cnt, 3);
    DAF(ctx->dt, C); DAF(ctx->dt_next, C); DAF(ctx->dt_bits, C); DAF(ctx->dtmax_bits, C);
    DAF(ctx->dt_part, N); DAF(ctx->dhdt, N); DAF(ctx->dbin, N);
    DAF(ctx->status, SPH_NSTATUS);
    DAF(ctx->counters, 5);
    if (ctx->cfg.precision == SPH_PREC_MIXED && ctx->cfg.theta_local > 0.0) {
        ctx->sg_cap = (int)std::min<size_t>(N, N / 8 + C + 64);
        DAF(ctx->sg_start, N); DAF(ctx->sg_count, N); DAF(ctx->sg_cloud, N);
        DAF(ctx->d_nsg, 1);
        DAF(ctx->g_sg, G);
        DAF(ctx->sg_nrem, (size_t)ctx->sg_cap);
        DAF(ctx->sg_pool, (size_t)SG_POOL * N);
        DAF(ctx->sgL, (size_t)SG_LSTRIDE * ctx->sg_cap);
    }
    DAF(ctx->work, 16);
    DAF(ctx->red, std::max<size_t>(2 * N + 16, 8192));
    DAF(ctx->st_table, ST_N);
    if (cudaMemsetAsync(ctx->status, 0, SPH_NSTATUS * sizeof(long long), ctx->stream) ||
        cudaMemsetAsync(ctx->pot, 0, N * sizeof(double), ctx->stream) ||
        cudaMemsetAsync(ctx->agrav, 0, 3 * N * sizeof(double), ctx->stream) ||
        cudaMemsetAsync(ctx->asph, 0, 3 * N * sizeof(double), ctx->stream) ||
        cudaMemsetAsync(ctx->dt_bits, 0xff, C * sizeof(unsigned long long), ctx->stream) ||
        cudaMemsetAsync(ctx->dt, 0, C * sizeof(double), ctx->stream) ||
        cudaMemsetAsync(ctx->divV, 0, N * sizeof(double), ctx->stream) ||
        cudaMemsetAsync(ctx->curlV, 0, N * sizeof(double), ctx->stream) ||
        cudaMemsetAsync(ctx->corg, 0, 3 * C * sizeof(double), ctx->stream) ||
        cudaMemsetAsync(ctx->dmv_max, 0, (C + 1) * sizeof(unsigned long long), ctx->stream) ||
        cudaMemsetAsync(ctx->dmv, 0, N * sizeof(double), ctx->stream) ||
        cudaMemsetAsync(ctx->kept_cnt, 0, 3 * sizeof(int), ctx->stream))
        return fail(SPH_ERR_CUDA);
    if (cudaStreamSynchronize(ctx->stream) != cudaSuccess) return fail(SPH_ERR_CUDA);
#undef DAF
    *out = ctx;
    return SPH_OK;
}

void sph_ctx_destroy(sph_ctx *ctx) {
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    drop_graphs(ctx);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    if (ctx->stream_g) cudaStreamSynchronize(ctx->stream_g);
    for (void *p : ctx->allocs) cudaFree(p);
    if (ctx->tev_ok)
        for (int k = 0; k < 16; k++) cudaEventDestroy(ctx->tev[k]);
    if (ctx->ev_fork) cudaEventDestroy(ctx->ev_fork);
    if (ctx->ev_join) cudaEventDestroy(ctx->ev_join);
    if (ctx->stream_io) cudaStreamSynchronize(ctx->stream_io);
    for (int k = 0; k < 4; k++)
        if (ctx->ev_io[k]) cudaEventDestroy(ctx->ev_io[k]);
    if (ctx->io_stage) cudaFree(ctx->io_stage);
    if (ctx->stream_io) cudaStreamDestroy(ctx->stream_io);
    if (ctx->own_stream && ctx->stream) cudaStreamDestroy(ctx->stream);
    if (ctx->stream_g) cudaStreamDestroy(ctx->stream_g);
    delete ctx;
}

int sph_set_stream(sph_ctx *ctx, void *s) {
    int rc = enter(ctx);
    if (rc) return rc;
    CK(cudaStreamSynchronize(ctx->stream));
    if (ctx->own_stream) cudaStreamDestroy(ctx->stream);
    ctx->stream = (cudaStream_t)s;
    ctx->own_stream = false;
    drop_graphs(ctx);
    return SPH_OK;
}

int sph_sync(sph_ctx *ctx) {
    int rc = enter(ctx);
    if (rc) return rc;
    CK(cudaStreamSynchronize(ctx->stream_g));
    CK(cudaStreamSynchronize(ctx->stream));
    return SPH_OK;
}

const char *sph_last_error(sph_ctx *ctx) { return ctx ? ctx->err.c_str() : "null context"; }

int sph_get_config(sph_ctx *ctx, sph_config *out) {
    if (!ctx || !out) return SPH_ERR_ARG;
    *out = ctx->cfg;
    return SPH_OK;
}

int sph_set_params(sph_ctx *ctx, const sph_config *c) {
    if (!ctx || !c) return SPH_ERR_ARG;
    sph_config t = ctx->cfg;
    t.av_mode = c->av_mode; t.balsara = c->balsara; t.flags = c->flags;
    t.n_ngb = c->n_ngb; t.h_tol = c->h_tol; t.h_max_iter = c->h_max_iter;
    t.gamma = c->gamma; t.alpha = c->alpha; t.beta = c->beta; t.eta = c->eta;
    t.G = c->G; t.eps = c->eps; t.theta = c->theta; t.courant = c->courant;
    t.dt_max = c->dt_max; t.dt_fixed = c->dt_fixed;
    t.ngb_lanes = c->ngb_lanes; t.block_size = c->block_size; t.leaf_size = c->leaf_size;
    t.walk_blocks = c->walk_blocks;
    t.theta_small = c->theta_small; t.small_cell = c->small_cell;
    t.dt_mode = c->dt_mode;
    t.ext_sigma = c->ext_sigma;
    t.rebuild_every = c->rebuild_every;
    int rc = check_cfg(&t);
    if (rc) return rc;
    if (t.theta != ctx->cfg.theta || t.leaf_size != ctx->cfg.leaf_size ||
        t.theta_small != ctx->cfg.theta_small || t.small_cell != ctx->cfg.small_cell)
        ctx->tree_ok = false;
    ctx->cfg = t;
    drop_graphs(ctx);
    ctx->p2_dirty = true;
    return SPH_OK;
}

int64_t sph_device_bytes(sph_ctx *ctx) { return ctx ? ctx->dev_bytes : 0; }

int sph_load(sph_ctx *ctx, int32_t n, const int32_t *cloud, const double *x, const double *y,
             const double *z, const double *vx, const double *vy, const double *vz,
             const double *m, const double *h, const double *u, int32_t host) {
    int rc = enter(ctx);
    if (rc) return rc;
    if (n < 0 || (n > 0 && (!x || !y || !z || !m || !h || !u))) return SPH_ERR_ARG;
    if (n > ctx->cfg.n_max) return SPH_ERR_CAPACITY;
    drop_graphs(ctx);
    CK(cudaStreamSynchronize(ctx->stream));
    // clouds: counts per id on the host
    std::vector<int> cl(n > 0 ? n : 1, 0);
    if (cloud) {
        if (host) memcpy(cl.data(), cloud, sizeof(int) * n);
        else CK(cudaMemcpy(cl.data(), cloud, sizeof(int) * n, cudaMemcpyDeviceToHost));
    }
    int ncl = 1;
    for (int i = 0; i < n; i++) {
        if (cl[i] < 0 || cl[i] >= ctx->cfg.n_cloud_max) return SPH_ERR_CAPACITY;
        ncl = std::max(ncl, cl[i] + 1);
    }
    std::vector<int> cnt(ncl, 0);
    for (int i = 0; i < n; i++) cnt[cl[i]]++;
    ctx->cloud_start_h.assign(ncl + 1, 0);
    for (int k = 0; k < ncl; k++) ctx->cloud_start_h[k + 1] = ctx->cloud_start_h[k] + cnt[k];
    ctx->n = n;
    ctx->ncloud = ncl;
    ctx->ngroup = n + ncl;
    ctx->cur = 0;
    cudaStream_t s = ctx->stream;
    cudaMemcpyKind kind = host ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice;
    const double *src[ST_N] = {x, y, z, vx, vy, vz, m, h, u, nullptr};
    for (int k = 0; k < ST_N; k++) {
        if (n == 0) break;
        if (src[k]) CK(cudaMemcpyAsync(ctx->st[0][k], src[k], sizeof(double) * n, kind, s));
        else CK(cudaMemsetAsync(ctx->st[0][k], 0, sizeof(double) * n, s));
    }
    if (n > 0) {
        CK(cudaMemcpyAsync(ctx->cloud[0], cl.data(), sizeof(int) * n, cudaMemcpyHostToDevice, s));
        k_iota<<<div_up(n, 256), 256, 0, s>>>(n, ctx->id[0]);
    }
    CK(cudaMemcpyAsync(ctx->cloud_start, ctx->cloud_start_h.data(), sizeof(int) * (ncl + 1),
                       cudaMemcpyHostToDevice, s));
    CK(cudaMemsetAsync(ctx->d_ngroup, 0, sizeof(int), s));
    CK(cudaMemsetAsync(ctx->dt_bits, 0xff, sizeof(unsigned long long) * ncl, s));
    {
        std::vector<double> dt0(ncl, ctx->cfg.dt_fixed > 0 ? ctx->cfg.dt_fixed : 0.0);
        CK(cudaMemcpyAsync(ctx->dt, dt0.data(), sizeof(double) * ncl, cudaMemcpyHostToDevice, s));
    }
    if (n > 0) {
        CK(cudaMemsetAsync(ctx->asph, 0, 3 * sizeof(double) * n, s));
        CK(cudaMemsetAsync(ctx->agrav, 0, 3 * sizeof(double) * n, s));
        CK(cudaMemsetAsync(ctx->divV, 0, sizeof(double) * n, s));
        CK(cudaMemsetAsync(ctx->curlV, 0, sizeof(double) * n, s));
        CK(cudaMemsetAsync(ctx->pot, 0, sizeof(double) * n, s));
        rc = launch_pack_p1(ctx);
        if (rc) return rc;
    }
    CK(cudaStreamSynchronize(s));
    ctx->tree_ok = ctx->lists_ok = ctx->rho_ok = ctx->divcurl_ok = ctx->cand_ok = false;
    ctx->p2_dirty = true;
    ctx->prologue_done = false;
    ctx->step_count = 0;
    ctx->last_injected_id = -1;
    ctx->topo_ok = false;
    return ctx_check_launch(ctx, "load");
}

int32_t sph_count(sph_ctx *ctx) { return ctx ? ctx->n : -1; }
int32_t sph_cloud_count(sph_ctx *ctx) { return ctx ? ctx->ncloud : -1; }

int sph_get_field(sph_ctx *ctx, int32_t field, double *out, int32_t host, int32_t storage_order) {
    int rc = enter(ctx);
    if (rc) return rc;
    double *src = field_ptr(ctx, field);
    if (!src || !out) return SPH_ERR_ARG;
    const int n = ctx->n;
    if (n == 0) return SPH_OK;
    cudaStream_t s = ctx->stream;
    CK(cudaStreamSynchronize(ctx->stream_g));
    const double *from = src;
    if (!storage_order) {
        k_scatter_by_id<<<div_up(n, 256), 256, 0, s>>>(n, ctx->id[ctx->cur], src, ctx->red);
        from = ctx->red;
    }
    CK(cudaMemcpyAsync(out, from, sizeof(double) * n,
                       host ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice, s));
    CK(cudaStreamSynchronize(s));
    return ctx_check_launch(ctx, "get_field");
}

int sph_set_field(sph_ctx *ctx, int32_t field, const double *in, int32_t host,
                  int32_t storage_order) {
    int rc = enter(ctx);
    if (rc) return rc;
    double *dst = field_ptr(ctx, field);
    if (!dst || !in) return SPH_ERR_ARG;
    const int n = ctx->n;
    if (n == 0) return SPH_OK;
    cudaStream_t s = ctx->stream;
    cudaMemcpyKind kind = host ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice;
    if (storage_order) {
        CK(cudaMemcpyAsync(dst, in, sizeof(double) * n, kind, s));
    } else {
        CK(cudaMemcpyAsync(ctx->red, in, sizeof(double) * n, kind, s));
        k_gather_by_id<<<div_up(n, 256), 256, 0, s>>>(n, ctx->id[ctx->cur], ctx->red, dst);
    }
    if (field <= SPH_F_H) {
        rc = launch_pack_p1(ctx, true);
        if (rc) return rc;
        if (field <= SPH_F_Z || field == SPH_F_M) ctx->tree_ok = false;
        ctx->cand_ok = false;
    }
    if (field == SPH_F_H || (field >= SPH_F_RHO && field <= SPH_F_CURLV)) ctx->p2_dirty = true;
    CK(cudaStreamSynchronize(s));
    return ctx_check_launch(ctx, "set_field");
}

// several fields in one call: the copies (and the order permutations) are
// queued back to back on the context stream through one scratch array, the
// particle records are rebuilt once, and the call returns after one
// synchronisation
int sph_set_fields(sph_ctx *ctx, int32_t nfield, const int32_t *fields, const double *const *in,
                   int32_t host, int32_t storage_order) {
    int rc = enter(ctx);
    if (rc) return rc;
    if (nfield < 0 || (nfield > 0 && (!fields || !in))) return SPH_ERR_ARG;
    for (int k = 0; k < nfield; k++)
        if (!field_ptr(ctx, fields[k]) || !in[k]) return SPH_ERR_ARG;
    const int n = ctx->n;
    if (n == 0 || nfield == 0) return SPH_OK;
    cudaStream_t s = ctx->stream;
    const cudaMemcpyKind kind = host ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice;
    bool pack = false;
    for (int k = 0; k < nfield; k++) {
        const int field = fields[k];
        double *dst = field_ptr(ctx, field);
        if (storage_order) {
            CK(cudaMemcpyAsync(dst, in[k], sizeof(double) * n, kind, s));
        } else {
            CK(cudaMemcpyAsync(ctx->red, in[k], sizeof(double) * n, kind, s));
            k_gather_by_id<<<div_up(n, 256), 256, 0, s>>>(n, ctx->id[ctx->cur], ctx->red, dst);
        }
        if (field <= SPH_F_H) {
            pack = true;
            if (field <= SPH_F_Z || field == SPH_F_M) ctx->tree_ok = false;
            ctx->cand_ok = false;
        }
        if (field == SPH_F_H || (field >= SPH_F_RHO && field <= SPH_F_CURLV)) ctx->p2_dirty = true;
    }
    if (pack && (rc = launch_pack_p1(ctx, true))) return rc;
    CK(cudaStreamSynchronize(s));
    return ctx_check_launch(ctx, "set_fields");
}

int sph_get_fields(sph_ctx *ctx, int32_t nfield, const int32_t *fields, double *const *out,
                   int32_t host, int32_t storage_order) {
    int rc = enter(ctx);
    if (rc) return rc;
    if (nfield < 0 || (nfield > 0 && (!fields || !out))) return SPH_ERR_ARG;
    for (int k = 0; k < nfield; k++)
        if (!field_ptr(ctx, fields[k]) || !out[k]) return SPH_ERR_ARG;
    const int n = ctx->n;
    if (n == 0 || nfield == 0) return SPH_OK;
    cudaStream_t s = ctx->stream;
    CK(cudaStreamSynchronize(ctx->stream_g));
    const cudaMemcpyKind kind = host ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice;
    for (int k = 0; k < nfield; k++) {
        const double *from = field_ptr(ctx, fields[k]);
        if (!storage_order) {
            k_scatter_by_id<<<div_up(n, 256), 256, 0, s>>>(n, ctx->id[ctx->cur], from, ctx->red);
            from = ctx->red;
        }
        CK(cudaMemcpyAsync(out[k], from, sizeof(double) * n, kind, s));
    }
    CK(cudaStreamSynchronize(s));
    return ctx_check_launch(ctx, "get_fields");
}

int sph_get_ids(sph_ctx *ctx, int32_t *out, int32_t host) {
    int rc = enter(ctx);
    if (rc) return rc;
    if (!out) return SPH_ERR_ARG;
    if (ctx->n == 0) return SPH_OK;
    CK(cudaMemcpyAsync(out, ctx->id[ctx->cur], sizeof(int) * ctx->n,
                       host ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return SPH_OK;
}

int sph_get_status(sph_ctx *ctx, int64_t *out, int32_t reset) {
    int rc = enter(ctx);
    if (rc) return rc;
    if (!out) return SPH_ERR_ARG;
    CK(cudaStreamSynchronize(ctx->stream_g));
    CK(cudaMemcpyAsync(out, ctx->status, sizeof(long long) * SPH_NSTATUS, cudaMemcpyDeviceToHost,
                       ctx->stream));
    if (reset) CK(cudaMemsetAsync(ctx->status, 0, sizeof(long long) * SPH_NSTATUS, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return SPH_OK;
}

int sph_get_dt(sph_ctx *ctx, double *dt) {
    int rc = enter(ctx);
    if (rc) return rc;
    if (!dt) return SPH_ERR_ARG;
    CK(cudaMemcpyAsync(dt, ctx->dt, sizeof(double) * ctx->ncloud, cudaMemcpyDeviceToHost,
                       ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return SPH_OK;
}

int sph_set_dt(sph_ctx *ctx, const double *dt) {
    int rc = enter(ctx);
    if (rc) return rc;
    if (!dt) return SPH_ERR_ARG;
    CK(cudaMemcpyAsync(ctx->dt, dt, sizeof(double) * ctx->ncloud, cudaMemcpyHostToDevice,
                       ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return SPH_OK;
}

int sph_sort(sph_ctx *ctx) {
    int rc = enter(ctx);
    if (rc) return rc;
    drop_graphs(ctx);
    rc = launch_sort(ctx);
    ctx->tree_ok = ctx->lists_ok = ctx->rho_ok = ctx->divcurl_ok = ctx->cand_ok = false;
    ctx->p2_dirty = true;
    return rc;
}

int sph_get_sort(sph_ctx *ctx, uint64_t *keys, int32_t *perm, int32_t host) {
    int rc = enter(ctx);
    if (rc) return rc;
    const int n = ctx->n;
    if (n == 0) return SPH_OK;
    cudaMemcpyKind k = host ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice;
    if (keys) CK(cudaMemcpyAsync(keys, ctx->key_in, sizeof(uint64_t) * n, k, ctx->stream));
    if (perm) CK(cudaMemcpyAsync(perm, ctx->val[0], sizeof(int) * n, k, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return SPH_OK;
}

int sph_build_tree(sph_ctx *ctx) {
    int rc = enter(ctx);
    if (rc) return rc;
    return launch_tree(ctx);
}

int sph_get_tree(sph_ctx *ctx, double *node, int32_t *child, int32_t *first, int32_t *last,
                 double *open_r2, double *hmax, int32_t host) {
    int rc = enter(ctx);
    if (rc) return rc;
    if (!ctx->tree_ok) return SPH_ERR_STATE;
    const size_t nn = ctx->n > 0 ? 2 * (size_t)ctx->n - 1 : 0;
    if (nn == 0) return SPH_OK;
    cudaMemcpyKind k = host ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice;
    cudaStream_t s = ctx->stream;
    if (node) {
        // the step stores the build records of the group nodes and above
        // only: recompute the rest for the current topology first
        if (!ctx->records_all && (rc = launch_tree_records(ctx))) return rc;
        if ((rc = launch_leaf_records(ctx))) return rc;
        CK(cudaMemcpyAsync(node, ctx->node, 16 * sizeof(double) * nn, k, s));
    }
    if (child) CK(cudaMemcpyAsync(child, ctx->child, 2 * sizeof(int) * nn, k, s));
    if (first) CK(cudaMemcpyAsync(first, ctx->first, sizeof(int) * nn, k, s));
    if (last) CK(cudaMemcpyAsync(last, ctx->last, sizeof(int) * nn, k, s));
    if (open_r2) CK(cudaMemcpyAsync(open_r2, ctx->ropen2, sizeof(double) * nn, k, s));
    if (hmax) CK(cudaMemcpyAsync(hmax, ctx->hmax, sizeof(double) * nn, k, s));
    CK(cudaStreamSynchronize(s));
    return SPH_OK;
}

int sph_smoothing_h(sph_ctx *ctx) {
    int rc = enter(ctx);
    if (rc) return rc;
    if (!ctx->tree_ok) return SPH_ERR_STATE;
    drop_graphs(ctx);
    return launch_smoothing_h(ctx);
}

int sph_smoothing_h_count(sph_ctx *ctx, int32_t n_target, int32_t n_tol, double step_frac,
                          int32_t max_iter) {
    int rc = enter(ctx);
    if (rc) return rc;
    if (!ctx->tree_ok) return SPH_ERR_STATE;
    if (n_target < 1 || n_tol < 0 || n_tol >= n_target || n_target + n_tol > ctx->cfg.max_ngb ||
        !(step_frac > 0.0 && step_frac < 0.5) || max_iter < 1)
        return SPH_ERR_ARG;
    drop_graphs(ctx);
    return launch_smoothing_h_count(ctx, n_target, n_tol, step_frac, max_iter);
}

int sph_smoothing_length_kth(sph_ctx *ctx, int32_t k) {
    int rc = enter(ctx);
    if (rc) return rc;
    if (!ctx->tree_ok) return SPH_ERR_STATE;
    if (k < 0 || k + 1 > ctx->cfg.max_ngb) return SPH_ERR_ARG;
    drop_graphs(ctx);
    return launch_smoothing_kth(ctx, k);
}

int sph_neighbours(sph_ctx *ctx) {
    int rc = enter(ctx);
    if (rc) return rc;
    if (!ctx->tree_ok) return SPH_ERR_STATE;
    return launch_neighbours(ctx);
}

int sph_get_neighbours(sph_ctx *ctx, int64_t *off, int32_t *lst, int64_t cap, int32_t host) {
    int rc = enter(ctx);
    if (rc) return rc;
    if (!ctx->lists_ok) return SPH_ERR_STATE;
    if (!off) return SPH_ERR_ARG;
    const int n = ctx->n;
    std::vector<int> cnt(n);
    std::vector<long long> o(n + 1, 0);
    if (n) CK(cudaMemcpyAsync(cnt.data(), ctx->ngb_cnt, sizeof(int) * n, cudaMemcpyDeviceToHost,
                              ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    for (int i = 0; i < n; i++) o[i + 1] = o[i] + cnt[i];
    if (host) memcpy(off, o.data(), sizeof(long long) * (n + 1));
    else {
        CK(cudaMemcpyAsync(off, o.data(), sizeof(long long) * (n + 1), cudaMemcpyHostToDevice,
                           ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
    }
    if (!lst) return SPH_OK;
    if (o[n] > cap) return SPH_ERR_CAPACITY;
    long long *doff = nullptr;
    int *dl = nullptr;
    CK(cudaMalloc(&doff, sizeof(long long) * (n + 1)));
    CK(cudaMalloc(&dl, sizeof(int) * std::max<long long>(o[n], 1)));
    CK(cudaMemcpyAsync(doff, o.data(), sizeof(long long) * (n + 1), cudaMemcpyHostToDevice,
                       ctx->stream));
    rc = launch_export_neighbours(ctx, (int64_t *)doff, dl, o[n]);
    if (!rc) {
        CK(cudaMemcpyAsync(lst, dl, sizeof(int) * o[n],
                           host ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice, ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
    }
    cudaFree(doff);
    cudaFree(dl);
    return rc;
}

int sph_density(sph_ctx *ctx) {
    int rc = enter(ctx);
    if (rc) return rc;
    if (!ctx->lists_ok) return SPH_ERR_STATE;
    return launch_density(ctx);
}

int sph_divcurl(sph_ctx *ctx) {
    int rc = enter(ctx);
    if (rc) return rc;
    if (!ctx->lists_ok) return SPH_ERR_STATE;
    if (ctx->p2_dirty) {
        rc = launch_repack_p2(ctx);
        if (rc) return rc;
    }
    return launch_divcurl(ctx);
}

int sph_forces(sph_ctx *ctx) {
    int rc = enter(ctx);
    if (rc) return rc;
    if (!ctx->lists_ok) return SPH_ERR_STATE;
    return launch_forces(ctx, true, (ctx->cfg.flags & SPH_FLAG_DUDT_FUSED) != 0, false);
}

int sph_dudt(sph_ctx *ctx) {
    int rc = enter(ctx);
    if (rc) return rc;
    if (!ctx->lists_ok) return SPH_ERR_STATE;
    return launch_forces(ctx, false, true, false);
}

int sph_gravity(sph_ctx *ctx) {
    int rc = enter(ctx);
    if (rc) return rc;
    if (!ctx->tree_ok) return SPH_ERR_STATE;
    return launch_gravity(ctx, ctx->stream, (ctx->cfg.flags & SPH_FLAG_POTENTIAL) != 0);
}

static int direct_common(sph_ctx *ctx, const double *eps, int32_t nt, const int32_t *targets,
                         double *out, int32_t host, int width, int nbeg = 0, int nend = -1) {
    int rc = enter(ctx);
    if (rc) return rc;
    if (nt < 0 || (nt > 0 && (!targets || !out))) return SPH_ERR_ARG;
    if (nt == 0) return SPH_OK;
    for (int t = 0; host && t < nt; t++)
        if (targets[t] < 0 || targets[t] >= ctx->n) return SPH_ERR_ARG;
    int *dt_ = nullptr;
    double *dout = nullptr, *deps = nullptr;
    CK(cudaMalloc(&dt_, sizeof(int) * nt));
    CK(cudaMalloc(&dout, sizeof(double) * width * nt));
    cudaMemcpyKind kin = host ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice;
    // copies on the context's non-blocking stream, ordered before the kernels
    CK(cudaMemcpyAsync(dt_, targets, sizeof(int) * nt, kin, ctx->stream));
    if (eps) {
        CK(cudaMalloc(&deps, sizeof(double) * ctx->n));
        CK(cudaMemcpyAsync(deps, eps, sizeof(double) * ctx->n, kin, ctx->stream));
        // eps is given in the caller's original order: bring it to storage order
        k_gather_by_id<<<div_up(ctx->n, 256), 256, 0, ctx->stream>>>(ctx->n, ctx->id[ctx->cur],
                                                                      deps, ctx->red);
        rc = launch_gravity_direct_spline(ctx, ctx->red, nt, dt_, dout, nbeg,
                                          nend < 0 ? ctx->n : nend);
    } else {
        rc = launch_gravity_direct(ctx, nt, dt_, dout);
    }
    if (!rc) {
        CK(cudaMemcpyAsync(out, dout, sizeof(double) * width * nt,
                           host ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice, ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
    }
    cudaFree(dt_);
    cudaFree(dout);
    if (deps) cudaFree(deps);
    return rc;
}

int sph_gravity_direct(sph_ctx *ctx, int32_t nt, const int32_t *targets, double *out, int32_t host) {
    return direct_common(ctx, nullptr, nt, targets, out, host, 4);
}

int sph_gravity_direct_spline(sph_ctx *ctx, const double *eps, int32_t nt, const int32_t *targets,
                              double *out, int32_t host) {
    if (!eps) return SPH_ERR_ARG;
    return direct_common(ctx, eps, nt, targets, out, host, 3);
}

int sph_gravity_direct_spline_rows(sph_ctx *ctx, const double *eps, int32_t nbeg, int32_t nend,
                                   double *out, int32_t host) {
    int rc = enter(ctx);
    if (rc) return rc;
    const int n = ctx->n;
    if (!eps || !out || nbeg < 0 || nend < nbeg || nend > n) return SPH_ERR_ARG;
    if (n == 0) return SPH_OK;
    // every stored particle is a target; the result is scattered back to the
    // caller's original order row by row
    std::vector<int> all(n);
    std::iota(all.begin(), all.end(), 0);
    std::vector<double> st(3 * (size_t)n), orig(3 * (size_t)n);
    rc = direct_common(ctx, eps, n, all.data(), st.data(), 1, 3, nbeg, nend);
    if (rc) return rc;
    std::vector<int> id(n);
    CK(cudaMemcpy(id.data(), ctx->id[ctx->cur], sizeof(int) * n, cudaMemcpyDeviceToHost));
    for (int s = 0; s < n; s++)
        for (int k = 0; k < 3; k++) orig[3 * (size_t)id[s] + k] = st[3 * (size_t)s + k];
    if (host) memcpy(out, orig.data(), sizeof(double) * 3 * n);
    else CK(cudaMemcpy(out, orig.data(), sizeof(double) * 3 * n, cudaMemcpyHostToDevice));
    return SPH_OK;
}

int sph_kick(sph_ctx *ctx, double fac) {
    int rc = enter(ctx);
    if (rc) return rc;
    return launch_kick(ctx, fac, false);
}

int sph_drift(sph_ctx *ctx) {
    int rc = enter(ctx);
    if (rc) return rc;
    ctx->tree_ok = ctx->lists_ok = ctx->cand_ok = false;
    return launch_drift(ctx);
}

int sph_update_u(sph_ctx *ctx, int32_t first) {
    int rc = enter(ctx);
    if (rc) return rc;
    return launch_update_u(ctx, first != 0);
}

int sph_cfl_dt(sph_ctx *ctx, double *dt) {
    int rc = enter(ctx);
    if (rc) return rc;
    rc = launch_cfl(ctx);
    if (rc) return rc;
    if (dt) return sph_get_dt(ctx, dt);
    return SPH_OK;
}

int sph_dt_individual(sph_ctx *ctx, double *dt, double *dhdt, int32_t *bin, int32_t host) {
    int rc = enter(ctx);
    if (rc) return rc;
    if (!ctx->lists_ok || !ctx->rho_ok) return SPH_ERR_STATE;
    CK(cudaStreamSynchronize(ctx->stream_g));
    if ((rc = launch_dt_individual(ctx))) return rc;
    if ((rc = launch_dt_bins(ctx))) return rc;
    if ((rc = launch_dt_commit(ctx))) return rc;
    const int n = ctx->n;
    cudaStream_t s = ctx->stream;
    const cudaMemcpyKind k = host ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice;
    const int *id = ctx->id[ctx->cur];
    double *buf = ctx->red;
    if (n > 0 && dt) {
        k_scatter_by_id<<<div_up(n, 256), 256, 0, s>>>(n, id, ctx->dt_part, buf);
        CK(cudaMemcpyAsync(dt, buf, sizeof(double) * n, k, s));
        CK(cudaStreamSynchronize(s));
    }
    if (n > 0 && dhdt) {
        k_scatter_by_id<<<div_up(n, 256), 256, 0, s>>>(n, id, ctx->dhdt, buf);
        CK(cudaMemcpyAsync(dhdt, buf, sizeof(double) * n, k, s));
        CK(cudaStreamSynchronize(s));
    }
    if (n > 0 && bin) {
        k_scatter_int_by_id<<<div_up(n, 256), 256, 0, s>>>(n, id, ctx->dbin, (int *)buf);
        CK(cudaMemcpyAsync(bin, buf, sizeof(int) * n, k, s));
        CK(cudaStreamSynchronize(s));
    }
    CK(cudaStreamSynchronize(s));
    return ctx_check_launch(ctx, "dt_individual");
}

int sph_outflow_inject(sph_ctx *ctx, const sph_outflow_params *p, double *leftover_mass,
                       int32_t *n_added) {
    int rc = enter(ctx);
    if (rc) return rc;
    if (!p || !leftover_mass) return SPH_ERR_ARG;
    if (n_added) *n_added = 0;
    if (ctx->ncloud < 1 || p->cloud != ctx->ncloud - 1) return SPH_ERR_ARG;
    if (!(p->m_particle > 0.0) || !(p->mdot >= 0.0) || !(p->r_max >= 0.0) ||
        !(p->h_first > 0.0) || !(*leftover_mass >= 0.0))
        return SPH_ERR_ARG;
    double dt = 0.0;
    CK(cudaStreamSynchronize(ctx->stream_g));
    CK(cudaMemcpyAsync(&dt, ctx->dt + p->cloud, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    double mass = p->mdot * dt + *leftover_mass;
    const double pairs_d = floor(mass / (2.0 * p->m_particle));
    if (pairs_d < 0.0 || pairs_d > (double)(ctx->cfg.n_max - ctx->n) / 2.0) return SPH_ERR_CAPACITY;
    const int npairs = (int)pairs_d;
    if (npairs > 0) {
        drop_graphs(ctx);
        rc = launch_inject_pairs(ctx, npairs, p->seed, p->cloud, p->r_max, p->v_in, p->m_particle,
                                 p->u_inject, ctx->last_injected_id, p->h_first);
        if (rc) return rc;
        const int n1 = ctx->n + 2 * npairs;
        ctx->cloud_start_h[ctx->ncloud] = n1;
        CK(cudaMemcpyAsync(ctx->cloud_start + ctx->ncloud, &ctx->cloud_start_h[ctx->ncloud],
                           sizeof(int), cudaMemcpyHostToDevice, ctx->stream));
        ctx->n = n1;
        ctx->ngroup = n1 + ctx->ncloud;
        ctx->last_injected_id = n1 - 1;
        if ((rc = launch_pack_p1(ctx))) return rc;
        CK(cudaStreamSynchronize(ctx->stream));
        ctx->tree_ok = ctx->lists_ok = ctx->rho_ok = ctx->divcurl_ok = ctx->cand_ok = false;
        ctx->topo_ok = false;  // new particles: the next step sorts and splits again
        ctx->p2_dirty = true;
        mass -= 2.0 * p->m_particle * npairs;
    }
    *leftover_mass = mass;
    if (n_added) *n_added = 2 * npairs;
    return ctx_check_launch(ctx, "outflow_inject");
}

int sph_energies(sph_ctx *ctx, double *out10) {
    int rc = enter(ctx);
    if (rc) return rc;
    if (!out10) return SPH_ERR_ARG;
    CK(cudaStreamSynchronize(ctx->stream_g));
    return launch_energies(ctx, out10);
}

int sph_get_far_cells(sph_ctx *ctx, int64_t *out) {
    int rc = enter(ctx);
    if (rc) return rc;
    if (!out) return SPH_ERR_ARG;
    CK(cudaStreamSynchronize(ctx->stream_g));
    long long c[2];
    CK(cudaMemcpyAsync(c, ctx->counters + 2, 2 * sizeof(long long), cudaMemcpyDeviceToHost,
                       ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    *out = c[0] + c[1];
    return SPH_OK;
}

int sph_get_supergroup_stats(sph_ctx *ctx, int64_t *out2) {
    int rc = enter(ctx);
    if (rc) return rc;
    if (!out2) return SPH_ERR_ARG;
    CK(cudaStreamSynchronize(ctx->stream_g));
    CK(cudaMemcpyAsync(out2, ctx->counters + 3, 2 * sizeof(long long), cudaMemcpyDeviceToHost,
                       ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return SPH_OK;
}

int sph_get_counters(sph_ctx *ctx, int64_t *out2) {
    int rc = enter(ctx);
    if (rc) return rc;
    if (!out2) return SPH_ERR_ARG;
    CK(cudaStreamSynchronize(ctx->stream_g));
    CK(cudaMemcpyAsync(out2, ctx->counters, 2 * sizeof(long long), cudaMemcpyDeviceToHost,
                       ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return SPH_OK;
}

int sph_prologue(sph_ctx *ctx) {
    int rc = enter(ctx);
    if (rc) return rc;
    drop_graphs(ctx);
    const bool pot = ctx->cfg.flags & SPH_FLAG_POTENTIAL;
    ctx->prologue_done = false;
    if ((rc = launch_sort(ctx))) return rc;
    if ((rc = launch_tree(ctx))) return rc;
    if ((rc = launch_gravity(ctx, ctx->stream, pot))) return rc;
    if ((rc = launch_smoothing_h(ctx))) return rc;
    if ((rc = launch_neighbours(ctx))) return rc;
    if ((rc = launch_density_divcurl(ctx))) return rc;
    if ((rc = launch_forces(ctx, true, true, false))) return rc;
    // first dt (fixed, Courant or individual), then u += du/dt dt
    // (sph_mpi4_v4.py:240-244)
    if (ctx->cfg.dt_fixed <= 0.0 && ctx->cfg.dt_mode == SPH_DT_INDIVIDUAL) {
        if ((rc = launch_dt_individual(ctx))) return rc;
        if ((rc = launch_dt_commit(ctx))) return rc;
    } else if ((rc = launch_cfl(ctx))) {
        return rc;
    }
    if ((rc = launch_update_u(ctx, true))) return rc;
    CK(cudaStreamSynchronize(ctx->stream));
    ctx->prologue_done = true;
    return ctx_check_launch(ctx, "prologue");
}

}  // extern "C"

namespace {

// one step on ctx->stream: the body in eager mode, else the CUDA graph of
// the current buffer parity and step kind (captured on first use).  Every
// rebuild_every-th step (and the first after the topology was invalidated)
// sorts and rebuilds the tree; the steps between refit it.
int step_launch(sph_ctx *ctx) {
    int rc;
    const int every = ctx->cfg.rebuild_every;
    const bool refit = every > 1 && ctx->topo_ok && ctx->refits + 1 < every;
    if (ctx->cfg.flags & SPH_FLAG_NO_GRAPH) {
        if ((rc = step_body(ctx, refit))) return rc;
    } else {
        const int par = ctx->cur;
        cudaGraphExec_t &gx = ctx->graph[par][refit ? 1 : 0];
        if (!gx) {
            cudaGraph_t g = nullptr;
            CK(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
            rc = step_body(ctx, refit);
            cudaError_t e = cudaStreamEndCapture(ctx->stream, &g);
            ctx->cur = par;  // capture did not run anything: restore the parity
            if (rc) {
                if (g) cudaGraphDestroy(g);
                return rc;
            }
            if (e != cudaSuccess) return ctx_fail(ctx, e, "cudaStreamEndCapture", __LINE__);
            e = cudaGraphInstantiate(&gx, g, 0);
            {
                size_t nn = 0;
                cudaGraphGetNodes(g, nullptr, &nn);
                std::vector<cudaGraphNode_t> nodes(nn);
                if (nn) cudaGraphGetNodes(g, nodes.data(), &nn);
                int kc = 0;
                for (size_t q = 0; q < nn; q++) {
                    cudaGraphNodeType t;
                    if (cudaGraphNodeGetType(nodes[q], &t) == cudaSuccess &&
                        t == cudaGraphNodeTypeKernel)
                        kc++;
                }
                ctx->graph_kernels = kc;
                ctx->graph_nk[par][refit ? 1 : 0] = kc;
            }
            cudaGraphDestroy(g);
            if (e != cudaSuccess) return ctx_fail(ctx, e, "cudaGraphInstantiate", __LINE__);
        }
        CK(cudaGraphLaunch(gx, ctx->stream));
        ctx->graph_kernels_launched += ctx->graph_nk[par][refit ? 1 : 0];
        ctx->rows_host = true;  // every step ends with the rows of its h iteration
        if (!refit) ctx->cur = par ^ 1;
    }
    if (refit) {
        ctx->refits++;
    } else {
        ctx->refits = 0;
        ctx->topo_ok = true;
    }
    ctx->step_count++;
    return SPH_OK;
}

// the step's event after which a field holds its value at the end of the
// step: positions and masses after the sort (the drift came before it), h
// after the neighbour pass, velocities after the closing kick, the rest at
// the end
int io_event(int field) {
    if (field <= SPH_F_Z || field == SPH_F_M) return 0;
    if (field == SPH_F_H) return 1;
    if (field <= SPH_F_VZ) return 2;
    return 3;
}

}  // namespace

extern "C" {

int sph_step(sph_ctx *ctx, int32_t nsteps) {
    int rc = enter(ctx);
    if (rc) return rc;
    if (nsteps < 0) return SPH_ERR_ARG;
    if (!ctx->prologue_done) return SPH_ERR_STATE;
    if (ctx->n == 0) return SPH_OK;
    for (int k = 0; k < nsteps; k++)
        if ((rc = step_launch(ctx))) return rc;
    ctx->tree_ok = ctx->lists_ok = ctx->rho_ok = ctx->divcurl_ok = true;
    return ctx_check_launch(ctx, "step");
}

int sph_step_io(sph_ctx *ctx, int32_t nin, const int32_t *fin, const double *const *in,
                int32_t nout, const int32_t *fout, double *const *out) {
    int rc = enter(ctx);
    if (rc) return rc;
    if (nin < 0 || nout < 0 || (nin > 0 && (!fin || !in)) || (nout > 0 && (!fout || !out)))
        return SPH_ERR_ARG;
    for (int k = 0; k < nin; k++)
        if (!field_ptr(ctx, fin[k]) || !in[k]) return SPH_ERR_ARG;
    for (int k = 0; k < nout; k++)
        if (!field_ptr(ctx, fout[k]) || !out[k]) return SPH_ERR_ARG;
    if (!ctx->prologue_done) return SPH_ERR_STATE;
    const int n = ctx->n;
    if (n == 0) return SPH_OK;
    // one staging slot of n_max doubles per field of the larger list, and the
    // copy stream, made on first use
    const int slots = std::max(std::max(nin, nout), 1);
    if (slots > ctx->io_slots) {
        CK(cudaStreamSynchronize(ctx->stream));
        if (ctx->stream_io) CK(cudaStreamSynchronize(ctx->stream_io));
        if (ctx->io_stage) cudaFree(ctx->io_stage);
        ctx->io_stage = nullptr;
        ctx->io_slots = 0;
        void *p = nullptr;
        cudaError_t e = cudaMalloc(&p, sizeof(double) * (size_t)slots * ctx->cfg.n_max);
        if (e != cudaSuccess) return ctx_fail(ctx, e, "cudaMalloc", __LINE__);
        ctx->io_stage = (double *)p;
        ctx->io_slots = slots;
    }
    if (!ctx->stream_io) {
        int lo = 0, hi = 0;
        cudaDeviceGetStreamPriorityRange(&lo, &hi);
        CK(cudaStreamCreateWithPriority(&ctx->stream_io, cudaStreamNonBlocking, hi));
    }
    cudaStream_t s = ctx->stream;
    // in: every copy first (back to back on the copy engine), then the
    // scatters into storage order; the step's first kernels need them all
    for (int k = 0; k < nin; k++)
        CK(cudaMemcpyAsync(ctx->io_stage + (size_t)k * n, in[k], sizeof(double) * n,
                           cudaMemcpyHostToDevice, s));
    bool pack = false;
    for (int k = 0; k < nin; k++) {
        const int field = fin[k];
        k_gather_by_id<<<div_up(n, 256), 256, 0, s>>>(n, ctx->id[ctx->cur],
                                                       ctx->io_stage + (size_t)k * n,
                                                       field_ptr(ctx, field));
        if (field <= SPH_F_H) {
            pack = true;
            if (field <= SPH_F_Z || field == SPH_F_M) ctx->tree_ok = false;
            ctx->cand_ok = false;
        }
        if (field == SPH_F_H || (field >= SPH_F_RHO && field <= SPH_F_CURLV)) ctx->p2_dirty = true;
    }
    if (pack && (rc = launch_pack_p1(ctx, true))) return rc;
    if ((rc = step_launch(ctx))) return rc;
    ctx->tree_ok = ctx->lists_ok = ctx->rho_ok = ctx->divcurl_ok = true;
    // out: on the copy stream, each field gathered into caller order and
    // copied out as soon as the step has written its last value; the rest
    // of the step runs meanwhile.  ctx->cur is the step's output buffer.
    int waited = -1;
    for (int ev = 0; ev < 4; ev++) {
        for (int k = 0; k < nout; k++) {
            if (io_event(fout[k]) != ev) continue;
            if (waited < ev) {
                CK(cudaStreamWaitEvent(ctx->stream_io, ctx->ev_io[ev], 0));
                waited = ev;
            }
            double *stage = ctx->io_stage + (size_t)k * n;
            k_scatter_by_id<<<div_up(n, 256), 256, 0, ctx->stream_io>>>(n, ctx->id[ctx->cur],
                                                                        field_ptr(ctx, fout[k]),
                                                                        stage);
            CK(cudaMemcpyAsync(out[k], stage, sizeof(double) * n, cudaMemcpyDeviceToHost,
                               ctx->stream_io));
        }
    }
    CK(cudaStreamSynchronize(ctx->stream_io));
    CK(cudaStreamSynchronize(ctx->stream_g));
    CK(cudaStreamSynchronize(s));
    return ctx_check_launch(ctx, "step_io");
}

int sph_get_phase_times(sph_ctx *ctx, float *ms) {
    int rc = enter(ctx);
    if (rc) return rc;
    if (!ms) return SPH_ERR_ARG;
    if (!ctx->tev_ok) return SPH_ERR_STATE;
    CK(cudaStreamSynchronize(ctx->stream_g));
    CK(cudaStreamSynchronize(ctx->stream));
    for (int k = 0; k < 11; k++) CK(cudaEventElapsedTime(&ms[k], ctx->tev[k], ctx->tev[k + 1]));
    CK(cudaEventElapsedTime(&ms[11], ctx->tev[13], ctx->tev[14]));
    return SPH_NPHASE;
}

__global__ void k_dbg_w(int n, const double4 *p0, const void *p1, int mixed, double *out0,
                        double *out1) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    out0[i] = p0[i].w;
    out1[i] = mixed ? (double)((const float4 *)p1)[i].w : ((const double4 *)p1)[i].w;
}

int sph_debug_copy(sph_ctx *ctx, int32_t which, void *out, int32_t host) {
    int rc = enter(ctx);
    if (rc) return rc;
    if (!out || which < 0 || which > 6) return SPH_ERR_ARG;
    if (which == 6) {
        CK(cudaStreamSynchronize(ctx->stream));
        CK(cudaMemcpy(out, ctx->lflag, sizeof(int) * (ctx->n + 1),
                      host ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice));
        return SPH_OK;
    }
    if (which >= 4) {
        const int n = ctx->n;
        k_dbg_w<<<div_up(n, 256), 256, 0, ctx->stream>>>(n, ctx->p0, ctx->p1,
                                                        ctx->cfg.precision == SPH_PREC_MIXED,
                                                        ctx->red, ctx->red + n);
        CK(cudaStreamSynchronize(ctx->stream));
        CK(cudaMemcpy(out, ctx->red + (which == 4 ? 0 : n), sizeof(double) * n,
                      host ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice));
        return SPH_OK;
    }
    const void *src = which == 0 ? (const void *)ctx->cand_cnt
                      : which == 1 ? (const void *)ctx->ngb_cnt
                      : which == 2 ? (const void *)ctx->retry
                                   : (const void *)ctx->hcand;
    const size_t bytes = (which == 3 ? sizeof(double) : sizeof(int)) * ctx->n;
    CK(cudaStreamSynchronize(ctx->stream));
    CK(cudaMemcpy(out, src, bytes, host ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice));
    return SPH_OK;
}

int sph_time_steps(sph_ctx *ctx, int32_t nsteps, float *ms) {
    int rc = enter(ctx);
    if (rc) return rc;
    if (!ms || nsteps < 0) return SPH_ERR_ARG;
    cudaEvent_t a, b;
    CK(cudaEventCreate(&a));
    if (cudaEventCreate(&b) != cudaSuccess) {
        cudaEventDestroy(a);
        return SPH_ERR_CUDA;
    }
    cudaError_t e = cudaEventRecord(a, ctx->stream);
    if (e == cudaSuccess) rc = sph_step(ctx, nsteps);
    if (e == cudaSuccess && rc == SPH_OK) {
        // the step's gravity stream has joined the main stream inside each step
        e = cudaEventRecord(b, ctx->stream);
        if (e == cudaSuccess) e = cudaEventSynchronize(b);
        if (e == cudaSuccess) e = cudaEventElapsedTime(ms, a, b);
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    if (rc) return rc;
    if (e != cudaSuccess) return ctx_fail(ctx, e, "time_steps", __LINE__);
    return SPH_OK;
}

int sph_graph_kernel_count(sph_ctx *ctx, int32_t *count) {
    if (!ctx || !count) return SPH_ERR_ARG;
    *count = ctx->graph_kernels;
    return SPH_OK;
}

int sph_graph_kernels_launched(sph_ctx *ctx, int64_t *count, int32_t reset) {
    if (!ctx || !count) return SPH_ERR_ARG;
    *count = ctx->graph_kernels_launched;
    if (reset) ctx->graph_kernels_launched = 0;
    return SPH_OK;
}

int sph_rows_kept(sph_ctx *ctx, int64_t *kept) {
    int rc = enter(ctx);
    if (rc) return rc;
    if (!kept) return SPH_ERR_ARG;
    *kept = 0;
    if (!ctx->kept_counted) return SPH_OK;
    int v = 0;
    CK(cudaStreamSynchronize(ctx->stream));
    CK(cudaMemcpy(&v, ctx->kept_cnt, sizeof(int), cudaMemcpyDeviceToHost));
    *kept = v;
    return SPH_OK;
}

int sph_measure_fp32_peak(sph_ctx *ctx, double *tflops) {
    int rc = enter(ctx);
    if (rc) return rc;
    if (!tflops) return SPH_ERR_ARG;
    const int blocks = ctx->num_sms * 8, threads = 256, iters = 4096;
    cudaEvent_t a, b;
    CK(cudaEventCreate(&a));
    CK(cudaEventCreate(&b));
    float *dummy = (float *)ctx->red;
    const double flops = 2.0 * 8 * 16 * (double)iters * blocks * threads;
    double best = 0.0;
    // scalar and packed FMA chains; the larger rate is the peak
    for (int packed = 0; packed < 2; packed++) {
        auto launch = [&](int it) {
            if (packed) k_fma2_peak<<<blocks, threads, 0, ctx->stream>>>(dummy, it, 0.999f, 0.001f);
            else k_fma_peak<<<blocks, threads, 0, ctx->stream>>>(dummy, it, 0.999f, 0.001f);
        };
        launch(64);  // warm-up
        CK(cudaEventRecord(a, ctx->stream));
        launch(iters);
        CK(cudaEventRecord(b, ctx->stream));
        CK(cudaEventSynchronize(b));
        float ms = 0.f;
        CK(cudaEventElapsedTime(&ms, a, b));
        best = std::max(best, (packed ? 2.0 : 1.0) * flops / (ms * 1e-3) / 1e12);
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    *tflops = best;
    return ctx_check_launch(ctx, "fp32_peak");
}

}  // extern "C"
