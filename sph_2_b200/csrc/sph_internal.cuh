// sph_internal.cuh -- shared definitions of libsphb200 (sm_100a).
//
// Layout of the particle state in HBM (storage order = Morton order after
// every sph_sort):
//   * FP64 SoA masters, double-buffered for the permutation at each sort:
//       x y z vx vy vz m h u dudt_prev  + int32 id (original index), cloud
//   * FP64 SoA results of the current step (single buffer):
//       rho P c divV curlV a_sph[3] a_grav[3] dudt vsig pot
//   * packed j-records read by the neighbour passes (one sector or less per
//     neighbour gather):
//       p0 = double4 (x, y, z, h)              -- FP64 in both precisions
//       p1 = Real4   (vx, vy, vz, m)
//       p2 = Real4   (rho, P/rho^2, c, f_balsara)
//       pw = Real4   (x, y, z, m)              -- gravity walk particles
//   * tree: 2N-1 nodes (internal 0..N-2, leaf of particle p at N-1+p), FP64
//     records of 16 doubles for the build, Real4 x3 walk records.
//   * neighbour rows: int32 [N][max_ngb] row-major + counts.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <map>
#include <string>
#include <utility>
#include <vector>

#include "../../include/sph_b200.h"

#define SPH_PI 3.14159265358979323846
#define SPH_SIG (1.0 / SPH_PI)

#define CK(call)                                                         \
    do {                                                                 \
        cudaError_t e_ = (call);                                         \
        if (e_ != cudaSuccess) return ctx_fail(ctx, e_, #call, __LINE__); \
    } while (0)

// ---- state field indices of the double-buffered persistent SoA ----
// ST_HNB: the largest h among the particle's list neighbours at the last list
// build (widens its next candidate search so that its list is complete from
// its own candidates)
enum { ST_X, ST_Y, ST_Z, ST_VX, ST_VY, ST_VZ, ST_M, ST_H, ST_U, ST_DUDT_PREV, ST_HNB, ST_N };

struct sph_ctx {
    sph_config cfg;
    int device = 0;
    int num_sms = 148;
    cudaStream_t stream = nullptr, stream_g = nullptr;
    bool own_stream = false;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    // points of the step after which fields are final (recorded in every
    // step): positions and masses (after the sort), h (after the neighbour
    // pass), velocities (after the closing kick), everything (the end)
    cudaEvent_t ev_io[4] = {};
    cudaStream_t stream_io = nullptr;   // copies of sph_step_io (created on first use)
    double *io_stage = nullptr;         // io_slots x n_max doubles (allocated on first use)
    int io_slots = 0;
    std::string err;
    int n = 0, ncloud = 0;
    std::vector<int> cloud_start_h;  // ncloud+1
    int64_t dev_bytes = 0;
    std::vector<void *> allocs;

    // persistent state, double buffered
    double *st[2][ST_N] = {};
    double **st_table = nullptr;  // device copy of one buffer's field pointers
    int last_injected_id = -1;    // original id of the last particle injected (-1: none)
    int *id[2] = {}, *cloud[2] = {};
    int cur = 0;

    // per-step results
    double *rho = nullptr, *P = nullptr, *c = nullptr, *divV = nullptr, *curlV = nullptr;
    double *asph = nullptr, *agrav = nullptr;  // 3*N each (x block, y block, z block)
    double *dudt = nullptr, *vsig = nullptr, *pot = nullptr;

    // packed records
    double4 *p0 = nullptr;
    void *p1 = nullptr, *p2 = nullptr, *pw = nullptr;
    bool p2_dirty = true;

    // sort
    unsigned long long *key[2] = {};
    int *val[2] = {};
    unsigned long long *key_in = nullptr;  // keys of the storage order before the last sort
    int *perm = nullptr;         // permutation of the last sort
    unsigned *hist = nullptr;    // radix histograms
    int sort_blocks = 0;
    unsigned long long *box = nullptr;  // per cloud 6 ordered-uint64 (min xyz, max xyz)
    // per cloud: the origin of the mixed walk's FP32 coordinates (x, y, z; the
    // centre of the cloud's box at the last sort, 0 before the first)
    double *corg = nullptr;
    int *cloud_start = nullptr;         // device copy

    // tree
    int *child = nullptr, *parent = nullptr, *first = nullptr, *last = nullptr, *flag = nullptr;
    double *node = nullptr, *hmax = nullptr, *ropen2 = nullptr;
    void *node_box = nullptr;  // float4 [2][2*n_max], rounded outward: (box min, h_max), (box max, 0)
    // Real4 walk records per node: wA (com, r_open^2), wB (Qxx, Qyy, Qzz, M),
    // wC (Qxy, Qxz, Qyz, trace); wL (first, count, left, right child)
    void *wA = nullptr, *wB = nullptr, *wC = nullptr;
    int4 *wL = nullptr;
    int *croot = nullptr;                              // per cloud root node
    int *gstart = nullptr, *gcount = nullptr, *groot_g = nullptr;  // groups: start, size, cloud id
    int *gnode = nullptr;                       // group -> tree node
    int *gmark = nullptr, *gpos = nullptr, *gnode_at = nullptr, *scan_tmp = nullptr;
    int *d_ngroup = nullptr;                    // number of groups (device)
    int ngroup = 0;                             // capacity of the group table
    // super-groups of the mixed walk with group expansions (theta_local > 0):
    // maximal tree nodes of at most SGROUP_MAX particles of one cloud, each
    // walked once for the far cells common to its groups (null otherwise)
    int *sg_start = nullptr, *sg_count = nullptr, *sg_cloud = nullptr;
    int *d_nsg = nullptr;                       // number of super-groups (device)
    int *g_sg = nullptr;                        // group -> super-group
    int *sg_nrem = nullptr;                     // nodes left to the groups, -1: none (walk from the root)
    int *sg_pool = nullptr;                     // those nodes, SG_POOL per particle from the first particle
    float *sgL = nullptr;                       // per super-group: expansion coefficients and centre
    int sg_cap = 0;                             // super-groups with an index below this have records
    bool tree_ok = false;

    // neighbours
    int *ngb = nullptr, *ngb_cnt = nullptr;
    int *cand_idx = nullptr;  // candidate slots j of the h iteration, max_ngb per particle
    int *cand_cnt = nullptr;
    int *lflag = nullptr;     // n+3: per particle "needs the tree search", "all do", "any does",
                              // how many are listed in mlist
    int *mlist = nullptr;     // the particles the fused list pass marked, each once
    bool cand_ok = false;     // candidate rows match the current order, positions and h
    int *retry = nullptr;        // per particle: 1 search, 2 or 3 keep the row, 0 done
    int *hiter = nullptr;        // per particle: iterations of the count iteration so far
    double *hcand = nullptr;     // candidate radius / 2 used per particle
    double *hover = nullptr;     // smallest candidate radius / 2 whose row overflowed this call
    // candidate rows kept between the h iterations of refit steps: a row
    // searched at radius 2 hsr still holds every particle within
    // 2 hsr - dmv_i - (the largest dmv_j nearby) of the particle's position
    double *hsr = nullptr;  // per particle: radius / 2 of the search that wrote its row (0: none)
    double *dmv = nullptr;  // per particle: distance moved through the packed records since the
                            // last h iteration that searched every particle
    unsigned long long *dmv_max = nullptr;  // per cloud: the largest dmv (FP64 bits)
    float *gdm = nullptr;   // per particle: the largest dmv of its group (rounded up)
    int *rows_ok = nullptr;  // device flag: the rows, hsr and dmv belong to the storage order
    bool rows_host = false;  // host view of rows_ok, for the choice of launches only
    int *kept_cnt = nullptr;     // [0] particles whose row the last h iteration kept (3 ints)
    bool kept_counted = false;   // that count belongs to the last h iteration
    bool lists_ok = false, rho_ok = false, divcurl_ok = false;

    // time step, status, counters
    double *dt = nullptr, *dt_next = nullptr;  // per cloud
    unsigned long long *dt_bits = nullptr;     // per cloud ordered min
    unsigned long long *dtmax_bits = nullptr;  // per cloud ordered max of the individual steps
    double *dt_part = nullptr, *dhdt = nullptr; // per particle: individual step, dh/dt
    int *dbin = nullptr;                        // per particle: power-of-two bin of its step
    long long *status = nullptr;               // SPH_NSTATUS
    unsigned long long *counters = nullptr;    // walk: cells, particles
    unsigned *work = nullptr;                  // work counters for persistent kernels (16)
    std::map<std::pair<const void *, int>, int> occupancy;  // resident blocks per SM per kernel
    double *red = nullptr;                     // reduction scratch

    // cooling
    bool cool_ok = false;
    sph_cooling_params cool{};
    double *cool_table = nullptr;  // n_bins+1
    float *mlp = nullptr;          // FP32 master params (SPH_MLP_NPARAM) + norm (8)
    void *mlp_bf16 = nullptr;      // packed BF16 weights for the tensor-core kernels
    float *mlp_grad = nullptr, *mlp_m = nullptr, *mlp_v = nullptr;
    float *mlp_scratch = nullptr;
    int *cool_list = nullptr;      // surrogate fallback rows (n_max) + their count
    // table cooling: grids (kpc, nH, Z, T, time), u after each time, ion
    // fractions, and the ion fractions of the last call per storage slot
    bool tab_ok = false;
    sph_cool_table_params tab{};
    int tab_dims[6] = {};
    float *tab_grid = nullptr, *tab_uev = nullptr, *tab_frac = nullptr, *ion = nullptr;
    int mlp_step = 0;
    bool mlp_ok = false;

    // phase timing events of sph_step (SPH_FLAG_TIMING)
    cudaEvent_t tev[16] = {};
    bool tev_ok = false;
    int graph_kernels = 0;

    // step graphs (one per buffer parity)
    // step graphs per buffer parity, full rebuild [0] or refit [1]
    cudaGraphExec_t graph[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};
    // the tree topology (child / parent / first / last, groups, super-groups)
    // matches the storage order and particle set, so a step may refit it
    bool topo_ok = false;
    int refits = 0;  // refit steps since the last full rebuild
    bool records_all = false;  // every node's 16-double build record is current
    int graph_nk[2][2] = {{0, 0}, {0, 0}};  // kernel nodes of each step graph
    int64_t graph_kernels_launched = 0;     // kernel nodes of the graphs launched
    bool graph_valid = false;
    bool prologue_done = false;
    bool in_step = false;  // the walk being queued is sph_step's (beside the SPH passes)
    int64_t step_count = 0;
};

int ctx_fail(sph_ctx *ctx, cudaError_t e, const char *what, int line);
void drop_graphs(sph_ctx *ctx);  // the step graphs are re-captured at the next sph_step
int ctx_check_launch(sph_ctx *ctx, const char *what);

// ----------------------------------------------------------------------------
// device helpers
// ----------------------------------------------------------------------------
template <class R> struct R4;
template <> struct R4<float> { typedef float4 T; };
template <> struct R4<double> { typedef double4 T; };

__device__ __forceinline__ double xmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double xadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double xsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double xdiv(double a, double b) { return __ddiv_rn(a, b); }

// ordered mapping double <-> uint64 (monotone), for atomic min/max of doubles
__device__ __forceinline__ unsigned long long dbl_to_ord(double d) {
    unsigned long long b = (unsigned long long)__double_as_longlong(d);
    return (b & 0x8000000000000000ULL) ? ~b : (b | 0x8000000000000000ULL);
}
// FP32 walk coordinates are taken relative to the cloud's origin, so their
// rounding scales with the cloud's size, not with its distance from 0; the
// FP64 walk keeps absolute coordinates
template <class R> struct WalkOrigin {
    __device__ __forceinline__ static double off(const double *, int) { return 0.0; }
};
template <> struct WalkOrigin<float> {
    __device__ __forceinline__ static double off(const double *org, int d) { return org[d]; }
};

__host__ __device__ __forceinline__ double ord_to_dbl(unsigned long long o) {
    unsigned long long b = (o & 0x8000000000000000ULL) ? (o & 0x7fffffffffffffffULL) : ~o;
#ifdef __CUDA_ARCH__
    return __longlong_as_double((long long)b);
#else
    double d;
    memcpy(&d, &b, 8);
    return d;
#endif
}

// exact neighbour predicate |r|^2 <= (hi+hj)^2, rounding as written
__device__ __forceinline__ bool ngb_pred(double xi, double yi, double zi, double hi, double xj,
                                         double yj, double zj, double hj) {
    double dx = xsub(xi, xj), dy = xsub(yi, yj), dz = xsub(zi, zj);
    double r2 = xadd(xmul(dx, dx), xmul(dy, dy));
    r2 = xadd(r2, xmul(dz, dz));
    double s = xadd(hi, hj);
    return r2 <= xmul(s, s);
}

// a / b in the neighbour sums: the fast single-precision divide (about 2 ulp)
// in FP32, where the sums' own rounding is far larger; IEEE division in FP64
template <class R> __device__ __forceinline__ R qdiv(R a, R b) { return a / b; }
template <> __device__ __forceinline__ float qdiv<float>(float a, float b) { return __fdividef(a, b); }
// sqrt(x) the same way: x * rsqrt(x) in FP32 (0 at x = 0), IEEE sqrt in FP64
template <class R> __device__ __forceinline__ R qsqrt(R x) { return sqrt(x); }
template <> __device__ __forceinline__ float qsqrt<float>(float x) { return x > 0.f ? x * rsqrtf(x) : 0.f; }

// M4 cubic spline (sigma = 1/pi, support 2h): W and nW with gradW = nW * dr
// (libsx.py:69-80, shear.py:109-121; the q+1e-20 guard of the reference)
template <class R>
__device__ __forceinline__ R kern_w(R q, R inv_h3) {
    if (q <= R(1)) return R(SPH_SIG) * inv_h3 * (R(1) - R(1.5) * q * q + R(0.75) * q * q * q);
    if (q <= R(2)) {
        R t = R(2) - q;
        return R(SPH_SIG) * inv_h3 * R(0.25) * t * t * t;
    }
    return R(0);
}
template <class R>
__device__ __forceinline__ R kern_nw(R q, R inv_h5) {
    if (q <= R(1)) return R(SPH_SIG) * inv_h5 * (R(-3) + R(2.25) * q);
    if (q <= R(2)) {
        R t = R(2) - q;
        return qdiv<R>(R(-0.75 * SPH_SIG) * inv_h5 * t * t, q + R(1e-20));
    }
    return R(0);
}

// Kahan-compensated accumulator for FP32, plain sum for FP64
template <class R> struct KSum {
    R s = R(0);
    __device__ __forceinline__ void add(R x) { s += x; }
    __device__ __forceinline__ double value() const { return (double)s; }
};
template <> struct KSum<float> {
    float s = 0.f, c = 0.f;
    __device__ __forceinline__ void add(float x) {
        float y = __fsub_rn(x, c);
        float t = __fadd_rn(s, y);
        c = __fsub_rn(__fsub_rn(t, s), y);
        s = t;
    }
    __device__ __forceinline__ double value() const { return (double)s - (double)c; }
};

// sum over the `lanes`-wide segment (lanes a power of two <= 32), all lanes
// of the warp must call; result identical on every lane of the segment
template <int LANES>
__device__ __forceinline__ double seg_sum(double v) {
#pragma unroll
    for (int o = LANES / 2; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31;
    return __shfl_sync(0xffffffffu, v, lane & ~(LANES - 1));
}
template <int LANES>
__device__ __forceinline__ double seg_max(double v) {
#pragma unroll
    for (int o = LANES / 2; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

__device__ __forceinline__ void status_add(long long *status, int which, long long v) {
    atomicAdd((unsigned long long *)&status[which], (unsigned long long)v);
}

// per-cloud minimum of t over the warp: one atomic per warp when the warp
// holds one cloud (clouds are contiguous in storage order), else one per
// lane.  Every lane of the warp calls; t = 0 marks a lane with no estimate.
__device__ __forceinline__ void cloud_min(unsigned long long *dt_bits, bool valid, int c, double t) {
    unsigned long long v = (valid && t > 0.0) ? dbl_to_ord(t) : ~0ULL;
    const int cc = valid ? c : -1;
    const int c0 = __shfl_sync(0xffffffffu, cc, 0);
    if (__all_sync(0xffffffffu, !valid || cc == c0)) {
#pragma unroll
        for (int o = 16; o; o >>= 1) {
            const unsigned long long w = __shfl_xor_sync(0xffffffffu, v, o);
            v = w < v ? w : v;
        }
        if ((threadIdx.x & 31) == 0 && v != ~0ULL) atomicMin(&dt_bits[c0], v);
    } else if (v != ~0ULL) {
        atomicMin(&dt_bits[cc], v);
    }
}

// Work queue of the persistent group kernels: with a counter (queue mode)
// every warp takes its next group from an atomic counter, so a persistent
// grid of one block per resident slot drains the (cloud, group) list in order
// however uneven the groups' costs are; without one (null) the warp strides
// over the groups by the grid size.  All lanes of the warp call both.
__device__ __forceinline__ int q_first(unsigned *q, int static_first) {
    if (!q) return static_first;
    int g = 0;
    if ((threadIdx.x & 31) == 0) g = (int)atomicAdd(q, 1u);
    return __shfl_sync(0xffffffffu, g, 0);
}
__device__ __forceinline__ int q_next(unsigned *q, int g, int stride) {
    return q ? q_first(q, 0) : g + stride;
}
// work-counter slots (sph_ctx::work) of the queued kernels
enum { WQ_WALK = 0, WQ_SG_WALK = 1, WQ_SEARCH = 2, WQ_N = 3 };

// ---- host-side launch helpers implemented per translation unit ----
int launch_sort(sph_ctx *ctx);
int launch_sort_refit(sph_ctx *ctx);
int launch_scan(sph_ctx *ctx, const int *in, int *out, int n, int *total);
int launch_groups(sph_ctx *ctx);
int launch_leaf_records(sph_ctx *ctx);  // the leaves' 16-double records (export only)
constexpr int SGROUP_MAX = 128;  // particles per super-group
constexpr int SG_POOL = 8;       // node slots per particle of a super-group
constexpr int SG_LSTRIDE = 40;   // floats per super-group record: 35 coefficients, pad, centre
int persistent_grid(sph_ctx *ctx, const void *kernel, int block, size_t smem);
// grid and queue counter of a group kernel: the persistent grid with its
// counter zeroed on the stream, or the static grid and no counter when
// SPH_FLAG_STATIC_GRID is set
int queue_launch(sph_ctx *ctx, cudaStream_t s, int slot, const void *kernel, int block,
                 int static_grid, int *grid, unsigned **queue);
// all_records false: the 16-double build records of the nodes inside the
// groups are not stored (only sph_get_tree reads them; it rebuilds them)
int launch_tree(sph_ctx *ctx, bool all_records = true);
int launch_tree_refit(sph_ctx *ctx, bool all_records = true);
int launch_tree_records(sph_ctx *ctx);
int launch_refit_hmax(sph_ctx *ctx, const int *need = nullptr);
int launch_smoothing_h(sph_ctx *ctx);
int launch_smoothing_h_count(sph_ctx *ctx, int n_target, int n_tol, double frac, int max_iter);
int launch_smoothing_kth(sph_ctx *ctx, int k);
int launch_neighbours(sph_ctx *ctx);
int launch_density(sph_ctx *ctx);
int launch_divcurl(sph_ctx *ctx);
int launch_density_divcurl(sph_ctx *ctx);
int launch_lists_density(sph_ctx *ctx);
int launch_lists_marked(sph_ctx *ctx);
int launch_forces(sph_ctx *ctx, bool want_acc, bool want_du, bool update_u);
int launch_repack_p2(sph_ctx *ctx);
int launch_gravity(sph_ctx *ctx, cudaStream_t s, bool pot);
int launch_gravity_direct(sph_ctx *ctx, int nt, const int *targets_dev, double *out_dev);
int launch_gravity_direct_spline(sph_ctx *ctx, const double *eps_dev, int nt,
                                 const int *targets_dev, double *out_dev, int nbeg, int nend);
int launch_kick(sph_ctx *ctx, double fac, bool cfl);
int launch_drift(sph_ctx *ctx);
int launch_kick_drift(sph_ctx *ctx);
int launch_update_u(sph_ctx *ctx, bool first);
int launch_cfl(sph_ctx *ctx);
int launch_external_potential(sph_ctx *ctx, cudaStream_t s);
int launch_inject_pairs(sph_ctx *ctx, int npairs, unsigned long long seed, int cloud,
                        double r_max, double v_in, double m, double u, int h_id, double h_first);
int launch_dt_individual(sph_ctx *ctx);
int launch_dt_bins(sph_ctx *ctx);
int launch_dt_commit(sph_ctx *ctx);
int launch_energies(sph_ctx *ctx, double *out10_host);
int launch_pack_p1(sph_ctx *ctx, bool track = false);
int launch_rows_invalidate(sph_ctx *ctx);
int launch_export_neighbours(sph_ctx *ctx, int64_t *off_dev, int *lst_dev, int64_t cap);
int launch_cooling_exact(sph_ctx *ctx);
int launch_cooling_table(sph_ctx *ctx);
int launch_cooling_mlp(sph_ctx *ctx);
int launch_cool_solve(sph_ctx *ctx, int n, const double *rho, const double *u_old,
                      const double *dt, double *u_new, int *iters);
int mlp_forward_dev(sph_ctx *ctx, int n, const float *X, float *y);
int mlp_grad_dev(sph_ctx *ctx, int n, const float *X, const float *t, float *grad, float *loss);
int mlp_train_dev(sph_ctx *ctx, int n, const float *X, const float *t, int batch, int nsteps,
                  float lr, float *loss);
int mlp_pack(sph_ctx *ctx);

static inline int div_up(long long a, long long b) { return (int)((a + b - 1) / b); }
