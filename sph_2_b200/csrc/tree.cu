// tree.cu -- Karras (2012) binary radix tree over the sorted Morton keys and
// the deterministic FP64 bottom-up pass (mass, centre of mass, quadrupole
// second moments, particle box, h_max, opening radius).
//
// Replaces the reference octree (bh_tree_iteration_v2.h:29-450): a single
// <<<1,256>>> block inserting bodies under atomicCAS child locks with
// atomicAdd'ed masses (nondeterministic), a separate centre-of-mass kernel and
// a busy-waiting tree-order sort.  Here the topology is one thread per
// internal node; the nodes inside a walk group (at most 32 particles of one
// cloud) are summed directly over their particle range in index order, one
// lane each, and the nodes above the groups are combined bottom-up with the
// left child always first, so every node record is the same bit pattern on
// every run and equals the oracle's.  The Morton order is the walk order.
#include <cuda/atomic>

#include "sph_internal.cuh"

namespace {

__device__ __forceinline__ int delta_pref(const unsigned long long *__restrict__ k, int n, int i,
                                          int j) {
    if (j < 0 || j > n - 1) return -1;
    unsigned long long a = k[i], b = k[j];
    if (a == b) return 64 + __clz((unsigned)i ^ (unsigned)j);
    return __clzll(a ^ b);
}

__global__ void k_karras(const unsigned long long *__restrict__ key, const int *__restrict__ cloud,
                         int n, int *__restrict__ child, int *__restrict__ parent,
                         int *__restrict__ first, int *__restrict__ last, int *__restrict__ croot,
                         int4 *__restrict__ wL) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n - 1) return;
    int d = (delta_pref(key, n, i, i + 1) - delta_pref(key, n, i, i - 1)) > 0 ? 1 : -1;
    int dmin = delta_pref(key, n, i, i - d);
    int lmax = 2;
    while (delta_pref(key, n, i, i + lmax * d) > dmin) lmax *= 2;
    int l = 0;
    for (int t = lmax / 2; t >= 1; t /= 2)
        if (delta_pref(key, n, i, i + (l + t) * d) > dmin) l += t;
    int j = i + l * d;
    int dnode = delta_pref(key, n, i, j);
    int s = 0;
    for (int t = (l + 1) / 2;; t = (t + 1) / 2) {
        if (delta_pref(key, n, i, i + (s + t) * d) > dnode) s += t;
        if (t == 1) break;
    }
    int gam = i + s * d + (d < 0 ? -1 : 0);
    int lo = min(i, j), hi = max(i, j);
    int L = (lo == gam) ? n - 1 + gam : gam;
    int R = (hi == gam + 1) ? n - 1 + gam + 1 : gam + 1;
    child[2 * i] = L;
    child[2 * i + 1] = R;
    parent[L] = i;
    parent[R] = i;
    first[i] = lo;
    last[i] = hi;
    wL[i] = make_int4(lo, hi - lo + 1, L, R);
    int c = cloud[lo];
    if (cloud[hi] == c && (lo == 0 || cloud[lo - 1] != c) && (hi == n - 1 || cloud[hi + 1] != c))
        croot[c] = i;
}

// clouds of one particle: their root is the leaf
__global__ void k_single_roots(const int *__restrict__ cstart, int ncloud, int n, int *croot) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= ncloud) return;
    if (cstart[k + 1] - cstart[k] == 1) croot[k] = n - 1 + cstart[k];
}

template <class R>
__device__ __forceinline__ void write_walk(int nd, const double *o, double r2, double hm,
                                           typename R4<R>::T *wA, typename R4<R>::T *wB,
                                           typename R4<R>::T *wC, const double *org) {
    typename R4<R>::T a, b, c;
    a.x = (R)(o[0] - WalkOrigin<R>::off(org, 0));
    a.y = (R)(o[1] - WalkOrigin<R>::off(org, 1));
    a.z = (R)(o[2] - WalkOrigin<R>::off(org, 2));
    a.w = (R)r2;
    b.x = (R)o[4]; b.y = (R)o[5]; b.z = (R)o[6]; b.w = (R)o[3];
    c.x = (R)o[7]; c.y = (R)o[8]; c.z = (R)o[9];
    c.w = (R)(o[4] + o[5] + o[6]);  // trace of the second moments
    (void)hm;
    wA[nd] = a;
    wB[nd] = b;
    wC[nd] = c;
}

// opening radius^2 of a node: (l/theta + |com - box centre|)^2, l = largest side
__device__ __forceinline__ double open_r2(const double *o, double theta) {
    double l = fmax(xsub(o[13], o[10]), fmax(xsub(o[14], o[11]), xsub(o[15], o[12])));
    double cx = xmul(xadd(o[10], o[13]), 0.5), cy = xmul(xadd(o[11], o[14]), 0.5),
           cz = xmul(xadd(o[12], o[15]), 0.5);
    double ex = xsub(o[0], cx), ey = xsub(o[1], cy), ez = xsub(o[2], cz);
    double d2 = xadd(xmul(ex, ex), xmul(ey, ey));
    d2 = xadd(d2, xmul(ez, ez));
    double r = xadd(xdiv(l, theta), __dsqrt_rn(d2));
    return xmul(r, r);
}

// search-box records in FP32, rounded outward: (min down, h_max up), (max up)
__device__ __forceinline__ float4 box_lo(double x, double y, double z, double hm) {
    return make_float4(__double2float_rd(x), __double2float_rd(y), __double2float_rd(z),
                       __double2float_ru(hm));
}
__device__ __forceinline__ float4 box_hi(double x, double y, double z) {
    return make_float4(__double2float_ru(x), __double2float_ru(y), __double2float_ru(z), 0.f);
}

template <class R>
__global__ void k_leaves(int n, const double *__restrict__ x, const double *__restrict__ y,
                         const double *__restrict__ z, const double *__restrict__ h,
                         double *__restrict__ hmax, double *__restrict__ ropen2,
                         float4 *__restrict__ sA, float4 *__restrict__ sB, int *__restrict__ flag,
                         int *__restrict__ first, int *__restrict__ last, int *__restrict__ child,
                         typename R4<R>::T *wA, int4 *__restrict__ wL,
                         const int *__restrict__ cloud, const double *__restrict__ corg) {
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    int nd = n - 1 + p;
    // a leaf is never accepted as a cell (count 1): the walks read its com
    // and count only, and the climb and the export rebuild its 16-double
    // record from the particle (leaf_record)
    const double xp = x[p], yp = y[p], zp = z[p];
    hmax[nd] = h[p];
    ropen2[nd] = 0.0;
    sA[nd] = box_lo(xp, yp, zp, h[p]);
    sB[nd] = box_hi(xp, yp, zp);
    first[nd] = p;
    last[nd] = p;
    child[2 * nd] = -1;
    child[2 * nd + 1] = -1;
    wL[nd] = make_int4(p, 1, -1, -1);
    typename R4<R>::T a;
    const double *org = corg + 3 * cloud[p];
    a.x = (R)(xp - WalkOrigin<R>::off(org, 0));
    a.y = (R)(yp - WalkOrigin<R>::off(org, 1));
    a.z = (R)(zp - WalkOrigin<R>::off(org, 2));
    a.w = (R)0;
    wA[nd] = a;
    if (p < n - 1) flag[p] = 0;
}

// the 16-double record of a leaf (particle p): com and box at the particle,
// its mass, no second moments
__device__ __forceinline__ void leaf_record(int p, const double *__restrict__ x,
                                            const double *__restrict__ y,
                                            const double *__restrict__ z,
                                            const double *__restrict__ m, double *o) {
    o[0] = o[10] = o[13] = x[p];
    o[1] = o[11] = o[14] = y[p];
    o[2] = o[12] = o[15] = z[p];
    o[3] = m[p];
    for (int q = 4; q < 10; q++) o[q] = 0.0;
}

// leaf records into the node array (for the export)
__global__ void k_leaf_records(int n, const double *__restrict__ x, const double *__restrict__ y,
                               const double *__restrict__ z, const double *__restrict__ m,
                               double *__restrict__ node) {
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    double o[16];
    leaf_record(p, x, y, z, m, o);
    double *dst = node + (size_t)16 * (n - 1 + p);
    for (int q = 0; q < 16; q++) dst[q] = o[q];
}

__device__ __forceinline__ void combine(double *o, const double *a, const double *b) {
    double M = xadd(a[3], b[3]);
    double c[3];
    for (int d = 0; d < 3; d++) c[d] = xdiv(xadd(xmul(a[3], a[d]), xmul(b[3], b[d])), M);
    double da[3] = {xsub(a[0], c[0]), xsub(a[1], c[1]), xsub(a[2], c[2])};
    double db[3] = {xsub(b[0], c[0]), xsub(b[1], c[1]), xsub(b[2], c[2])};
    const int ia[6] = {0, 1, 2, 0, 0, 1}, ib[6] = {0, 1, 2, 1, 2, 2};
#pragma unroll
    for (int q = 0; q < 6; q++) {
        double ta = xadd(a[4 + q], xmul(xmul(a[3], da[ia[q]]), da[ib[q]]));
        double tb = xadd(b[4 + q], xmul(xmul(b[3], db[ia[q]]), db[ib[q]]));
        o[4 + q] = xadd(ta, tb);
    }
    o[0] = c[0]; o[1] = c[1]; o[2] = c[2]; o[3] = M;
    for (int d = 0; d < 3; d++) {
        o[10 + d] = fmin(a[10 + d], b[10 + d]);
        o[13 + d] = fmax(a[13 + d], b[13 + d]);
    }
}

// opening angles: theta_small for the cells of at most small_cell particles
struct Opening {
    double theta, theta_small;
    int small_cell;
    __device__ __forceinline__ double at(int count) const {
        return theta_small > 0.0 && count <= small_cell ? theta_small : theta;
    }
};

// the records of node nd from its combined moments o and h_max hm
// (record false: the 16-double build record is not stored; the walks and
// searches read only the other records)
template <class R>
__device__ __forceinline__ void store_node(int nd, const double *o, double hm, double theta,
                                           double *node, double *hmax, double *ropen2,
                                           float4 *sA, float4 *sB, typename R4<R>::T *wA,
                                           typename R4<R>::T *wB, typename R4<R>::T *wC,
                                           const double *org, bool record = true) {
    const double r2 = open_r2(o, theta);
    if (record) {
        double *dst = node + (size_t)16 * nd;
        for (int q = 0; q < 16; q++) dst[q] = o[q];
    }
    hmax[nd] = hm;
    ropen2[nd] = r2;
    sA[nd] = box_lo(o[10], o[11], o[12], hm);
    sB[nd] = box_hi(o[13], o[14], o[15]);
    write_walk<R>(nd, o, r2, hm, wA, wB, wC, org);
}

// the internal nodes inside each group (the nodes of at most 32 particles of
// one cloud): one warp per group, the group's particles in shared memory,
// each lane one internal node summed directly over its particle range in
// index order -- mass, com = sum(m x) / M, second moments sum((m d_a) d_b)
// about the com, box -- the oracle's direct_moments.  A group of c >= 2
// particles from s0 owns the c - 1 internal nodes base .. base + c - 2 of
// the radix tree, base = s0 when the group's node is s0 (a right child: its
// index is its first particle) and s0 + 1 when it is s0 + c - 1 (a left
// child); every descendant's index lies strictly inside the range.
constexpr int GUP_WARPS = 4;
template <class R>
__global__ void __launch_bounds__(GUP_WARPS * 32)
    k_group_up(int n, const int *__restrict__ ngroup_p, const int *__restrict__ gstart,
               const int *__restrict__ gcount, const int *__restrict__ gnode,
               const int *__restrict__ first, const int *__restrict__ last,
               const double *__restrict__ x, const double *__restrict__ y,
               const double *__restrict__ z, const double *__restrict__ m,
               const double *__restrict__ h, double *node, double *hmax, double *ropen2,
               float4 *sA, float4 *sB, Opening op, typename R4<R>::T *wA,
               typename R4<R>::T *wB, typename R4<R>::T *wC,
               const int *__restrict__ cloud, const double *__restrict__ corg,
               int all_records) {
    __shared__ double px[GUP_WARPS][32], py[GUP_WARPS][32], pz[GUP_WARPS][32],
        pm[GUP_WARPS][32], ph[GUP_WARPS][32];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int ngroup = *ngroup_p;
    for (int g = blockIdx.x * GUP_WARPS + w; g < ngroup; g += gridDim.x * GUP_WARPS) {
        const int s0 = gstart[g], c = gcount[g];
        if (c < 2) continue;  // a single particle: its leaf is the group's node
        if (lane < c) {
            px[w][lane] = x[s0 + lane];
            py[w][lane] = y[s0 + lane];
            pz[w][lane] = z[s0 + lane];
            pm[w][lane] = m[s0 + lane];
            ph[w][lane] = h[s0 + lane];
        }
        __syncwarp();
        if (lane < c - 1) {
            const int nd = (gnode[g] == s0 ? s0 : s0 + 1) + lane;
            const int f = max(first[nd] - s0, 0), l = min(last[nd] - s0, c - 1);
            double M = 0.0, sx = 0.0, sy = 0.0, sz = 0.0, hm = ph[w][f];
            double o[16];
            o[10] = o[13] = px[w][f];
            o[11] = o[14] = py[w][f];
            o[12] = o[15] = pz[w][f];
            for (int k = f; k <= l; k++) {
                const double xk = px[w][k], yk = py[w][k], zk = pz[w][k], mk = pm[w][k];
                M = xadd(M, mk);
                sx = xadd(sx, xmul(mk, xk));
                sy = xadd(sy, xmul(mk, yk));
                sz = xadd(sz, xmul(mk, zk));
                o[10] = fmin(o[10], xk); o[11] = fmin(o[11], yk); o[12] = fmin(o[12], zk);
                o[13] = fmax(o[13], xk); o[14] = fmax(o[14], yk); o[15] = fmax(o[15], zk);
                hm = fmax(hm, ph[w][k]);
            }
            const double cx = xdiv(sx, M), cy = xdiv(sy, M), cz = xdiv(sz, M);
            double qxx = 0.0, qyy = 0.0, qzz = 0.0, qxy = 0.0, qxz = 0.0, qyz = 0.0;
            for (int k = f; k <= l; k++) {
                const double dx = xsub(px[w][k], cx), dy = xsub(py[w][k], cy),
                             dz = xsub(pz[w][k], cz);
                const double mk = pm[w][k];
                const double tx = xmul(mk, dx), ty = xmul(mk, dy), tz = xmul(mk, dz);
                qxx = xadd(qxx, xmul(tx, dx)); qxy = xadd(qxy, xmul(tx, dy));
                qxz = xadd(qxz, xmul(tx, dz)); qyy = xadd(qyy, xmul(ty, dy));
                qyz = xadd(qyz, xmul(ty, dz)); qzz = xadd(qzz, xmul(tz, dz));
            }
            o[0] = cx; o[1] = cy; o[2] = cz; o[3] = M;
            o[4] = qxx; o[5] = qyy; o[6] = qzz; o[7] = qxy; o[8] = qxz; o[9] = qyz;
            // the climb reads the 16-double record of the group's own node
            // only; the others are for sph_get_tree
            store_node<R>(nd, o, hm, op.at(l - f + 1), node, hmax, ropen2, sA, sB, wA, wB, wC,
                          corg + 3 * cloud[s0], all_records || nd == gnode[g]);
        }
        __syncwarp();
    }
}

// one thread per group climbs from the group's node; the second child to
// finish combines its parent
template <class R>
__global__ void k_bottom_up(int n, const int *__restrict__ ngroup_p,
                            const int *__restrict__ gnode, const int *__restrict__ parent,
                            const int *__restrict__ child, const double *__restrict__ x,
                            const double *__restrict__ y, const double *__restrict__ z,
                            const double *__restrict__ m, double *node, double *hmax,
                            double *ropen2, float4 *sA, float4 *sB, int *flag, Opening op,
                            const int4 *__restrict__ wL, typename R4<R>::T *wA,
                            typename R4<R>::T *wB, typename R4<R>::T *wC,
                            const int *__restrict__ cloud, const double *__restrict__ corg) {
    int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= *ngroup_p || n < 2) return;
    int nd = parent[gnode[g]];
    while (nd >= 0) {
        // acquire-release on the arrival counter: the first thread's node
        // record is visible to the second, which combines the two
        cuda::atomic_ref<int, cuda::thread_scope_device> arrived(flag[nd]);
        if (arrived.fetch_add(1, cuda::memory_order_acq_rel) == 0) return;
        arrived.store(0, cuda::memory_order_relaxed);  // ready for the next pass
        int L = child[2 * nd], Rr = child[2 * nd + 1];
        double a[16], b[16], o[16];
        if (L >= n - 1) {
            leaf_record(L - (n - 1), x, y, z, m, a);
        } else {
            const double *pa = node + (size_t)16 * L;
            for (int q = 0; q < 16; q++) a[q] = __ldcg(pa + q);
        }
        if (Rr >= n - 1) {
            leaf_record(Rr - (n - 1), x, y, z, m, b);
        } else {
            const double *pb = node + (size_t)16 * Rr;
            for (int q = 0; q < 16; q++) b[q] = __ldcg(pb + q);
        }
        combine(o, a, b);
        double hm = fmax(__ldcg(hmax + L), __ldcg(hmax + Rr));
        store_node<R>(nd, o, hm, op.at(wL[nd].y), node, hmax, ropen2, sA, sB, wA, wB, wC,
                      corg + 3 * cloud[wL[nd].x]);
        nd = parent[nd];
    }
}

// h_max refit after the smoothing lengths changed
// need (may be null): skip the refit when *need == 0 (no tree search follows)
// The leaves and the internal nodes inside each group: one warp per group,
// h of its particles in shared memory, each internal node the maximum over
// its particle range (the same nodes as k_group_up)
__global__ void __launch_bounds__(GUP_WARPS * 32)
    k_refit_groups(int n, const int *__restrict__ ngroup_p, const int *__restrict__ gstart,
                   const int *__restrict__ gcount, const int *__restrict__ gnode,
                   const int *__restrict__ first, const int *__restrict__ last,
                   const double *__restrict__ h, double *hmax, float4 *sA,
                   const int *__restrict__ need) {
    __shared__ double sh[GUP_WARPS][32];
    if (need && !*need) return;
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int ngroup = *ngroup_p;
    for (int g = blockIdx.x * GUP_WARPS + w; g < ngroup; g += gridDim.x * GUP_WARPS) {
        const int s0 = gstart[g], c = gcount[g];
        if (lane < c) {
            const double hp = h[s0 + lane];
            sh[w][lane] = hp;
            hmax[n - 1 + s0 + lane] = hp;
            sA[n - 1 + s0 + lane].w = __double2float_ru(hp);
        }
        __syncwarp();
        if (c >= 2 && lane < c - 1) {
            const int nd = (gnode[g] == s0 ? s0 : s0 + 1) + lane;
            const int f = max(first[nd] - s0, 0), l = min(last[nd] - s0, c - 1);
            double hm = sh[w][f];
            for (int k = f + 1; k <= l; k++) hm = fmax(hm, sh[w][k]);
            hmax[nd] = hm;
            sA[nd].w = __double2float_ru(hm);
        }
        __syncwarp();
    }
}

// above the groups: one thread per group climbs from the group's node; the
// second arrival combines and clears the counter for the next pass
__global__ void k_refit_up(int n, const int *__restrict__ ngroup_p, const int *__restrict__ gnode,
                           const int *__restrict__ parent, const int *__restrict__ child,
                           double *hmax, float4 *sA, int *flag, const int *__restrict__ need) {
    int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= *ngroup_p || n < 2 || (need && !*need)) return;
    int nd = parent[gnode[g]];
    while (nd >= 0) {
        cuda::atomic_ref<int, cuda::thread_scope_device> arrived(flag[nd]);
        if (arrived.fetch_add(1, cuda::memory_order_acq_rel) == 0) return;
        arrived.store(0, cuda::memory_order_relaxed);
        double hm = fmax(__ldcg(hmax + child[2 * nd]), __ldcg(hmax + child[2 * nd + 1]));
        hmax[nd] = hm;
        sA[nd].w = __double2float_ru(hm);
        nd = parent[nd];
    }
}

}  // namespace

namespace {

// leaf records, then the moments, boxes and walk records of the nodes inside
// the groups and of those above them (groups: the tables of the current
// topology, rebuilt first when `groups`)
int tree_records(sph_ctx *ctx, bool groups, bool all_records) {
    const int n = ctx->n;
    cudaStream_t s = ctx->stream;
    const int c = ctx->cur;
    float4 *boxA = (float4 *)ctx->node_box;
    float4 *boxB = boxA + (2 * (size_t)ctx->cfg.n_max);
    const int ggrid = max(1, div_up(div_up(n, 16) + ctx->ncloud, GUP_WARPS));
    const Opening op{ctx->cfg.theta, ctx->cfg.theta_small, ctx->cfg.small_cell};
    int rc;
    if (ctx->cfg.precision == SPH_PREC_MIXED) {
        k_leaves<float><<<div_up(n, 256), 256, 0, s>>>(
            n, ctx->st[c][ST_X], ctx->st[c][ST_Y], ctx->st[c][ST_Z], ctx->st[c][ST_H], ctx->hmax,
            ctx->ropen2, boxA, boxB, ctx->flag, ctx->first, ctx->last, ctx->child, (float4 *)ctx->wA,
            ctx->wL, ctx->cloud[c], ctx->corg);
        if (groups && (rc = launch_groups(ctx))) return rc;
        k_group_up<float><<<ggrid, GUP_WARPS * 32, 0, s>>>(
            n, ctx->d_ngroup, ctx->gstart, ctx->gcount, ctx->gnode, ctx->first, ctx->last,
            ctx->st[c][ST_X], ctx->st[c][ST_Y], ctx->st[c][ST_Z], ctx->st[c][ST_M],
            ctx->st[c][ST_H], ctx->node, ctx->hmax, ctx->ropen2, boxA, boxB, op,
            (float4 *)ctx->wA, (float4 *)ctx->wB, (float4 *)ctx->wC, ctx->cloud[c], ctx->corg,
            all_records ? 1 : 0);
        k_bottom_up<float><<<div_up(n, 256), 256, 0, s>>>(
            n, ctx->d_ngroup, ctx->gnode, ctx->parent, ctx->child, ctx->st[c][ST_X],
            ctx->st[c][ST_Y], ctx->st[c][ST_Z], ctx->st[c][ST_M], ctx->node, ctx->hmax,
            ctx->ropen2, boxA, boxB, ctx->flag, op, ctx->wL, (float4 *)ctx->wA,
            (float4 *)ctx->wB, (float4 *)ctx->wC, ctx->cloud[c], ctx->corg);
    } else {
        k_leaves<double><<<div_up(n, 256), 256, 0, s>>>(
            n, ctx->st[c][ST_X], ctx->st[c][ST_Y], ctx->st[c][ST_Z], ctx->st[c][ST_H], ctx->hmax,
            ctx->ropen2, boxA, boxB, ctx->flag, ctx->first, ctx->last, ctx->child, (double4 *)ctx->wA,
            ctx->wL, ctx->cloud[c], ctx->corg);
        if (groups && (rc = launch_groups(ctx))) return rc;
        k_group_up<double><<<ggrid, GUP_WARPS * 32, 0, s>>>(
            n, ctx->d_ngroup, ctx->gstart, ctx->gcount, ctx->gnode, ctx->first, ctx->last,
            ctx->st[c][ST_X], ctx->st[c][ST_Y], ctx->st[c][ST_Z], ctx->st[c][ST_M],
            ctx->st[c][ST_H], ctx->node, ctx->hmax, ctx->ropen2, boxA, boxB, op,
            (double4 *)ctx->wA, (double4 *)ctx->wB, (double4 *)ctx->wC, ctx->cloud[c], ctx->corg,
            all_records ? 1 : 0);
        k_bottom_up<double><<<div_up(n, 256), 256, 0, s>>>(
            n, ctx->d_ngroup, ctx->gnode, ctx->parent, ctx->child, ctx->st[c][ST_X],
            ctx->st[c][ST_Y], ctx->st[c][ST_Z], ctx->st[c][ST_M], ctx->node, ctx->hmax,
            ctx->ropen2, boxA, boxB, ctx->flag, op, ctx->wL, (double4 *)ctx->wA,
            (double4 *)ctx->wB, (double4 *)ctx->wC, ctx->cloud[c], ctx->corg);
    }
    return SPH_OK;
}

}  // namespace

int launch_tree(sph_ctx *ctx, bool all_records) {
    ctx->cand_ok = false;
    const int n = ctx->n;
    if (n <= 0) return SPH_OK;
    cudaStream_t s = ctx->stream;
    const int c = ctx->cur;
    const unsigned long long *key = ctx->key[0];
    if (n > 1)
        k_karras<<<div_up(n - 1, 256), 256, 0, s>>>(key, ctx->cloud[c], n, ctx->child, ctx->parent,
                                                    ctx->first, ctx->last, ctx->croot, ctx->wL);
    k_single_roots<<<div_up(ctx->ncloud, 128), 128, 0, s>>>(ctx->cloud_start, ctx->ncloud, n,
                                                            ctx->croot);
    // the root has no parent
    CK(cudaMemsetAsync(ctx->parent, 0xff, sizeof(int), s));
    // leaf records (they complete the leaves' first / last the groups read),
    // the groups, the nodes inside the groups, then the climb above them
    int rc = tree_records(ctx, true, all_records);
    if (rc) return rc;
    ctx->tree_ok = true;
    ctx->topo_ok = true;
    ctx->refits = 0;
    ctx->records_all = all_records;
    return ctx_check_launch(ctx, "tree");
}

// every record of every node for the current topology (sph_get_tree after a
// step, which stores the build records of the group nodes and above only)
int launch_tree_records(sph_ctx *ctx) {
    if (ctx->n <= 0) return SPH_OK;
    int rc = tree_records(ctx, false, true);
    if (rc) return rc;
    ctx->records_all = true;
    return ctx_check_launch(ctx, "tree records");
}

// The tree of a refit step: the topology, groups and super-groups of the last
// full build (the storage order has not changed since), every record of every
// node recomputed from the drifted particles.  The boxes may be looser than a
// fresh split would give, never wrong.
int launch_tree_refit(sph_ctx *ctx, bool all_records) {
    ctx->cand_ok = false;
    if (ctx->n <= 0) return SPH_OK;
    if (!ctx->topo_ok) return SPH_ERR_STATE;
    int rc = tree_records(ctx, false, all_records);
    if (rc) return rc;
    ctx->tree_ok = true;
    ctx->records_all = all_records;
    return ctx_check_launch(ctx, "tree refit");
}

int launch_leaf_records(sph_ctx *ctx) {
    const int n = ctx->n, c = ctx->cur;
    if (n <= 0) return SPH_OK;
    k_leaf_records<<<div_up(n, 256), 256, 0, ctx->stream>>>(
        n, ctx->st[c][ST_X], ctx->st[c][ST_Y], ctx->st[c][ST_Z], ctx->st[c][ST_M], ctx->node);
    return ctx_check_launch(ctx, "leaf records");
}

int launch_refit_hmax(sph_ctx *ctx, const int *need) {
    const int n = ctx->n;
    if (n <= 0) return SPH_OK;
    cudaStream_t s = ctx->stream;
    float4 *boxA = (float4 *)ctx->node_box;
    const int ggrid = max(1, div_up(div_up(n, 16) + ctx->ncloud, GUP_WARPS));
    k_refit_groups<<<ggrid, GUP_WARPS * 32, 0, s>>>(n, ctx->d_ngroup, ctx->gstart, ctx->gcount,
                                                    ctx->gnode, ctx->first, ctx->last,
                                                    ctx->st[ctx->cur][ST_H], ctx->hmax, boxA, need);
    k_refit_up<<<div_up(n, 256), 256, 0, s>>>(n, ctx->d_ngroup, ctx->gnode, ctx->parent,
                                              ctx->child, ctx->hmax, boxA, ctx->flag, need);
    return ctx_check_launch(ctx, "refit");
}
