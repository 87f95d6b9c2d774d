// sort.cu -- per-cloud bounding box, 63-bit Morton keys, stable LSD radix
// sort and the permutation of the particle state into key order.
//
// Replaces compute_bounding_box_kernel (bh_tree_iteration_v2.h:76-145: one
// block, a global spin lock, box accumulators started at 0) and the 10^3-cell
// counting sort CountBodies/ComputeOffset/GroupBodies (ngb_v3.h:58-117, with
// an atomicAdd-ordered, nondeterministic result).  Here the box is an exact
// FP64 min/max (order independent), keys are computed with the roundings
// spelled out so they equal the oracle's bit for bit, and the sort is stable
// so the permutation is a pure function of (keys, storage order).
#include "sph_internal.cuh"

namespace {

constexpr int SORT_THREADS = 256;
constexpr int SORT_ITEMS = 8;
constexpr int SORT_TILE = SORT_THREADS * SORT_ITEMS;

__device__ __forceinline__ unsigned long long warp_min_u64(unsigned long long v) {
    for (int o = 16; o > 0; o >>= 1) {
        unsigned long long w = __shfl_xor_sync(0xffffffffu, v, o);
        v = w < v ? w : v;
    }
    return v;
}
__device__ __forceinline__ unsigned long long warp_max_u64(unsigned long long v) {
    for (int o = 16; o > 0; o >>= 1) {
        unsigned long long w = __shfl_xor_sync(0xffffffffu, v, o);
        v = w > v ? w : v;
    }
    return v;
}

// box[6*c + 0..2] = ordered min, [3..5] = ordered max; reset to (~0, 0)
__global__ void k_box_reset(unsigned long long *box, int ncloud) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < 6 * ncloud) box[i] = (i % 6) < 3 ? ~0ULL : 0ULL;
}

__global__ void k_box(const double *__restrict__ x, const double *__restrict__ y,
                      const double *__restrict__ z, const int *__restrict__ cloud, int n,
                      unsigned long long *box, long long *status) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    bool ok = i < n;
    int c = ok ? cloud[i] : -1;
    unsigned long long o[3];
    double p[3] = {ok ? x[i] : 0.0, ok ? y[i] : 0.0, ok ? z[i] : 0.0};
    bool fin = isfinite(p[0]) && isfinite(p[1]) && isfinite(p[2]);
    if (ok && !fin) status_add(status, SPH_S_NONFINITE, 1);
    for (int d = 0; d < 3; d++) o[d] = dbl_to_ord(p[d]);
    // one set of atomics per block when the whole block holds one cloud (the
    // usual case: clouds are contiguous), else per warp or per particle
    __shared__ unsigned long long smn[3][8], smx[3][8];
    __shared__ int scl[8];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    unsigned same = __match_any_sync(0xffffffffu, c);
    const bool uni = same == 0xffffffffu && c >= 0;
    if (uni) {
        for (int d = 0; d < 3; d++) {
            const unsigned long long mn = warp_min_u64(o[d]), mx = warp_max_u64(o[d]);
            if (lane == 0) {
                smn[d][w] = mn;
                smx[d][w] = mx;
            }
        }
    } else if (ok) {
        for (int d = 0; d < 3; d++) {
            atomicMin(&box[6 * c + d], o[d]);
            atomicMax(&box[6 * c + 3 + d], o[d]);
        }
    }
    if (lane == 0) scl[w] = uni ? c : -1;
    __syncthreads();
    const int nw = blockDim.x >> 5;
    if (threadIdx.x == 0) {
        bool block_uni = scl[0] >= 0;
        for (int k = 1; k < nw; k++) block_uni = block_uni && scl[k] == scl[0];
        if (block_uni) {
            for (int d = 0; d < 3; d++) {
                unsigned long long mn = smn[d][0], mx = smx[d][0];
                for (int k = 1; k < nw; k++) {
                    mn = smn[d][k] < mn ? smn[d][k] : mn;
                    mx = smx[d][k] > mx ? smx[d][k] : mx;
                }
                atomicMin(&box[6 * scl[0] + d], mn);
                atomicMax(&box[6 * scl[0] + 3 + d], mx);
            }
        } else {
            for (int k = 0; k < nw; k++)
                if (scl[k] >= 0)
                    for (int d = 0; d < 3; d++) {
                        atomicMin(&box[6 * scl[k] + d], smn[d][k]);
                        atomicMax(&box[6 * scl[k] + 3 + d], smx[d][k]);
                    }
        }
    }
}

__device__ __forceinline__ unsigned long long spread3(unsigned long long v) {
    v &= 0x1fffffULL;
    v = (v | v << 32) & 0x1f00000000ffffULL;
    v = (v | v << 16) & 0x1f0000ff0000ffULL;
    v = (v | v << 8) & 0x100f00f00f00f00fULL;
    v = (v | v << 4) & 0x10c30c30c30c30c3ULL;
    v = (v | v << 2) & 0x1249249249249249ULL;
    return v;
}

__device__ __forceinline__ unsigned long long cell_coord(double x, double lo, double ext, int bits) {
    double t = xdiv(xsub(x, lo), ext);
    double s = xmul(t, (double)(1ULL << bits));
    unsigned long long c = s <= 0.0 ? 0ULL : (unsigned long long)s;
    unsigned long long cmax = (1ULL << bits) - 1ULL;
    return c > cmax ? cmax : c;
}

// key = (cloud << 3*bits) | interleave(ix, iy, iz), x in the top bit of each
// triple; cubic cells of side ext/2^bits with ext the box's largest side
__global__ void k_keys(const double *__restrict__ x, const double *__restrict__ y,
                       const double *__restrict__ z, const int *__restrict__ cloud, int n,
                       const unsigned long long *__restrict__ box, int bits,
                       unsigned long long *__restrict__ key) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int c = cloud[i];
    double lo[3], hi[3];
    for (int d = 0; d < 3; d++) {
        lo[d] = ord_to_dbl(box[6 * c + d]);
        hi[d] = ord_to_dbl(box[6 * c + 3 + d]);
    }
    double ext = fmax(xsub(hi[0], lo[0]), fmax(xsub(hi[1], lo[1]), xsub(hi[2], lo[2])));
    if (!(ext > 0.0)) ext = 1.0;
    unsigned long long ix = cell_coord(x[i], lo[0], ext, bits);
    unsigned long long iy = cell_coord(y[i], lo[1], ext, bits);
    unsigned long long iz = cell_coord(z[i], lo[2], ext, bits);
    key[i] = ((unsigned long long)c << (3 * bits)) | (spread3(ix) << 2) | (spread3(iy) << 1) |
             spread3(iz);
}

// ---- LSD radix sort, 8-bit digits ----
// hist layout: hist[d * nb + b] (digit major) so one scan per digit gives the
// block offsets; tot[d] = count of digit d over all blocks.
__global__ void __launch_bounds__(SORT_THREADS)
    k_radix_hist(const unsigned long long *__restrict__ kin, int n, int shift, int nb,
                 unsigned *__restrict__ hist) {
    __shared__ unsigned h[256];
    int t = threadIdx.x;
    h[t] = 0;
    __syncthreads();
    int base = blockIdx.x * SORT_TILE;
#pragma unroll
    for (int k = 0; k < SORT_ITEMS; k++) {
        int idx = base + k * SORT_THREADS + t;
        if (idx < n) atomicAdd(&h[(unsigned)(kin[idx] >> shift) & 255u], 1u);
    }
    __syncthreads();
    hist[t * nb + blockIdx.x] = h[t];
}

// one block per digit: exclusive scan of hist[d*nb .. d*nb+nb-1] in place
__global__ void __launch_bounds__(256) k_radix_scan(unsigned *hist, int nb, unsigned *tot) {
    __shared__ unsigned part[256];
    int d = blockIdx.x, t = threadIdx.x;
    unsigned *row = hist + (size_t)d * nb;
    int per = (nb + 255) / 256;
    int a = t * per, b = min(nb, a + per);
    unsigned s = 0;
    for (int i = a; i < b; i++) s += row[i];
    part[t] = s;
    __syncthreads();
    // inclusive scan of the 256 partials (Hillis-Steele)
    for (int o = 1; o < 256; o <<= 1) {
        unsigned v = t >= o ? part[t - o] : 0;
        __syncthreads();
        part[t] += v;
        __syncthreads();
    }
    unsigned run = t ? part[t - 1] : 0;
    for (int i = a; i < b; i++) {
        unsigned v = row[i];
        row[i] = run;
        run += v;
    }
    if (t == 255) tot[d] = part[255];
}

// Stable scatter.  Item k of thread t of block b is element b*TILE + k*256 + t,
// so the loop over k (and warps, lanes) walks the tile in storage order; the
// rank of an element among equal digits is (count in earlier k) + (count in
// earlier warps of this k) + (lower lanes of its warp with the same digit).
__global__ void __launch_bounds__(SORT_THREADS)
    k_radix_scatter(const unsigned long long *__restrict__ kin, const int *__restrict__ vin,
                    unsigned long long *__restrict__ kout, int *__restrict__ vout, int n,
                    int shift, int nb, const unsigned *__restrict__ hist,
                    const unsigned *__restrict__ tot) {
    constexpr int NW = SORT_THREADS / 32;
    __shared__ unsigned s_base[256];
    __shared__ unsigned s_run[256];
    __shared__ unsigned s_cnt[NW][257];
    int t = threadIdx.x, w = t >> 5, lane = t & 31;
    // exclusive scan of the digit totals
    s_run[t] = tot[t];
    __syncthreads();
    for (int o = 1; o < 256; o <<= 1) {
        unsigned v = t >= o ? s_run[t - o] : 0;
        __syncthreads();
        s_run[t] += v;
        __syncthreads();
    }
    unsigned excl = s_run[t] - tot[t];
    __syncthreads();
    s_base[t] = excl + hist[t * nb + blockIdx.x];
    s_run[t] = 0;
    const unsigned lt = (1u << lane) - 1u;
    int base = blockIdx.x * SORT_TILE;
    for (int k = 0; k < SORT_ITEMS; k++) {
        int idx = base + k * SORT_THREADS + t;
        bool ok = idx < n;
        unsigned long long key = ok ? kin[idx] : 0ULL;
        int val = ok ? (vin ? vin[idx] : idx) : 0;
        unsigned d = ok ? (unsigned)(key >> shift) & 255u : 256u;
        for (int j = lane; j < 257; j += 32) s_cnt[w][j] = 0;
        __syncthreads();
        unsigned peers = __match_any_sync(0xffffffffu, d);
        unsigned r = __popc(peers & lt);
        if (r == 0) s_cnt[w][d] = __popc(peers);
        __syncthreads();
        unsigned pre = r;
        if (ok) {
            pre += s_run[d];
            for (int ww = 0; ww < w; ww++) pre += s_cnt[ww][d];
        }
        __syncthreads();
        {
            unsigned add = 0;
            for (int ww = 0; ww < NW; ww++) add += s_cnt[ww][t];
            s_run[t] += add;
        }
        if (ok) {
            unsigned pos = s_base[d] + pre;
            kout[pos] = key;
            vout[pos] = val;
        }
        __syncthreads();  // s_cnt is cleared again by the next item
    }
}

// origin of each cloud's FP32 walk coordinates: the centre of its box (0
// for a cloud without a finite box)
__global__ void k_origin(const unsigned long long *__restrict__ box, int ncloud,
                         double *__restrict__ corg) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= ncloud) return;
    for (int d = 0; d < 3; d++) {
        const double lo = ord_to_dbl(box[6 * c + d]), hi = ord_to_dbl(box[6 * c + 3 + d]);
        corg[3 * c + d] = lo <= hi ? 0.5 * (lo + hi) : 0.0;
    }
}

struct PermTab {
    const double *src[ST_N];
    double *dst[ST_N];
};

template <class R>
__global__ void k_permute(int n, const int *__restrict__ perm, const PermTab tab, const int *__restrict__ id_in,
                          const int *__restrict__ cl_in, int *__restrict__ id_out,
                          int *__restrict__ cl_out, double4 *__restrict__ p0,
                          typename R4<R>::T *__restrict__ p1, typename R4<R>::T *__restrict__ pw,
                          const double *__restrict__ corg) {
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    int o = perm[s];
    double v[ST_N];
#pragma unroll
    for (int k = 0; k < ST_N; k++) v[k] = tab.src[k][o];
#pragma unroll
    for (int k = 0; k < ST_N; k++) tab.dst[k][s] = v[k];
    const int cl = cl_in[o];
    id_out[s] = id_in[o];
    cl_out[s] = cl;
    p0[s] = make_double4(v[ST_X], v[ST_Y], v[ST_Z], v[ST_H]);
    typename R4<R>::T a, b;
    a.x = (R)v[ST_VX]; a.y = (R)v[ST_VY]; a.z = (R)v[ST_VZ]; a.w = (R)v[ST_M];
    const double *org = corg + 3 * cl;
    b.x = (R)(v[ST_X] - WalkOrigin<R>::off(org, 0));
    b.y = (R)(v[ST_Y] - WalkOrigin<R>::off(org, 1));
    b.z = (R)(v[ST_Z] - WalkOrigin<R>::off(org, 2));
    b.w = (R)v[ST_M];
    p1[s] = a;
    pw[s] = b;
}

}  // namespace

static int morton_bits_for(int ncloud) {
    int cb = 0;
    while ((1 << cb) < ncloud) cb++;
    return (63 - cb) / 3;
}

// The first phase of a refit step: the per-cloud boxes (non-finite check and
// the origin of the FP32 walk coordinates) and the packed records of the
// drifted particles, in the storage order of the last sort.
int launch_sort_refit(sph_ctx *ctx) {
    ctx->cand_ok = false;
    const int n = ctx->n;
    if (n <= 0) return SPH_OK;
    cudaStream_t s = ctx->stream;
    double *const *st = ctx->st[ctx->cur];
    k_box_reset<<<div_up(6 * ctx->ncloud, 256), 256, 0, s>>>(ctx->box, ctx->ncloud);
    k_box<<<div_up(n, 256), 256, 0, s>>>(st[ST_X], st[ST_Y], st[ST_Z], ctx->cloud[ctx->cur], n,
                                         ctx->box, ctx->status);
    k_origin<<<div_up(ctx->ncloud, 128), 128, 0, s>>>(ctx->box, ctx->ncloud, ctx->corg);
    // same order: the drift is added to the distances moved
    int rc = launch_pack_p1(ctx, true);
    if (rc) return rc;
    return ctx_check_launch(ctx, "sort refit");
}

int launch_sort(sph_ctx *ctx) {
    ctx->cand_ok = false;
    ctx->topo_ok = false;  // the next tree build splits the new order
    // the candidate rows hold storage indices of the old order
    int rc0 = launch_rows_invalidate(ctx);
    if (rc0) return rc0;
    const int n = ctx->n;
    if (n <= 0) return SPH_OK;
    cudaStream_t s = ctx->stream;
    const int c = ctx->cur;
    double *const *st = ctx->st[c];
    k_box_reset<<<div_up(6 * ctx->ncloud, 256), 256, 0, s>>>(ctx->box, ctx->ncloud);
    k_box<<<div_up(n, 256), 256, 0, s>>>(st[ST_X], st[ST_Y], st[ST_Z], ctx->cloud[c], n, ctx->box,
                                         ctx->status);
    k_origin<<<div_up(ctx->ncloud, 128), 128, 0, s>>>(ctx->box, ctx->ncloud, ctx->corg);
    const int bits = morton_bits_for(ctx->ncloud);
    k_keys<<<div_up(n, 256), 256, 0, s>>>(st[ST_X], st[ST_Y], st[ST_Z], ctx->cloud[c], n, ctx->box,
                                          bits, ctx->key_in);
    const int used = 63;
    const int passes = (used + 7) / 8;
    const int nb = div_up(n, SORT_TILE);
    unsigned *tot = ctx->hist + (size_t)256 * nb;
    const unsigned long long *kin = ctx->key_in;
    const int *vin = nullptr;
    int outb = 1;
    for (int p = 0; p < passes; p++) {
        int shift = 8 * p;
        unsigned long long *kout = ctx->key[outb];
        int *vout = ctx->val[outb];
        k_radix_hist<<<nb, SORT_THREADS, 0, s>>>(kin, n, shift, nb, ctx->hist);
        k_radix_scan<<<256, 256, 0, s>>>(ctx->hist, nb, tot);
        k_radix_scatter<<<nb, SORT_THREADS, 0, s>>>(kin, vin, kout, vout, n, shift, nb, ctx->hist,
                                                    tot);
        kin = kout;
        vin = vout;
        outb ^= 1;
    }
    // passes is even, so the sorted keys/values end in buffer 0
    static_assert(((63 + 7) / 8) % 2 == 0, "radix pass count must be even");
    ctx->perm = ctx->val[0];
    const int d = c ^ 1;
    PermTab tab;
    for (int k = 0; k < ST_N; k++) {
        tab.src[k] = ctx->st[c][k];
        tab.dst[k] = ctx->st[d][k];
    }
    if (ctx->cfg.precision == SPH_PREC_MIXED)
        k_permute<float><<<div_up(n, 256), 256, 0, s>>>(n, ctx->perm, tab, ctx->id[c],
                                                        ctx->cloud[c], ctx->id[d], ctx->cloud[d],
                                                        ctx->p0, (float4 *)ctx->p1, (float4 *)ctx->pw,
                                                        ctx->corg);
    else
        k_permute<double><<<div_up(n, 256), 256, 0, s>>>(n, ctx->perm, tab, ctx->id[c],
                                                         ctx->cloud[c], ctx->id[d], ctx->cloud[d],
                                                         ctx->p0, (double4 *)ctx->p1,
                                                         (double4 *)ctx->pw, ctx->corg);
    ctx->cur = d;
    return ctx_check_launch(ctx, "sort");
}
