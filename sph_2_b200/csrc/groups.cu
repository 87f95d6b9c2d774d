// groups.cu -- walk/search groups from the radix tree, and a device prefix sum.
//
// A group is a maximal tree node holding at most GROUP_MAX (32) particles of
// one cloud: its parent holds more than 32 particles or particles of several
// clouds.  These nodes partition the particles into Morton-contiguous runs that
// are compact in space by construction (a node's particles share a key
// prefix), unlike fixed 32-particle chunks of the Morton order, which can span
// a jump of the curve across the domain.  Groups are numbered in Morton order
// by a prefix sum over "group starts", so the table is deterministic; its size
// stays on the device (ctx->d_ngroup) for the persistent kernels and graphs.
#include "sph_internal.cuh"

namespace {

constexpr int SCAN_B = 1024;

__global__ void k_mark_groups(int n, const int *__restrict__ first, const int *__restrict__ last,
                              const int *__restrict__ parent, const int *__restrict__ cloud,
                              int gmax, int *__restrict__ mark, int *__restrict__ gnode) {
    const int nn = 2 * n - 1;
    int nd = blockIdx.x * blockDim.x + threadIdx.x;
    if (nd >= nn) return;
    const int f = first[nd], l = last[nd];
    if (l - f + 1 > gmax || cloud[f] != cloud[l]) return;
    const int p = parent[nd];
    bool top = p < 0;
    if (!top) {
        const int pf = first[p], pl = last[p];
        top = (pl - pf + 1 > gmax) || cloud[pf] != cloud[pl];
    }
    if (top) {
        mark[f] = 1;
        gnode[f] = nd;
    }
}

// exclusive scan, three passes: block sums, scan of the block sums (one block),
// block-local scan plus offset
__global__ void __launch_bounds__(SCAN_B) k_scan_reduce(const int *__restrict__ in, int n,
                                                        int *__restrict__ bsum) {
    __shared__ int s[SCAN_B / 32];
    int i = blockIdx.x * SCAN_B + threadIdx.x;
    int v = i < n ? in[i] : 0;
    for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x < 32) {
        int w = s[threadIdx.x];
        for (int o = 16; o; o >>= 1) w += __shfl_xor_sync(0xffffffffu, w, o);
        if (threadIdx.x == 0) bsum[blockIdx.x] = w;
    }
}

__device__ __forceinline__ int block_excl_scan(int v, int *s, int *total) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int x = v;
    for (int o = 1; o < 32; o <<= 1) {
        int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) s[w] = x;
    __syncthreads();
    if (w == 0) {
        int t = lane < (int)(blockDim.x >> 5) ? s[lane] : 0;
        for (int o = 1; o < 32; o <<= 1) {
            int y = __shfl_up_sync(0xffffffffu, t, o);
            if (lane >= o) t += y;
        }
        s[lane] = t;
    }
    __syncthreads();
    int res = x - v + (w ? s[w - 1] : 0);
    if (total) *total = s[(blockDim.x >> 5) - 1];
    __syncthreads();
    return res;
}

// one block scans the block sums in chunks of SCAN_B
__global__ void __launch_bounds__(SCAN_B) k_scan_bsums(int *bsum, int nb, int *total) {
    __shared__ int s[32];
    int run = 0;
    for (int base = 0; base < nb; base += SCAN_B) {
        int i = base + threadIdx.x;
        int v = i < nb ? bsum[i] : 0;
        int tot;
        int e = block_excl_scan(v, s, &tot);
        if (i < nb) bsum[i] = run + e;
        run += tot;
    }
    if (threadIdx.x == 0 && total) *total = run;
}

__global__ void __launch_bounds__(SCAN_B) k_scan_final(const int *__restrict__ in, int n,
                                                       const int *__restrict__ bsum,
                                                       int *__restrict__ out) {
    __shared__ int s[32];
    int i = blockIdx.x * SCAN_B + threadIdx.x;
    int v = i < n ? in[i] : 0;
    int e = block_excl_scan(v, s, nullptr);
    if (i < n) out[i] = e + bsum[blockIdx.x];
}

__global__ void k_write_groups(int n, const int *__restrict__ mark, const int *__restrict__ pos,
                               const int *__restrict__ gnode_at, const int *__restrict__ first,
                               const int *__restrict__ last, const int *__restrict__ cloud,
                               int *__restrict__ gstart, int *__restrict__ gcount,
                               int *__restrict__ gcloud, int *__restrict__ gnode) {
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n || !mark[p]) return;
    const int g = pos[p];
    const int nd = gnode_at[p];
    gstart[g] = p;
    gcount[g] = last[nd] - first[nd] + 1;
    gcloud[g] = cloud[p];
    gnode[g] = nd;
}

// super-group table (no tree node output)
__global__ void k_write_sgroups(int n, const int *__restrict__ mark, const int *__restrict__ pos,
                                const int *__restrict__ node_at, const int *__restrict__ first,
                                const int *__restrict__ last, const int *__restrict__ cloud,
                                int *__restrict__ sstart, int *__restrict__ scount,
                                int *__restrict__ scloud) {
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n || !mark[p]) return;
    const int s = pos[p];
    const int nd = node_at[p];
    sstart[s] = p;
    scount[s] = last[nd] - first[nd] + 1;
    scloud[s] = cloud[p];
}

// super-group of each group: the last super-group starting at or before the
// group's first particle (super-groups are unions of whole groups)
__global__ void k_group_sg(int n, const int *__restrict__ ngroup_p, const int *__restrict__ gstart,
                           const int *__restrict__ smark, const int *__restrict__ spos,
                           int *__restrict__ g_sg) {
    int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= *ngroup_p) return;
    const int p = gstart[g];
    g_sg[g] = spos[p] + smark[p] - 1;
}

}  // namespace

int launch_scan(sph_ctx *ctx, const int *in, int *out, int n, int *total) {
    cudaStream_t s = ctx->stream;
    const int nb = div_up(n, SCAN_B);
    int *bsum = ctx->scan_tmp;
    k_scan_reduce<<<nb, SCAN_B, 0, s>>>(in, n, bsum);
    k_scan_bsums<<<1, SCAN_B, 0, s>>>(bsum, nb, total);
    k_scan_final<<<nb, SCAN_B, 0, s>>>(in, n, bsum, out);
    return ctx_check_launch(ctx, "scan");
}

int launch_groups(sph_ctx *ctx) {
    const int n = ctx->n;
    if (n <= 0) return SPH_OK;
    cudaStream_t s = ctx->stream;
    CK(cudaMemsetAsync(ctx->gmark, 0, sizeof(int) * n, s));
    k_mark_groups<<<div_up(2 * n - 1, 256), 256, 0, s>>>(n, ctx->first, ctx->last, ctx->parent,
                                                          ctx->cloud[ctx->cur], 32, ctx->gmark,
                                                          ctx->gnode_at);
    int rc = launch_scan(ctx, ctx->gmark, ctx->gpos, n, ctx->d_ngroup);
    if (rc) return rc;
    k_write_groups<<<div_up(n, 256), 256, 0, s>>>(n, ctx->gmark, ctx->gpos, ctx->gnode_at,
                                                  ctx->first, ctx->last, ctx->cloud[ctx->cur],
                                                  ctx->gstart, ctx->gcount, ctx->groot_g,
                                                  ctx->gnode);
    if (ctx->g_sg) {
        // super-groups, in the marking arrays the group table no longer needs
        CK(cudaMemsetAsync(ctx->gmark, 0, sizeof(int) * n, s));
        k_mark_groups<<<div_up(2 * n - 1, 256), 256, 0, s>>>(n, ctx->first, ctx->last,
                                                              ctx->parent, ctx->cloud[ctx->cur],
                                                              SGROUP_MAX, ctx->gmark,
                                                              ctx->gnode_at);
        rc = launch_scan(ctx, ctx->gmark, ctx->gpos, n, ctx->d_nsg);
        if (rc) return rc;
        k_write_sgroups<<<div_up(n, 256), 256, 0, s>>>(n, ctx->gmark, ctx->gpos, ctx->gnode_at,
                                                       ctx->first, ctx->last, ctx->cloud[ctx->cur],
                                                       ctx->sg_start, ctx->sg_count, ctx->sg_cloud);
        k_group_sg<<<div_up(n, 256), 256, 0, s>>>(n, ctx->d_ngroup, ctx->gstart, ctx->gmark,
                                                  ctx->gpos, ctx->g_sg);
    }
    return ctx_check_launch(ctx, "groups");
}

extern "C" int sph_get_groups(sph_ctx *ctx, int32_t *ngroup, int32_t *gstart, int32_t *gcount,
                              int32_t host) {
    if (!ctx || !ngroup) return SPH_ERR_ARG;
    cudaSetDevice(ctx->device);
    if (!ctx->tree_ok) return SPH_ERR_STATE;
    int ng = 0;
    CK(cudaMemcpyAsync(&ng, ctx->d_ngroup, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    *ngroup = ng;
    cudaMemcpyKind k = host ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice;
    if (gstart && ng) CK(cudaMemcpyAsync(gstart, ctx->gstart, sizeof(int) * ng, k, ctx->stream));
    if (gcount && ng) CK(cudaMemcpyAsync(gcount, ctx->gcount, sizeof(int) * ng, k, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return SPH_OK;
}
