// noalloc.cu -- Morton keys and their stable sort order for caller-provided
// positions, with no device allocation.
//
// Who needs it: a caller that may not (or cannot) allocate device memory when
// it wants the particle order -- for instance code whose device memory is all
// owned by another framework's caching allocator, or that runs where a
// cudaMalloc would implicitly synchronise the device or fail without a
// recovery path.  A context (sph_ctx_create) allocates all of its buffers up
// front for its full capacity; this entry point instead uses one fixed scratch
// array compiled into the library, so the caller passes only its inputs and
// outputs.
//
// The scratch array lives in device global memory for as long as the library
// stays loaded: every GPU that loads the library holds it until the process
// exits.  All calls share it, so calls that overlap on the GPU (different
// streams or threads without ordering between them) race on it; the contents
// left by one call are not used by the next (the box is cleared at the start
// of every call, every histogram and buffer entry read is written first).
//
// The keys, box and stable LSD radix passes follow the same definitions as the
// context path (sort.cu) for one cloud: key = interleave of 21-bit cell
// coordinates in the cube spanned by the particles' box, x in the top bit of
// each triple; equal keys keep their input order.
#include <mutex>

#include "sph_internal.cuh"

namespace {

constexpr int NA_THREADS = 256;
constexpr int NA_ITEMS = 8;
constexpr int NA_TILE = NA_THREADS * NA_ITEMS;
constexpr int NA_MAX_N = SPH_NOALLOC_MAX_N;
constexpr int NA_MAX_BLOCKS = (NA_MAX_N + NA_TILE - 1) / NA_TILE;

// scratch layout (bytes): two key buffers, two value buffers, histograms
// (256 digits x blocks + 256 totals), box (6 ordered uint64)
constexpr size_t NA_KEYS = sizeof(unsigned long long) * NA_MAX_N;
constexpr size_t NA_VALS = sizeof(int) * NA_MAX_N;
constexpr size_t NA_HIST = sizeof(unsigned) * (256 * (size_t)NA_MAX_BLOCKS + 256);
constexpr size_t NA_OFF_K0 = 0;
constexpr size_t NA_OFF_K1 = NA_OFF_K0 + NA_KEYS;
constexpr size_t NA_OFF_V0 = NA_OFF_K1 + NA_KEYS;
constexpr size_t NA_OFF_V1 = NA_OFF_V0 + NA_VALS;
constexpr size_t NA_OFF_H = NA_OFF_V1 + NA_VALS;
constexpr size_t NA_OFF_BOX = (NA_OFF_H + NA_HIST + 255) / 256 * 256;
constexpr size_t NA_BYTES = NA_OFF_BOX + 6 * sizeof(unsigned long long);

static __device__ __align__(256) unsigned char g_noalloc_scratch[NA_BYTES];

__global__ void na_box_reset(unsigned long long *box) {
    int i = threadIdx.x;
    if (i < 6) box[i] = i < 3 ? ~0ULL : 0ULL;
}

__global__ void na_box(const double *__restrict__ x, const double *__restrict__ y,
                       const double *__restrict__ z, int n, unsigned long long *box) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool ok = i < n;
    unsigned long long mn[3], mx[3];
    const double p[3] = {ok ? x[i] : 0.0, ok ? y[i] : 0.0, ok ? z[i] : 0.0};
    for (int d = 0; d < 3; d++) {
        mn[d] = ok ? dbl_to_ord(p[d]) : ~0ULL;
        mx[d] = ok ? dbl_to_ord(p[d]) : 0ULL;
        for (int o = 16; o; o >>= 1) {
            unsigned long long a = __shfl_xor_sync(0xffffffffu, mn[d], o);
            unsigned long long b = __shfl_xor_sync(0xffffffffu, mx[d], o);
            mn[d] = a < mn[d] ? a : mn[d];
            mx[d] = b > mx[d] ? b : mx[d];
        }
    }
    if ((threadIdx.x & 31) == 0)
        for (int d = 0; d < 3; d++) {
            atomicMin(&box[d], mn[d]);
            atomicMax(&box[3 + d], mx[d]);
        }
}

__device__ __forceinline__ unsigned long long na_spread3(unsigned long long v) {
    v &= 0x1fffffULL;
    v = (v | v << 32) & 0x1f00000000ffffULL;
    v = (v | v << 16) & 0x1f0000ff0000ffULL;
    v = (v | v << 8) & 0x100f00f00f00f00fULL;
    v = (v | v << 4) & 0x10c30c30c30c30c3ULL;
    v = (v | v << 2) & 0x1249249249249249ULL;
    return v;
}

__device__ __forceinline__ unsigned long long na_cell(double x, double lo, double ext) {
    const double t = xdiv(xsub(x, lo), ext);
    const double s = xmul(t, 2097152.0);
    unsigned long long c = s <= 0.0 ? 0ULL : (unsigned long long)s;
    return c > 2097151ULL ? 2097151ULL : c;
}

__global__ void na_keys(const double *__restrict__ x, const double *__restrict__ y,
                        const double *__restrict__ z, int n, const unsigned long long *box,
                        unsigned long long *__restrict__ key) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double lo[3], hi[3];
    for (int d = 0; d < 3; d++) {
        lo[d] = ord_to_dbl(box[d]);
        hi[d] = ord_to_dbl(box[3 + d]);
    }
    double ext = fmax(xsub(hi[0], lo[0]), fmax(xsub(hi[1], lo[1]), xsub(hi[2], lo[2])));
    if (!(ext > 0.0)) ext = 1.0;
    key[i] = (na_spread3(na_cell(x[i], lo[0], ext)) << 2) |
             (na_spread3(na_cell(y[i], lo[1], ext)) << 1) | na_spread3(na_cell(z[i], lo[2], ext));
}

__global__ void __launch_bounds__(NA_THREADS)
    na_hist(const unsigned long long *__restrict__ kin, int n, int shift, int nb,
            unsigned *__restrict__ hist) {
    __shared__ unsigned h[256];
    const int t = threadIdx.x;
    h[t] = 0;
    __syncthreads();
    const int base = blockIdx.x * NA_TILE;
    for (int k = 0; k < NA_ITEMS; k++) {
        const int idx = base + k * NA_THREADS + t;
        if (idx < n) atomicAdd(&h[(unsigned)(kin[idx] >> shift) & 255u], 1u);
    }
    __syncthreads();
    hist[t * nb + blockIdx.x] = h[t];
}

__global__ void __launch_bounds__(256) na_scan(unsigned *hist, int nb, unsigned *tot) {
    __shared__ unsigned part[256];
    const int d = blockIdx.x, t = threadIdx.x;
    unsigned *row = hist + (size_t)d * nb;
    const int per = (nb + 255) / 256;
    const int a = t * per, b = min(nb, a + per);
    unsigned s = 0;
    for (int i = a; i < b; i++) s += row[i];
    part[t] = s;
    __syncthreads();
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

__global__ void __launch_bounds__(NA_THREADS)
    na_scatter(const unsigned long long *__restrict__ kin, const int *__restrict__ vin,
               unsigned long long *__restrict__ kout, int *__restrict__ vout, int n, int shift,
               int nb, const unsigned *__restrict__ hist, const unsigned *__restrict__ tot) {
    constexpr int NW = NA_THREADS / 32;
    __shared__ unsigned s_base[256];
    __shared__ unsigned s_run[256];
    __shared__ unsigned s_cnt[NW][257];
    const int t = threadIdx.x, w = t >> 5, lane = t & 31;
    s_run[t] = tot[t];
    __syncthreads();
    for (int o = 1; o < 256; o <<= 1) {
        unsigned v = t >= o ? s_run[t - o] : 0;
        __syncthreads();
        s_run[t] += v;
        __syncthreads();
    }
    const unsigned excl = s_run[t] - tot[t];
    __syncthreads();
    s_base[t] = excl + hist[t * nb + blockIdx.x];
    s_run[t] = 0;
    const unsigned lt = (1u << lane) - 1u;
    const int base = blockIdx.x * NA_TILE;
    for (int k = 0; k < NA_ITEMS; k++) {
        const int idx = base + k * NA_THREADS + t;
        const bool ok = idx < n;
        const unsigned long long key = ok ? kin[idx] : 0ULL;
        const int val = ok ? (vin ? vin[idx] : idx) : 0;
        const unsigned d = ok ? (unsigned)(key >> shift) & 255u : 256u;
        for (int j = lane; j < 257; j += 32) s_cnt[w][j] = 0;
        __syncthreads();
        const unsigned peers = __match_any_sync(0xffffffffu, d);
        const unsigned r = __popc(peers & lt);
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
            const unsigned pos = s_base[d] + pre;
            kout[pos] = key;
            vout[pos] = val;
        }
        __syncthreads();
    }
}

// device address of the scratch array, fetched once per device and kept for
// the life of the process: a caller that resets the device (cudaDeviceReset)
// or otherwise destroys its primary context must reload the library before it
// calls this entry point again, since the address belongs to the old context
std::mutex g_na_mutex;
void *g_na_ptr[256] = {};

int na_scratch(int dev, unsigned char **out) {
    if (dev < 0 || dev >= 256) return SPH_ERR_ARG;
    std::lock_guard<std::mutex> lock(g_na_mutex);
    if (!g_na_ptr[dev]) {
        void *p = nullptr;
        if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) return SPH_ERR_CUDA;
        g_na_ptr[dev] = p;
    }
    *out = (unsigned char *)g_na_ptr[dev];
    return SPH_OK;
}

}  // namespace

extern "C" int sph_morton_sort_noalloc(const double *x, const double *y, const double *z,
                                       int32_t n, uint64_t *keys, int32_t *perm,
                                       void *cuda_stream) {
    if (n < 0) return SPH_ERR_ARG;
    if (n > NA_MAX_N) return SPH_ERR_CAPACITY;
    if (n == 0) return SPH_OK;
    if (!x || !y || !z || !keys || !perm) return SPH_ERR_ARG;
    // an error left pending by the caller's earlier work is not ours to
    // report or to clear: refuse to launch and leave it for the caller
    if (cudaPeekAtLastError() != cudaSuccess) return SPH_ERR_CUDA;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return SPH_ERR_CUDA;
    unsigned char *base = nullptr;
    int rc = na_scratch(dev, &base);
    if (rc) return rc;
    cudaStream_t s = (cudaStream_t)cuda_stream;
    unsigned long long *kbuf[2] = {(unsigned long long *)(base + NA_OFF_K0),
                                   (unsigned long long *)(base + NA_OFF_K1)};
    int *vbuf[2] = {(int *)(base + NA_OFF_V0), (int *)(base + NA_OFF_V1)};
    unsigned *hist = (unsigned *)(base + NA_OFF_H);
    unsigned long long *box = (unsigned long long *)(base + NA_OFF_BOX);
    const int nb = (n + NA_TILE - 1) / NA_TILE;
    unsigned *tot = hist + (size_t)256 * nb;
    unsigned long long *ukeys = (unsigned long long *)keys;

    na_box_reset<<<1, 32, 0, s>>>(box);
    na_box<<<(n + 255) / 256, 256, 0, s>>>(x, y, z, n, box);
    na_keys<<<(n + 255) / 256, 256, 0, s>>>(x, y, z, n, box, ukeys);
    // 8 passes of 8 bits; the input keys stay untouched in the caller's array,
    // the last pass writes the permutation straight into perm
    const unsigned long long *kin = ukeys;
    const int *vin = nullptr;
    for (int p = 0; p < 8; p++) {
        unsigned long long *kout = kbuf[p & 1];
        int *vout = p == 7 ? perm : vbuf[p & 1];
        na_hist<<<nb, NA_THREADS, 0, s>>>(kin, n, 8 * p, nb, hist);
        na_scan<<<256, 256, 0, s>>>(hist, nb, tot);
        na_scatter<<<nb, NA_THREADS, 0, s>>>(kin, vin, kout, vout, n, 8 * p, nb, hist, tot);
        kin = kout;
        vin = vout;
    }
    // no error was pending on entry, so one found now comes from these launches
    return cudaGetLastError() == cudaSuccess ? SPH_OK : SPH_ERR_CUDA;
}
