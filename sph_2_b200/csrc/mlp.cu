// mlp.cu -- the cooling surrogate: a 3 -> 64 -> 64 -> 1 MLP (tanh-GELU),
// BF16 operands with FP32 accumulation on the tensor cores.  Inference (the
// in-step surrogate, the standalone solves and sph_mlp_forward) runs its 64 x 64
// layer on tcgen05.mma with a TMEM accumulator, 128 rows per CTA (namespace
// tc below); training (forward + backward of minibatches, weight gradients from
// transposed activations) uses the warp-level mma.sync.aligned.m16n8k16 bf16
// fragments, and SPH_FLAG_MLP_WARP_MMA selects them for inference too.  All
// kernels are written here, with Adam, and the in-step use: predict
// dlog10(u) = log10(u_new/u_old) from (log10 rho, log10 u, log10 dt) [cgs],
// estimate the error of the prediction with the Newton residual of the
// implicit equation after up to four Newton steps from it, and fall back
// to the exact solver where it exceeds the tolerance or where the implicit
// equation is not monotone between u_old and the prediction (there it can have
// several roots and the surrogate may have found another one).  No reference counterpart: the reference always runs the
// bisection (myPhotoLibsGPU.h:615-686) or a table lookup (hcoolingx,
// hfvCLibs_v7_hfv_v2.h:1240-1418).
//
// Parameters (FP32 masters, SPH_MLP_NPARAM): W1[3][64] b1[64] W2[64][64]
// b2[64] W3[64] b3 -- layer k computes z = a W + b with a the row vector of
// the previous layer -- followed by norm[8] = (mean[3], scale[3], y_mean,
// y_scale).  Packed BF16 operand tables: W1t[64][16] (out x in, K padded to
// 16), W2t[64][64] (out x in) for the forward pass, W2[64][64] (in x out) for
// the backward pass.
//
// MMA fragment layout (per lane, gid = lane/4, tig = lane%4): A 16x16 holds
// rows gid, gid+8 at columns 2tig..2tig+1 and 2tig+8..+9; B 16x8 holds
// k = 2tig..+1 and 2tig+8..+9 at column gid; C 16x8 holds rows gid, gid+8 at
// columns 2tig..+1.  Two adjacent C tiles of one layer are exactly the A
// fragment of the next layer's K step, so activations stay in registers.
#include <cuda_bf16.h>

#include "cooling.cuh"

namespace {

constexpr int H = 64;
constexpr int NP = SPH_MLP_NPARAM;
constexpr int OFF_W1 = 0, OFF_B1 = 192, OFF_W2 = 256, OFF_B2 = 4352, OFF_W3 = 4416, OFF_B3 = 4480;
constexpr int PK_W1T = 0, PK_W2T = 1024, PK_W2 = 1024 + 4096, PK_N = 1024 + 2 * 4096;
constexpr unsigned FULL = 0xffffffffu;

__device__ __forceinline__ void mma16816(float *d, const unsigned *a, const unsigned *b) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
        "{%8,%9}, {%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

__device__ __forceinline__ unsigned pack2(float lo, float hi) {
    __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<unsigned *>(&v);
}
__device__ __forceinline__ unsigned ld32(const __nv_bfloat16 *p) {
    return *reinterpret_cast<const unsigned *>(p);
}

// tanh form of GELU and its derivative
__device__ __forceinline__ float gelu(float z) {
    const float k = 0.7978845608028654f;
    return 0.5f * z * (1.0f + tanhf(k * (z + 0.044715f * z * z * z)));
}
// the same with the hardware tanh approximation (tanh.approx.f32, relative
// error about 2^-11, below the BF16 rounding of the activations it feeds):
// used by the in-step inference only; training and the reference forward
// keep tanhf
__device__ __forceinline__ float gelu_fast(float z) {
    const float k = 0.7978845608028654f;
    float t;
    asm("tanh.approx.f32 %0, %1;" : "=f"(t) : "f"(k * (z + 0.044715f * z * z * z)));
    return 0.5f * z * (1.0f + t);
}
template <bool FAST> __device__ __forceinline__ float act(float z) { return FAST ? gelu_fast(z) : gelu(z); }
__device__ __forceinline__ float gelu_grad(float z) {
    const float k = 0.7978845608028654f;
    const float t = tanhf(k * (z + 0.044715f * z * z * z));
    return 0.5f * (1.0f + t) + 0.5f * z * (1.0f - t * t) * k * (1.0f + 3.0f * 0.044715f * z * z);
}

struct MlpSmem {
    __nv_bfloat16 w[PK_N];     // W1t, W2t, W2
    float b1[H], b2[H], w3[H], b3;
};

__device__ __forceinline__ void load_weights(MlpSmem &S, const __nv_bfloat16 *pk, const float *P) {
    for (int k = threadIdx.x; k < PK_N / 2; k += blockDim.x)
        reinterpret_cast<unsigned *>(S.w)[k] = reinterpret_cast<const unsigned *>(pk)[k];
    for (int k = threadIdx.x; k < H; k += blockDim.x) {
        S.b1[k] = P[OFF_B1 + k];
        S.b2[k] = P[OFF_B2 + k];
        S.w3[k] = P[OFF_W3 + k];
    }
    if (threadIdx.x == 0) S.b3 = P[OFF_B3];
    __syncthreads();
}

// forward of one 16-row tile: ax = A fragment of X (16 x 16, 3 real columns);
// z1, z2 pre-activations (C fragments), y for rows gid and gid+8
template <bool FAST = false>
__device__ __forceinline__ void tile_forward(const MlpSmem &S, const unsigned *ax, float z1[8][4],
                                             float z2[8][4], float &y0, float &y1) {
    const int lane = threadIdx.x & 31, gid = lane >> 2, tig = lane & 3;
    const __nv_bfloat16 *W1t = S.w + PK_W1T, *W2t = S.w + PK_W2T;
#pragma unroll
    for (int nt = 0; nt < 8; nt++) {
        const int col = nt * 8 + 2 * tig;
        z1[nt][0] = S.b1[col]; z1[nt][1] = S.b1[col + 1];
        z1[nt][2] = S.b1[col]; z1[nt][3] = S.b1[col + 1];
        const __nv_bfloat16 *wb = W1t + (nt * 8 + gid) * 16 + 2 * tig;
        const unsigned b[2] = {ld32(wb), ld32(wb + 8)};
        mma16816(z1[nt], ax, b);
    }
    unsigned a2[4][4];
#pragma unroll
    for (int kk = 0; kk < 4; kk++) {
        a2[kk][0] = pack2(act<FAST>(z1[2 * kk][0]), act<FAST>(z1[2 * kk][1]));
        a2[kk][1] = pack2(act<FAST>(z1[2 * kk][2]), act<FAST>(z1[2 * kk][3]));
        a2[kk][2] = pack2(act<FAST>(z1[2 * kk + 1][0]), act<FAST>(z1[2 * kk + 1][1]));
        a2[kk][3] = pack2(act<FAST>(z1[2 * kk + 1][2]), act<FAST>(z1[2 * kk + 1][3]));
    }
    float s0 = 0.f, s1 = 0.f;
#pragma unroll
    for (int nt = 0; nt < 8; nt++) {
        const int col = nt * 8 + 2 * tig;
        z2[nt][0] = S.b2[col]; z2[nt][1] = S.b2[col + 1];
        z2[nt][2] = S.b2[col]; z2[nt][3] = S.b2[col + 1];
#pragma unroll
        for (int kk = 0; kk < 4; kk++) {
            const __nv_bfloat16 *wb = W2t + (nt * 8 + gid) * 64 + kk * 16 + 2 * tig;
            const unsigned b[2] = {ld32(wb), ld32(wb + 8)};
            mma16816(z2[nt], a2[kk], b);
        }
        s0 += act<FAST>(z2[nt][0]) * S.w3[col] + act<FAST>(z2[nt][1]) * S.w3[col + 1];
        s1 += act<FAST>(z2[nt][2]) * S.w3[col] + act<FAST>(z2[nt][3]) * S.w3[col + 1];
    }
    s0 += __shfl_xor_sync(FULL, s0, 1);
    s0 += __shfl_xor_sync(FULL, s0, 2);
    s1 += __shfl_xor_sync(FULL, s1, 1);
    s1 += __shfl_xor_sync(FULL, s1, 2);
    y0 = s0 + S.b3;
    y1 = s1 + S.b3;
}

// A fragment of a 16-row tile of X staged row-major as bf16 [16][16]
__device__ __forceinline__ void x_fragment(const __nv_bfloat16 *X16, unsigned *ax) {
    const int lane = threadIdx.x & 31, gid = lane >> 2, tig = lane & 3;
    ax[0] = ld32(X16 + gid * 16 + 2 * tig);
    ax[1] = ld32(X16 + (gid + 8) * 16 + 2 * tig);
    ax[2] = ld32(X16 + gid * 16 + 2 * tig + 8);
    ax[3] = ld32(X16 + (gid + 8) * 16 + 2 * tig + 8);
}

__global__ void k_mlp_pack(const float *__restrict__ P, __nv_bfloat16 *__restrict__ pk) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < 1024) {  // W1t[j][c]
        const int j = t / 16, c = t % 16;
        pk[PK_W1T + t] = __float2bfloat16_rn(c < 3 ? P[OFF_W1 + c * H + j] : 0.f);
    } else if (t < 1024 + 4096) {  // W2t[j][i] = W2[i][j]
        const int u = t - 1024, j = u / 64, i = u % 64;
        pk[PK_W2T + u] = __float2bfloat16_rn(P[OFF_W2 + i * H + j]);
    } else if (t < PK_N) {  // W2[i][j]
        const int u = t - 1024 - 4096;
        pk[PK_W2 + u] = __float2bfloat16_rn(P[OFF_W2 + u]);
    }
}

// forward on n rows of normalised X[n][3] -> y[n]; one warp per 16-row tile
__global__ void __launch_bounds__(128)
    k_mlp_forward(int n, const float *__restrict__ X, float *__restrict__ y,
                  const __nv_bfloat16 *__restrict__ pk, const float *__restrict__ P) {
    __shared__ MlpSmem S;
    __shared__ __align__(16) __nv_bfloat16 xs[4][16 * 16];
    load_weights(S, pk, P);
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int ntile = (n + 15) / 16;
    for (int tile = blockIdx.x * 4 + w; tile < ntile; tile += gridDim.x * 4) {
        const int r0 = tile * 16;
        for (int e = lane; e < 256; e += 32) {
            const int r = e / 16, c = e % 16;
            const int row = r0 + r;
            xs[w][e] = __float2bfloat16_rn((c < 3 && row < n) ? X[3 * row + c] : 0.f);
        }
        __syncwarp();
        unsigned ax[4];
        x_fragment(xs[w], ax);
        float z1[8][4], z2[8][4], y0, y1;
        tile_forward(S, ax, z1, z2, y0, y1);
        const int gid = lane >> 2, tig = lane & 3;
        if (tig == 0) {
            if (r0 + gid < n) y[r0 + gid] = y0;
            if (r0 + gid + 8 < n) y[r0 + gid + 8] = y1;
        }
        __syncwarp();
    }
}

// gradient of L = 0.5/n_total * sum (y - t)^2 over this launch's rows, added
// into grad (FP32, pre-zeroed); loss added into *loss
constexpr int GR = 256;        // rows per block
constexpr int LD = GR + 8;     // padded row stride of the transposed tiles
struct GradSmem {
    MlpSmem W;
    __nv_bfloat16 X[GR * 16];  // row-major [r][c]
    __nv_bfloat16 Xt[16 * LD]; // [c][r]
    __nv_bfloat16 At1[H * LD]; // gelu(z1) transposed [i][r]
    __nv_bfloat16 dZ2t[H * LD];
    __nv_bfloat16 dZ1t[H * LD];
    float gb1[H], gb2[H], gw3[H], gb3, loss;
};

__global__ void __launch_bounds__(128)
    k_mlp_grad(int n, const float *__restrict__ X, const float *__restrict__ T, float inv_n,
               const __nv_bfloat16 *__restrict__ pk, const float *__restrict__ P,
               float *__restrict__ grad, float *__restrict__ loss) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    GradSmem &S = *reinterpret_cast<GradSmem *>(smem_raw);
    load_weights(S.W, pk, P);
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31, gid = lane >> 2, tig = lane & 3;
    const int rb = blockIdx.x * GR;
    for (int e = threadIdx.x; e < GR * 16; e += blockDim.x) {
        const int r = e / 16, c = e % 16;
        const float v = (c < 3 && rb + r < n) ? X[3 * (rb + r) + c] : 0.f;
        const __nv_bfloat16 bv = __float2bfloat16_rn(v);
        S.X[e] = bv;
        S.Xt[c * LD + r] = bv;
    }
    for (int k = threadIdx.x; k < H; k += blockDim.x) S.gb1[k] = S.gb2[k] = S.gw3[k] = 0.f;
    if (threadIdx.x == 0) S.gb3 = S.loss = 0.f;
    __syncthreads();
    const __nv_bfloat16 *W2 = S.W.w + PK_W2;
    float pb3 = 0.f, pl = 0.f;
    for (int tile = w; tile < GR / 16; tile += 4) {
        const int r0 = tile * 16;
        unsigned ax[4];
        x_fragment(S.X + r0 * 16, ax);
        float z1[8][4], z2[8][4], y0, y1;
        tile_forward(S.W, ax, z1, z2, y0, y1);
        const bool ok0 = rb + r0 + gid < n, ok1 = rb + r0 + gid + 8 < n;
        const float e0 = ok0 ? y0 - T[rb + r0 + gid] : 0.f;
        const float e1 = ok1 ? y1 - T[rb + r0 + gid + 8] : 0.f;
        const float dy0 = e0 * inv_n, dy1 = e1 * inv_n;
        if (tig == 0) {
            pl += 0.5f * inv_n * (e0 * e0 + e1 * e1);
            pb3 += dy0 + dy1;
        }
        // dZ2, bias/W3 partials, transposed tiles for the weight GEMMs
        float dz2[8][4];
#pragma unroll
        for (int nt = 0; nt < 8; nt++) {
            const int col = nt * 8 + 2 * tig;
            const float w30 = S.W.w3[col], w31 = S.W.w3[col + 1];
            dz2[nt][0] = dy0 * w30 * gelu_grad(z2[nt][0]);
            dz2[nt][1] = dy0 * w31 * gelu_grad(z2[nt][1]);
            dz2[nt][2] = dy1 * w30 * gelu_grad(z2[nt][2]);
            dz2[nt][3] = dy1 * w31 * gelu_grad(z2[nt][3]);
            atomicAdd(&S.gw3[col], gelu(z2[nt][0]) * dy0 + gelu(z2[nt][2]) * dy1);
            atomicAdd(&S.gw3[col + 1], gelu(z2[nt][1]) * dy0 + gelu(z2[nt][3]) * dy1);
            atomicAdd(&S.gb2[col], dz2[nt][0] + dz2[nt][2]);
            atomicAdd(&S.gb2[col + 1], dz2[nt][1] + dz2[nt][3]);
            const int ra = r0 + gid, rc = r0 + gid + 8;
            S.At1[col * LD + ra] = __float2bfloat16_rn(gelu(z1[nt][0]));
            S.At1[(col + 1) * LD + ra] = __float2bfloat16_rn(gelu(z1[nt][1]));
            S.At1[col * LD + rc] = __float2bfloat16_rn(gelu(z1[nt][2]));
            S.At1[(col + 1) * LD + rc] = __float2bfloat16_rn(gelu(z1[nt][3]));
            S.dZ2t[col * LD + ra] = __float2bfloat16_rn(dz2[nt][0]);
            S.dZ2t[(col + 1) * LD + ra] = __float2bfloat16_rn(dz2[nt][1]);
            S.dZ2t[col * LD + rc] = __float2bfloat16_rn(dz2[nt][2]);
            S.dZ2t[(col + 1) * LD + rc] = __float2bfloat16_rn(dz2[nt][3]);
        }
        // dA1 = dZ2 W2^T  (B[k=j][n=i] = W2[i][j], stored [i][j])
        unsigned ad[4][4];
#pragma unroll
        for (int kk = 0; kk < 4; kk++) {
            ad[kk][0] = pack2(dz2[2 * kk][0], dz2[2 * kk][1]);
            ad[kk][1] = pack2(dz2[2 * kk][2], dz2[2 * kk][3]);
            ad[kk][2] = pack2(dz2[2 * kk + 1][0], dz2[2 * kk + 1][1]);
            ad[kk][3] = pack2(dz2[2 * kk + 1][2], dz2[2 * kk + 1][3]);
        }
#pragma unroll
        for (int nt = 0; nt < 8; nt++) {
            float da[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
            for (int kk = 0; kk < 4; kk++) {
                const __nv_bfloat16 *wb = W2 + (nt * 8 + gid) * 64 + kk * 16 + 2 * tig;
                const unsigned b[2] = {ld32(wb), ld32(wb + 8)};
                mma16816(da, ad[kk], b);
            }
            const int col = nt * 8 + 2 * tig;
            const float d0 = da[0] * gelu_grad(z1[nt][0]), d1 = da[1] * gelu_grad(z1[nt][1]);
            const float d2 = da[2] * gelu_grad(z1[nt][2]), d3 = da[3] * gelu_grad(z1[nt][3]);
            atomicAdd(&S.gb1[col], d0 + d2);
            atomicAdd(&S.gb1[col + 1], d1 + d3);
            const int ra = r0 + gid, rc = r0 + gid + 8;
            S.dZ1t[col * LD + ra] = __float2bfloat16_rn(d0);
            S.dZ1t[(col + 1) * LD + ra] = __float2bfloat16_rn(d1);
            S.dZ1t[col * LD + rc] = __float2bfloat16_rn(d2);
            S.dZ1t[(col + 1) * LD + rc] = __float2bfloat16_rn(d3);
        }
    }
    if (tig == 0) {
        atomicAdd(&S.gb3, pb3);
        atomicAdd(&S.loss, pl);
    }
    __syncthreads();
    // dW2[i][j] = sum_r A1[r][i] dZ2[r][j]: warp w owns rows i = 16w..16w+15
    {
        float acc[8][4];
#pragma unroll
        for (int nt = 0; nt < 8; nt++) acc[nt][0] = acc[nt][1] = acc[nt][2] = acc[nt][3] = 0.f;
        const int i0 = 16 * w;
        for (int kk = 0; kk < GR / 16; kk++) {
            const __nv_bfloat16 *ap = S.At1 + (i0 + gid) * LD + kk * 16 + 2 * tig;
            const unsigned a[4] = {ld32(ap), ld32(ap + 8 * LD), ld32(ap + 8), ld32(ap + 8 * LD + 8)};
#pragma unroll
            for (int nt = 0; nt < 8; nt++) {
                const __nv_bfloat16 *bp = S.dZ2t + (nt * 8 + gid) * LD + kk * 16 + 2 * tig;
                const unsigned b[2] = {ld32(bp), ld32(bp + 8)};
                mma16816(acc[nt], a, b);
            }
        }
#pragma unroll
        for (int nt = 0; nt < 8; nt++) {
            const int j = nt * 8 + 2 * tig;
            atomicAdd(&grad[OFF_W2 + (i0 + gid) * H + j], acc[nt][0]);
            atomicAdd(&grad[OFF_W2 + (i0 + gid) * H + j + 1], acc[nt][1]);
            atomicAdd(&grad[OFF_W2 + (i0 + gid + 8) * H + j], acc[nt][2]);
            atomicAdd(&grad[OFF_W2 + (i0 + gid + 8) * H + j + 1], acc[nt][3]);
        }
    }
    // dW1[c][j] = sum_r X[r][c] dZ1[r][j]: warp w owns columns j = 16w..16w+15
    {
        float acc[2][4] = {{0.f, 0.f, 0.f, 0.f}, {0.f, 0.f, 0.f, 0.f}};
        for (int kk = 0; kk < GR / 16; kk++) {
            const __nv_bfloat16 *ap = S.Xt + gid * LD + kk * 16 + 2 * tig;
            const unsigned a[4] = {ld32(ap), ld32(ap + 8 * LD), ld32(ap + 8), ld32(ap + 8 * LD + 8)};
#pragma unroll
            for (int q = 0; q < 2; q++) {
                const __nv_bfloat16 *bp = S.dZ1t + ((2 * w + q) * 8 + gid) * LD + kk * 16 + 2 * tig;
                const unsigned b[2] = {ld32(bp), ld32(bp + 8)};
                mma16816(acc[q], a, b);
            }
        }
        if (gid < 3)
#pragma unroll
            for (int q = 0; q < 2; q++) {
                const int j = (2 * w + q) * 8 + 2 * tig;
                atomicAdd(&grad[OFF_W1 + gid * H + j], acc[q][0]);
                atomicAdd(&grad[OFF_W1 + gid * H + j + 1], acc[q][1]);
            }
    }
    for (int k = threadIdx.x; k < H; k += blockDim.x) {
        atomicAdd(&grad[OFF_B1 + k], S.gb1[k]);
        atomicAdd(&grad[OFF_B2 + k], S.gb2[k]);
        atomicAdd(&grad[OFF_W3 + k], S.gw3[k]);
    }
    if (threadIdx.x == 0) {
        atomicAdd(&grad[OFF_B3], S.gb3);
        atomicAdd(loss, S.loss);
    }
}

__global__ void k_adam(float *__restrict__ P, const float *__restrict__ g, float *__restrict__ m,
                       float *__restrict__ v, float lr, float b1, float b2, float eps, float c1,
                       float c2) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= NP) return;
    const float gk = g[k];
    const float mk = b1 * m[k] + (1.f - b1) * gk;
    const float vk = b2 * v[k] + (1.f - b2) * gk * gk;
    m[k] = mk;
    v[k] = vk;
    P[k] -= lr * (mk / c1) / (sqrtf(vk / c2) + eps);
}

// Surrogate prediction for the 32 rows of one warp (two 16-row MMA tiles):
// features (log10 rho, log10 u, log10 dt) staged through shared memory, the
// network's dlog10(u) returned for the lane's own row.
__device__ __forceinline__ float predict32(const MlpSmem &S, __nv_bfloat16 *xs, float *ys,
                                           const float *norm, bool own, double rho_c, double u0,
                                           double dt_c) {
    const int lane = threadIdx.x & 31, gid = lane >> 2, tig = lane & 3;
    for (int e = lane; e < 512; e += 32) xs[e] = __float2bfloat16_rn(0.f);
    __syncwarp();
    if (own) {
        // FP32 logarithms: the features are rounded to BF16 next
        xs[lane * 16 + 0] = __float2bfloat16_rn((log10f((float)rho_c) - norm[0]) / norm[3]);
        xs[lane * 16 + 1] = __float2bfloat16_rn((log10f((float)u0) - norm[1]) / norm[4]);
        xs[lane * 16 + 2] = __float2bfloat16_rn((log10f((float)dt_c) - norm[2]) / norm[5]);
    }
    __syncwarp();
#pragma unroll 1
    for (int t = 0; t < 2; t++) {
        unsigned ax[4];
        x_fragment(xs + t * 256, ax);
        float z1[8][4], z2[8][4], y0, y1;
        tile_forward<true>(S, ax, z1, z2, y0, y1);
        if (tig == 0) {
            ys[t * 16 + gid] = y0;
            ys[t * 16 + gid + 8] = y1;
        }
    }
    __syncwarp();
    const float y = ys[lane];
    __syncwarp();
    return y;
}

// Rows the surrogate does not answer go to a list (list[cap] counts them) that
// k_cool_list solves exactly with full warps; a row that finds the list full
// is solved in place.
__device__ __forceinline__ bool to_list(int *list, int cap, int i) {
    const int k = atomicAdd(&list[cap], 1);
    if (k < cap) {
        list[k] = i;
        return true;
    }
    return false;
}

// In-step cooling with the surrogate: one warp per 32 particles.  Rows whose
// estimated error exceeds err_tol (or whose estimate is void) are solved
// exactly by k_cool_list.
__global__ void __launch_bounds__(128)
    k_cool_mlp(CoolDev c, int n, const double *__restrict__ rho, double *__restrict__ u,
               const int *__restrict__ cloud, const double *__restrict__ dt, double ur, double uu,
               double ut, const __nv_bfloat16 *__restrict__ pk, const float *__restrict__ P,
               double err_tol, int *__restrict__ list, int cap, long long *status) {
    __shared__ MlpSmem S;
    __shared__ __align__(16) __nv_bfloat16 xs[4][32 * 16];
    __shared__ float ys[4][32];
    load_weights(S, pk, P);
    const float *norm = P + NP;
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int ntile = (n + 31) / 32;
    for (int tile = blockIdx.x * 4 + w; tile < ntile; tile += gridDim.x * 4) {
        const int i = tile * 32 + lane;
        const bool own = i < n;
        double rho_c = 1.0, u0 = 1.0, dt_c = 1.0;
        if (own) {
            rho_c = rho[i] * ur;
            u0 = u[i] * uu;
            dt_c = dt[cloud[i]] * ut;
        }
        const float y = predict32(S, xs[w], ys[w], norm, own, rho_c, u0, dt_c);
        if (own) {
            const double dl = (double)y * norm[7] + norm[6];
            double un = u0 * (double)__exp10f((float)dl), est;
            cool_newton_polish_f(c, rho_c, u0, dt_c, &un, &est, err_tol);
            if (cool_accept_f(c, rho_c, u0, dt_c, un, est, err_tol)) {
                u[i] = un / uu;
            } else {
                status_add(status, SPH_S_MLP_FALLBACK, 1);
                if (!to_list(list, cap, i)) {
                    if (cool_solve(c, rho_c, u0, dt_c, &un) < 0) status_add(status, SPH_S_COOL_NOCONV, 1);
                    u[i] = un / uu;
                }
            }
        }
    }
}

// exact solves of the listed in-step rows (u still holds u_old there)
__global__ void k_cool_list(CoolDev c, const int *__restrict__ list, int cap,
                            const double *__restrict__ rho, double *__restrict__ u,
                            const int *__restrict__ cloud, const double *__restrict__ dt, double ur,
                            double uu, double ut, long long *status) {
    const int cnt = min(list[cap], cap);
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < cnt; k += gridDim.x * blockDim.x) {
        const int i = list[k];
        double un;
        if (cool_solve(c, rho[i] * ur, u[i] * uu, dt[cloud[i]] * ut, &un) < 0)
            status_add(status, SPH_S_COOL_NOCONV, 1);
        u[i] = un / uu;
    }
}

// the same for standalone arrays (cgs), with the per-row fallback flag
__global__ void __launch_bounds__(128)
    k_cool_mlp_arrays(CoolDev c, int n, const double *__restrict__ rho,
                      const double *__restrict__ u_old, const double *__restrict__ dtv,
                      double *__restrict__ u_new, int *__restrict__ fell_back,
                      const __nv_bfloat16 *__restrict__ pk, const float *__restrict__ P,
                      double err_tol, int *__restrict__ list, int cap) {
    __shared__ MlpSmem S;
    __shared__ __align__(16) __nv_bfloat16 xs[4][32 * 16];
    __shared__ float ys[4][32];
    load_weights(S, pk, P);
    const float *norm = P + NP;
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int ntile = (n + 31) / 32;
    for (int tile = blockIdx.x * 4 + w; tile < ntile; tile += gridDim.x * 4) {
        const int i = tile * 32 + lane;
        const bool own = i < n;
        const double r = own ? rho[i] : 1.0, u0 = own ? u_old[i] : 1.0, d = own ? dtv[i] : 1.0;
        const float y = predict32(S, xs[w], ys[w], norm, own, r, u0, d);
        if (own) {
            const double dl = (double)y * norm[7] + norm[6];
            double un = u0 * (double)__exp10f((float)dl), est;
            cool_newton_polish_f(c, r, u0, d, &un, &est, err_tol);
            int fb = 0;
            if (cool_accept_f(c, r, u0, d, un, est, err_tol)) {
                u_new[i] = un;
            } else {
                fb = 1;
                if (!to_list(list, cap, i)) {
                    cool_solve(c, r, u0, d, &un);
                    u_new[i] = un;
                }
            }
            if (fell_back) fell_back[i] = fb;
        }
    }
}

__global__ void k_cool_list_arrays(CoolDev c, const int *__restrict__ list, int cap,
                                   const double *__restrict__ rho, const double *__restrict__ u_old,
                                   const double *__restrict__ dtv, double *__restrict__ u_new) {
    const int cnt = min(list[cap], cap);
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < cnt; k += gridDim.x * blockDim.x) {
        const int i = list[k];
        double un;
        cool_solve(c, rho[i], u_old[i], dtv[i], &un);
        u_new[i] = un;
    }
}

// ---------------------------------------------------------------------------
// Inference on the 5th-generation tensor cores (tcgen05): 128 rows per CTA.
// Layer 1 (3 -> 64) runs on the CUDA cores, one thread per row, from the BF16
// weights, and writes its BF16 activations into shared memory as operand A of
// layer 2 (128 x 64, K-major, no swizzle: 8-row x 16-byte core matrices, the
// K-adjacent ones 128 B apart, the M-adjacent ones 1024 B apart).  W2t is
// operand B in the same layout (64 x 64).  One thread issues the four K = 16
// steps of tcgen05.mma kind::f16 (BF16 x BF16 -> FP32, M = 128, N = 64) into a
// 64-column TMEM accumulator and commits them to an mbarrier; every thread
// then reads its row (TMEM lane = row) with tcgen05.ld, adds b2, applies GELU
// and the layer-3 dot product in FP32.  The waits are bounded: a wait that
// gives up counts in SPH_S_WAIT_TIMEOUT and the CTA sends its remaining rows
// to the exact solver.
namespace tc {

constexpr int ROWS = 128;
constexpr int COLS = 64;          // TMEM columns of the accumulator
constexpr int SPIN = 1 << 22;     // try_wait polls before a wait gives up

struct alignas(128) Smem {
    __nv_bfloat16 a[ROWS * H];    // layer-2 operand A, core-matrix layout
    __nv_bfloat16 b[H * H];       // W2t, core-matrix layout
    float w1[3][H], b1[H], b2[H], w3[H], b3;
    unsigned long long mbar;
    unsigned tmem;
};
// dynamic shared memory per CTA: at most 7 CTAs share an SM, 7 x 64 TMEM
// columns of the 512
constexpr int SMEM_BYTES = 32 * 1024;
static_assert(sizeof(Smem) <= SMEM_BYTES, "tcgen05 MLP tile does not fit");

__device__ __forceinline__ unsigned saddr(const void *p) {
    return (unsigned)__cvta_generic_to_shared(p);
}
// byte offset of element (row, k) in the core-matrix layout of a K = 64 operand
__device__ __forceinline__ unsigned cm_off(int row, int k) {
    return (row >> 3) * 1024 + (k >> 3) * 128 + (row & 7) * 16 + (k & 7) * 2;
}
// shared-memory matrix descriptor (no swizzle, K-major): start, leading
// (K-direction) and stride (M/N-direction) byte offsets in 16-byte units,
// descriptor version 1
__device__ __forceinline__ unsigned long long sdesc(unsigned addr) {
    return (unsigned long long)((addr >> 4) & 0x3FFF) | ((unsigned long long)(128 >> 4) << 16) |
           ((unsigned long long)(1024 >> 4) << 32) | (1ull << 46);
}
// instruction descriptor: FP32 accumulator, BF16 A and B, both K-major,
// N = 64, M = 128
constexpr unsigned IDESC = (1u << 4) | (1u << 7) | (1u << 10) | ((unsigned)(H >> 3) << 17) |
                           ((unsigned)(ROWS >> 4) << 24);

__device__ __forceinline__ void mma(unsigned d, unsigned long long a, unsigned long long b, int acc) {
    asm volatile(
        "{\n.reg .pred p;\nsetp.ne.b32 p, %4, 0;\n"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(d),
        "l"(a), "l"(b), "r"(IDESC), "r"(acc));
}
__device__ __forceinline__ void commit(unsigned mbar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar)
                 : "memory");
}
__device__ __forceinline__ bool try_wait(unsigned mbar, unsigned phase) {
    unsigned ok;
    asm volatile(
        "{\n.reg .pred p;\nmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        "selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(mbar), "r"(phase)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_smem_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
// 16 consecutive FP32 columns of this thread's TMEM lane
__device__ __forceinline__ void ld16(unsigned taddr, float *v) {
    unsigned r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
          "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
#pragma unroll
    for (int q = 0; q < 16; q++) v[q] = __uint_as_float(r[q]);
}
__device__ __forceinline__ void wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// weights into shared memory, TMEM allocation (warp 0), mbarrier set-up
__device__ __forceinline__ void setup(Smem &S, const __nv_bfloat16 *pk, const float *P) {
    const int t = threadIdx.x;
    for (int e = t; e < H * H; e += blockDim.x) {
        const int nn = e / H, k = e % H;  // W2t[n][k]
        *reinterpret_cast<__nv_bfloat16 *>(reinterpret_cast<char *>(S.b) + cm_off(nn, k)) =
            pk[PK_W2T + e];
    }
    for (int e = t; e < 3 * H; e += blockDim.x) {
        const int c = e / H, j = e % H;
        S.w1[c][j] = __bfloat162float(pk[PK_W1T + j * 16 + c]);
    }
    for (int j = t; j < H; j += blockDim.x) {
        S.b1[j] = P[OFF_B1 + j];
        S.b2[j] = P[OFF_B2 + j];
        S.w3[j] = P[OFF_W3 + j];
    }
    if (t == 0) {
        S.b3 = P[OFF_B3];
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(saddr(&S.mbar)));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (t < 32) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         saddr(&S.tmem)),
                     "r"(COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    fence_smem_async();
    fence_before();
    __syncthreads();
    fence_after();
}

__device__ __forceinline__ void teardown(Smem &S) {
    fence_before();
    __syncthreads();
    fence_after();
    if (threadIdx.x < 32)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(S.tmem), "r"(COLS));
}

// One tile: x = this thread's normalised features (rounded to BF16 like the
// warp-level path), returns y; ok = false when the wait gave up (then the
// caller treats the row as unanswered).  All threads of the CTA call it.
template <bool FAST>
__device__ __forceinline__ float predict(Smem &S, const float x[3], unsigned &phase, bool &ok,
                                         long long *status) {
    const int r = threadIdx.x;
    float xb[3];
#pragma unroll
    for (int c = 0; c < 3; c++) xb[c] = __bfloat162float(__float2bfloat16_rn(x[c]));
    char *arow = reinterpret_cast<char *>(S.a);
#pragma unroll
    for (int k8 = 0; k8 < H / 8; k8++) {
        unsigned pkd[4];
#pragma unroll
        for (int q = 0; q < 4; q++) {
            const int j = 8 * k8 + 2 * q;
            const float z0 = S.b1[j] + xb[0] * S.w1[0][j] + xb[1] * S.w1[1][j] + xb[2] * S.w1[2][j];
            const float z1 = S.b1[j + 1] + xb[0] * S.w1[0][j + 1] + xb[1] * S.w1[1][j + 1] +
                             xb[2] * S.w1[2][j + 1];
            pkd[q] = pack2(act<FAST>(z0), act<FAST>(z1));
        }
        *reinterpret_cast<uint4 *>(arow + cm_off(r, 8 * k8)) = make_uint4(pkd[0], pkd[1], pkd[2], pkd[3]);
    }
    fence_smem_async();
    __syncthreads();
    const unsigned mbar = saddr(&S.mbar);
    if (r == 0 && ok) {
        fence_after();
        const unsigned a0 = saddr(S.a), b0 = saddr(S.b);
#pragma unroll
        for (int ks = 0; ks < H / 16; ks++) mma(S.tmem, sdesc(a0 + 256 * ks), sdesc(b0 + 256 * ks), ks > 0);
        commit(mbar);
    }
    bool done = !ok;
    for (int it = 0; it < SPIN && !done; it++) done = try_wait(mbar, phase);
    const bool timed_out = !__syncthreads_and(done) || !ok;
    float y = 0.f;
    if (!timed_out) {
        phase ^= 1u;
        fence_after();
        const unsigned tl = S.tmem + ((unsigned)(32 * (r >> 5)) << 16);
        float acc = S.b3;
#pragma unroll
        for (int c16 = 0; c16 < H / 16; c16++) {
            float v[16];
            ld16(tl + 16 * c16, v);
            wait_ld();
#pragma unroll
            for (int q = 0; q < 16; q++) acc += act<FAST>(v[q] + S.b2[16 * c16 + q]) * S.w3[16 * c16 + q];
        }
        y = acc;
    } else if (ok) {
        ok = false;  // this CTA stops using the tensor cores
        if (r == 0) status_add(status, SPH_S_WAIT_TIMEOUT, 1);
    }
    fence_before();
    __syncthreads();  // TMEM and operand A are free for the next tile
    return y;
}

}  // namespace tc

__global__ void __launch_bounds__(tc::ROWS)
    k_mlp_forward_tc(int n, const float *__restrict__ X, float *__restrict__ y,
                     const __nv_bfloat16 *__restrict__ pk, const float *__restrict__ P,
                     long long *status) {
    extern __shared__ __align__(1024) unsigned char tc_smem[];
    tc::Smem &S = *reinterpret_cast<tc::Smem *>(tc_smem);
    tc::setup(S, pk, P);
    unsigned phase = 0;
    bool ok = true;
    const int ntile = (n + tc::ROWS - 1) / tc::ROWS;
    for (int tile = blockIdx.x; tile < ntile; tile += gridDim.x) {
        const int i = tile * tc::ROWS + threadIdx.x;
        float x[3] = {0.f, 0.f, 0.f};
        if (i < n) x[0] = X[3 * i], x[1] = X[3 * i + 1], x[2] = X[3 * i + 2];
        const float v = tc::predict<false>(S, x, phase, ok, status);
        if (i < n) y[i] = ok ? v : NAN;
    }
    tc::teardown(S);
}

// in-step cooling with the tensor-core surrogate, 128 rows per CTA
__global__ void __launch_bounds__(tc::ROWS)
    k_cool_mlp_tc(CoolDev c, int n, const double *__restrict__ rho, double *__restrict__ u,
                  const int *__restrict__ cloud, const double *__restrict__ dt, double ur,
                  double uu, double ut, const __nv_bfloat16 *__restrict__ pk,
                  const float *__restrict__ P, double err_tol, int *__restrict__ list, int cap,
                  long long *status) {
    extern __shared__ __align__(1024) unsigned char tc_smem[];
    tc::Smem &S = *reinterpret_cast<tc::Smem *>(tc_smem);
    tc::setup(S, pk, P);
    const float *norm = P + NP;
    unsigned phase = 0;
    bool ok = true;
    const int ntile = (n + tc::ROWS - 1) / tc::ROWS;
    for (int tile = blockIdx.x; tile < ntile; tile += gridDim.x) {
        const int i = tile * tc::ROWS + threadIdx.x;
        const bool own = i < n;
        double rho_c = 1.0, u0 = 1.0, dt_c = 1.0;
        if (own) {
            rho_c = rho[i] * ur;
            u0 = u[i] * uu;
            dt_c = dt[cloud[i]] * ut;
        }
        const float x[3] = {(log10f((float)rho_c) - norm[0]) / norm[3],
                            (log10f((float)u0) - norm[1]) / norm[4],
                            (log10f((float)dt_c) - norm[2]) / norm[5]};
        const float y = tc::predict<true>(S, x, phase, ok, status);
        if (own) {
            double un = u0, est = INFINITY;
            if (ok) {
                un = u0 * (double)__exp10f(y * norm[7] + norm[6]);
                cool_newton_polish_f(c, rho_c, u0, dt_c, &un, &est, err_tol);
            }
            if (ok && cool_accept_f(c, rho_c, u0, dt_c, un, est, err_tol)) {
                u[i] = un / uu;
            } else {
                status_add(status, SPH_S_MLP_FALLBACK, 1);
                if (!to_list(list, cap, i)) {
                    if (cool_solve(c, rho_c, u0, dt_c, &un) < 0) status_add(status, SPH_S_COOL_NOCONV, 1);
                    u[i] = un / uu;
                }
            }
        }
    }
    tc::teardown(S);
}

// the same for standalone arrays (cgs), with the per-row fallback flag
__global__ void __launch_bounds__(tc::ROWS)
    k_cool_mlp_arrays_tc(CoolDev c, int n, const double *__restrict__ rho,
                         const double *__restrict__ u_old, const double *__restrict__ dtv,
                         double *__restrict__ u_new, int *__restrict__ fell_back,
                         const __nv_bfloat16 *__restrict__ pk, const float *__restrict__ P,
                         double err_tol, int *__restrict__ list, int cap, long long *status) {
    extern __shared__ __align__(1024) unsigned char tc_smem[];
    tc::Smem &S = *reinterpret_cast<tc::Smem *>(tc_smem);
    tc::setup(S, pk, P);
    const float *norm = P + NP;
    unsigned phase = 0;
    bool ok = true;
    const int ntile = (n + tc::ROWS - 1) / tc::ROWS;
    for (int tile = blockIdx.x; tile < ntile; tile += gridDim.x) {
        const int i = tile * tc::ROWS + threadIdx.x;
        const bool own = i < n;
        const double r = own ? rho[i] : 1.0, u0 = own ? u_old[i] : 1.0, d = own ? dtv[i] : 1.0;
        const float x[3] = {(log10f((float)r) - norm[0]) / norm[3],
                            (log10f((float)u0) - norm[1]) / norm[4],
                            (log10f((float)d) - norm[2]) / norm[5]};
        const float y = tc::predict<true>(S, x, phase, ok, status);
        if (own) {
            double un = u0, est = INFINITY;
            if (ok) {
                un = u0 * (double)__exp10f(y * norm[7] + norm[6]);
                cool_newton_polish_f(c, r, u0, d, &un, &est, err_tol);
            }
            int fb = 0;
            if (ok && cool_accept_f(c, r, u0, d, un, est, err_tol)) {
                u_new[i] = un;
            } else {
                fb = 1;
                if (!to_list(list, cap, i)) {
                    cool_solve(c, r, u0, d, &un);
                    u_new[i] = un;
                }
            }
            if (fell_back) fell_back[i] = fb;
        }
    }
    tc::teardown(S);
}

// grid of a tensor-core MLP kernel: at most 7 CTAs per SM (TMEM columns)
int tc_grid(sph_ctx *ctx, int n) {
    return max(1, min(div_up(n, tc::ROWS), ctx->num_sms * 7));
}
bool use_tc(const sph_ctx *ctx) { return !(ctx->cfg.flags & SPH_FLAG_MLP_WARP_MMA); }

int grid_for(sph_ctx *ctx, int n) { return max(1, min(div_up(div_up(n, 16), 4), ctx->num_sms * 8)); }
int grid32_for(sph_ctx *ctx, int n) { return max(1, min(div_up(div_up(n, 32), 4), ctx->num_sms * 8)); }

int ensure_mlp(sph_ctx *ctx) {
    if (ctx->mlp) return SPH_OK;
    void *q = nullptr;
    const size_t bytes = sizeof(float) * (NP + 8) + sizeof(float) * NP * 3 + sizeof(float) * 8 +
                         sizeof(__nv_bfloat16) * PK_N;
    CK(cudaMalloc(&q, bytes));
    {
        // fallback rows of the surrogate (n_max entries + a counter)
        void *l = nullptr;
        CK(cudaMalloc(&l, sizeof(int) * ((size_t)ctx->cfg.n_max + 1)));
        ctx->allocs.push_back(l);
        ctx->dev_bytes += sizeof(int) * ((size_t)ctx->cfg.n_max + 1);
        ctx->cool_list = (int *)l;
    }
    CK(cudaMemsetAsync(q, 0, bytes, ctx->stream));  // ordered before the parameter copies
    ctx->allocs.push_back(q);
    ctx->dev_bytes += bytes;
    float *f = (float *)q;
    ctx->mlp = f;                    // params + norm
    ctx->mlp_grad = f + NP + 8;      // grad
    ctx->mlp_m = ctx->mlp_grad + NP;
    ctx->mlp_v = ctx->mlp_m + NP;
    ctx->mlp_scratch = ctx->mlp_v + NP;  // loss (+7 spare)
    ctx->mlp_bf16 = (void *)(ctx->mlp_scratch + 8);
    return SPH_OK;
}

}  // namespace

int mlp_pack(sph_ctx *ctx) {
    k_mlp_pack<<<div_up(PK_N, 256), 256, 0, ctx->stream>>>(ctx->mlp,
                                                            (__nv_bfloat16 *)ctx->mlp_bf16);
    return ctx_check_launch(ctx, "mlp_pack");
}

int mlp_forward_dev(sph_ctx *ctx, int n, const float *X, float *y) {
    if (n <= 0) return SPH_OK;
    if (use_tc(ctx))
        k_mlp_forward_tc<<<tc_grid(ctx, n), tc::ROWS, tc::SMEM_BYTES, ctx->stream>>>(
            n, X, y, (const __nv_bfloat16 *)ctx->mlp_bf16, ctx->mlp, ctx->status);
    else
        k_mlp_forward<<<grid_for(ctx, n), 128, 0, ctx->stream>>>(
            n, X, y, (const __nv_bfloat16 *)ctx->mlp_bf16, ctx->mlp);
    return ctx_check_launch(ctx, "mlp_forward");
}

static int grad_launch(sph_ctx *ctx, int n, const float *X, const float *t, float inv_n) {
    const size_t sm = sizeof(GradSmem);
    static bool attr = false;
    if (!attr) {
        CK(cudaFuncSetAttribute(k_mlp_grad, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
        attr = true;
    }
    k_mlp_grad<<<div_up(n, GR), 128, sm, ctx->stream>>>(
        n, X, t, inv_n, (const __nv_bfloat16 *)ctx->mlp_bf16, ctx->mlp, ctx->mlp_grad,
        ctx->mlp_scratch);
    return ctx_check_launch(ctx, "mlp_grad");
}

int mlp_grad_dev(sph_ctx *ctx, int n, const float *X, const float *t, float *grad, float *loss) {
    if (n <= 0) return SPH_ERR_ARG;
    CK(cudaMemsetAsync(ctx->mlp_grad, 0, sizeof(float) * NP, ctx->stream));
    CK(cudaMemsetAsync(ctx->mlp_scratch, 0, sizeof(float), ctx->stream));
    int rc = grad_launch(ctx, n, X, t, 1.0f / n);
    if (rc) return rc;
    if (grad) CK(cudaMemcpyAsync(grad, ctx->mlp_grad, sizeof(float) * NP, cudaMemcpyDeviceToDevice,
                                 ctx->stream));
    if (loss) CK(cudaMemcpyAsync(loss, ctx->mlp_scratch, sizeof(float), cudaMemcpyDeviceToDevice,
                                 ctx->stream));
    return SPH_OK;
}

int mlp_train_dev(sph_ctx *ctx, int n, const float *X, const float *t, int batch, int nsteps,
                  float lr, float *loss_out) {
    if (n <= 0 || batch <= 0 || nsteps < 0) return SPH_ERR_ARG;
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    const int nb = max(1, n / batch);
    for (int s = 0; s < nsteps; s++) {
        const int b = s % nb;
        const int rows = min(batch, n - b * batch);
        CK(cudaMemsetAsync(ctx->mlp_grad, 0, sizeof(float) * NP, ctx->stream));
        CK(cudaMemsetAsync(ctx->mlp_scratch, 0, sizeof(float), ctx->stream));
        int rc = grad_launch(ctx, rows, X + 3 * (size_t)b * batch, t + (size_t)b * batch, 1.0f / rows);
        if (rc) return rc;
        ctx->mlp_step++;
        const float c1 = 1.f - powf(b1, (float)ctx->mlp_step), c2 = 1.f - powf(b2, (float)ctx->mlp_step);
        k_adam<<<div_up(NP, 256), 256, 0, ctx->stream>>>(ctx->mlp, ctx->mlp_grad, ctx->mlp_m,
                                                         ctx->mlp_v, lr, b1, b2, eps, c1, c2);
        rc = mlp_pack(ctx);
        if (rc) return rc;
    }
    if (loss_out)
        CK(cudaMemcpyAsync(loss_out, ctx->mlp_scratch, sizeof(float), cudaMemcpyDeviceToHost,
                           ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return SPH_OK;
}

int launch_cooling_mlp(sph_ctx *ctx) {
    if (!ctx->cool_ok || !ctx->mlp_ok) return SPH_ERR_STATE;
    const int n = ctx->n, c = ctx->cur;
    if (n <= 0) return SPH_OK;
    const int cap = ctx->cfg.n_max;
    CK(cudaMemsetAsync(ctx->cool_list + cap, 0, sizeof(int), ctx->stream));
    if (use_tc(ctx))
        k_cool_mlp_tc<<<tc_grid(ctx, n), tc::ROWS, tc::SMEM_BYTES, ctx->stream>>>(
            cool_dev_of(ctx), n, ctx->rho, ctx->st[c][ST_U], ctx->cloud[c], ctx->dt,
            ctx->cool.unit_rho, ctx->cool.unit_u, ctx->cool.unit_t,
            (const __nv_bfloat16 *)ctx->mlp_bf16, ctx->mlp, ctx->cool.mlp_err_tol, ctx->cool_list,
            cap, ctx->status);
    else
        k_cool_mlp<<<grid32_for(ctx, n), 128, 0, ctx->stream>>>(
            cool_dev_of(ctx), n, ctx->rho, ctx->st[c][ST_U], ctx->cloud[c], ctx->dt,
            ctx->cool.unit_rho, ctx->cool.unit_u, ctx->cool.unit_t,
            (const __nv_bfloat16 *)ctx->mlp_bf16, ctx->mlp, ctx->cool.mlp_err_tol, ctx->cool_list,
            cap, ctx->status);
    k_cool_list<<<ctx->num_sms * 4, 128, 0, ctx->stream>>>(
        cool_dev_of(ctx), ctx->cool_list, cap, ctx->rho, ctx->st[c][ST_U], ctx->cloud[c], ctx->dt,
        ctx->cool.unit_rho, ctx->cool.unit_u, ctx->cool.unit_t, ctx->status);
    return ctx_check_launch(ctx, "cooling_mlp");
}

extern "C" {

int sph_mlp_set(sph_ctx *ctx, const float *params, const float *norm, int32_t host) {
    if (!ctx || !params || !norm) return SPH_ERR_ARG;
    cudaSetDevice(ctx->device);
    int rc = ensure_mlp(ctx);
    if (rc) return rc;
    cudaMemcpyKind k = host ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice;
    CK(cudaMemcpyAsync(ctx->mlp, params, sizeof(float) * NP, k, ctx->stream));
    CK(cudaMemcpyAsync(ctx->mlp + NP, norm, sizeof(float) * 8, k, ctx->stream));
    CK(cudaMemsetAsync(ctx->mlp_m, 0, sizeof(float) * NP * 2, ctx->stream));
    ctx->mlp_step = 0;
    rc = mlp_pack(ctx);
    if (rc) return rc;
    CK(cudaStreamSynchronize(ctx->stream));
    ctx->mlp_ok = true;
    return SPH_OK;
}

int sph_mlp_get(sph_ctx *ctx, float *params, float *norm, int32_t host) {
    if (!ctx || !ctx->mlp_ok) return SPH_ERR_STATE;
    cudaSetDevice(ctx->device);
    cudaMemcpyKind k = host ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice;
    CK(cudaStreamSynchronize(ctx->stream));
    if (params) CK(cudaMemcpy(params, ctx->mlp, sizeof(float) * NP, k));
    if (norm) CK(cudaMemcpy(norm, ctx->mlp + NP, sizeof(float) * 8, k));
    return SPH_OK;
}

static int to_device(sph_ctx *ctx, const void *src, size_t bytes, int host, void **dst) {
    *dst = nullptr;
    if (!host) {
        *dst = (void *)src;
        return SPH_OK;
    }
    CK(cudaMalloc(dst, bytes));
    // on the context's (non-blocking) stream, so the kernel that reads it is ordered after it
    CK(cudaMemcpyAsync(*dst, src, bytes, cudaMemcpyHostToDevice, ctx->stream));
    return SPH_OK;
}

int sph_mlp_forward(sph_ctx *ctx, int32_t n, const float *X, float *y, int32_t host) {
    if (!ctx || n < 0 || (n && (!X || !y))) return SPH_ERR_ARG;
    if (!ctx->mlp_ok) return SPH_ERR_STATE;
    if (n == 0) return SPH_OK;
    cudaSetDevice(ctx->device);
    void *dX = nullptr, *dy = nullptr;
    int rc = to_device(ctx, X, sizeof(float) * 3 * n, host, &dX);
    if (rc) return rc;
    if (host) CK(cudaMalloc(&dy, sizeof(float) * n));
    else dy = y;
    rc = mlp_forward_dev(ctx, n, (const float *)dX, (float *)dy);
    if (!rc && host) {
        CK(cudaStreamSynchronize(ctx->stream));
        CK(cudaMemcpy(y, dy, sizeof(float) * n, cudaMemcpyDeviceToHost));
    }
    if (host) {
        cudaFree(dX);
        cudaFree(dy);
    }
    return rc;
}

int sph_mlp_grad(sph_ctx *ctx, int32_t n, const float *X, const float *t, float *grad, float *loss,
                 int32_t host) {
    if (!ctx || n <= 0 || !X || !t) return SPH_ERR_ARG;
    if (!ctx->mlp_ok) return SPH_ERR_STATE;
    cudaSetDevice(ctx->device);
    void *dX = nullptr, *dt = nullptr;
    int rc = to_device(ctx, X, sizeof(float) * 3 * n, host, &dX);
    if (!rc) rc = to_device(ctx, t, sizeof(float) * n, host, &dt);
    if (!rc) rc = mlp_grad_dev(ctx, n, (const float *)dX, (const float *)dt, nullptr, nullptr);
    if (!rc) {
        CK(cudaStreamSynchronize(ctx->stream));
        cudaMemcpyKind k = host ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice;
        if (grad) CK(cudaMemcpy(grad, ctx->mlp_grad, sizeof(float) * NP, k));
        if (loss) CK(cudaMemcpy(loss, ctx->mlp_scratch, sizeof(float), k));
    }
    if (host) {
        cudaFree(dX);
        cudaFree(dt);
    }
    return rc;
}

int sph_mlp_train(sph_ctx *ctx, int32_t n, const float *X, const float *t, int32_t batch,
                  int32_t nsteps, float lr, float *loss) {
    if (!ctx || !X || !t) return SPH_ERR_ARG;
    if (!ctx->mlp_ok) return SPH_ERR_STATE;
    cudaSetDevice(ctx->device);
    return mlp_train_dev(ctx, n, X, t, batch, nsteps, lr, loss);
}

int sph_cool_solve_mlp(sph_ctx *ctx, int32_t n, const double *rho, const double *u_old,
                       const double *dt, double *u_new, int32_t *fell_back) {
    if (!ctx || n < 0) return SPH_ERR_ARG;
    if (!ctx->cool_ok || !ctx->mlp_ok) return SPH_ERR_STATE;
    if (n == 0) return SPH_OK;
    cudaSetDevice(ctx->device);
    const int cap = ctx->cfg.n_max;
    CK(cudaMemsetAsync(ctx->cool_list + cap, 0, sizeof(int), ctx->stream));
    if (use_tc(ctx))
        k_cool_mlp_arrays_tc<<<tc_grid(ctx, n), tc::ROWS, tc::SMEM_BYTES, ctx->stream>>>(
            cool_dev_of(ctx), n, rho, u_old, dt, u_new, fell_back,
            (const __nv_bfloat16 *)ctx->mlp_bf16, ctx->mlp, ctx->cool.mlp_err_tol, ctx->cool_list,
            cap, ctx->status);
    else
        k_cool_mlp_arrays<<<grid32_for(ctx, n), 128, 0, ctx->stream>>>(
            cool_dev_of(ctx), n, rho, u_old, dt, u_new, fell_back,
            (const __nv_bfloat16 *)ctx->mlp_bf16, ctx->mlp, ctx->cool.mlp_err_tol, ctx->cool_list,
            cap);
    k_cool_list_arrays<<<ctx->num_sms * 4, 128, 0, ctx->stream>>>(cool_dev_of(ctx), ctx->cool_list,
                                                                 cap, rho, u_old, dt, u_new);
    return ctx_check_launch(ctx, "cool_solve_mlp");
}

}  // extern "C"
