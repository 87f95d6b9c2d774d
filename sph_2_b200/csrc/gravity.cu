// gravity.cu -- Barnes-Hut walk (monopole + quadrupole, Plummer softening)
// and FP64 direct summation.
//
// Replaces compute_forces_kernel (bh_tree_iteration_v2.h:454-588): one warp
// stack per warp of 64 entries, a per-thread __all_sync opening vote with
// dp = 0.25 depth (theta_eff ~ 0.707), monopole only, spline softening with
// eps_i only, G = 1.  And the O(N^2) direct sums acc_g (hfvCLibs_v7_hfv_v2.h:
// 532-584) / getAcc_g_smth_mimj_mpi (MPI_sph/sph_code/libsx.py:910-947).
//
// Walk: one warp per group (a maximal tree node of at most 32 particles of
// one cloud), grid-stride over the groups.  The warp walks the tree 32 nodes
// per round (LIFO stack in shared memory) testing each node against the
// group's box: a node is accepted when the squared distance from its centre of
// mass to the box is >= r_open^2 (r_open = l/theta + |com - box centre|, theta
// possibly wider for small cells, see tree.cu), opened otherwise; opened
// buckets (<= leaf_size particles) go to a particle list.  Accepted nodes and
// bucket particles are staged 32 at a time in shared memory and every lane
// evaluates all 32 against its own particle, so the interaction loop is
// branch-free FP32 (mixed) or FP64 (plain) FMA work with one reciprocal square
// root per interaction.  In FP32 every instruction evaluates two staged
// entries at once with the packed f32x2 arithmetic of sm_100 (__ffma2_rn /
// __fmul2_rn), which halves the issued instructions of this issue-bound loop.
// Each 32-term chunk is summed plainly and added to a plain accumulator.
// The FP32 walk with theta_local > 0 also sends far accepted cells through
// per-group Taylor expansions, and starts each group from its super-group's
// node list with the super-group's own expansion (k_sg_walk).
#include <type_traits>

#include "sph_internal.cuh"

namespace {

constexpr int WALK_WARPS = 4;
// coefficients of the group local expansion: field (3), its gradient J
// (xx yy zz xy xz yz), the monopole's second derivatives H (xxx yyy zzz xxy
// xxz yyx yyz zzx zzy xyz), the potential, and the monopole's third
// derivatives T (xxxx yyyy zzzz xxxy xxxz yyyx yyyz zzzx zzzy xxyy xxzz yyzz
// xxyz yyxz zzxy)
constexpr int NLOC = 35;
#ifndef SPH_WALK_STACK
#define SPH_WALK_STACK 512
#endif
constexpr int WSTK = SPH_WALK_STACK;

constexpr unsigned FULL = 0xffffffffu;

template <class R> struct PlainSum {
    R s = R(0);
    __device__ __forceinline__ void add(R x) { s += x; }
    __device__ __forceinline__ double value() const { return (double)s; }
};

template <class R> __device__ __forceinline__ R rsq(R x);
template <> __device__ __forceinline__ float rsq<float>(float x) { return rsqrtf(x); }
template <> __device__ __forceinline__ double rsq<double>(double x) { return rsqrt(x); }

// pending bucket particles: ranges of consecutive slots, range r starting at
// slot rf[r] and at offset rs[r] of the pending stream (rs ascending; at most
// 31 carried ranges + 32 appended by one round)
constexpr int NRANGE = 64;

template <class R> struct WalkSmem {
    int stk[WSTK];
    int clist[64];
    int rf[NRANGE], rs[NRANGE];
    typename R4<R>::T sa[32], sb[32], sc[32];
};

// FP32 staging as one array per field, so that a 64-bit shared load gives the
// field of two consecutive entries for the packed f32x2 arithmetic
struct WalkSmemF {
    int stk[WSTK];
    int clist[64];
    int rf[NRANGE], rs[NRANGE];
    // cells: com x y z, -mass, Qxx Qyy Qzz Qxy Qxz Qyz, trace
    __align__(8) float f[11][32];
    // far cells of the group's local expansion: their node ids, per-lane
    // partial sums of the coefficients (one column per lane) and the totals
    int flist[64];
    float red[NLOC][32];
    float ltot[NLOC];
};

// super-group records read by the group walk (g_sg null: none)
struct SgArgs {
    const int *g_sg, *start, *nrem, *pool;
    const float *L;
    int cap;
};

// super-group pre-walk: stack, far-cell list, per-lane coefficient columns
struct SgSmem {
    int stk[WSTK];
    int flist[96];
    float red[NLOC][32];
};

__device__ __forceinline__ float2 f2(float a) { return make_float2(a, a); }
__device__ __forceinline__ float2 ld2(const float *p) { return *reinterpret_cast<const float2 *>(p); }

template <class R> __device__ __forceinline__ R wmin(R v) {
    for (int o = 16; o; o >>= 1) v = fmin(v, __shfl_xor_sync(FULL, v, o));
    return v;
}
template <class R> __device__ __forceinline__ R wmax(R v) {
    for (int o = 16; o; o >>= 1) v = fmax(v, __shfl_xor_sync(FULL, v, o));
    return v;
}

// squared distance from point c to the box, rounding as the oracle's box_dist2
__device__ __forceinline__ double box_d2(double x0, double y0, double z0, double x1, double y1,
                                         double z1, double cx, double cy, double cz) {
    double a, b, v, tx, ty, tz;
    a = xsub(x0, cx); b = xsub(cx, x1); v = a > b ? a : b; tx = v > 0.0 ? v : 0.0;
    a = xsub(y0, cy); b = xsub(cy, y1); v = a > b ? a : b; ty = v > 0.0 ? v : 0.0;
    a = xsub(z0, cz); b = xsub(cz, z1); v = a > b ? a : b; tz = v > 0.0 ? v : 0.0;
    double s = xadd(xmul(tx, tx), xmul(ty, ty));
    return xadd(s, xmul(tz, tz));
}
__device__ __forceinline__ float box_d2(float x0, float y0, float z0, float x1, float y1, float z1,
                                        float cx, float cy, float cz) {
    float tx = fmaxf(fmaxf(x0 - cx, cx - x1), 0.f);
    float ty = fmaxf(fmaxf(y0 - cy, cy - y1), 0.f);
    float tz = fmaxf(fmaxf(z0 - cz, cz - z1), 0.f);
    return tx * tx + ty * ty + tz * tz;
}

// Local (Taylor) coefficients at the group centre x0 of one far cell (com c,
// mass M, second moments Q about c, trace tr), r = x0 - c, Plummer-softened:
// the monopole + quadrupole field and its gradient J_ij = d a_i / d r_j, the
// monopole's second derivatives H_ijk, and the potential.  With
// g_n = (r^2 + eps^2)^(-n/2):
//   a   = (-M g3 + 1.5 tr g5 - 7.5 (r.Q.r) g7) r + 3 g5 Q.r
//   J   = delta (A - M g3) + r r^T (B + 3 M g5) + 3 g5 Q - 15 g7 (r (Qr)^T + (Qr) r^T),
//         A = 1.5 tr g5 - 7.5 (r.Q.r) g7,  B = -7.5 tr g7 + 52.5 (r.Q.r) g9
//   H   = 3 M g5 (delta_ij r_k + delta_ik r_j + delta_jk r_i) - 15 M g7 r_i r_j r_k
//   phi = -(M g1 + 0.5 (3 (r.Q.r) g5 - tr g3))
//   T   = 3 M g5 d4 - 15 M g7 d2rr + 105 M g9 r_i r_j r_k r_l, with
//         d4 = d_ij d_kl + d_ik d_jl + d_il d_jk and d2rr the six d_ab r_c r_d
//         terms over the pairings of (ijkl)
__device__ __forceinline__ void far_coeffs(float rx, float ry, float rz, float eps2, float M,
                                           float qxx, float qyy, float qzz, float qxy, float qxz,
                                           float qyz, float tr, float *L) {
    const float s2 = rx * rx + ry * ry + rz * rz + eps2;
    const float g1 = rsqrtf(s2), gi2 = g1 * g1;
    const float g3 = g1 * gi2, g5 = g3 * gi2, g7 = g5 * gi2, g9 = g7 * gi2;
    const float qx = qxx * rx + qxy * ry + qxz * rz;
    const float qy = qxy * rx + qyy * ry + qyz * rz;
    const float qz = qxz * rx + qyz * ry + qzz * rz;
    const float dqd = rx * qx + ry * qy + rz * qz;
    const float A = 1.5f * tr * g5 - 7.5f * dqd * g7;
    const float sc = A - M * g3;
    const float t5 = 3.f * g5;
    L[0] = sc * rx + t5 * qx;
    L[1] = sc * ry + t5 * qy;
    L[2] = sc * rz + t5 * qz;
    const float Bm = -7.5f * tr * g7 + 52.5f * dqd * g9 + 3.f * M * g5;
    const float c15 = 15.f * g7;
    L[3] = sc + rx * rx * Bm + t5 * qxx - 2.f * c15 * rx * qx;
    L[4] = sc + ry * ry * Bm + t5 * qyy - 2.f * c15 * ry * qy;
    L[5] = sc + rz * rz * Bm + t5 * qzz - 2.f * c15 * rz * qz;
    L[6] = rx * ry * Bm + t5 * qxy - c15 * (rx * qy + ry * qx);
    L[7] = rx * rz * Bm + t5 * qxz - c15 * (rx * qz + rz * qx);
    L[8] = ry * rz * Bm + t5 * qyz - c15 * (ry * qz + rz * qy);
    const float a3 = 3.f * M * g5, b7 = 15.f * M * g7;
    const float ex = a3 - b7 * rx * rx, ey = a3 - b7 * ry * ry, ez = a3 - b7 * rz * rz;
    L[9] = rx * (ex + 2.f * a3);   // xxx
    L[10] = ry * (ey + 2.f * a3);  // yyy
    L[11] = rz * (ez + 2.f * a3);  // zzz
    L[12] = ry * ex;               // xxy
    L[13] = rz * ex;               // xxz
    L[14] = rx * ey;               // yyx
    L[15] = rz * ey;               // yyz
    L[16] = rx * ez;               // zzx
    L[17] = ry * ez;               // zzy
    L[18] = -b7 * rx * ry * rz;    // xyz
    L[19] = -(M * g1 + 0.5f * (3.f * dqd * g5 - tr * g3));
    const float p9 = 105.f * M * g9, X = rx * rx, Y = ry * ry, Z = rz * rz;
    const float cx = p9 * X - 3.f * b7, cy = p9 * Y - 3.f * b7, cz = p9 * Z - 3.f * b7;
    const float dx = p9 * X - b7, dy = p9 * Y - b7, dz = p9 * Z - b7;
    const float xy = rx * ry, xz = rx * rz, yz = ry * rz;
    L[20] = X * (cx - 3.f * b7) + 3.f * a3;  // xxxx
    L[21] = Y * (cy - 3.f * b7) + 3.f * a3;  // yyyy
    L[22] = Z * (cz - 3.f * b7) + 3.f * a3;  // zzzz
    L[23] = xy * cx;                         // xxxy
    L[24] = xz * cx;                         // xxxz
    L[25] = xy * cy;                         // yyyx
    L[26] = yz * cy;                         // yyyz
    L[27] = xz * cz;                         // zzzx
    L[28] = yz * cz;                         // zzzy
    L[29] = X * dy - b7 * Y + a3;            // xxyy
    L[30] = X * dz - b7 * Z + a3;            // xxzz
    L[31] = Y * dz - b7 * Z + a3;            // yyzz
    L[32] = yz * dx;                         // xxyz
    L[33] = xz * dy;                         // yyxz
    L[34] = xy * dz;                         // zzxy
}

// far cells flist[lane], flist[lane + 32], ... (below m <= 32 PER) into this
// lane's column of the partial coefficient sums of an expansion at
// (x0, y0, z0), summed in registers first (one shared-memory update per
// coefficient)
template <int PER>
__device__ __forceinline__ void far_add(float (*red)[32], int lane, const int *flist, int m,
                                        float x0, float y0, float z0, float eps2,
                                        const float4 *__restrict__ wA,
                                        const float4 *__restrict__ wB,
                                        const float4 *__restrict__ wC) {
    if (lane >= m) return;
    float acc[NLOC];
    {
        const int nd = flist[lane];
        const float4 a = wA[nd], b = wB[nd], c = wC[nd];
        far_coeffs(x0 - a.x, y0 - a.y, z0 - a.z, eps2, b.w, b.x, b.y, b.z, c.x, c.y, c.z, c.w,
                   acc);
    }
#pragma unroll 1
    for (int k = lane + 32; k < m && k < 32 * PER; k += 32) {
        float Lc[NLOC];
        const int nd = flist[k];
        const float4 a = wA[nd], b = wB[nd], c = wC[nd];
        far_coeffs(x0 - a.x, y0 - a.y, z0 - a.z, eps2, b.w, b.x, b.y, b.z, c.x, c.y, c.z, c.w, Lc);
#pragma unroll
        for (int q = 0; q < NLOC; q++) acc[q] += Lc[q];
    }
#pragma unroll
    for (int q = 0; q < NLOC; q++) red[q][lane] += acc[q];
}

// value of the local expansion at offset u from the group centre: the field
// a0 + J u + H:uu/2 + T:uuu/6 and the potential phi0 - a0.u - u.J.u/2
__device__ __forceinline__ void far_eval(const float *L, float ux, float uy, float uz, float &ax,
                                         float &ay, float &az, float &phi) {
    const float jx = L[3] * ux + L[6] * uy + L[7] * uz;
    const float jy = L[6] * ux + L[4] * uy + L[8] * uz;
    const float jz = L[7] * ux + L[8] * uy + L[5] * uz;
    const float xx = ux * ux, yy = uy * uy, zz = uz * uz, xy = ux * uy, xz = ux * uz, yz = uy * uz;
    const float hx = L[9] * xx + L[14] * yy + L[16] * zz + 2.f * (L[12] * xy + L[13] * xz + L[18] * yz);
    const float hy = L[12] * xx + L[10] * yy + L[17] * zz + 2.f * (L[14] * xy + L[18] * xz + L[15] * yz);
    const float hz = L[13] * xx + L[15] * yy + L[11] * zz + 2.f * (L[18] * xy + L[16] * xz + L[17] * yz);
    const float xxx = xx * ux, yyy = yy * uy, zzz = zz * uz, xxy = xx * uy, xxz = xx * uz;
    const float xyy = yy * ux, yyz = yy * uz, xzz = zz * ux, yzz = zz * uy, xyz = xy * uz;
    const float tx = L[20] * xxx + L[25] * yyy + L[27] * zzz + 6.f * L[32] * xyz +
                     3.f * (L[23] * xxy + L[24] * xxz + L[29] * xyy + L[30] * xzz + L[33] * yyz + L[34] * yzz);
    const float ty = L[23] * xxx + L[21] * yyy + L[28] * zzz + 6.f * L[33] * xyz +
                     3.f * (L[29] * xxy + L[32] * xxz + L[25] * xyy + L[34] * xzz + L[26] * yyz + L[31] * yzz);
    const float tz = L[24] * xxx + L[26] * yyy + L[22] * zzz + 6.f * L[34] * xyz +
                     3.f * (L[32] * xxy + L[30] * xxz + L[33] * xyy + L[27] * xzz + L[31] * yyz + L[28] * yzz);
    const float s6 = 1.f / 6.f;
    ax = L[0] + jx + 0.5f * hx + s6 * tx;
    ay = L[1] + jy + 0.5f * hy + s6 * ty;
    az = L[2] + jz + 0.5f * hz + s6 * tz;
    phi = L[19] - (L[0] * ux + L[1] * uy + L[2] * uz) - 0.5f * (ux * jx + uy * jy + uz * jz);
}

template <class R, bool POT>
__global__ void __launch_bounds__(WALK_WARPS * 32, std::is_same<R, float>::value && !POT ? 6 : 1)
    k_walk(const int *__restrict__ ngroup_p, const int *__restrict__ gstart, const int *__restrict__ gcount,
           const int *__restrict__ gcloud, const int *__restrict__ croot,
           const typename R4<R>::T *__restrict__ pw, const typename R4<R>::T *__restrict__ wA,
           const typename R4<R>::T *__restrict__ wB, const typename R4<R>::T *__restrict__ wC,
           const int4 *__restrict__ wL, int leaf_size, R eps2, double G, int n,
           double *__restrict__ agrav, double *__restrict__ pot, unsigned *work,
           unsigned long long *counters, long long *status, float theta_local, SgArgs sg) {
    typedef typename R4<R>::T V4;
    constexpr bool PACKED = std::is_same<R, float>::value;
    typedef typename std::conditional<PACKED, WalkSmemF, WalkSmem<R>>::type SM;
    __shared__ SM smem[WALK_WARPS];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    SM &S = smem[w];
    const unsigned lt = (1u << lane) - 1u;
    int maxsp = 0;
    const int ngroup = *ngroup_p;
    // grid-stride over groups: many short blocks, so the block scheduler can
    // interleave this compute-bound walk with the memory-bound SPH passes
    // running on the other stream
    for (int g = q_first(work, blockIdx.x * WALK_WARPS + w); g < ngroup;
         g = q_next(work, g, gridDim.x * WALK_WARPS)) {
        const int s0 = gstart[g], gc = gcount[g];
        const bool act = lane < gc;
        const int i = s0 + (act ? lane : 0);
        const V4 pi = pw[i];
        const R bx0 = wmin<R>(act ? pi.x : R(INFINITY)), by0 = wmin<R>(act ? pi.y : R(INFINITY)),
                bz0 = wmin<R>(act ? pi.z : R(INFINITY));
        const R bx1 = wmax<R>(act ? pi.x : R(-INFINITY)), by1 = wmax<R>(act ? pi.y : R(-INFINITY)),
                bz1 = wmax<R>(act ? pi.z : R(-INFINITY));
        // each chunk's sum (at most 32 terms) joins a plain accumulator of
        // the walk's precision: in FP32 the compensated form measured 1.7 %
        // slower (the registers of its correction terms) for a change of
        // 1.3e-7 in the acceleration, against the opening angle's 1e-4
        PlainSum<R> ax, ay, az, ph;
        int nC = 0, nP = 0, nF = 0;
        int sp = 1, nc = 0, np = 0, nr = 0, nfar = 0;
        bool overflow = false;
        // the super-group's node list replaces the root when it has one
        int rpos = 0, nrem = 0, sgi = -1;
        const int *rem = nullptr;
        if constexpr (PACKED) {
            if (sg.g_sg) {
                const int s = sg.g_sg[g];
                const int k = s < sg.cap ? sg.nrem[s] : -1;
                if (k >= 0) {
                    sgi = s;
                    nrem = k;
                    rem = sg.pool + (size_t)sg.start[s] * SG_POOL;
                    sp = 0;
                    // the super-group's expansion at its own centre, first
                    const float *Ls = sg.L + (size_t)s * SG_LSTRIDE;
                    float Lt[NLOC];
#pragma unroll
                    for (int q = 0; q < NLOC; q++) Lt[q] = Ls[q];
                    float fax, fay, faz, fph;
                    far_eval(Lt, pi.x - Ls[36], pi.y - Ls[37], pi.z - Ls[38], fax, fay, faz, fph);
                    ax.add(fax);
                    ay.add(fay);
                    az.add(faz);
                    if (POT) ph.add(fph);
                }
            }
        }
        if (lane == 0 && sgi < 0) S.stk[0] = croot[gcloud[g]];
        // local expansion (FP32 walk, theta_local > 0): accepted cells whose
        // com is at least R_g / theta_local from the group centre x0 (R_g the
        // group's radius about x0) enter a Taylor expansion at x0 once per
        // group instead of being evaluated for every particle
        R fx0 = R(0), fy0 = R(0), fz0 = R(0), rfar2 = R(INFINITY);
        if constexpr (PACKED) {
            if (theta_local > 0.f) {
                fx0 = 0.5f * (bx0 + bx1);
                fy0 = 0.5f * (by0 + by1);
                fz0 = 0.5f * (bz0 + bz1);
                const float ux = pi.x - fx0, uy = pi.y - fy0, uz = pi.z - fz0;
                const float rg2 = wmax<float>(act ? ux * ux + uy * uy + uz * uz : 0.f);
                rfar2 = rg2 / (theta_local * theta_local);
#pragma unroll
                for (int q = 0; q < NLOC; q++) S.red[q][lane] = 0.f;
            }
        }
        __syncwarp();

        auto flush_cells = [&](int m) {
          if constexpr (PACKED) {
            // two cells per lane per instruction (f32x2); odd chunks are padded
            // with a massless, moment-free entry that contributes zero
            const int m2 = (m + 1) & ~1;
            if (lane < m2) {
                float4 a = make_float4(0.f, 0.f, 0.f, 0.f), b = a, c = a;
                if (lane < m) {
                    const int nd = S.clist[lane];
                    a = wA[nd];
                    b = wB[nd];
                    c = wC[nd];
                }
                S.f[0][lane] = a.x; S.f[1][lane] = a.y; S.f[2][lane] = a.z; S.f[3][lane] = -b.w;
                S.f[4][lane] = b.x; S.f[5][lane] = b.y; S.f[6][lane] = b.z;
                S.f[7][lane] = c.x; S.f[8][lane] = c.y; S.f[9][lane] = c.z; S.f[10][lane] = c.w;
            }
            __syncwarp();
            const float2 px = f2(pi.x), py = f2(pi.y), pz = f2(pi.z), e2 = f2(eps2);
            const float2 m1 = f2(-1.f), c15 = f2(1.5f), cm75 = f2(-7.5f), c3 = f2(3.f);
            float2 sx = f2(0.f), sy = f2(0.f), sz = f2(0.f), spp = f2(0.f);
#pragma unroll 4
            for (int k = 0; k < m2; k += 2) {
                const float2 dx = __ffma2_rn(ld2(&S.f[0][k]), m1, px);
                const float2 dy = __ffma2_rn(ld2(&S.f[1][k]), m1, py);
                const float2 dz = __ffma2_rn(ld2(&S.f[2][k]), m1, pz);
                float2 r2 = __ffma2_rn(dx, dx, e2);
                r2 = __ffma2_rn(dy, dy, r2);
                r2 = __ffma2_rn(dz, dz, r2);
                const float2 rinv = make_float2(rsqrtf(r2.x), rsqrtf(r2.y));
                const float2 ri2 = __fmul2_rn(rinv, rinv);
                const float2 g3 = __fmul2_rn(rinv, ri2), g5 = __fmul2_rn(g3, ri2),
                             g7 = __fmul2_rn(g5, ri2);
                const float2 qxx = ld2(&S.f[4][k]), qyy = ld2(&S.f[5][k]), qzz = ld2(&S.f[6][k]);
                const float2 qxy = ld2(&S.f[7][k]), qxz = ld2(&S.f[8][k]), qyz = ld2(&S.f[9][k]);
                const float2 qx = __ffma2_rn(qxx, dx, __ffma2_rn(qxy, dy, __fmul2_rn(qxz, dz)));
                const float2 qy = __ffma2_rn(qxy, dx, __ffma2_rn(qyy, dy, __fmul2_rn(qyz, dz)));
                const float2 qz = __ffma2_rn(qxz, dx, __ffma2_rn(qyz, dy, __fmul2_rn(qzz, dz)));
                const float2 dqd = __ffma2_rn(dx, qx, __ffma2_rn(dy, qy, __fmul2_rn(dz, qz)));
                const float2 tr = ld2(&S.f[10][k]), nm = ld2(&S.f[3][k]);
                const float2 a7 = __fmul2_rn(dqd, g7), b5 = __fmul2_rn(tr, g5);
                // s = -M g3 + 1.5 tr g5 - 7.5 dqd g7
                const float2 sc = __ffma2_rn(b5, c15, __ffma2_rn(a7, cm75, __fmul2_rn(nm, g3)));
                const float2 t5 = __fmul2_rn(g5, c3);
                sx = __ffma2_rn(t5, qx, __ffma2_rn(sc, dx, sx));
                sy = __ffma2_rn(t5, qy, __ffma2_rn(sc, dy, sy));
                sz = __ffma2_rn(t5, qz, __ffma2_rn(sc, dz, sz));
                if (POT) {
                    // -(M rinv + 0.5 (3 dqd g5 - tr g3))
                    const float2 hq = __ffma2_rn(__fmul2_rn(dqd, g5), f2(1.5f),
                                                 __fmul2_rn(__fmul2_rn(tr, g3), f2(-0.5f)));
                    spp = __ffma2_rn(nm, rinv, spp);
                    spp = __ffma2_rn(hq, m1, spp);
                }
            }
            ax.add(sx.x + sx.y); ay.add(sy.x + sy.y); az.add(sz.x + sz.y);
            if (POT) ph.add(spp.x + spp.y);
            nC += m;
            __syncwarp();
          } else {
            if (lane < m) {
                int nd = S.clist[lane];
                S.sa[lane] = wA[nd];
                S.sb[lane] = wB[nd];
                S.sc[lane] = wC[nd];
            }
            __syncwarp();
            R sx = 0, sy = 0, sz = 0, sp_ = 0;
#pragma unroll 4
            for (int k = 0; k < m; k++) {
                const V4 a = S.sa[k], b = S.sb[k], c = S.sc[k];
                const R dx = pi.x - a.x, dy = pi.y - a.y, dz = pi.z - a.z;
                const R r2 = dx * dx + dy * dy + dz * dz + eps2;
                const R rinv = rsq<R>(r2);
                const R ri2 = rinv * rinv;
                const R g3 = rinv * ri2, g5 = g3 * ri2, g7 = g5 * ri2;
                const R qx = b.x * dx + c.x * dy + c.y * dz;
                const R qy = c.x * dx + b.y * dy + c.z * dz;
                const R qz = c.y * dx + c.z * dy + b.z * dz;
                const R dqd = dx * qx + dy * qy + dz * qz;
                const R tr = c.w;
                const R s = -b.w * g3 + R(1.5) * tr * g5 - R(7.5) * dqd * g7;
                const R t5 = R(3) * g5;
                sx += s * dx + t5 * qx;
                sy += s * dy + t5 * qy;
                sz += s * dz + t5 * qz;
                if (POT) sp_ -= b.w * rinv + R(0.5) * (R(3) * dqd * g5 - tr * g3);
            }
            ax.add(sx); ay.add(sy); az.add(sz);
            if (POT) ph.add(sp_);
            nC += m;
            __syncwarp();
          }
        };
        // far cells: one per lane, added into the lane's own column of
        // partial coefficient sums (summed over the warp once per group)
        auto flush_far = [&](int m) {
          if constexpr (PACKED) {
            far_add<1>(S.red, lane, S.flist, m, fx0, fy0, fz0, eps2, wA, wB, wC);
            nF += m;
            __syncwarp();
          }
        };
        // slot of the particle at offset t of the pending stream: the last
        // range starting at or before t (nr <= NRANGE)
        auto part_slot = [&](int t) {
            int r = 0;
#pragma unroll
            for (int step = NRANGE / 2; step; step >>= 1) {
                const int c = r + step;
                if (c < nr && S.rs[c] <= t) r = c;
            }
            return S.rf[r] + (t - S.rs[r]);
        };
        // the m pending particles from stream offset h
        auto flush_parts = [&](int m, int h) {
          if constexpr (PACKED) {
            const int m2 = (m + 1) & ~1;
            if (lane < m2) {
                float4 a = make_float4(0.f, 0.f, 0.f, 0.f);
                if (lane < m) a = pw[part_slot(h + lane)];
                S.f[0][lane] = a.x; S.f[1][lane] = a.y; S.f[2][lane] = a.z; S.f[3][lane] = -a.w;
            }
            __syncwarp();
            const float2 px = f2(pi.x), py = f2(pi.y), pz = f2(pi.z), e2 = f2(eps2);
            const float2 m1 = f2(-1.f);
            float2 sx = f2(0.f), sy = f2(0.f), sz = f2(0.f), spp = f2(0.f);
#pragma unroll 4
            for (int k = 0; k < m2; k += 2) {
                const float2 dx = __ffma2_rn(ld2(&S.f[0][k]), m1, px);
                const float2 dy = __ffma2_rn(ld2(&S.f[1][k]), m1, py);
                const float2 dz = __ffma2_rn(ld2(&S.f[2][k]), m1, pz);
                const float2 nm = ld2(&S.f[3][k]);  // -m
                float2 r2 = __ffma2_rn(dx, dx, e2);
                r2 = __ffma2_rn(dy, dy, r2);
                r2 = __ffma2_rn(dz, dz, r2);
                const float2 rinv = make_float2(rsqrtf(r2.x), rsqrtf(r2.y));
                const float2 nmr = __fmul2_rn(nm, rinv);
                const float2 g = __fmul2_rn(nmr, __fmul2_rn(rinv, rinv));  // -m / r^3
                sx = __ffma2_rn(g, dx, sx);
                sy = __ffma2_rn(g, dy, sy);
                sz = __ffma2_rn(g, dz, sz);
                if (POT) spp = __fadd2_rn(spp, nmr);
            }
            ax.add(sx.x + sx.y); ay.add(sy.x + sy.y); az.add(sz.x + sz.y);
            if (POT) ph.add(spp.x + spp.y);
            nP += m;
            __syncwarp();
          } else {
            if (lane < m) S.sa[lane] = pw[part_slot(h + lane)];
            __syncwarp();
            R sx = 0, sy = 0, sz = 0, sp_ = 0;
#pragma unroll 8
            for (int k = 0; k < m; k++) {
                const V4 a = S.sa[k];
                const R dx = pi.x - a.x, dy = pi.y - a.y, dz = pi.z - a.z;
                const R r2 = dx * dx + dy * dy + dz * dz + eps2;
                const R rinv = rsq<R>(r2);
                const R gg = a.w * rinv * rinv * rinv;
                sx -= gg * dx;
                sy -= gg * dy;
                sz -= gg * dz;
                if (POT) sp_ -= a.w * rinv;
            }
            ax.add(sx); ay.add(sy); az.add(sz);
            if (POT) ph.add(sp_);
            nP += m;
            __syncwarp();
          }
        };

        while (sp > 0 || rpos < nrem || nc > 0 || np > 0) {
            if (sp == 0 && rpos < nrem) {
                // next 32 nodes of the super-group's list
                const int take = min(nrem - rpos, 32);
                if (lane < take) S.stk[lane] = rem[rpos + lane];
                rpos += take;
                sp = take;
                __syncwarp();
            }
            if (sp > 0) {
                const int take = min(sp, 32);
                sp -= take;
                int nd = 0, f = 0, cn = 0;
                bool accept = false, open = false, far = false;
                int cl = 0, cr = 0;
                if (lane < take) {
                    nd = S.stk[sp + lane];
                    // the two 16-byte records a node visit needs, issued together
                    const V4 a = wA[nd];
                    const int4 L = wL[nd];
                    f = L.x;
                    cn = L.y;
                    cl = L.z;
                    cr = L.w;
                    const R d2 = box_d2(bx0, by0, bz0, bx1, by1, bz1, a.x, a.y, a.z);
                    accept = d2 >= a.w && cn > 1;
                    open = !accept;
                    if constexpr (PACKED) {
                        if (accept && theta_local > 0.f) {
                            const float dx = a.x - fx0, dy = a.y - fy0, dz = a.z - fz0;
                            far = dx * dx + dy * dy + dz * dz >= rfar2;
                        }
                    }
                }
                __syncwarp();
                const bool bucket = open && cn <= leaf_size;
                const bool inner = open && cn > leaf_size;
                // accepted cells: near ones to the per-particle list, far
                // ones (local expansion) to the far list
                const unsigned am = __ballot_sync(FULL, accept && !far);
                if (accept && !far) S.clist[nc + __popc(am & lt)] = nd;
                nc += __popc(am);
                if constexpr (PACKED) {
                    const unsigned fm = __ballot_sync(FULL, far);
                    if (far) S.flist[nfar + __popc(fm & lt)] = nd;
                    nfar += __popc(fm);
                    __syncwarp();
                    if (nfar >= 32) {
                        flush_far(32);
                        const int v = S.flist[32 + lane];
                        __syncwarp();
                        if (lane + 32 < nfar) S.flist[lane] = v;
                        nfar -= 32;
                        __syncwarp();
                    }
                }
                // children of opened inner nodes
                const unsigned im = __ballot_sync(FULL, inner);
                const int npush = 2 * __popc(im);
                if (sp + npush <= WSTK) {
                    if (inner) {
                        const int pos = sp + 2 * __popc(im & lt);
                        S.stk[pos] = cr;
                        S.stk[pos + 1] = cl;
                    }
                    sp += npush;
                    maxsp = max(maxsp, sp);
                } else {
                    overflow = true;
                }
                unsigned bm = __ballot_sync(FULL, bucket);
                __syncwarp();
                while (nc >= 32) {
                    flush_cells(32);
                    int v = S.clist[32 + lane];
                    __syncwarp();
                    if (lane + 32 < nc) S.clist[lane] = v;
                    nc -= 32;
                    __syncwarp();
                }
                if (bm) {
                    // opened buckets join the pending stream in lane order:
                    // one range per bucket at the scanned offset
                    const int cnt = bucket ? cn : 0;
                    int incl = cnt;
#pragma unroll
                    for (int o = 1; o < 32; o <<= 1) {
                        const int t = __shfl_up_sync(FULL, incl, o);
                        if (lane >= o) incl += t;
                    }
                    if (bucket) {
                        const int r = nr + __popc(bm & lt);
                        S.rf[r] = f;
                        S.rs[r] = np + incl - cnt;
                    }
                    nr += __popc(bm);
                    np += __shfl_sync(FULL, incl, 31);
                    __syncwarp();
                    if (np >= 32) {
                        int h = 0;
                        do {
                            flush_parts(32, h);
                            h += 32;
                        } while (np - h >= 32);
                        np -= h;
                        // keep the ranges from the one holding offset h on,
                        // their offsets taken from h (<= 31 of them: each
                        // keeps at least one of the < 32 pending particles)
                        int r0 = 0;
                        if (np > 0) {
#pragma unroll
                            for (int step = NRANGE / 2; step; step >>= 1) {
                                const int c = r0 + step;
                                if (c < nr && S.rs[c] <= h) r0 = c;
                            }
                        } else {
                            r0 = nr;
                        }
                        const int keep = nr - r0;
                        int vf = 0, vs = 0;
                        if (lane < keep) {
                            vf = S.rf[r0 + lane];
                            vs = S.rs[r0 + lane] - h;
                        }
                        __syncwarp();
                        if (lane < keep) {
                            S.rf[lane] = vf;
                            S.rs[lane] = vs;
                        }
                        nr = keep;
                        __syncwarp();
                    }
                }
            }
            if (sp == 0 && rpos >= nrem) {
                if (nc > 0) { flush_cells(nc); nc = 0; }
                if (np > 0) { flush_parts(np, 0); np = 0; nr = 0; }
                if (nfar > 0) { flush_far(nfar); nfar = 0; }
            }
        }
        if constexpr (PACKED) {
            if (nF > 0) {
                __syncwarp();
                for (int q = lane; q < NLOC; q += 32) {  // Kahan sum of the 32 lane columns
                    KSum<float> t;
                    for (int k = 0; k < 32; k++) t.add(S.red[q][k]);
                    S.ltot[q] = (float)t.value();
                }
                __syncwarp();
                float Lt[NLOC];
#pragma unroll
                for (int q = 0; q < NLOC; q++) Lt[q] = S.ltot[q];
                float fax, fay, faz, fph;
                far_eval(Lt, pi.x - fx0, pi.y - fy0, pi.z - fz0, fax, fay, faz, fph);
                ax.add(fax);
                ay.add(fay);
                az.add(faz);
                if (POT) ph.add(fph);
            }
        }
        if (act) {
            const double self = POT ? (double)(pi.w * rsq<R>(eps2)) : 0.0;
            agrav[i] = G * ax.value();
            agrav[(size_t)n + i] = G * ay.value();
            agrav[2 * (size_t)n + i] = G * az.value();
            if (POT) pot[i] = G * (ph.value() + self);
        }
        if (lane == 0) {
            atomicAdd(&counters[0], (unsigned long long)nC * gc);
            atomicAdd(&counters[1], (unsigned long long)nP * gc);
            atomicAdd(&counters[2], (unsigned long long)nF);
            if (overflow) status_add(status, SPH_S_STACK_OVERFLOW, 1);
        }
    }
    if (lane == 0) atomicMax((unsigned long long *)&status[7], (unsigned long long)maxsp);
}

// Super-group pre-walk of the FP32 walk with group expansions: one warp per
// super-group (a maximal tree node of at most SGROUP_MAX particles of one
// cloud) walks the tree with the super-group's box.  Accepted cells whose com
// lies at least R / theta_local from the box centre c (R the super-group's
// radius about c) enter the super-group's Taylor expansion at c, which every
// particle of its groups evaluates.  Accepted cells nearer than that, buckets,
// and nodes of at most SGROUP_MAX particles that fail the acceptance test go
// to the node list its groups walk instead of the root (a group's box lies
// inside the super-group's, so the group accepts at least what this walk
// accepts); larger nodes that fail it are opened here.  A list longer than
// SG_POOL slots per particle, or a stack overflow, leaves the super-group
// without a record (nrem -1): its groups then walk from the root.
// (the expansion carries the potential too, so one kernel serves both)
__global__ void __launch_bounds__(WALK_WARPS * 32, 6)
    k_sg_walk(const int *__restrict__ nsg_p, int cap, const int *__restrict__ sstart,
              const int *__restrict__ scount, const int *__restrict__ scloud,
              const int *__restrict__ croot, const float4 *__restrict__ pw,
              const float4 *__restrict__ wA, const float4 *__restrict__ wB,
              const float4 *__restrict__ wC, const int4 *__restrict__ wL, float eps2,
              float theta_local, int *__restrict__ pool, int *__restrict__ nrem_out,
              float *__restrict__ sgL, unsigned long long *counters, unsigned *queue) {
    __shared__ SgSmem smem[WALK_WARPS];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    SgSmem &S = smem[w];
    const unsigned lt = (1u << lane) - 1u;
    const int nsg = min(*nsg_p, cap);
    for (int s = q_first(queue, blockIdx.x * WALK_WARPS + w); s < nsg;
         s = q_next(queue, s, gridDim.x * WALK_WARPS)) {
        const int s0 = sstart[s], sc = scount[s];
        if (sc <= 32) {
            // a single group: nothing to share, the group walks from the root
            if (lane == 0) nrem_out[s] = -1;
            continue;
        }
        float bx0 = INFINITY, by0 = INFINITY, bz0 = INFINITY;
        float bx1 = -INFINITY, by1 = -INFINITY, bz1 = -INFINITY;
        for (int k = lane; k < sc; k += 32) {
            const float4 p = pw[s0 + k];
            bx0 = fminf(bx0, p.x); by0 = fminf(by0, p.y); bz0 = fminf(bz0, p.z);
            bx1 = fmaxf(bx1, p.x); by1 = fmaxf(by1, p.y); bz1 = fmaxf(bz1, p.z);
        }
        bx0 = wmin<float>(bx0); by0 = wmin<float>(by0); bz0 = wmin<float>(bz0);
        bx1 = wmax<float>(bx1); by1 = wmax<float>(by1); bz1 = wmax<float>(bz1);
        const float cx = 0.5f * (bx0 + bx1), cy = 0.5f * (by0 + by1), cz = 0.5f * (bz0 + bz1);
        float r2 = 0.f;
        for (int k = lane; k < sc; k += 32) {
            const float4 p = pw[s0 + k];
            const float dx = p.x - cx, dy = p.y - cy, dz = p.z - cz;
            r2 = fmaxf(r2, dx * dx + dy * dy + dz * dz);
        }
        const float rfar2 = wmax<float>(r2) / (theta_local * theta_local);
#pragma unroll
        for (int q = 0; q < NLOC; q++) S.red[q][lane] = 0.f;
        int *rem = pool + (size_t)s0 * SG_POOL;
        const int remcap = sc * SG_POOL;
        int sp = 1, nrem = 0, nfar = 0;
        long long nF = 0;
        bool bad = false;
        if (lane == 0) S.stk[0] = croot[scloud[s]];
        __syncwarp();
        while (sp > 0 && !bad) {
            const int take = min(sp, 32);
            sp -= take;
            int nd = 0, cl = 0, cr = 0;
            bool far = false, keep = false, open = false;
            if (lane < take) {
                nd = S.stk[sp + lane];
                const float4 a = wA[nd];
                const int4 L = wL[nd];
                cl = L.z;
                cr = L.w;
                const float d2 = box_d2(bx0, by0, bz0, bx1, by1, bz1, a.x, a.y, a.z);
                if (d2 >= a.w && L.y > 1) {
                    const float dx = a.x - cx, dy = a.y - cy, dz = a.z - cz;
                    far = dx * dx + dy * dy + dz * dz >= rfar2;
                    keep = !far;
                } else {
                    open = L.y > SGROUP_MAX;
                    keep = !open;
                }
            }
            __syncwarp();
            const unsigned km = __ballot_sync(FULL, keep);
            if (nrem + __popc(km) > remcap) {
                bad = true;
            } else if (keep) {
                rem[nrem + __popc(km & lt)] = nd;
            }
            nrem += __popc(km);
            const unsigned fm = __ballot_sync(FULL, far);
            if (far) S.flist[nfar + __popc(fm & lt)] = nd;
            nfar += __popc(fm);
            __syncwarp();
            if (nfar >= 64) {
                far_add<2>(S.red, lane, S.flist, 64, cx, cy, cz, eps2, wA, wB, wC);
                nF += 64;
                const int v = S.flist[64 + lane];
                __syncwarp();
                if (lane + 64 < nfar) S.flist[lane] = v;
                nfar -= 64;
            }
            const unsigned om = __ballot_sync(FULL, open);
            const int npush = 2 * __popc(om);
            if (sp + npush <= WSTK) {
                if (open) {
                    const int pos = sp + 2 * __popc(om & lt);
                    S.stk[pos] = cr;
                    S.stk[pos + 1] = cl;
                }
                sp += npush;
            } else {
                bad = true;
            }
            __syncwarp();
        }
        if (!bad) {
            far_add<3>(S.red, lane, S.flist, nfar, cx, cy, cz, eps2, wA, wB, wC);
            nF += nfar;
            __syncwarp();
            float *Ls = sgL + (size_t)s * SG_LSTRIDE;
            for (int q = lane; q < NLOC; q += 32) {  // Kahan sum of the 32 lane columns
                KSum<float> t;
                for (int k = 0; k < 32; k++) t.add(S.red[q][k]);
                Ls[q] = (float)t.value();
            }
            if (lane == 0) {
                Ls[36] = cx;
                Ls[37] = cy;
                Ls[38] = cz;
            }
        }
        if (lane == 0) {
            nrem_out[s] = bad ? -1 : nrem;
            if (bad) atomicAdd(&counters[4], 1ull);
            else atomicAdd(&counters[3], (unsigned long long)nF);
        }
        __syncwarp();
    }
}

// FP64 Plummer direct sum onto targets from all particles of the same cloud
__global__ void __launch_bounds__(256)
    k_direct(int nt, const int *__restrict__ targets, const double4 *__restrict__ p0,
             const double *__restrict__ m, const int *__restrict__ cloud,
             const int *__restrict__ cstart, double eps2, double G, double *__restrict__ out) {
    __shared__ double4 sh[256];
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const bool ok = t < nt;
    const int i = ok ? targets[t] : targets[0];
    // all targets of a block must share a cloud for the tiling; loop over the
    // union of the clouds present (normally one)
    const int ci = cloud[i];
    const double4 pi = p0[i];
    double ax = 0, ay = 0, az = 0, ph = 0;
    int cmin = ci, cmax = ci;
    for (int o = 16; o; o >>= 1) {
        cmin = min(cmin, __shfl_xor_sync(0xffffffffu, cmin, o));
        cmax = max(cmax, __shfl_xor_sync(0xffffffffu, cmax, o));
    }
    __shared__ int bmin, bmax;
    if (threadIdx.x == 0) { bmin = 1 << 30; bmax = -1; }
    __syncthreads();
    if ((threadIdx.x & 31) == 0) { atomicMin(&bmin, cmin); atomicMax(&bmax, cmax); }
    __syncthreads();
    const int j0 = cstart[bmin], j1 = cstart[bmax + 1];
    for (int base = j0; base < j1; base += 256) {
        const int j = base + threadIdx.x;
        if (j < j1) {
            double4 q = p0[j];
            q.w = m[j];
            sh[threadIdx.x] = q;
        }
        __syncthreads();
        const int lim = min(256, j1 - base);
        for (int k = 0; k < lim; k++) {
            const int jj = base + k;
            if (jj == i || cloud[jj] != ci) continue;
            const double4 q = sh[k];
            const double dx = pi.x - q.x, dy = pi.y - q.y, dz = pi.z - q.z;
            const double r2 = dx * dx + dy * dy + dz * dz + eps2;
            const double rinv = 1.0 / sqrt(r2);
            const double gg = q.w * rinv * rinv * rinv;
            ax -= gg * dx; ay -= gg * dy; az -= gg * dz;
            ph -= q.w * rinv;
        }
        __syncthreads();
    }
    if (ok) {
        out[4 * t] = G * ax; out[4 * t + 1] = G * ay; out[4 * t + 2] = G * az; out[4 * t + 3] = G * ph;
    }
}

// spline-softened pair factor of libsx.py:924-934 (eps_ij = mean of eps)
__device__ __forceinline__ double fk_spline(double rr, double e) {
    const double q = rr / e;
    const double inv_r3 = 1.0 / (rr * rr * rr);
    if (q <= 1.0) return (1.0 / (e * e * e)) * ((4.0 / 3.0) - (6.0 / 5.0) * q * q + 0.5 * q * q * q);
    if (q <= 2.0) {
        const double q3 = q * q * q;
        return inv_r3 * ((-1.0 / 15.0) + (8.0 / 3.0) * q3 - 3.0 * q3 * q + (6.0 / 5.0) * q3 * q * q -
                         (1.0 / 6.0) * q3 * q3);
    }
    return inv_r3;
}

// With ids (original particle indices) the sum is the reference's partial
// field of the rows [nbeg, nend): the pairs (a, b), a < b in original index
// with a in the rows, add to both particles (libsx.py:914-945), so target i
// takes source s when s > i and i is a row, or s < i and s is a row.
// ids == null: every s != i.
__global__ void __launch_bounds__(256)
    k_direct_spline(int nt, const int *__restrict__ targets, const double4 *__restrict__ p0,
                    const double *__restrict__ m, const double *__restrict__ eps, int n, double G,
                    double *__restrict__ out, const int *__restrict__ ids, int nbeg, int nend) {
    __shared__ double4 sh[256];
    __shared__ double se[256];
    __shared__ int sid[256];
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const bool ok = t < nt;
    const int i = ok ? targets[t] : targets[0];
    const double4 pi = p0[i];
    const double ei = eps[i];
    const int idi = ids ? ids[i] : 0;
    const bool irow = idi >= nbeg && idi < nend;
    double ax = 0, ay = 0, az = 0;
    for (int base = 0; base < n; base += 256) {
        const int j = base + threadIdx.x;
        if (j < n) {
            double4 q = p0[j];
            q.w = m[j];
            sh[threadIdx.x] = q;
            se[threadIdx.x] = eps[j];
            sid[threadIdx.x] = ids ? ids[j] : 0;
        }
        __syncthreads();
        const int lim = min(256, n - base);
        for (int k = 0; k < lim; k++) {
            if (base + k == i) continue;
            if (ids) {
                const int ids_ = sid[k];
                if (!((ids_ > idi && irow) || (ids_ < idi && ids_ >= nbeg && ids_ < nend))) continue;
            }
            const double4 q = sh[k];
            const double dx = q.x - pi.x, dy = q.y - pi.y, dz = q.z - pi.z;
            const double rr = sqrt(dx * dx + dy * dy + dz * dz);
            const double fk = fk_spline(rr, 0.5 * (ei + se[k]));
            ax += fk * dx * q.w; ay += fk * dy * q.w; az += fk * dz * q.w;
        }
        __syncthreads();
    }
    if (ok) { out[3 * t] = G * ax; out[3 * t + 1] = G * ay; out[3 * t + 2] = G * az; }
}

template <class R, bool POT>
int run_walk(sph_ctx *ctx, cudaStream_t s) {
    // groups hold 1..32 particles (about 20 on average); size the grid for
    // one group per warp at 16 particles per group, the rest by grid stride
    int grid0 = max(1, div_up(div_up(ctx->n, 16) + ctx->ncloud, WALK_WARPS));
    // inside the step the walk runs beside the SPH passes of the other
    // stream: 4 of the FP32 walk's 6 resident blocks per SM leave room for
    // them (N = 1M: step 6.21 -> 6.15 ms, the walk alone 2.29 -> 2.66 ms)
    int per_sm = ctx->cfg.walk_blocks;
    if (per_sm == 0 && ctx->in_step && std::is_same<R, float>::value) per_sm = 4;
    if (per_sm > 0) grid0 = min(grid0, ctx->num_sms * per_sm);
    const R eps2 = (R)(ctx->cfg.eps * ctx->cfg.eps);
    SgArgs sg{};
    int rc;
    if constexpr (std::is_same<R, float>::value) {
        if (ctx->g_sg && ctx->cfg.theta_local > 0.0) {
            int sgrid;
            unsigned *sq;
            rc = queue_launch(ctx, s, WQ_SG_WALK, (const void *)k_sg_walk, WALK_WARPS * 32,
                              max(1, div_up(div_up(ctx->n, 64) + ctx->ncloud, WALK_WARPS)), &sgrid, &sq);
            if (rc) return rc;
            k_sg_walk<<<sgrid, WALK_WARPS * 32, 0, s>>>(
                ctx->d_nsg, ctx->sg_cap, ctx->sg_start, ctx->sg_count, ctx->sg_cloud, ctx->croot,
                (const float4 *)ctx->pw, (const float4 *)ctx->wA, (const float4 *)ctx->wB,
                (const float4 *)ctx->wC, ctx->wL, eps2, (float)ctx->cfg.theta_local, ctx->sg_pool,
                ctx->sg_nrem, ctx->sgL, ctx->counters, sq);
            sg.g_sg = ctx->g_sg;
            sg.start = ctx->sg_start;
            sg.nrem = ctx->sg_nrem;
            sg.pool = ctx->sg_pool;
            sg.L = ctx->sgL;
            sg.cap = ctx->sg_cap;
        }
    }
    int grid;
    unsigned *wq;
    rc = queue_launch(ctx, s, WQ_WALK, (const void *)k_walk<R, POT>, WALK_WARPS * 32, grid0, &grid,
                      &wq);
    if (rc) return rc;
    k_walk<R, POT><<<grid, WALK_WARPS * 32, 0, s>>>(
        ctx->d_ngroup, ctx->gstart, ctx->gcount, ctx->groot_g, ctx->croot,
        (const typename R4<R>::T *)ctx->pw, (const typename R4<R>::T *)ctx->wA,
        (const typename R4<R>::T *)ctx->wB, (const typename R4<R>::T *)ctx->wC, ctx->wL,
        ctx->cfg.leaf_size, eps2, ctx->cfg.G, ctx->n, ctx->agrav, ctx->pot,
        wq, ctx->counters, ctx->status, (float)ctx->cfg.theta_local, sg);
    return SPH_OK;
}

}  // namespace

int launch_gravity(sph_ctx *ctx, cudaStream_t s, bool pot) {
    if (ctx->n <= 0) return SPH_OK;
    CK(cudaMemsetAsync(ctx->counters, 0, 5 * sizeof(unsigned long long), s));
    int rc;
    if (ctx->cfg.precision == SPH_PREC_MIXED)
        rc = pot ? run_walk<float, true>(ctx, s) : run_walk<float, false>(ctx, s);
    else
        rc = pot ? run_walk<double, true>(ctx, s) : run_walk<double, false>(ctx, s);
    if (rc) return rc;
    if ((rc = launch_external_potential(ctx, s))) return rc;
    return ctx_check_launch(ctx, "gravity");
}

int launch_gravity_direct(sph_ctx *ctx, int nt, const int *targets, double *out) {
    if (nt <= 0) return SPH_OK;
    k_direct<<<div_up(nt, 256), 256, 0, ctx->stream>>>(nt, targets, ctx->p0, ctx->st[ctx->cur][ST_M],
                                                       ctx->cloud[ctx->cur], ctx->cloud_start,
                                                       ctx->cfg.eps * ctx->cfg.eps, ctx->cfg.G, out);
    return ctx_check_launch(ctx, "gravity_direct");
}

int launch_gravity_direct_spline(sph_ctx *ctx, const double *eps, int nt, const int *targets,
                                 double *out, int nbeg, int nend) {
    if (nt <= 0) return SPH_OK;
    const bool rows = !(nbeg == 0 && nend == ctx->n);
    k_direct_spline<<<div_up(nt, 256), 256, 0, ctx->stream>>>(
        nt, targets, ctx->p0, ctx->st[ctx->cur][ST_M], eps, ctx->n, ctx->cfg.G, out,
        rows ? ctx->id[ctx->cur] : nullptr, nbeg, nend);
    return ctx_check_launch(ctx, "gravity_direct_spline");
}
