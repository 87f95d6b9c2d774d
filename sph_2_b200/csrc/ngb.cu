// ngb.cu -- neighbour search over the radix tree and the Newton
// smoothing-length iteration.
//
// Replaces ngbDB_new_v2 (ngb_v3.h:124-238: a per-thread scan of 27 cells of a
// 10^3 grid, radius grown until 70-190 candidates, atomics-ordered output,
// host exit on failure) and smoothing_h_ngb (hfvCLibs_v7_hfv_v2.h:367-455: a
// count-based +-coeff*2h iteration of up to 200 rounds over the list).
//
// Search: one warp per group (a tree node of at most 32 Morton-contiguous
// particles of one cloud).  The warp walks the tree 32 nodes at a time with the
// group's box (LIFO stack in shared memory); buckets that can hold neighbours
// are flattened into a shared list of candidate particles, staged 32 at a time
// in shared memory, and every lane tests the staged candidates against its own
// particle.  Rows are written in traversal order (deterministic);
// sph_get_neighbours exports them sorted.
//
// h iteration (fused with the candidate search): the search writes each
// lane's candidate slots into its particle's row (max_ngb entries) and
// accumulates the kernel sums of the first Newton evaluation on the way; every
// lane then runs a bracketed Newton iteration on (4pi/3)(2h)^3 rho(h) = n_ngb m
// with FP64 updates and convergence test, gathering its row again only for
// the rare second and later evaluations.  Particles whose h outgrows the
// candidate radius are flagged and searched again in the next round; a row
// that overflows shrinks the radius instead.  Between sorts a group keeps its
// rows without a search while the distances its particles and the particles
// near them moved since the rows' search leave the rows complete for a
// radius above 2 h (refit steps move particles by 1e-4 to 1e-2 h each).
#include <climits>

#include "sph_internal.cuh"

namespace {

constexpr int SEARCH_WARPS = 4;
constexpr int SSTK = 512;
constexpr unsigned FULL = 0xffffffffu;
// pending bucket particles: ranges of consecutive slots, range r starting at
// slot rf[r] and at offset rs[r] of the pending stream (rs ascending; at most
// 31 carried ranges + 32 appended by one round)
constexpr int NRANGE = 64;

struct SearchSmem {
    int stk[SSTK];
    int flat[32];  // slots of the chunk being processed
    int rf[NRANGE], rs[NRANGE];
    double4 stage[32];
    double smass[32];
    // FP32 copies of the staged positions relative to the group's centre and
    // of their h, one array per field (four entries per 128-bit load)
    __align__(8) float fx[32];
    __align__(8) float fy[32];
    __align__(8) float fz[32];
    __align__(8) float fh[32];
    // the same per candidate (x, y, z, m) for the hit loop of the h iteration
    float4 fq[32];
};

__device__ __forceinline__ float2 ldf2(const float *p) { return *reinterpret_cast<const float2 *>(p); }
__device__ __forceinline__ float4 ldf4(const float *p) { return *reinterpret_cast<const float4 *>(p); }
__device__ __forceinline__ float2 lo2(float4 v) { return make_float2(v.x, v.y); }
__device__ __forceinline__ float2 hi2(float4 v) { return make_float2(v.z, v.w); }
__device__ __forceinline__ float2 bc2(float a) { return make_float2(a, a); }

template <class R> struct R2;
template <> struct R2<float> { typedef float2 T; };
template <> struct R2<double> { typedef double2 T; };

// Sums of the h iteration at one trial h: S = sum m_j w(q), D = sum m_j
// w'(q)-form (q = r_ij / h, M4 kernel without its 1/(pi h^3) factor)
template <class R> struct HSums {
    KSum<R> S, D;
    R inv_h;
    // kernel terms at distance r, branch-free in the B-spline form of the
    // two pieces: with a = (2 - q)+ and b = (1 - q)+,
    //   w  = a^3 / 4 - b^3                    (1 - 1.5 q^2 + 0.75 q^3 up to q = 1)
    //   dw = 1.5 a^2 (1 - q) - 3 b^2 (1 - 2q)  (3 - 7.5 q^2 + 4.5 q^3 up to q = 1)
    // both zero from q = 2 on
    __device__ __forceinline__ void terms(R r, R &w, R &dw) const {
        const R q = r * inv_h;
        const R a = fmax(R(2) - q, R(0)), b = fmax(R(1) - q, R(0));
        const R a2 = a * a, b2 = b * b;
        w = fma(R(0.25) * a2, a, -(b2 * b));
        dw = fma(R(1.5) * a2, R(1) - q, R(-3) * b2 * fma(R(-2), q, R(1)));
    }
    __device__ __forceinline__ void add(R r, R m) {
        const R q = r * inv_h;
        if (q < R(2)) {
            R w, dw;
            if (q <= R(1)) {
                w = R(1) - R(1.5) * q * q + R(0.75) * q * q * q;
                dw = R(3) - R(7.5) * q * q + R(4.5) * q * q * q;
            } else {
                const R t = R(2) - q;
                w = R(0.25) * t * t * t;
                dw = R(1.5) * t * t * (R(1) - q);
            }
            S.add(m * w);
            D.add(m * dw);
        }
    }
};

// |r_ij| in the sums' type: the difference taken in FP64, then rounded
template <class R>
__device__ __forceinline__ R pair_r(const double4 &pi, const double4 &pj) {
    const R rx = (R)(pi.x - pj.x), ry = (R)(pi.y - pj.y), rz = (R)(pi.z - pj.z);
    return qsqrt<R>(rx * rx + ry * ry + rz * rz);
}

__device__ __forceinline__ double wmin(double v) {
    for (int o = 16; o; o >>= 1) v = fmin(v, __shfl_xor_sync(FULL, v, o));
    return v;
}
__device__ __forceinline__ double wmax(double v) {
    for (int o = 16; o; o >>= 1) v = fmax(v, __shfl_xor_sync(FULL, v, o));
    return v;
}

struct SearchArgs {
    const int *gstart, *gcount, *gcloud, *croot;
    double4 *p0;
    // node boxes in FP32 rounded outward: (min rounded down, h_max rounded
    // up), (max rounded up, 0)
    const float4 *sA, *sB;
    const int4 *wL;  // per node: first particle, count, left and right child
    int leaf_size, K;
    int *rows, *cnt;
    int *ngb_cnt;  // list counts written by k_lists_cand (cnt holds candidate counts)
    double *hnb;   // per particle: the largest h_j of its list (written by the list builds)
    // candidate rows of the h iteration: the slots j inside the particle's
    // candidate radius, max_ngb entries per particle (row i at i K)
    int *cidx;
    const void *p1;  // Real4 (v, m)
    // exact search restricted to the particles with only[i] != 0, or to all
    // of them when *only_all != 0 (null: every particle)
    const int *only, *only_all;
    // with only: the marked particles also listed (mlist, *mcount entries);
    // k_lists then runs only when *only_all, k_lists_list otherwise
    const int *mlist, *mcount;
    long long *status;
};

// Walk the tree for group g and write the rows of the active lanes.
// MODE 0: candidates r^2 <= ri^2 (ri = 2 hc_i, the h iteration's gather radius)
//         with the first Newton evaluation's kernel sums
// MODE 1: exact lists |r|^2 <= (h_i + h_j)^2
// MODE 2: candidates r^2 <= ri^2 alone (the count iteration)
template <int MODE, class R = double>
__device__ __forceinline__ void group_search(SearchSmem &S, const SearchArgs &A, int g, bool act,
                                             int i, const double4 &pi, double ri,
                                             HSums<R> *hs = nullptr) {
    typedef typename R4<R>::T V4;
    const int lane = threadIdx.x & 31;
    const unsigned lt = (1u << lane) - 1u;
    const double gx0 = wmin(act ? pi.x : INFINITY), gy0 = wmin(act ? pi.y : INFINITY),
                 gz0 = wmin(act ? pi.z : INFINITY);
    const double gx1 = wmax(act ? pi.x : -INFINITY), gy1 = wmax(act ? pi.y : -INFINITY),
                 gz1 = wmax(act ? pi.z : -INFINITY);
    const double rmax = wmax(act ? ri : 0.0);
    const double ri2 = ri * ri;
    const int K = A.K;
    // the traversal's box test in FP32 with directed rounding: the group box
    // rounded outward, the gap between the boxes rounded down and the reach
    // rounded up, so a node is opened whenever the FP64 test would open it
    const float fgx0 = __double2float_rd(gx0), fgy0 = __double2float_rd(gy0),
                fgz0 = __double2float_rd(gz0);
    const float fgx1 = __double2float_ru(gx1), fgy1 = __double2float_ru(gy1),
                fgz1 = __double2float_ru(gz1);
    const float frmax = fmaxf(__double2float_ru(rmax), 1e-18f);
    // candidate row of particle i: entries [i K, i K + K)
    const size_t cbase = MODE != 1 ? (size_t)i * K : 0;
    int count = 0;
    double hnb = 0.0;
    int sp = 1, nflat = 0, nr = 0;
    bool overflow = false;
    if (lane == 0) S.stk[0] = A.croot[A.gcloud[g]];
    __syncwarp();

    // FP32 prefilter: distances relative to the group's centre, compared
    // with the threshold widened by a margin; the candidates it passes get
    // the exact FP64 test, so the rows are the same as an FP64-only scan.
    // The relative error of the FP32 r^2 is at most about 2^-21 (2E/R + 3)
    // (E the group's half-diagonal, R the search radius: the coordinates are
    // rounded at their distance from the centre, which is at most E + R), so
    // the margin is 1e-4 plus a bound of that size: 1e-4 alone while E stays
    // below about 100 R, wider for a sparse group.
    const double cx = 0.5 * (gx0 + gx1), cy = 0.5 * (gy0 + gy1), cz = 0.5 * (gz0 + gz1);
    const double ex = 0.5 * sqrt((gx1 - gx0) * (gx1 - gx0) + (gy1 - gy0) * (gy1 - gy0) +
                                 (gz1 - gz0) * (gz1 - gz0));
    const double rsearch = MODE == 1 ? pi.w : ri;
    const float mrg = (float)(1e-4 + ldexp(2.0 * ex / fmax(rsearch, 1e-300) + 3.0, -20));
    const float2 pfx = bc2((float)(pi.x - cx)), pfy = bc2((float)(pi.y - cy)),
                 pfz = bc2((float)(pi.z - cz));
    const float2 ri2f = bc2((float)ri2 * (1.f + mrg)), hif = bc2((float)pi.w);
    // FP32 h iteration: a candidate whose FP32 distance is below the
    // threshold narrowed by the same margin is inside in FP64 too and skips
    // the FP64 test; its kernel terms use the FP32 relative coordinates and
    // are summed plainly over the chunk (at most 32 terms), then added to the
    // Kahan sums
    constexpr bool FAST = MODE == 0 && std::is_same<R, float>::value;
    const float2 ri2lo = bc2((float)ri2 * (1.f - mrg));
    const float2 m1 = bc2(-1.f), nwiden = bc2(-(1.f + mrg)), nri2f = bc2(-ri2f.x);

    // slot of the particle at offset t of the pending stream: the last range
    // starting at or before t
    auto part_slot = [&](int t) {
        int r = 0;
#pragma unroll
        for (int step = NRANGE / 2; step; step >>= 1) {
            const int c = r + step;
            if (c < nr && S.rs[c] <= t) r = c;
        }
        return S.rf[r] + (t - S.rs[r]);
    };
    // the m pending candidates from stream offset h
    auto process = [&](int m, int h) {
        if (lane < m) {
            const int j = part_slot(h + lane);
            S.flat[lane] = j;
            const double4 q = A.p0[j];
            S.stage[lane] = q;
            const float qx = (float)(q.x - cx), qy = (float)(q.y - cy), qz = (float)(q.z - cz);
            S.fx[lane] = qx;
            S.fy[lane] = qy;
            S.fz[lane] = qz;
            if (FAST) {
                const float mj = (float)((const V4 *)A.p1)[j].w;
                S.fh[lane] = mj;
                S.fq[lane] = make_float4(qx, qy, qz, mj);
            } else {
                S.fh[lane] = (float)q.w;
            }
            if (MODE == 0 && !FAST) S.smass[lane] = (double)((const V4 *)A.p1)[j].w;
        } else if (lane < ((m + 3) & ~3)) {
            // the tail of a chunk up to a multiple of four: entries that
            // never pass
            S.fx[lane] = S.fy[lane] = S.fz[lane] = INFINITY;
            S.fh[lane] = 0.f;
        }
        __syncwarp();
        const int m4 = (m + 3) & ~3;
        unsigned hit = 0;
        if (act) {
            // d = r^2 - lim accumulated from -lim: a set sign bit is a hit
            // (within a few ulps of the widened threshold, which lies outside
            // the true radius, a candidate may count either way); the sign
            // bits are shifted into acc one per candidate, the newest at bit 0
            unsigned acc = 0;
            auto pair = [&](float2 qx, float2 qy, float2 qz, float2 qh) {
                const float2 dx = __ffma2_rn(qx, m1, pfx);
                const float2 dy = __ffma2_rn(qy, m1, pfy);
                const float2 dz = __ffma2_rn(qz, m1, pfz);
                float2 nlim = nri2f;
                if (MODE == 1) {
                    const float2 sh = __fadd2_rn(hif, qh);
                    nlim = __fmul2_rn(__fmul2_rn(sh, sh), nwiden);
                }
                const float2 d = __ffma2_rn(dz, dz, __ffma2_rn(dy, dy, __ffma2_rn(dx, dx, nlim)));
                acc = __funnelshift_l(__float_as_uint(d.x), acc, 1);
                acc = __funnelshift_l(__float_as_uint(d.y), acc, 1);
            };
            if ((reinterpret_cast<uintptr_t>(S.fx) & 15u) == 0) {
                // four candidates per 128-bit shared load
#pragma unroll 2
                for (int k = 0; k < m4; k += 4) {
                    const float4 X = ldf4(&S.fx[k]), Y = ldf4(&S.fy[k]), Z = ldf4(&S.fz[k]);
                    const float4 H = MODE == 1 ? ldf4(&S.fh[k]) : X;
                    pair(lo2(X), lo2(Y), lo2(Z), lo2(H));
                    pair(hi2(X), hi2(Y), hi2(Z), hi2(H));
                }
            } else {
                // (a shared array placed on an 8-byte boundary only)
#pragma unroll 4
                for (int k = 0; k < m4; k += 2)
                    pair(ldf2(&S.fx[k]), ldf2(&S.fy[k]), ldf2(&S.fz[k]),
                         MODE == 1 ? ldf2(&S.fh[k]) : bc2(0.f));
            }
            // candidate k's sign bit is at bit m4 - 1 - k (m4 = m rounded up
            // to a multiple of four, 4..32; the padding entries never pass)
            hit = (__brev(acc) >> (32 - m4)) & (0xffffffffu >> (32 - m4));
        }
        R cs = R(0), cd = R(0);
        if (FAST) {
            // two hits per trip (independent chains for the scheduler), the
            // sums and the row entries in the same order as one per trip
            auto exact_in = [&](int k) {
                const double4 pj = S.stage[k];
                const double dx = pi.x - pj.x, dy = pi.y - pj.y, dz = pi.z - pj.z;
                return dx * dx + dy * dy + dz * dz <= ri2;
            };
            while (hit) {
                const int k1 = __ffs(hit) - 1;
                hit &= hit - 1;
                const bool two = hit != 0;
                const int k2 = two ? __ffs(hit) - 1 : k1;
                hit &= hit - 1;
                // the prefilter's FP32 r^2, rounded the same way: below the
                // narrowed threshold the candidate is inside in FP64 too
                const float4 c1 = S.fq[k1], c2 = S.fq[k2];
                const float ax = pfx.x - c1.x, ay = pfy.x - c1.y, az = pfz.x - c1.z;
                const float bx = pfx.x - c2.x, by = pfy.x - c2.y, bz = pfz.x - c2.z;
                const float r2a = fmaf(az, az, fmaf(ay, ay, ax * ax));
                const float r2b = fmaf(bz, bz, fmaf(by, by, bx * bx));
                bool in1 = r2a <= ri2lo.x, in2 = two && r2b <= ri2lo.x;
                if (!in1) in1 = exact_in(k1);
                if (two && !in2) in2 = exact_in(k2);
                // r = r^2 rsqrt(r^2 + 1e-30): the same r for the candidates'
                // r^2 (far above 1e-30), 0 for the particle itself
                R w1, dw1, w2, dw2;
                hs->terms(r2a * rsqrtf(r2a + 1e-30f), w1, dw1);
                hs->terms(r2b * rsqrtf(r2b + 1e-30f), w2, dw2);
                if (in1) {
                    cs = fmaf(c1.w, w1, cs);
                    cd = fmaf(c1.w, dw1, cd);
                    if (count < K) A.cidx[cbase + count] = S.flat[k1];
                    count++;
                }
                if (in2) {
                    cs = fmaf(c2.w, w2, cs);
                    cd = fmaf(c2.w, dw2, cd);
                    if (count < K) A.cidx[cbase + count] = S.flat[k2];
                    count++;
                }
            }
        }
        while (!FAST && hit) {
            const int k = __ffs(hit) - 1;
            hit &= hit - 1;
            const double4 pj = S.stage[k];
            if (MODE != 1) {
                const double dx = pi.x - pj.x, dy = pi.y - pj.y, dz = pi.z - pj.z;
                if (dx * dx + dy * dy + dz * dz <= ri2) {
                    // the first Newton evaluation (at h = pi.w) rides on the
                    // search: rows are only re-read by later iterations
                    if (MODE == 0) hs->add(pair_r<R>(pi, pj), (R)S.smass[k]);
                    if (count < K) A.cidx[cbase + count] = S.flat[k];
                    count++;
                }
            } else {
                if (ngb_pred(pi.x, pi.y, pi.z, pi.w, pj.x, pj.y, pj.z, pj.w)) {
                    if (count < K) A.rows[(size_t)i * K + count] = S.flat[k];
                    count++;
                    hnb = fmax(hnb, pj.w);
                }
            }
        }
        if (FAST) {
            hs->S.add(cs);
            hs->D.add(cd);
        }
        __syncwarp();
    };

    while (sp > 0 || nflat > 0) {
        if (sp > 0) {
            const int take = min(sp, 32);
            sp -= take;
            int nd = 0, f = 0, cn = 0, cl = 0, cr = 0;
            bool open = false;
            if (lane < take) {
                nd = S.stk[sp + lane];
                const float4 a = A.sA[nd], b = A.sB[nd];
                const int4 L = A.wL[nd];
                f = L.x;
                cn = L.y;
                cl = L.z;
                cr = L.w;
                const float ex = fmaxf(fmaxf(__fsub_rd(a.x, fgx1), __fsub_rd(fgx0, b.x)), 0.f);
                const float ey = fmaxf(fmaxf(__fsub_rd(a.y, fgy1), __fsub_rd(fgy0, b.y)), 0.f);
                const float ez = fmaxf(fmaxf(__fsub_rd(a.z, fgz1), __fsub_rd(fgz0, b.z)), 0.f);
                const float d2 = __fmaf_rd(ez, ez, __fmaf_rd(ey, ey, __fmul_rd(ex, ex)));
                const float reach = MODE != 1 ? frmax : __fadd_ru(a.w, frmax);
                open = d2 <= __fmul_ru(__fmul_ru(reach, reach), 1.000001f);
            }
            __syncwarp();
            const bool leafy = cn <= A.leaf_size;
            const unsigned pm = __ballot_sync(FULL, open && !leafy);
            const int npush = 2 * __popc(pm);
            if (sp + npush <= SSTK) {
                if (open && !leafy) {
                    int pos = sp + 2 * __popc(pm & lt);
                    S.stk[pos] = cr;
                    S.stk[pos + 1] = cl;
                }
                sp += npush;
            } else {
                overflow = true;
            }
            const bool bucket = open && leafy;
            const unsigned lm = __ballot_sync(FULL, bucket);
            __syncwarp();
            if (lm) {
                // opened buckets join the pending stream in lane order: one
                // range per bucket at the scanned offset
                const int cnt = bucket ? cn : 0;
                int incl = cnt;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const int t = __shfl_up_sync(FULL, incl, o);
                    if (lane >= o) incl += t;
                }
                if (bucket) {
                    const int r = nr + __popc(lm & lt);
                    S.rf[r] = f;
                    S.rs[r] = nflat + incl - cnt;
                }
                nr += __popc(lm);
                nflat += __shfl_sync(FULL, incl, 31);
                __syncwarp();
                if (nflat >= 32) {
                    int h = 0;
                    do {
                        process(32, h);
                        h += 32;
                    } while (nflat - h >= 32);
                    nflat -= h;
                    // keep the ranges from the one holding offset h on, their
                    // offsets taken from h (<= 31 of them: each keeps at
                    // least one of the < 32 pending candidates)
                    int r0 = nr;
                    if (nflat > 0) {
                        r0 = 0;
#pragma unroll
                        for (int step = NRANGE / 2; step; step >>= 1) {
                            const int c = r0 + step;
                            if (c < nr && S.rs[c] <= h) r0 = c;
                        }
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
        if (sp == 0 && nflat > 0) {
            process(nflat, 0);
            nflat = 0;
            nr = 0;
        }
    }
    if (act) {
        if (MODE != 1) {
            // the full count: the Newton step shrinks the gather radius of a
            // row that did not fit instead of iterating on a truncated one
            A.cnt[i] = count;
        } else {
            A.cnt[i] = min(count, K);
            if (count > K) status_add(A.status, SPH_S_NGB_OVERFLOW, 1);
            A.hnb[i] = hnb;
        }
    }
    if (overflow && lane == 0) status_add(A.status, SPH_S_STACK_OVERFLOW, 1);
    __syncwarp();
}

// exact lists for every particle
__global__ void __launch_bounds__(SEARCH_WARPS * 32)
    k_lists(const int *__restrict__ ngroup_p, SearchArgs A, unsigned *queue) {
    __shared__ SearchSmem smem[SEARCH_WARPS];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int ngroup = *ngroup_p;
    if (A.mlist && !*A.only_all) return;  // the listed particles: k_lists_list
    for (int g = q_first(queue, blockIdx.x * SEARCH_WARPS + w); g < ngroup;
         g = q_next(queue, g, gridDim.x * SEARCH_WARPS)) {
        const int s0 = A.gstart[g], gc = A.gcount[g];
        bool act = lane < gc;
        const int i = s0 + (act ? lane : 0);
        if (A.only && !*A.only_all) {
            act = act && A.only[i];
            if (!__any_sync(FULL, act)) continue;
        }
        const double4 pi = A.p0[i];
        group_search<1>(smem[w], A, g, act, i, pi, pi.w);
    }
}

// exact lists for the listed particles (A.mlist, *A.mcount entries; nothing
// when *A.only_all, which k_lists covers): one warp per particle, its own box
// (the search of one lane), the cloud root of the group holding it
__global__ void __launch_bounds__(SEARCH_WARPS * 32)
    k_lists_list(const int *__restrict__ ngroup_p, SearchArgs A) {
    __shared__ SearchSmem smem[SEARCH_WARPS];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (*A.only_all) return;
    const int m = *A.mcount, ngroup = *ngroup_p;
    for (int e = blockIdx.x * SEARCH_WARPS + w; e < m; e += gridDim.x * SEARCH_WARPS) {
        const int i = A.mlist[e];
        // the group holding i: the last one starting at or before it
        int lo = 0, hi = ngroup - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (A.gstart[mid] <= i) lo = mid;
            else hi = mid - 1;
        }
        const double4 pi = A.p0[i];
        group_search<1>(smem[w], A, lo, lane == 0, i, pi, pi.w);
    }
}

// Exact lists from the candidate rows of the h iteration.  A pair with
// |r| <= h_i + h_j lies inside 2 max(h_i, h_j), so it sits in the candidate
// row of the particle with the larger h (2 h <= 2 hc, the radius of that
// particle's last candidate search).  Each lane filters its own row with the
// exact predicate (same rounding as the tree search); where a pair's partner
// j did not hold i in its own row (|r| beyond 2 hc_j, with a margin for
// rounding), j's list may miss i and j is marked for the tree search.  A row
// that is not a complete candidate set (overflow, or h above the candidate
// radius after the last round) sends every particle to the tree search.
__global__ void __launch_bounds__(SEARCH_WARPS * 32, 6)
    k_lists_cand(const int *__restrict__ ngroup_p, SearchArgs A, const double *__restrict__ hc,
                 int *__restrict__ full, int *__restrict__ full_all, int *__restrict__ full_any) {
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int ngroup = *ngroup_p;
    const int K = A.K;
    for (int g = blockIdx.x * SEARCH_WARPS + w; g < ngroup; g += gridDim.x * SEARCH_WARPS) {
        const int s0 = A.gstart[g], gc = A.gcount[g];
        if (lane >= gc) continue;
        const int i = s0 + lane;
        const double4 pi = A.p0[i];
        const int craw = A.cnt[i];
        if (craw > K || !(pi.w <= hc[i])) {
            *full_all = 1;
            *full_any = 1;
            continue;
        }
        const int *crow = A.cidx + (size_t)i * K;
        const double4 *__restrict__ p0 = A.p0;
        int count = 0;
        double hnb = 0.0;
        // four candidates per round: their index, position and radius loads
        // are issued together (the loop is bound by gather latency)
        constexpr int U = 4;
        for (int k0 = 0; k0 < craw; k0 += U) {
            int jj[U];
            double4 pj[U];
            double hj[U];
#pragma unroll
            for (int u = 0; u < U; u++) jj[u] = k0 + u < craw ? __ldg(&crow[k0 + u]) : i;
#pragma unroll
            for (int u = 0; u < U; u++) {
                pj[u] = p0[jj[u]];
                hj[u] = __ldg(&hc[jj[u]]);
            }
#pragma unroll
            for (int u = 0; u < U; u++) {
                if (k0 + u < craw && ngb_pred(pi.x, pi.y, pi.z, pi.w, pj[u].x, pj[u].y, pj[u].z, pj[u].w)) {
                    if (count < K) A.rows[(size_t)i * K + count] = jj[u];
                    count++;
                    hnb = fmax(hnb, pj[u].w);
                    const double dx = pi.x - pj[u].x, dy = pi.y - pj[u].y, dz = pi.z - pj[u].z;
                    const double rj = 2.0 * hj[u];
                    if (dx * dx + dy * dy + dz * dz > rj * rj * (1.0 - 1e-9)) {
                        full[jj[u]] = 1;
                        *full_any = 1;
                    }
                }
            }
        }
        A.ngb_cnt[i] = min(count, K);
        if (count > K) status_add(A.status, SPH_S_NGB_OVERFLOW, 1);
        A.hnb[i] = hnb;
    }
}

// candidate radius 2 hc: a margin `grow` over h for the iteration, widened
// to reach h_i + 1.05 h_nb (the largest neighbour h of the last list build) so
// that the next list is complete from the particle's own candidates, at most
// to 2 (1.5 h)
__device__ __forceinline__ double cand_half_radius(double h, double hnb, double grow) {
    return fmax(h * grow, fmin(0.5 * (h + 1.05 * hnb), 1.5 * h));
}

// the smallest room a kept row must leave above h: a Newton root beyond it
// sends the particle to the search; and the reach it must keep towards the
// largest neighbour h of the last list build (times REACH), below which the
// list pass would send that neighbour to a tree search: at most REACH_CAP h,
// just below the 1.5 h that caps a search's own reach
#ifndef SPH_REUSE_ROOM
#define SPH_REUSE_ROOM 1.01
#endif
#ifndef SPH_REUSE_REACH
#define SPH_REUSE_REACH 1.01
#endif
#ifndef SPH_REUSE_REACH_CAP
#define SPH_REUSE_REACH_CAP 1.48
#endif

// the radius / 2 a kept row must still cover
__device__ __forceinline__ double reuse_need(double h, double hnb) {
    return fmax(h * SPH_REUSE_ROOM,
                fmin(0.5 * (h + SPH_REUSE_REACH * hnb), SPH_REUSE_REACH_CAP * h));
}

// Row reuse.  A search at radius 2 hsr_i listed every j within 2 hsr_i of
// particle i's position then.  Since that search i moved at most dmv_i and
// every j at most dmv_j, so the row still lists every j now within
// 2 hsr_i - dmv_i - M of i, M the largest dmv_j of the particles now that
// close: half of that is the particle's candidate radius hc without a
// search.  M = the cloud's largest dmv decides here (retry 2); where that is
// too coarse but the particle's own move leaves room (retry 3), the first
// search round bounds M by the particles of the tree nodes near its group.
// An h iteration that searches every particle (the rows dropped, reuse off,
// or the last attempt kept fewer than an eighth of the rows) restarts the
// distances moved, so the next one can keep rows again.
struct ReuseArgs {
    int on;                     // rows may be kept
    const int *rows_ok;         // device flag: the rows belong to the storage order
    const double *hsr;
    double *dmv;
    unsigned long long *dmv_max;
    const int *cloud;
    int *kept;                  // rows kept: [0] this h iteration, [1] the last attempt
                                // (INT_MAX after a full search), [2] this one attempts
};

// the kept-row counts moved on by one h iteration (one thread)
__global__ void k_kept_shift(int *kept) {
    kept[1] = kept[2] ? kept[0] : INT_MAX;
    kept[0] = 0;
    kept[2] = 0;
}

__global__ void k_h_init(int n, const double *__restrict__ h, const double *__restrict__ hnb,
                         double *__restrict__ hc, int *__restrict__ retry, double grow,
                         double *__restrict__ hover, ReuseArgs U) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double hi = h[i], hn = hnb[i];
    double c = cand_half_radius(hi, hn, grow);
    int r = 1;
    const bool attempt = U.on && *U.rows_ok && U.kept[1] >= n / 8;
    if (U.kept && i == 0) U.kept[2] = attempt ? 1 : 0;
    if (attempt) {
        const double hs = U.hsr[i], own = U.dmv[i];
        const double cl = __longlong_as_double((long long)U.dmv_max[U.cloud[i]]);
        const double keep = (hs - 0.5 * (own + cl)) * (1.0 - 1e-12);
        const double need = reuse_need(hi, hn);
        if (hs > 0.0 && keep >= need) {
            c = keep;
            r = 2;
        } else if (hs > 0.0 && (hs - 0.5 * own) * (1.0 - 1e-12) >= need) {
            r = 3;
        }
    } else if (U.dmv) {
        U.dmv[i] = 0.0;
        if (i == 0 || U.cloud[i] != U.cloud[i - 1]) U.dmv_max[U.cloud[i]] = 0ull;
    }
    hc[i] = c;
    retry[i] = r;
    if (hover) hover[i] = INFINITY;
}

// per particle: the largest distance moved in its group, rounded up to FP32
// (every tree node of at most 32 particles lies inside one group); one warp
// per group
__global__ void k_group_moved(const int *__restrict__ ngroup_p, const int *__restrict__ gstart,
                              const int *__restrict__ gcount, const double *__restrict__ dmv,
                              float *__restrict__ gdm) {
    const int lane = threadIdx.x & 31;
    const int ngroup = *ngroup_p;
    const int nw = gridDim.x * (blockDim.x >> 5);
    for (int g = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); g < ngroup; g += nw) {
        const int s0 = gstart[g], gc = gcount[g];
        double d = lane < gc ? dmv[s0 + lane] : 0.0;
        for (int o = 16; o; o >>= 1) d = fmax(d, __shfl_xor_sync(FULL, d, o));
        if (lane < gc) gdm[s0 + lane] = __double2float_ru(d);
    }
}

// The largest distance moved (gdm) over the particles of the tree nodes of
// the cloud whose boxes come within frmax of the box [fg0, fg1] (boxes as the
// search tests them, rounded outward): every particle now that close to the
// box is in one of them.  INFINITY as soon as it passes lim, or if the
// stack would overflow.
__device__ float moved_near(SearchSmem &S, const SearchArgs &A, int root, float fgx0, float fgy0,
                           float fgz0, float fgx1, float fgy1, float fgz1, float frmax, float lim,
                           const float *__restrict__ gdm) {
    const int lane = threadIdx.x & 31;
    const unsigned lt = (1u << lane) - 1u;
    const float reach2 = __fmul_ru(__fmul_ru(frmax, frmax), 1.000001f);
    int sp = 1;
    if (lane == 0) S.stk[0] = root;
    __syncwarp();
    float m = 0.f;
    bool bad = false;
    while (sp > 0) {
        const int take = min(sp, 32);
        sp -= take;
        int f = 0, cn = 0, cl = 0, cr = 0;
        bool open = false;
        if (lane < take) {
            const int nd = S.stk[sp + lane];
            const float4 a = A.sA[nd], b = A.sB[nd];
            const int4 L = A.wL[nd];
            f = L.x;
            cn = L.y;
            cl = L.z;
            cr = L.w;
            const float ex = fmaxf(fmaxf(__fsub_rd(a.x, fgx1), __fsub_rd(fgx0, b.x)), 0.f);
            const float ey = fmaxf(fmaxf(__fsub_rd(a.y, fgy1), __fsub_rd(fgy0, b.y)), 0.f);
            const float ez = fmaxf(fmaxf(__fsub_rd(a.z, fgz1), __fsub_rd(fgz0, b.z)), 0.f);
            const float d2 = __fmaf_rd(ez, ez, __fmaf_rd(ey, ey, __fmul_rd(ex, ex)));
            open = d2 <= reach2;
        }
        __syncwarp();
        const bool small = cn <= 32;
        if (open && small) m = fmaxf(m, gdm[f]);
        const unsigned pm = __ballot_sync(FULL, open && !small);
        const int npush = 2 * __popc(pm);
        if (sp + npush > SSTK || __any_sync(FULL, m > lim)) {
            bad = true;
            break;
        }
        if (open && !small) {
            const int pos = sp + 2 * __popc(pm & lt);
            S.stk[pos] = cr;
            S.stk[pos + 1] = cl;
        }
        sp += npush;
        __syncwarp();
    }
    __syncwarp();
    for (int o = 16; o; o >>= 1) m = fmaxf(m, __shfl_xor_sync(FULL, m, o));
    return bad ? INFINITY : m;
}

struct NewtonArgs {
    const void *p1;  // Real4 (v, m)
    double *h_out, *hc;
    double *hover;   // per particle: the smallest candidate radius / 2 whose row overflowed
    double *hsr;     // per particle: radius / 2 of the search that wrote the row (0: incomplete)
    const double *hnb;
    const double *dmv;  // distances moved (with hsr: the bound of a kept row)
    const float *gdm;   // per particle: its group's largest dmv, rounded up
    int *kept;       // count of the particles that kept their row (null: not counted)
    int *retry;
    double n_ngb, tol, grow, regrow;
    int max_iter, last_round;
};

// Newton iteration of the particle of every active lane, FP32 or FP64 kernel
// sums with FP64 update and convergence test.  The first evaluation (at
// h = pi.w), S0 and D0, comes from the search (searched) or from the kept
// row; later ones, rare once h has settled from step to step, gather the
// candidates again through the particle's slot row in the same order, so
// they sum the same terms in the same order.  No warp collectives: lanes run
// independent iteration counts.
template <class R>
__device__ __forceinline__ void newton_lane(const SearchArgs &A, const NewtonArgs &B, int i,
                                            const double4 &pi, const int *row, double S0,
                                            double D0, bool searched) {
    typedef typename R4<R>::T V4;
    const V4 *p1 = (const V4 *)B.p1;
    const int craw = A.cnt[i];
    if (searched) B.hsr[i] = craw > A.K ? 0.0 : B.hc[i];
    if (craw > A.K) {
        // more candidates inside 2 hc than the row holds: the sums would miss
        // some, so remember that radius, shrink hc towards a three-quarter
        // full row and search again; h restarts at most just below the new
        // radius
        if (!B.last_round) {
            B.hover[i] = fmin(B.hover[i], B.hc[i]);
            const double hc = B.hc[i] * fmax(0.5, cbrt(0.75 * A.K / (double)craw));
            const double h0 = fmin(pi.w, hc / B.grow);
            B.hc[i] = hc;
            B.retry[i] = 1;
            B.h_out[i] = h0;
            A.p0[i].w = h0;
            status_add(A.status, SPH_S_H_RETRY, 1);
        } else {
            B.retry[i] = 0;
            status_add(A.status, SPH_S_NGB_OVERFLOW, 1);
            status_add(A.status, SPH_S_H_NOCONV, 1);
        }
        return;
    }
    const int c = craw;
    const double mi = (double)p1[i].w;
    const double cap = B.hc[i];
    const double cfac = 4.0 * SPH_PI / 3.0 * 8.0;
    double h = pi.w, lo = 0.0, hi = INFINITY;
    bool ok = false, need = false;
    for (int it = 1; it <= B.max_iter; it++) {
        if (h > cap) {  // 2h would pass the candidate radius 2*cap
            need = true;
            break;
        }
        double Ssum, Dsum;
        if (it == 1) {
            Ssum = S0;
            Dsum = D0;
        } else {
            HSums<R> hs;
            hs.inv_h = R(1.0 / h);
            for (int k = 0; k < c; k++) {
                const int j = row[k];
                hs.add(pair_r<R>(pi, A.p0[j]), (R)(double)p1[j].w);
            }
            Ssum = hs.S.value();
            Dsum = hs.D.value();
        }
        const double h3 = h * h * h;
        const double rho = SPH_SIG / h3 * Ssum;
        const double drho = -SPH_SIG / (h3 * h) * Dsum;
        const double f = cfac * h3 * rho - B.n_ngb * mi;
        const double fp = cfac * h * h * (3.0 * rho + h * drho);
        if (f < 0.0) lo = h; else hi = h;
        double hn = fp > 0.0 ? h - f / fp : -1.0;
        // a Newton step below the tolerance is accepted before any bracket
        // test: in FP64 it can round to exactly h (= a bracket end); one that
        // ends beyond the candidate radius needs the wider search first
        if (fp > 0.0 && fabs(f / fp) < B.tol * h) {
            h = hn;
            if (h > cap) need = true;
            else ok = true;
            break;
        }
        // at most a factor 1.25 per iteration (keeps retries inside the rows)
        if (hn > 1.25 * h) hn = 1.25 * h;
        if (hn > 0.0 && hn < h / 1.25) hn = h / 1.25;
        if (!(hn > lo && hn < hi)) {
            if (hi == INFINITY) hn = 1.25 * h;
            else if (lo == 0.0) hn = h / 1.25;
            else hn = 0.5 * (lo + hi);
        }
        // an iterate beyond the candidate radius first tries the radius
        // itself, where the row still holds every term: only a root beyond
        // it sends the particle to another search (an overshooting Newton
        // step alone used to)
        bool clamped = false;
        if (hn > cap && h < cap) {
            hn = cap;
            clamped = true;
        }
        const double dh = hn - h;
        h = hn;
        if (!clamped && fabs(dh) < B.tol * fabs(h - dh)) {
            if (h > cap) need = true;
            else ok = true;
            break;
        }
    }
    if (need && !B.last_round) {
        // a wider search, kept below a radius whose row already overflowed;
        // a kept row that h outgrew is searched at the usual radius
        const double ov = B.hover[i];
        const double g = searched ? h * B.regrow : cand_half_radius(h, B.hnb[i], B.grow);
        B.hc[i] = h < ov ? fmin(g, h + 0.5 * (ov - h)) : g;
        B.retry[i] = 1;
    } else {
        B.retry[i] = 0;
        if (!ok) status_add(A.status, SPH_S_H_NOCONV, 1);
    }
    if (need) status_add(A.status, SPH_S_H_RETRY, 1);
    B.h_out[i] = h;
    A.p0[i].w = h;  // p0 is written only by the lane owning particle i
}

// the first Newton evaluation of the kept rows of a group: four lanes per
// row over interleaved entries (terms beyond 2 h are zero), eight rows at a
// time, each row's sums handed to the lane of its particle
template <class R>
__device__ __forceinline__ void kept_sums(const SearchArgs &A, const NewtonArgs &B, int s0, int gc,
                                       double &S0, double &D0) {
    typedef typename R4<R>::T V4;
    const int lane = threadIdx.x & 31, q = lane >> 2, sl = lane & 3;
    S0 = 0.0;
    D0 = 0.0;
    for (int p = 0; p < gc; p += 8) {
        HSums<R> hk;
        hk.inv_h = R(1);
        if (p + q < gc) {
            const int ii = s0 + p + q;
            const double4 pp = A.p0[ii];
            hk.inv_h = R(1.0 / pp.w);
            const int c = A.cnt[ii];
            const int *rw = A.cidx + (size_t)ii * A.K;
            for (int k = sl; k < c; k += 4) {
                const int j = rw[k];
                hk.add(pair_r<R>(pp, A.p0[j]), (R)(double)((const V4 *)B.p1)[j].w);
            }
        }
        const double sS = seg_sum<4>(hk.S.value()), sD = seg_sum<4>(hk.D.value());
        const int src = ((lane - p) & 7) * 4;
        const double tS = __shfl_sync(FULL, sS, src), tD = __shfl_sync(FULL, sD, src);
        if (lane >= p && lane < p + 8) {
            S0 = tS;
            D0 = tD;
        }
    }
}

// candidate search + Newton iteration for the flagged particles of each group
// (retry 1), and in the first round the Newton iteration from the kept rows
// (retry 2 and 3) in the same warps, so both share the persistent grid that
// runs beside the gravity walk (latency-bound: 8 blocks per SM, 64
// registers, measured faster than 95)
template <class R>
__global__ void __launch_bounds__(SEARCH_WARPS * 32, 8)
    k_cand_newton(const int *__restrict__ ngroup_p, SearchArgs A, NewtonArgs B, unsigned *queue) {
    typedef typename R4<R>::T V4;
    __shared__ SearchSmem smem[SEARCH_WARPS];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int ngroup = *ngroup_p;
    for (int g = q_first(queue, blockIdx.x * SEARCH_WARPS + w); g < ngroup;
         g = q_next(queue, g, gridDim.x * SEARCH_WARPS)) {
        const int s0 = A.gstart[g], gc = A.gcount[g];
        const bool in = lane < gc;
        const int i = s0 + (in ? lane : 0);
        const int rt = in ? B.retry[i] : 0;
        const double4 pi = A.p0[i];
        // a group keeps its rows only as a whole: a lane gathering its row
        // alone would hold up the warp's search for the others
        bool part = __any_sync(FULL, rt == 1);
        if (!part && __any_sync(FULL, rt == 3)) {
            // the moves of the particles near the group decide: M, bounded
            // over the tree nodes within the largest kept radius of the
            // group's box, must leave each lane's row the radius it needs
            const bool l3 = rt == 3;
            const double hs = l3 ? B.hsr[i] : 0.0, own = l3 ? B.dmv[i] : 0.0;
            const double lim =
                l3 ? 2.0 * (hs - reuse_need(pi.w, B.hnb[i]) / (1.0 - 1e-12)) - own : INFINITY;
            const float flim = __double2float_rd(wmin(lim));
            const float fgx0 = __double2float_rd(wmin(l3 ? pi.x : INFINITY)),
                        fgy0 = __double2float_rd(wmin(l3 ? pi.y : INFINITY)),
                        fgz0 = __double2float_rd(wmin(l3 ? pi.z : INFINITY));
            const float fgx1 = __double2float_ru(wmax(l3 ? pi.x : -INFINITY)),
                        fgy1 = __double2float_ru(wmax(l3 ? pi.y : -INFINITY)),
                        fgz1 = __double2float_ru(wmax(l3 ? pi.z : -INFINITY));
            const float frmax = __double2float_ru(wmax(2.0 * hs));
            const float M = flim >= 0.f ? moved_near(smem[w], A, A.croot[A.gcloud[g]], fgx0, fgy0,
                                                     fgz0, fgx1, fgy1, fgz1, frmax, flim, B.gdm)
                                        : INFINITY;
            if (M <= flim) {
                if (l3) B.hc[i] = (hs - 0.5 * (own + (double)M)) * (1.0 - 1e-12);
            } else {
                part = true;
            }
        }
        const bool act = rt == 1 || (rt >= 2 && part), keep = rt >= 2 && !part;
        const unsigned todo = __ballot_sync(FULL, act);
        const unsigned km = __ballot_sync(FULL, keep);
        if (!todo && !km) continue;
        if (km && lane == 0 && B.kept) atomicAdd(B.kept, __popc(km));
        const int *row = A.cidx + (size_t)i * A.K;
        double hci = act ? B.hc[i] : 0.0;
        if (rt >= 2 && part) {
            // searched after all, at the usual radius
            hci = cand_half_radius(pi.w, B.hnb[i], B.grow);
            B.hc[i] = hci;
        }
        HSums<R> hs;
        hs.inv_h = R(1.0 / pi.w);
        if (todo) group_search<0, R>(smem[w], A, g, act, i, pi, 2.0 * hci, &hs);
        if (act) {
            // each lane reads back only the row entries it wrote itself
            newton_lane<R>(A, B, i, pi, row, hs.S.value(), hs.D.value(), true);
        }
        if (km) {
            // the group kept its rows (first round only; no lane searches)
            double S0, D0;
            kept_sums<R>(A, B, s0, gc, S0, D0);
            if (keep) newton_lane<R>(A, B, i, pi, row, S0, D0, false);
        }
        __syncwarp();
    }
}

// The reference's count iteration (h_smooth_fast_mpi, MPI_sph/sph_code/
// libsx.py:854-902) for the particle of one lane: with d_j = |r_j - r_i|
// (self included) and n(h) = #{j : d_j < 2 h}, h <- h - f h while n(h) > hi_n
// and h <- h + f h while n(h) < lo_n.  Its only state is h, so a particle
// whose 2 h would pass its candidate radius 2 hc stops, stores h and
// resumes in the next round with a wider radius: the sequence of h is that
// of one uninterrupted iteration.  d_j is rounded as the reference writes it
// (dx = x_j - x_i, dx dx + dy dy, + dz dz, correctly rounded square root),
// so the result is bit-exact with it on the same positions.
struct CountArgs {
    double *h_out, *hc;
    int *retry, *iters;
    int lo_n, hi_n, max_iter, last_round;
    double frac, grow;
};

__device__ __forceinline__ double ref_dist(const double4 &pi, const double4 &pj) {
    const double dx = xsub(pj.x, pi.x), dy = xsub(pj.y, pi.y), dz = xsub(pj.z, pi.z);
    return __dsqrt_rn(xadd(xadd(xmul(dx, dx), xmul(dy, dy)), xmul(dz, dz)));
}

__device__ __forceinline__ void count_lane(const SearchArgs &A, const CountArgs &B, int i,
                                           const double4 &pi, const int *row) {
    const int craw = A.cnt[i];
    double h = pi.w;
    int it = B.iters[i];
    const double cap = B.hc[i];
    bool ok = false, done = false, again = false;
    if (craw > A.K) {
        // the row cannot hold every candidate: narrow the radius towards a
        // half-full row and search again
        B.hc[i] = cap * fmax(0.5, cbrt(0.5 * A.K / (double)craw));
        again = true;
    } else {
        // every j with d_j < 2 lim is in the row: the search's r^2 test is
        // not rounded as d_j is, so lim keeps a margin below the radius
        const double lim = cap * (1.0 - 1e-12);
        if (h > lim) {
            // h beyond the complete radius: n(h) >= n(lim), so while n(lim)
            // is above the window every decrement is the reference's own
            const double l2 = 2.0 * lim;
            int nin = 0;
            for (int k = 0; k < craw; k++) nin += ref_dist(pi, A.p0[row[k]]) < l2;
            if (nin > B.hi_n) {
                while (h > lim) {
                    h = xsub(h, xmul(B.frac, h));
                    if (++it > B.max_iter) {
                        done = true;
                        break;
                    }
                }
            } else {
                B.hc[i] = h * B.grow;  // too few inside: search wider
                again = true;
            }
        }
        while (!done && !again && h <= lim) {
            const double h2 = 2.0 * h;
            int nn = 0;
            for (int k = 0; k < craw; k++) nn += ref_dist(pi, A.p0[row[k]]) < h2;
            if (nn > B.hi_n) {
                h = xsub(h, xmul(B.frac, h));
            } else if (nn < B.lo_n) {
                h = xadd(h, xmul(B.frac, h));
            } else {
                ok = true;
                break;
            }
            if (++it > B.max_iter) done = true;
        }
        if (!ok && !done && !again) {
            B.hc[i] = h * B.grow;  // h passed the radius: search again, wider
            again = true;
        }
    }
    if (again) status_add(A.status, SPH_S_H_RETRY, 1);
    again = again && !B.last_round;
    B.retry[i] = again ? 1 : 0;
    if (!ok && !again) status_add(A.status, SPH_S_H_NOCONV, 1);
    B.iters[i] = it;
    B.h_out[i] = h;
    A.p0[i].w = h;
}

// candidate search + count iteration for the flagged particles of each group
__global__ void __launch_bounds__(SEARCH_WARPS * 32, 8)
    k_cand_count(const int *__restrict__ ngroup_p, SearchArgs A, CountArgs B, unsigned *queue) {
    __shared__ SearchSmem smem[SEARCH_WARPS];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int ngroup = *ngroup_p;
    for (int g = q_first(queue, blockIdx.x * SEARCH_WARPS + w); g < ngroup;
         g = q_next(queue, g, gridDim.x * SEARCH_WARPS)) {
        const int s0 = A.gstart[g], gc = A.gcount[g];
        bool act = lane < gc;
        const int i = s0 + (act ? lane : 0);
        act = act && B.retry[i];
        if (!__ballot_sync(FULL, act)) continue;
        const double4 pi = A.p0[i];
        group_search<2, double>(smem[w], A, g, act, i, pi, 2.0 * B.hc[i]);
        if (act) count_lane(A, B, i, pi, A.cidx + (size_t)i * A.K);
        __syncwarp();
    }
}

// Half the k-th smallest distance (self at index 0) of the particle of one
// lane (smoothing_length_mpi, MPI_sph/sph_code/libsx.py:777-800: np.sort(dist)
// [50] / 2).  With a complete row (every j with d_j <= 2 hc) holding at least
// k + 1 entries, the k-th smallest distance overall is the row's; it is found
// by bisection over the bit patterns of the row's distances (non-negative
// doubles order like their patterns), so the value is one of the distances,
// rounded as the reference computes them.  A row with too few entries widens
// the radius, one that overflows narrows it, and the particle searches again.
__device__ __forceinline__ void kth_lane(const SearchArgs &A, const CountArgs &B, int i,
                                         const double4 &pi, const int *row, int k) {
    const int craw = A.cnt[i];
    const double cap = B.hc[i];
    bool again = false;
    if (craw > A.K) {
        B.hc[i] = cap * fmax(0.5, cbrt(0.75 * A.K / (double)craw));
        again = true;
    } else if (craw < k + 1) {
        B.hc[i] = cap * (craw > 0 ? fmin(2.0, fmax(1.1, cbrt(1.5 * (k + 1) / (double)craw))) : 2.0);
        again = true;
    } else {
        // every row entry lies within 2 cap up to the rounding of the
        // search's r^2 test; hi bounds them all
        unsigned long long lo = 0,
                           hi = (unsigned long long)__double_as_longlong(2.0 * cap * (1.0 + 1e-9));
        for (int it = 0; it < 64 && lo < hi; it++) {
            const unsigned long long mid = lo + (hi - lo) / 2;
            const double v = __longlong_as_double((long long)mid);
            int c = 0;
            for (int q = 0; q < craw; q++) c += ref_dist(pi, A.p0[row[q]]) <= v;
            if (c >= k + 1) hi = mid;
            else lo = mid + 1;
        }
        const double d = __longlong_as_double((long long)lo);
        if (d > 2.0 * cap * (1.0 - 1e-12)) {
            // at the radius itself a particle outside the row could be nearer
            // by a rounding: search again, wider
            B.hc[i] = cap * 1.1;
            again = true;
        } else {
            B.h_out[i] = 0.5 * d;
            A.p0[i].w = 0.5 * d;
        }
    }
    if (again) status_add(A.status, SPH_S_H_RETRY, 1);
    const bool retry = again && !B.last_round;
    B.retry[i] = retry ? 1 : 0;
    if (again && !retry) status_add(A.status, SPH_S_H_NOCONV, 1);
}

__global__ void __launch_bounds__(SEARCH_WARPS * 32, 8)
    k_cand_kth(const int *__restrict__ ngroup_p, SearchArgs A, CountArgs B, int k, unsigned *queue) {
    __shared__ SearchSmem smem[SEARCH_WARPS];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int ngroup = *ngroup_p;
    for (int g = q_first(queue, blockIdx.x * SEARCH_WARPS + w); g < ngroup;
         g = q_next(queue, g, gridDim.x * SEARCH_WARPS)) {
        const int s0 = A.gstart[g], gc = A.gcount[g];
        bool act = lane < gc;
        const int i = s0 + (act ? lane : 0);
        act = act && B.retry[i];
        if (!__ballot_sync(FULL, act)) continue;
        const double4 pi = A.p0[i];
        group_search<2, double>(smem[w], A, g, act, i, pi, 2.0 * B.hc[i]);
        if (act) kth_lane(A, B, i, pi, A.cidx + (size_t)i * A.K, k);
        __syncwarp();
    }
}

__global__ void k_zero_int(int n, int *__restrict__ a) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) a[i] = 0;
}

// canonical CSR export, each row sorted ascending
__global__ void k_export(int n, const int *__restrict__ rows, const int *__restrict__ cnt, int K,
                         const long long *__restrict__ off, int *__restrict__ lst) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int c = cnt[i];
    int *o = lst + off[i];
    for (int k = 0; k < c; k++) {
        int v = rows[(size_t)i * K + k];
        int p = k;
        while (p > 0 && o[p - 1] > v) {
            o[p] = o[p - 1];
            p--;
        }
        o[p] = v;
    }
}

SearchArgs search_args(sph_ctx *ctx, int *rows, int *cnt) {
    SearchArgs A;
    A.gstart = ctx->gstart;
    A.gcount = ctx->gcount;
    A.gcloud = ctx->groot_g;
    A.croot = ctx->croot;
    A.p0 = ctx->p0;
    A.sA = (const float4 *)ctx->node_box;
    A.sB = A.sA + 2 * (size_t)ctx->cfg.n_max;
    A.wL = ctx->wL;
    A.leaf_size = ctx->cfg.leaf_size;
    A.K = ctx->cfg.max_ngb;
    A.rows = rows;
    A.cnt = cnt;
    A.cidx = ctx->cand_idx;
    A.ngb_cnt = ctx->ngb_cnt;
    A.hnb = ctx->st[ctx->cur][ST_HNB];
    A.only = nullptr;
    A.only_all = nullptr;
    A.mlist = nullptr;
    A.mcount = nullptr;
    A.p1 = ctx->p1;
    A.status = ctx->status;
    return A;
}

}  // namespace

// margin of the step's first candidate radius over h: h may grow by this
// factor inside the first search round before the particle is searched again
#ifndef SPH_H_GROW
#define SPH_H_GROW 1.05
#endif
static const double H_GROW = SPH_H_GROW;
// the wider margin of a repeated search (a few particles per step), so that
// the step's four rounds follow a growth of h by 1.05 x 1.25^3 = 2.05
static const double H_REGROW = 1.25;
// the margin of the count and k-th iterations, whose round counts are sized
// for it
static const double H_GROW_COUNT = 1.08;

int launch_smoothing_h(sph_ctx *ctx) {
    const int n = ctx->n;
    if (n <= 0) return SPH_OK;
    cudaStream_t s = ctx->stream;
    const int c = ctx->cur;
    // rows kept from the last h iteration when they can be: decided per
    // particle and group on the device; the host only knows whether to try
    const bool reuse = ctx->rows_host && !(ctx->cfg.flags & SPH_FLAG_NO_ROW_REUSE);
    ReuseArgs U;
    U.on = reuse ? 1 : 0;
    U.rows_ok = ctx->rows_ok;
    U.hsr = ctx->hsr;
    U.dmv = ctx->dmv;
    U.dmv_max = ctx->dmv_max;
    U.cloud = ctx->cloud[c];
    U.kept = ctx->kept_cnt;
    k_kept_shift<<<1, 1, 0, s>>>(ctx->kept_cnt);
    ctx->kept_counted = true;
    k_h_init<<<div_up(n, 256), 256, 0, s>>>(n, ctx->st[c][ST_H], ctx->st[c][ST_HNB], ctx->hcand,
                                            ctx->retry, H_GROW, ctx->hover, U);
    if (reuse)
        k_group_moved<<<ctx->num_sms * 4, 256, 0, s>>>(ctx->d_ngroup, ctx->gstart, ctx->gcount,
                                                       ctx->dmv, ctx->gdm);
    const int rounds = ctx->prologue_done ? 4 : 8;
    const int grid = max(1, div_up(div_up(n, 16) + ctx->ncloud, SEARCH_WARPS));
    SearchArgs A = search_args(ctx, nullptr, ctx->cand_cnt);
    NewtonArgs B;
    B.p1 = ctx->p1;
    B.h_out = ctx->st[c][ST_H];
    B.hc = ctx->hcand;
    B.hover = ctx->hover;
    B.hsr = ctx->hsr;
    B.hnb = ctx->st[c][ST_HNB];
    B.dmv = ctx->dmv;
    B.gdm = ctx->gdm;
    B.kept = ctx->kept_cnt;
    B.retry = ctx->retry;
    B.n_ngb = ctx->cfg.n_ngb;
    B.tol = ctx->cfg.h_tol;
    B.grow = H_GROW;
    B.regrow = H_REGROW;
    B.max_iter = ctx->cfg.h_max_iter;
    const bool mixed = ctx->cfg.precision == SPH_PREC_MIXED;
    const void *kern = mixed ? (const void *)k_cand_newton<float> : (const void *)k_cand_newton<double>;
    for (int r = 0; r < rounds; r++) {
        B.last_round = r == rounds - 1;
        int g;
        unsigned *q;
        int rc = queue_launch(ctx, s, WQ_SEARCH, kern, SEARCH_WARPS * 32, grid, &g, &q);
        if (rc) return rc;
        if (r > 0) {
            // the later rounds search again only for the few particles whose
            // h left the candidate radius: a fixed stride over the groups,
            // which most warps skip after one ballot, costs less than one
            // work-queue atomic per group (the first round keeps the queue:
            // after kept rows its share of searched groups ranges from none
            // to all)
            g = min(grid, ctx->num_sms * 8);
            q = nullptr;
        }
        if (mixed)
            k_cand_newton<float><<<g, SEARCH_WARPS * 32, 0, s>>>(ctx->d_ngroup, A, B, q);
        else
            k_cand_newton<double><<<g, SEARCH_WARPS * 32, 0, s>>>(ctx->d_ngroup, A, B, q);
    }
    // every row now lists the candidates of its hsr (or is marked incomplete)
    CK(cudaMemsetAsync(ctx->rows_ok, 1, sizeof(int), s));
    ctx->rows_host = true;
    ctx->lists_ok = false;
    ctx->cand_ok = true;
    return ctx_check_launch(ctx, "smoothing_h");
}

int launch_smoothing_h_count(sph_ctx *ctx, int n_target, int n_tol, double frac, int max_iter) {
    const int n = ctx->n;
    if (n <= 0) return SPH_OK;
    cudaStream_t s = ctx->stream;
    const int c = ctx->cur;
    // these iterations write the rows without their search radii
    int rc0 = launch_rows_invalidate(ctx);
    if (rc0) return rc0;
    ctx->kept_counted = false;
    k_h_init<<<div_up(n, 256), 256, 0, s>>>(n, ctx->st[c][ST_H], ctx->st[c][ST_HNB], ctx->hcand,
                                            ctx->retry, H_GROW_COUNT, nullptr, ReuseArgs{});
    k_zero_int<<<div_up(n, 256), 256, 0, s>>>(n, ctx->hiter);
    // each round widens the radius by H_GROW_COUNT; 0.3 % steps need about 26
    // iterations for that, so 16 rounds cover a 3.4x change of h
    const int rounds = 16;
    const int grid = max(1, div_up(div_up(n, 16) + ctx->ncloud, SEARCH_WARPS));
    SearchArgs A = search_args(ctx, nullptr, ctx->cand_cnt);
    CountArgs B;
    B.h_out = ctx->st[c][ST_H];
    B.hc = ctx->hcand;
    B.retry = ctx->retry;
    B.iters = ctx->hiter;
    B.lo_n = n_target - n_tol;
    B.hi_n = n_target + n_tol;
    B.max_iter = max_iter;
    B.frac = frac;
    B.grow = H_GROW_COUNT;
    for (int r = 0; r < rounds; r++) {
        B.last_round = r == rounds - 1;
        int g;
        unsigned *q;
        int rc = queue_launch(ctx, s, WQ_SEARCH, (const void *)k_cand_count, SEARCH_WARPS * 32,
                              grid, &g, &q);
        if (rc) return rc;
        k_cand_count<<<g, SEARCH_WARPS * 32, 0, s>>>(ctx->d_ngroup, A, B, q);
    }
    ctx->lists_ok = false;
    ctx->cand_ok = true;
    ctx->p2_dirty = true;
    return ctx_check_launch(ctx, "smoothing_h_count");
}

// h = half the k-th neighbour distance, the search radius started from the
// current h
int launch_smoothing_kth(sph_ctx *ctx, int k) {
    const int n = ctx->n;
    if (n <= 0) return SPH_OK;
    cudaStream_t s = ctx->stream;
    const int c = ctx->cur;
    // these iterations write the rows without their search radii
    int rc0 = launch_rows_invalidate(ctx);
    if (rc0) return rc0;
    ctx->kept_counted = false;
    k_h_init<<<div_up(n, 256), 256, 0, s>>>(n, ctx->st[c][ST_H], ctx->st[c][ST_HNB], ctx->hcand,
                                            ctx->retry, H_GROW_COUNT, nullptr, ReuseArgs{});
    const int grid = max(1, div_up(div_up(n, 16) + ctx->ncloud, SEARCH_WARPS));
    SearchArgs A = search_args(ctx, nullptr, ctx->cand_cnt);
    CountArgs B{};
    B.h_out = ctx->st[c][ST_H];
    B.hc = ctx->hcand;
    B.retry = ctx->retry;
    B.iters = ctx->hiter;
    B.grow = H_GROW_COUNT;
    const int rounds = 24;
    for (int r = 0; r < rounds; r++) {
        B.last_round = r == rounds - 1;
        int g;
        unsigned *q;
        int rc = queue_launch(ctx, s, WQ_SEARCH, (const void *)k_cand_kth, SEARCH_WARPS * 32, grid, &g, &q);
        if (rc) return rc;
        k_cand_kth<<<g, SEARCH_WARPS * 32, 0, s>>>(ctx->d_ngroup, A, B, k, q);
    }
    ctx->lists_ok = false;
    ctx->cand_ok = false;  // the rows are candidate sets of the search radius, not of h
    ctx->p2_dirty = true;
    return ctx_check_launch(ctx, "smoothing_kth");
}

int launch_neighbours(sph_ctx *ctx) {
    const int n = ctx->n;
    if (n <= 0) return SPH_OK;
    cudaStream_t s = ctx->stream;
    const int grid = max(1, div_up(div_up(n, 16) + ctx->ncloud, SEARCH_WARPS));
    SearchArgs A = search_args(ctx, ctx->ngb, ctx->ngb_cnt);
    if (ctx->cand_ok) {
        // lists from the candidate rows, then the tree search for the
        // particles whose rows cannot show that their list is complete
        CK(cudaMemsetAsync(ctx->lflag, 0, sizeof(int) * (n + 2), s));
        SearchArgs C = search_args(ctx, ctx->ngb, ctx->cand_cnt);
        k_lists_cand<<<grid, SEARCH_WARPS * 32, 0, s>>>(ctx->d_ngroup, C, ctx->hcand, ctx->lflag,
                                                       ctx->lflag + n, ctx->lflag + n + 1);
        A.only = ctx->lflag;
        A.only_all = ctx->lflag + n;
    }
    // node h_max only matters to the tree search: skipped when no list needs it
    int rc = launch_refit_hmax(ctx, ctx->cand_ok ? ctx->lflag + n + 1 : nullptr);
    if (rc) return rc;
    int g;
    unsigned *q;
    if ((rc = queue_launch(ctx, s, WQ_SEARCH, (const void *)k_lists, SEARCH_WARPS * 32, grid, &g, &q)))
        return rc;
    k_lists<<<g, SEARCH_WARPS * 32, 0, s>>>(ctx->d_ngroup, A, q);
    ctx->lists_ok = true;
    ctx->rho_ok = ctx->divcurl_ok = false;
    return ctx_check_launch(ctx, "neighbours");
}

// the tree search for the particles marked in ctx->lflag (all of them when
// lflag[n] is set), after the node h_max refit (skipped when nothing is marked)
int launch_lists_marked(sph_ctx *ctx) {
    const int n = ctx->n;
    if (n <= 0) return SPH_OK;
    const int grid = max(1, div_up(div_up(n, 16) + ctx->ncloud, SEARCH_WARPS));
    SearchArgs A = search_args(ctx, ctx->ngb, ctx->ngb_cnt);
    A.only = ctx->lflag;
    A.only_all = ctx->lflag + n;
    A.mlist = ctx->mlist;
    A.mcount = ctx->lflag + n + 2;
    int rc = launch_refit_hmax(ctx, ctx->lflag + n + 1);
    if (rc) return rc;
    int g;
    unsigned *q;
    if ((rc = queue_launch(ctx, ctx->stream, WQ_SEARCH, (const void *)k_lists, SEARCH_WARPS * 32,
                           grid, &g, &q)))
        return rc;
    k_lists<<<g, SEARCH_WARPS * 32, 0, ctx->stream>>>(ctx->d_ngroup, A, q);
    k_lists_list<<<ctx->num_sms * 2, SEARCH_WARPS * 32, 0, ctx->stream>>>(ctx->d_ngroup, A);
    return ctx_check_launch(ctx, "lists_marked");
}

int launch_export_neighbours(sph_ctx *ctx, int64_t *off_dev, int *lst_dev, int64_t cap) {
    (void)cap;
    const int n = ctx->n;
    if (n <= 0) return SPH_OK;
    k_export<<<div_up(n, 128), 128, 0, ctx->stream>>>(n, ctx->ngb, ctx->ngb_cnt, ctx->cfg.max_ngb,
                                                       (const long long *)off_dev, lst_dev);
    return ctx_check_launch(ctx, "export_neighbours");
}
