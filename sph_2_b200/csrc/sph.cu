// sph.cu -- the neighbour-sum passes: density (+ EOS), div/curl (+ Balsara
// factor), pressure/viscous acceleration with the signal velocity, du/dt.
//
// Replaces getDensity_ngb / getPressure_Adiabatic / getCsound_Adiabatic /
// div_curlVel_ngb / acc_sph_ngb / get_dU_ngb (hfvCLibs_v7_hfv_v2.h:474-916),
// each a thread per particle looping over a -1 padded row of 200 int slots
// with uncoalesced float loads, and the all-pairs numba loops of
// MPI_sph/sph_code/libsx.py:52-262 and shear.py:78-485 (same formulas).
//
// Mapping: LANES consecutive lanes own one particle (LANES = ngb_lanes, the
// "neighbour chunk width", 4..32).  They read that particle's row of the
// neighbour list contiguously and gather the neighbours' packed records
// (p0 = double4 x,y,z,h; p1 = Real4 v,m; p2 = Real4 rho,P/rho^2,c,f); rows are
// spatially local in Morton order so the gathers mostly hit L1/L2.  Partial
// sums are Kahan-compensated in FP32 (mixed) and reduced across the lanes in
// FP64.  Coordinate differences are always taken in FP64.
#include <type_traits>

#include "sph_internal.cuh"

// resident 256-thread blocks per SM asked of the FP32 list + density and
// force passes (register budget: 65536 / (256 x this)).  The force pass is
// gather-latency bound: 48 registers (5) run it 3 % faster than 58, 40 (6)
// spill; the list pass spills at 48
#ifndef SPH_LISTS_MINB
#define SPH_LISTS_MINB 1
#endif
#ifndef SPH_FORCE_MINB
#define SPH_FORCE_MINB 5
#endif

namespace {

template <class R, int LANES>
__global__ void __launch_bounds__(256)
    k_density(int n, const double4 *__restrict__ p0, const typename R4<R>::T *__restrict__ p1,
              typename R4<R>::T *__restrict__ p2, const int *__restrict__ rows,
              const int *__restrict__ cnt, int K, const double *__restrict__ u, double gamma,
              double *__restrict__ rho_out, double *__restrict__ P_out, double *__restrict__ c_out) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int i = (int)(t / LANES), sl = (int)(t % LANES);
    const bool valid = i < n;
    KSum<R> S;
    if (valid) {
        const double4 pi = p0[i];
        const int c = cnt[i];
        const int *row = rows + (size_t)i * K;
        for (int k = sl; k < c; k += LANES) {
            const int j = row[k];
            const double4 pj = p0[j];
            const R mj = p1[j].w;
            const R dx = (R)(pi.x - pj.x), dy = (R)(pi.y - pj.y), dz = (R)(pi.z - pj.z);
            const R rr = qsqrt<R>(dx * dx + dy * dy + dz * dz);
            const R hij = (R)(0.5 * (pi.w + pj.w));
            const R inv = qdiv<R>(R(1), hij);
            S.add(mj * kern_w<R>(rr * inv, inv * inv * inv));
        }
    }
    const double rho = seg_sum<LANES>(S.value());
    if (valid && sl == 0) {
        const double ui = u[i];
        const double P = (gamma - 1.0) * rho * ui;
        const double cs = sqrt(gamma * (gamma - 1.0) * ui);
        rho_out[i] = rho;
        P_out[i] = P;
        c_out[i] = cs;
        typename R4<R>::T q = p2[i];
        q.x = (R)rho;
        q.y = (R)(P / (rho * rho));
        q.z = (R)cs;
        p2[i] = q;
    }
}

template <class R, int LANES>
__global__ void __launch_bounds__(256)
    k_divcurl(int n, const double4 *__restrict__ p0, const typename R4<R>::T *__restrict__ p1,
              typename R4<R>::T *__restrict__ p2, const int *__restrict__ rows,
              const int *__restrict__ cnt, int K, const double *__restrict__ rho,
              const double *__restrict__ csnd, int balsara, double *__restrict__ divV,
              double *__restrict__ curlV) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int i = (int)(t / LANES), sl = (int)(t % LANES);
    const bool valid = i < n;
    KSum<R> s, cx, cy, cz;
    if (valid) {
        const double4 pi = p0[i];
        const typename R4<R>::T vi = p1[i];
        const int c = cnt[i];
        const int *row = rows + (size_t)i * K;
        for (int k = sl; k < c; k += LANES) {
            const int j = row[k];
            const double4 pj = p0[j];
            const typename R4<R>::T vj = p1[j];
            const R dx = (R)(pi.x - pj.x), dy = (R)(pi.y - pj.y), dz = (R)(pi.z - pj.z);
            const R rr = qsqrt<R>(dx * dx + dy * dy + dz * dz);
            const R hij = (R)(0.5 * (pi.w + pj.w));
            const R inv = qdiv<R>(R(1), hij);
            const R i2 = inv * inv;
            const R nW = kern_nw<R>(rr * inv, i2 * i2 * inv);
            const R gx = nW * dx, gy = nW * dy, gz = nW * dz;
            const R ux = vi.x - vj.x, uy = vi.y - vj.y, uz = vi.z - vj.z;
            const R mj = vj.w;
            s.add(-mj * (ux * gx + uy * gy + uz * gz));
            cx.add(mj * (uy * gz - uz * gy));
            cy.add(mj * (uz * gx - ux * gz));
            cz.add(mj * (ux * gy - uy * gx));
        }
    }
    const double S = seg_sum<LANES>(s.value());
    const double X = seg_sum<LANES>(cx.value()), Y = seg_sum<LANES>(cy.value()),
                 Z = seg_sum<LANES>(cz.value());
    if (valid && sl == 0) {
        const double inv_rho = 1.0 / rho[i];
        const double d = fabs(S * inv_rho);
        const double cv = sqrt(X * X + Y * Y + Z * Z) * inv_rho;
        divV[i] = d;
        curlV[i] = cv;
        typename R4<R>::T q = p2[i];
        q.w = balsara ? (R)(d / (d + cv + 0.0001 * csnd[i] / p0[i].w)) : R(0);
        p2[i] = q;
    }
}

// density, EOS, div v, |curl v| and the Balsara factor in one pass: the
// div/curl sums need only the particle's own density (sum m_j/rho_i ...), so
// they are accumulated unnormalised beside the density sum and divided by
// rho_i at the end
// density, EOS, div v, |curl v| and the packed p2 record of particle i from
// its list, on the LANES lanes of its segment (every lane of the warp calls:
// the segment sums are warp collectives; valid false: no particle)
template <class R, int LANES>
__device__ __forceinline__ void density_divcurl_one(
    bool valid, int i, int sl, const double4 *__restrict__ p0,
    const typename R4<R>::T *__restrict__ p1, typename R4<R>::T *__restrict__ p2,
    const int *__restrict__ rows, const int *__restrict__ cnt, int K, const double *__restrict__ u,
    double gamma, int balsara, double *__restrict__ rho_out, double *__restrict__ P_out,
    double *__restrict__ c_out, double *__restrict__ divV, double *__restrict__ curlV) {
    KSum<R> S, s, cx, cy, cz;
    double hi = 1.0;
    if (valid) {
        const double4 pi = p0[i];
        hi = pi.w;
        const typename R4<R>::T vi = p1[i];
        const int c = cnt[i];
        const int *row = rows + (size_t)i * K;
        for (int k = sl; k < c; k += LANES) {
            const int j = row[k];
            const double4 pj = p0[j];
            const typename R4<R>::T vj = p1[j];
            const R dx = (R)(pi.x - pj.x), dy = (R)(pi.y - pj.y), dz = (R)(pi.z - pj.z);
            const R rr = qsqrt<R>(dx * dx + dy * dy + dz * dz);
            const R hij = (R)(0.5 * (pi.w + pj.w));
            const R inv = qdiv<R>(R(1), hij);
            const R i2 = inv * inv;
            const R q = rr * inv;
            const R mj = vj.w;
            S.add(mj * kern_w<R>(q, i2 * inv));
            const R nW = kern_nw<R>(q, i2 * i2 * inv);
            const R gx = nW * dx, gy = nW * dy, gz = nW * dz;
            const R ux = vi.x - vj.x, uy = vi.y - vj.y, uz = vi.z - vj.z;
            s.add(-mj * (ux * gx + uy * gy + uz * gz));
            cx.add(mj * (uy * gz - uz * gy));
            cy.add(mj * (uz * gx - ux * gz));
            cz.add(mj * (ux * gy - uy * gx));
        }
    }
    const double rho = seg_sum<LANES>(S.value());
    const double Sd = seg_sum<LANES>(s.value());
    const double X = seg_sum<LANES>(cx.value()), Y = seg_sum<LANES>(cy.value()),
                 Z = seg_sum<LANES>(cz.value());
    if (valid && sl == 0) {
        const double ui = u[i];
        const double P = (gamma - 1.0) * rho * ui;
        const double cs = sqrt(gamma * (gamma - 1.0) * ui);
        const double inv_rho = 1.0 / rho;
        const double d = fabs(Sd * inv_rho);
        const double cv = sqrt(X * X + Y * Y + Z * Z) * inv_rho;
        rho_out[i] = rho;
        P_out[i] = P;
        c_out[i] = cs;
        divV[i] = d;
        curlV[i] = cv;
        typename R4<R>::T q;
        q.x = (R)rho;
        q.y = (R)(P / (rho * rho));
        q.z = (R)cs;
        q.w = balsara ? (R)(d / (d + cv + 0.0001 * cs / hi)) : R(0);
        p2[i] = q;
    }
}

template <class R, int LANES>
__global__ void __launch_bounds__(256)
    k_density_divcurl(int n, const double4 *__restrict__ p0,
                      const typename R4<R>::T *__restrict__ p1, typename R4<R>::T *__restrict__ p2,
                      const int *__restrict__ rows, const int *__restrict__ cnt, int K,
                      const double *__restrict__ u, double gamma, int balsara,
                      double *__restrict__ rho_out, double *__restrict__ P_out,
                      double *__restrict__ c_out, double *__restrict__ divV,
                      double *__restrict__ curlV) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int i = (int)(t / LANES), sl = (int)(t % LANES);
    density_divcurl_one<R, LANES>(i < n, i, sl, p0, p1, p2, rows, cnt, K, u, gamma, balsara,
                                  rho_out, P_out, c_out, divV, curlV);
}

// The same for the particles the fused list pass sent to the tree search:
// the *mcount entries of mlist, or every particle when *all is set; a grid
// of a few blocks per SM strides over them, so a step that marks a hundred
// particles does not launch a thread per particle
template <class R, int LANES>
__global__ void __launch_bounds__(256)
    k_density_divcurl_list(int n, const int *__restrict__ mlist, const int *__restrict__ mcount,
                           const int *__restrict__ all, const double4 *__restrict__ p0,
                           const typename R4<R>::T *__restrict__ p1,
                           typename R4<R>::T *__restrict__ p2, const int *__restrict__ rows,
                           const int *__restrict__ cnt, int K, const double *__restrict__ u,
                           double gamma, int balsara, double *__restrict__ rho_out,
                           double *__restrict__ P_out, double *__restrict__ c_out,
                           double *__restrict__ divV, double *__restrict__ curlV) {
    const bool every = *all != 0;
    const int m = every ? n : *mcount;
    const long long stride = (long long)gridDim.x * blockDim.x;
    // the trip count is the same for every thread (the segment sums need
    // the whole warp)
    for (long long base = 0; base < (long long)m * LANES; base += stride) {
        const long long t = base + (long long)blockIdx.x * blockDim.x + threadIdx.x;
        const int e = (int)(t / LANES), sl = (int)(t % LANES);
        const bool ok = e < m;
        const int i = ok ? (every ? e : mlist[e]) : 0;
        density_divcurl_one<R, LANES>(ok, i, sl, p0, p1, p2, rows, cnt, K, u, gamma, balsara,
                                      rho_out, P_out, c_out, divV, curlV);
    }
}

// The exact lists and the density pass in one: each particle's LANES lanes
// walk its candidate row from the h iteration (rows i K .. i K + ccnt - 1),
// keep the pairs with |r| <= h_i + h_j (the FP64 predicate of the tree
// search), write them to the list row in candidate order (a segment ballot
// per round of LANES entries) and add their density, div and curl terms.  The
// list of a particle is complete from its own row unless a partner j with the
// larger h held it in its row only: such a j (|r| beyond 2 hc_j, with a margin
// for rounding) is marked for the tree search and its density recomputed
// from that list; a row that is not a complete candidate set (overflow, or h
// above the candidate radius) marks every particle.
template <class R, int LANES>
__global__ void __launch_bounds__(256, std::is_same<R, float>::value ? SPH_LISTS_MINB : 1)
    k_cand_density_divcurl(int n, const double4 *__restrict__ p0,
                           const typename R4<R>::T *__restrict__ p1,
                           typename R4<R>::T *__restrict__ p2, const int *__restrict__ crows,
                           const int *__restrict__ ccnt, const double *__restrict__ hc, int K,
                           int *__restrict__ rows, int *__restrict__ cnt, double *__restrict__ hnb,
                           int *__restrict__ full, int *__restrict__ full_all,
                           int *__restrict__ full_any, int *__restrict__ mlist,
                           int *__restrict__ mcount, long long *status,
                           const double *__restrict__ u, double gamma, int balsara,
                           double *__restrict__ rho_out, double *__restrict__ P_out,
                           double *__restrict__ c_out, double *__restrict__ divV,
                           double *__restrict__ curlV) {
    typedef typename R4<R>::T V4;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int i = (int)(t / LANES), sl = (int)(t % LANES);
    const int lane = threadIdx.x & 31;
    const unsigned seg = LANES == 32 ? 0xffffffffu : (((1u << LANES) - 1u) << (lane & ~(LANES - 1)));
    const unsigned below = (1u << lane) - 1u;
    const bool valid = i < n;
    KSum<R> S, s, cx, cy, cz;
    double hi = 1.0, hmx = 0.0;
    int craw = 0;
    double4 pi = make_double4(0.0, 0.0, 0.0, 1.0);
    V4 vi;
    vi.x = vi.y = vi.z = vi.w = R(0);
    if (valid) {
        pi = p0[i];
        hi = pi.w;
        vi = p1[i];
        craw = ccnt[i];
        if (!(craw <= K && pi.w <= hc[i])) {
            if (sl == 0) {
                *full_all = 1;
                *full_any = 1;
            }
            craw = 0;
        }
    }
    // one trip count for the warp: the segment ballot needs every lane
    int kmax = craw;
    for (int o = 16; o; o >>= 1) kmax = max(kmax, __shfl_xor_sync(0xffffffffu, kmax, o));
    const int *crow = crows + (size_t)(valid ? i : 0) * K;
    int count = 0;
    for (int k0 = 0; k0 < kmax; k0 += LANES) {
        const int k = k0 + sl;
        bool hit = false;
        int j = 0;
        double4 pj = pi;
        if (k < craw) {
            j = crow[k];
            pj = p0[j];
            hit = ngb_pred(pi.x, pi.y, pi.z, pi.w, pj.x, pj.y, pj.z, pj.w);
        }
        const unsigned m = __ballot_sync(0xffffffffu, hit) & seg;
        if (hit) {
            const int pos = count + __popc(m & below);
            if (pos < K) rows[(size_t)i * K + pos] = j;
            const V4 vj = p1[j];
            const R dx = (R)(pi.x - pj.x), dy = (R)(pi.y - pj.y), dz = (R)(pi.z - pj.z);
            const R rr = qsqrt<R>(dx * dx + dy * dy + dz * dz);
            const R hij = (R)(0.5 * (pi.w + pj.w));
            const R inv = qdiv<R>(R(1), hij);
            const R i2 = inv * inv;
            const R q = rr * inv;
            const R mj = vj.w;
            S.add(mj * kern_w<R>(q, i2 * inv));
            const R nW = kern_nw<R>(q, i2 * i2 * inv);
            const R gx = nW * dx, gy = nW * dy, gz = nW * dz;
            const R ux = vi.x - vj.x, uy = vi.y - vj.y, uz = vi.z - vj.z;
            s.add(-mj * (ux * gx + uy * gy + uz * gz));
            cx.add(mj * (uy * gz - uz * gy));
            cy.add(mj * (uz * gx - ux * gz));
            cz.add(mj * (ux * gy - uy * gx));
            hmx = fmax(hmx, pj.w);
            const double ex = pi.x - pj.x, ey = pi.y - pj.y, ez = pi.z - pj.z;
            const double rj = 2.0 * hc[j];
            if (ex * ex + ey * ey + ez * ez > rj * rj * (1.0 - 1e-9)) {
                // j joins the list of particles to search once
                if (atomicExch(&full[j], 1) == 0) mlist[atomicAdd(mcount, 1)] = j;
                *full_any = 1;
            }
        }
        count += __popc(m);
    }
    const double rho = seg_sum<LANES>(S.value());
    const double Sd = seg_sum<LANES>(s.value());
    const double X = seg_sum<LANES>(cx.value()), Y = seg_sum<LANES>(cy.value()),
                 Z = seg_sum<LANES>(cz.value());
    hmx = seg_max<LANES>(hmx);
    if (valid && sl == 0) {
        cnt[i] = min(count, K);
        if (count > K) status_add(status, SPH_S_NGB_OVERFLOW, 1);
        hnb[i] = hmx;
        const double ui = u[i];
        const double P = (gamma - 1.0) * rho * ui;
        const double cs = sqrt(gamma * (gamma - 1.0) * ui);
        const double inv_rho = 1.0 / rho;
        const double d = fabs(Sd * inv_rho);
        const double cv = sqrt(X * X + Y * Y + Z * Z) * inv_rho;
        rho_out[i] = rho;
        P_out[i] = P;
        c_out[i] = cs;
        divV[i] = d;
        curlV[i] = cv;
        typename R4<R>::T qq;
        qq.x = (R)rho;
        qq.y = (R)(P / (rho * rho));
        qq.z = (R)cs;
        qq.w = balsara ? (R)(d / (d + cv + 0.0001 * cs / hi)) : R(0);
        p2[i] = qq;
    }
}

// acc_i = -sum m_j (P_i/rho_i^2 + P_j/rho_j^2 + PI_ij) gradW_ij,
// du_i  =  sum m_j (P_i/rho_i^2 + PI_ij/2) v_ij . gradW_ij,
// vsig_i = max_j (c_i + c_j - 3 w_ij), w_ij = v_ij.r_ij/(r_ij + 1e-5).
template <class R, int LANES>
__global__ void __launch_bounds__(256, std::is_same<R, float>::value ? SPH_FORCE_MINB : 1)
    k_force(int n, const double4 *__restrict__ p0, const typename R4<R>::T *__restrict__ p1,
            const typename R4<R>::T *__restrict__ p2, const int *__restrict__ rows,
            const int *__restrict__ cnt, int K, int av_mode, int balsara, R alpha, R beta, R eta,
            int want_acc, int want_du, double *__restrict__ acc, double *__restrict__ dudt,
            double *__restrict__ vsig) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int i = (int)(t / LANES), sl = (int)(t % LANES);
    const bool valid = i < n;
    KSum<R> ax, ay, az, du;
    R vs = R(0);
    if (valid) {
        const double4 pi = p0[i];
        const typename R4<R>::T vi = p1[i], qi = p2[i];
        const int c = cnt[i];
        const int *row = rows + (size_t)i * K;
        const R eta2 = eta * eta;
        for (int k = sl; k < c; k += LANES) {
            const int j = row[k];
            const double4 pj = p0[j];
            const typename R4<R>::T vj = p1[j], qj = p2[j];
            const R dx = (R)(pi.x - pj.x), dy = (R)(pi.y - pj.y), dz = (R)(pi.z - pj.z);
            const R rr = qsqrt<R>(dx * dx + dy * dy + dz * dz);
            const R hij = (R)(0.5 * (pi.w + pj.w));
            const R inv = qdiv<R>(R(1), hij);
            const R i2 = inv * inv;
            const R nW = kern_nw<R>(rr * inv, i2 * i2 * inv);
            const R gx = nW * dx, gy = nW * dy, gz = nW * dz;
            const R ux = vi.x - vj.x, uy = vi.y - vj.y, uz = vi.z - vj.z;
            const R vr = ux * dx + uy * dy + uz * dz;
            const R w = qdiv<R>(vr, rr + R(1e-5));
            R PI = R(0);
            if (vr <= R(0)) {
                const R rhoij = R(0.5) * (qi.x + qj.x);
                if (av_mode == SPH_AV_MG83) {
                    const R cij = R(0.5) * (qi.z + qj.z);
                    const R mu = qdiv<R>(hij * vr, rr * rr + hij * hij * eta2);
                    PI = qdiv<R>(-alpha * cij * mu + beta * mu * mu, rhoij);
                } else {
                    const R sig = qi.z + qj.z - R(3) * w;
                    PI = qdiv<R>(R(-0.5) * alpha * sig * w, rhoij);
                }
            }
            if (balsara) PI = R(0.5) * (qi.w + qj.w) * PI;
            const R mj = vj.w;
            if (want_acc) {
                const R tt = mj * (qi.y + qj.y + PI);
                ax.add(-tt * gx);
                ay.add(-tt * gy);
                az.add(-tt * gz);
                vs = fmax(vs, qi.z + qj.z - R(3) * w);
            }
            if (want_du) du.add(mj * (qi.y + R(0.5) * PI) * (ux * gx + uy * gy + uz * gz));
        }
    }
    if (want_acc) {
        const double X = seg_sum<LANES>(ax.value()), Y = seg_sum<LANES>(ay.value()),
                     Z = seg_sum<LANES>(az.value());
        const double V = seg_max<LANES>((double)vs);
        if (valid && sl == 0) {
            acc[i] = X;
            acc[(size_t)n + i] = Y;
            acc[2 * (size_t)n + i] = Z;
            vsig[i] = V;
        }
    }
    if (want_du) {
        const double D = seg_sum<LANES>(du.value());
        if (valid && sl == 0) dudt[i] = D;
    }
}

template <class R>
__global__ void k_repack_p2(int n, const double *__restrict__ rho, const double *__restrict__ P,
                            const double *__restrict__ c, const double *__restrict__ divV,
                            const double *__restrict__ curlV, const double4 *__restrict__ p0,
                            int balsara, typename R4<R>::T *__restrict__ p2) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    typename R4<R>::T q;
    const double r = rho[i];
    q.x = (R)r;
    q.y = (R)(P[i] / (r * r));
    q.z = (R)c[i];
    const double d = divV[i], cv = curlV[i];
    q.w = balsara ? (R)(d / (d + cv + 0.0001 * c[i] / p0[i].w)) : R(0);
    p2[i] = q;
}

template <class R>
__global__ void k_pack_p1(int n, const double *__restrict__ vx, const double *__restrict__ vy,
                          const double *__restrict__ vz, const double *__restrict__ m,
                          const double *__restrict__ x, const double *__restrict__ y,
                          const double *__restrict__ z, const double *__restrict__ h,
                          typename R4<R>::T *__restrict__ p1, typename R4<R>::T *__restrict__ pw,
                          double4 *__restrict__ p0, const int *__restrict__ cloud,
                          const double *__restrict__ corg, double *__restrict__ dmv,
                          unsigned long long *__restrict__ dmv_max) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (dmv) {
        // the move of the record since the last pack, added to the particle's
        // distance moved and to its cloud's largest (warp maximum first; the
        // valid lanes of a warp are a prefix, so lane 0 is one of them)
        const bool ok = i < n;
        unsigned long long bits = 0ull;
        int cl = -1;
        if (ok) {
            const double4 o = p0[i];
            const double dx = x[i] - o.x, dy = y[i] - o.y, dz = z[i] - o.z;
            // rounded up: a bound, not an estimate
            const double d = sqrt(dx * dx + dy * dy + dz * dz) * (1.0 + 1e-12);
            const double D = dmv[i] + d;
            dmv[i] = D;
            bits = (unsigned long long)__double_as_longlong(D);
            cl = cloud[i];
        }
        const int c0 = __shfl_sync(0xffffffffu, cl, 0);
        if (__all_sync(0xffffffffu, !ok || cl == c0)) {
#pragma unroll
            for (int o = 16; o; o >>= 1) {
                const unsigned long long t = __shfl_xor_sync(0xffffffffu, bits, o);
                bits = t > bits ? t : bits;
            }
            if ((threadIdx.x & 31) == 0 && c0 >= 0) atomicMax(&dmv_max[c0], bits);
        } else if (ok) {
            atomicMax(&dmv_max[cl], bits);
        }
    }
    if (i >= n) return;
    typename R4<R>::T a, b;
    a.x = (R)vx[i]; a.y = (R)vy[i]; a.z = (R)vz[i]; a.w = (R)m[i];
    const double *org = corg + 3 * cloud[i];
    b.x = (R)(x[i] - WalkOrigin<R>::off(org, 0));
    b.y = (R)(y[i] - WalkOrigin<R>::off(org, 1));
    b.z = (R)(z[i] - WalkOrigin<R>::off(org, 2));
    b.w = (R)m[i];
    p1[i] = a;
    pw[i] = b;
    p0[i] = make_double4(x[i], y[i], z[i], h[i]);
}

template <class R, int L>
int run_density(sph_ctx *ctx) {
    const int n = ctx->n, c = ctx->cur;
    const int bs = ctx->cfg.block_size;
    k_density<R, L><<<div_up((long long)n * L, bs), bs, 0, ctx->stream>>>(
        n, ctx->p0, (const typename R4<R>::T *)ctx->p1, (typename R4<R>::T *)ctx->p2, ctx->ngb,
        ctx->ngb_cnt, ctx->cfg.max_ngb, ctx->st[c][ST_U], ctx->cfg.gamma, ctx->rho, ctx->P, ctx->c);
    return SPH_OK;
}
template <class R, int L>
int run_density_divcurl(sph_ctx *ctx) {
    const int n = ctx->n, c = ctx->cur;
    const int bs = ctx->cfg.block_size;
    k_density_divcurl<R, L><<<div_up((long long)n * L, bs), bs, 0, ctx->stream>>>(
        n, ctx->p0, (const typename R4<R>::T *)ctx->p1, (typename R4<R>::T *)ctx->p2, ctx->ngb,
        ctx->ngb_cnt, ctx->cfg.max_ngb, ctx->st[c][ST_U], ctx->cfg.gamma, ctx->cfg.balsara,
        ctx->rho, ctx->P, ctx->c, ctx->divV, ctx->curlV);
    return SPH_OK;
}
template <class R, int L>
int run_density_divcurl_marked(sph_ctx *ctx) {
    const int n = ctx->n, c = ctx->cur;
    const int bs = ctx->cfg.block_size;
    k_density_divcurl_list<R, L><<<ctx->num_sms * 4, bs, 0, ctx->stream>>>(
        n, ctx->mlist, ctx->lflag + n + 2, ctx->lflag + n, ctx->p0,
        (const typename R4<R>::T *)ctx->p1, (typename R4<R>::T *)ctx->p2, ctx->ngb, ctx->ngb_cnt,
        ctx->cfg.max_ngb, ctx->st[c][ST_U], ctx->cfg.gamma, ctx->cfg.balsara, ctx->rho, ctx->P,
        ctx->c, ctx->divV, ctx->curlV);
    return SPH_OK;
}
template <class R, int L>
int run_cand_density_divcurl(sph_ctx *ctx) {
    const int n = ctx->n, c = ctx->cur;
    const int bs = ctx->cfg.block_size;
    k_cand_density_divcurl<R, L><<<div_up((long long)n * L, bs), bs, 0, ctx->stream>>>(
        n, ctx->p0, (const typename R4<R>::T *)ctx->p1, (typename R4<R>::T *)ctx->p2,
        ctx->cand_idx, ctx->cand_cnt, ctx->hcand, ctx->cfg.max_ngb, ctx->ngb, ctx->ngb_cnt,
        ctx->st[c][ST_HNB], ctx->lflag, ctx->lflag + n, ctx->lflag + n + 1, ctx->mlist,
        ctx->lflag + n + 2, ctx->status,
        ctx->st[c][ST_U], ctx->cfg.gamma, ctx->cfg.balsara, ctx->rho, ctx->P, ctx->c, ctx->divV,
        ctx->curlV);
    return SPH_OK;
}
template <class R, int L>
int run_divcurl(sph_ctx *ctx) {
    const int n = ctx->n;
    const int bs = ctx->cfg.block_size;
    k_divcurl<R, L><<<div_up((long long)n * L, bs), bs, 0, ctx->stream>>>(
        n, ctx->p0, (const typename R4<R>::T *)ctx->p1, (typename R4<R>::T *)ctx->p2, ctx->ngb,
        ctx->ngb_cnt, ctx->cfg.max_ngb, ctx->rho, ctx->c, ctx->cfg.balsara, ctx->divV, ctx->curlV);
    return SPH_OK;
}
template <class R, int L>
int run_force(sph_ctx *ctx, bool acc, bool du) {
    const int n = ctx->n;
    const int bs = ctx->cfg.block_size;
    k_force<R, L><<<div_up((long long)n * L, bs), bs, 0, ctx->stream>>>(
        n, ctx->p0, (const typename R4<R>::T *)ctx->p1, (const typename R4<R>::T *)ctx->p2,
        ctx->ngb, ctx->ngb_cnt, ctx->cfg.max_ngb, ctx->cfg.av_mode, ctx->cfg.balsara,
        (R)ctx->cfg.alpha, (R)ctx->cfg.beta, (R)ctx->cfg.eta, acc ? 1 : 0, du ? 1 : 0, ctx->asph,
        ctx->dudt, ctx->vsig);
    return SPH_OK;
}

#define SPH_DISPATCH_LANES(FN, R, ctx, ...)                 \
    switch ((ctx)->cfg.ngb_lanes) {                         \
        case 1: rc = FN<R, 1>(ctx, ##__VA_ARGS__); break;   \
        case 2: rc = FN<R, 2>(ctx, ##__VA_ARGS__); break;   \
        case 4: rc = FN<R, 4>(ctx, ##__VA_ARGS__); break;   \
        case 8: rc = FN<R, 8>(ctx, ##__VA_ARGS__); break;   \
        case 16: rc = FN<R, 16>(ctx, ##__VA_ARGS__); break; \
        default: rc = FN<R, 32>(ctx, ##__VA_ARGS__); break; \
    }

}  // namespace

int launch_density(sph_ctx *ctx) {
    if (ctx->n <= 0) return SPH_OK;
    int rc;
    if (ctx->cfg.precision == SPH_PREC_MIXED) { SPH_DISPATCH_LANES(run_density, float, ctx); }
    else { SPH_DISPATCH_LANES(run_density, double, ctx); }
    if (rc) return rc;
    ctx->rho_ok = true;
    return ctx_check_launch(ctx, "density");
}

// Exact lists + density + EOS + div/curl + Balsara from the h iteration's
// candidate rows (the step's path once smoothing_h has run): the fused pass,
// the tree search for the particles it marks, and their density recomputed
// from those lists.
int launch_lists_density(sph_ctx *ctx) {
    const int n = ctx->n;
    if (n <= 0) return SPH_OK;
    if (!ctx->cand_ok) return SPH_ERR_STATE;
    CK(cudaMemsetAsync(ctx->lflag, 0, sizeof(int) * (n + 3), ctx->stream));
    int rc;
    if (ctx->cfg.precision == SPH_PREC_MIXED) { SPH_DISPATCH_LANES(run_cand_density_divcurl, float, ctx); }
    else { SPH_DISPATCH_LANES(run_cand_density_divcurl, double, ctx); }
    if (rc) return rc;
    if ((rc = launch_lists_marked(ctx))) return rc;
    if (ctx->cfg.precision == SPH_PREC_MIXED) {
        SPH_DISPATCH_LANES(run_density_divcurl_marked, float, ctx);
    } else {
        SPH_DISPATCH_LANES(run_density_divcurl_marked, double, ctx);
    }
    if (rc) return rc;
    ctx->lists_ok = ctx->rho_ok = ctx->divcurl_ok = true;
    ctx->p2_dirty = false;
    return ctx_check_launch(ctx, "lists_density");
}

int launch_density_divcurl(sph_ctx *ctx) {
    if (ctx->n <= 0) return SPH_OK;
    int rc;
    if (ctx->cfg.precision == SPH_PREC_MIXED) { SPH_DISPATCH_LANES(run_density_divcurl, float, ctx); }
    else { SPH_DISPATCH_LANES(run_density_divcurl, double, ctx); }
    if (rc) return rc;
    ctx->rho_ok = ctx->divcurl_ok = true;
    ctx->p2_dirty = false;
    return ctx_check_launch(ctx, "density_divcurl");
}

int launch_divcurl(sph_ctx *ctx) {
    if (ctx->n <= 0) return SPH_OK;
    int rc;
    if (ctx->cfg.precision == SPH_PREC_MIXED) { SPH_DISPATCH_LANES(run_divcurl, float, ctx); }
    else { SPH_DISPATCH_LANES(run_divcurl, double, ctx); }
    if (rc) return rc;
    ctx->divcurl_ok = true;
    ctx->p2_dirty = false;
    return ctx_check_launch(ctx, "divcurl");
}

int launch_repack_p2(sph_ctx *ctx) {
    const int n = ctx->n;
    if (n <= 0) return SPH_OK;
    if (ctx->cfg.precision == SPH_PREC_MIXED)
        k_repack_p2<float><<<div_up(n, 256), 256, 0, ctx->stream>>>(
            n, ctx->rho, ctx->P, ctx->c, ctx->divV, ctx->curlV, ctx->p0, ctx->cfg.balsara,
            (float4 *)ctx->p2);
    else
        k_repack_p2<double><<<div_up(n, 256), 256, 0, ctx->stream>>>(
            n, ctx->rho, ctx->P, ctx->c, ctx->divV, ctx->curlV, ctx->p0, ctx->cfg.balsara,
            (double4 *)ctx->p2);
    ctx->p2_dirty = false;
    return ctx_check_launch(ctx, "repack_p2");
}

// The candidate rows of the last h iteration no longer match the storage
// order or particle set: the next h iteration searches every particle.
int launch_rows_invalidate(sph_ctx *ctx) {
    ctx->rows_host = false;
    CK(cudaMemsetAsync(ctx->rows_ok, 0, sizeof(int), ctx->stream));
    return SPH_OK;
}

// track: the storage order is that of the last pack, so the records' moves
// are added to the distances moved (the candidate rows stay usable);
// otherwise the rows are dropped
int launch_pack_p1(sph_ctx *ctx, bool track) {
    const int n = ctx->n, c = ctx->cur;
    if (!track) {
        int rc = launch_rows_invalidate(ctx);
        if (rc) return rc;
    }
    if (n <= 0) return SPH_OK;
    double *const *st = ctx->st[c];
    double *dmv = track ? ctx->dmv : nullptr;
    if (ctx->cfg.precision == SPH_PREC_MIXED)
        k_pack_p1<float><<<div_up(n, 256), 256, 0, ctx->stream>>>(
            n, st[ST_VX], st[ST_VY], st[ST_VZ], st[ST_M], st[ST_X], st[ST_Y], st[ST_Z], st[ST_H],
            (float4 *)ctx->p1, (float4 *)ctx->pw, ctx->p0, ctx->cloud[c], ctx->corg, dmv,
            ctx->dmv_max);
    else
        k_pack_p1<double><<<div_up(n, 256), 256, 0, ctx->stream>>>(
            n, st[ST_VX], st[ST_VY], st[ST_VZ], st[ST_M], st[ST_X], st[ST_Y], st[ST_Z], st[ST_H],
            (double4 *)ctx->p1, (double4 *)ctx->pw, ctx->p0, ctx->cloud[c], ctx->corg, dmv,
            ctx->dmv_max);
    return ctx_check_launch(ctx, "pack_p1");
}

int launch_forces(sph_ctx *ctx, bool want_acc, bool want_du, bool update_u) {
    (void)update_u;
    if (ctx->n <= 0) return SPH_OK;
    if (ctx->p2_dirty) {
        int r = launch_repack_p2(ctx);
        if (r) return r;
    }
    int rc;
    if (ctx->cfg.precision == SPH_PREC_MIXED) { SPH_DISPATCH_LANES(run_force, float, ctx, want_acc, want_du); }
    else { SPH_DISPATCH_LANES(run_force, double, ctx, want_acc, want_du); }
    if (rc) return rc;
    return ctx_check_launch(ctx, "forces");
}
