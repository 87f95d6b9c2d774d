// timestep.cu -- individual (per-particle) time steps over the neighbour lists.
//
// Replaces dt_array_indiv_dt (Particles_in_BH_Tree_II/Evrard_test/
// hfvCLibs_v7_hfv_v2.h:999-1078).  The reference takes, for every particle i,
// the largest signal velocity c_i + c_j - 3 w_ij (w_ij = v_ij.r_ij /
// (|r_ij| + 1e-5), j = i included, starting from 0) over ALL N particles --
// an O(N^2) loop that is why its Evrard driver leaves the kernel disabled
// (EVR.cu:1716-1733) -- and then the smallest of six estimates:
//   dt_hyd = C h / max_j v_sig,ij          (Springel et al. 2005, eq. 16)
//   dt_cour = C h / (h |div v| + max(c, |v|)(1 + 0.6 alpha))   (Gadget-2 eq. 49)
//   dt_G1 = 0.4 sqrt(eps / |a_tot|),  dt_G2 = 0.4 eps / |v|    (Dave et al. 1997)
//   dt_f = sqrt(h / |a_grav|),  dt_kin = sqrt(h / |a_tot|)
// and dh/dt = h div v / 3 (Gadget-2, below eq. 31), with div v signed.
// Here the signal-velocity maximum runs over the particle's neighbour list
// (the pairs that interact through the kernel), so the kernel is one
// O(N_ngb) pass fused with the signed divergence it needs: LANES lanes per
// particle over its list row, the same lane layout as the force pass.  The
// per-cloud minimum becomes the next step (the reference's min_finder), and a
// second small kernel files each particle into a power-of-two bin below the
// largest step for drivers that advance particles on their own steps.
#include "sph_internal.cuh"

namespace {

template <class R, int LANES>
__global__ void __launch_bounds__(256)
    k_dt_indiv(int n, const double4 *__restrict__ p0, const typename R4<R>::T *__restrict__ p1,
               const typename R4<R>::T *__restrict__ p2, const int *__restrict__ rows,
               const int *__restrict__ cnt, int K, const double *__restrict__ rho,
               const double *__restrict__ c, const double *__restrict__ vx,
               const double *__restrict__ vy, const double *__restrict__ vz,
               const double *__restrict__ asph, const double *__restrict__ agrav,
               const int *__restrict__ cloud, double eps, double courant, double alpha,
               double *__restrict__ dt_out, double *__restrict__ dhdt_out,
               unsigned long long *__restrict__ dt_bits,
               unsigned long long *__restrict__ dtmax_bits) {
    typedef typename R4<R>::T V4;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int i = (int)(t / LANES), sl = (int)(t % LANES);
    const bool valid = i < n;
    R vmax = R(0);
    KSum<R> s;
    if (valid) {
        const double4 pi = p0[i];
        const V4 vi = p1[i];
        const R ci = p2[i].z;
        const int cn = cnt[i];
        const int *row = rows + (size_t)i * K;
        for (int k = sl; k < cn; k += LANES) {
            const int j = row[k];
            const double4 pj = p0[j];
            const V4 vj = p1[j];
            const R cj = p2[j].z;
            const R dx = (R)(pi.x - pj.x), dy = (R)(pi.y - pj.y), dz = (R)(pi.z - pj.z);
            const R rr = qsqrt<R>(dx * dx + dy * dy + dz * dz);
            const R ux = vi.x - vj.x, uy = vi.y - vj.y, uz = vi.z - vj.z;
            const R vr = ux * dx + uy * dy + uz * dz;
            const R w = qdiv<R>(vr, rr + R(1e-5));
            vmax = fmax(vmax, ci + cj - R(3) * w);
            const R hij = (R)(0.5 * (pi.w + pj.w));
            const R inv = qdiv<R>(R(1), hij);
            const R i2 = inv * inv;
            const R nW = kern_nw<R>(rr * inv, i2 * i2 * inv);
            s.add(-vj.w * nW * vr);
        }
    }
    const double vs = seg_max<LANES>((double)vmax);
    const double sd = seg_sum<LANES>(s.value());
    const bool lead = valid && sl == 0;
    int cl = 0;
    double dt = 0.0;
    if (lead) {
        const double hi = p0[i].w, ci = c[i];
        const double div = sd / rho[i];
        const double gx = agrav[i], gy = agrav[(size_t)n + i], gz = agrav[2 * (size_t)n + i];
        const double tx = asph[i] + gx, ty = asph[(size_t)n + i] + gy, tz = asph[2 * (size_t)n + i] + gz;
        const double ag = sqrt(gx * gx + gy * gy + gz * gz);
        const double at = sqrt(tx * tx + ty * ty + tz * tz);
        const double va = sqrt(vx[i] * vx[i] + vy[i] * vy[i] + vz[i] * vz[i]);
        // IEEE division: an estimate whose denominator is 0 is +inf and
        // drops out of the minimum, as in the reference
        const double dt_hyd = courant * hi / vs;
        const double dt_cour = courant * hi / (hi * fabs(div) + fmax(ci, va) * (1.0 + 0.6 * alpha));
        const double dt_g1 = 0.4 * sqrt(eps / at);
        const double dt_g2 = 0.4 * eps / va;
        const double dt_f = sqrt(hi / ag);
        const double dt_kin = sqrt(hi / at);
        dt = fmin(fmin(fmin(dt_hyd, dt_cour), fmin(dt_g1, dt_g2)), fmin(dt_f, dt_kin));
        dt_out[i] = dt;
        dhdt_out[i] = hi * div / 3.0;
        cl = cloud[i];
        if (!(dt > 0.0 && isfinite(dt))) dt = 0.0;
        if (dt > 0.0) atomicMax(&dtmax_bits[cl], dbl_to_ord(dt));
    }
    cloud_min(dt_bits, lead, cl, dt);
}

// bin k of particle i: the smallest k >= 0 with ref / 2^k <= dt_i, ref the
// largest step (dt_max if set, else the cloud's largest dt_i); -1 when dt_i
// is not a finite positive number
__global__ void k_dt_bins(int n, const double *__restrict__ dt, const int *__restrict__ cloud,
                          double dt_max, const unsigned long long *__restrict__ dtmax_bits,
                          int *__restrict__ bin) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double d = dt[i];
    if (!(d > 0.0 && isfinite(d))) {
        bin[i] = -1;
        return;
    }
    const unsigned long long b = dtmax_bits[cloud[i]];
    const double ref = dt_max > 0.0 ? dt_max : (b ? ord_to_dbl(b) : d);
    int k = 0;
    double s = ref;
    while (s > d && k < 62) {
        s *= 0.5;
        k++;
    }
    bin[i] = k;
}

template <class R, int L>
int run_dt_indiv(sph_ctx *ctx) {
    const int n = ctx->n, cur = ctx->cur;
    const int bs = ctx->cfg.block_size;
    double *const *st = ctx->st[cur];
    k_dt_indiv<R, L><<<div_up((long long)n * L, bs), bs, 0, ctx->stream>>>(
        n, ctx->p0, (const typename R4<R>::T *)ctx->p1, (const typename R4<R>::T *)ctx->p2,
        ctx->ngb, ctx->ngb_cnt, ctx->cfg.max_ngb, ctx->rho, ctx->c, st[ST_VX], st[ST_VY],
        st[ST_VZ], ctx->asph, ctx->agrav, ctx->cloud[cur], ctx->cfg.eps, ctx->cfg.courant,
        ctx->cfg.alpha, ctx->dt_part, ctx->dhdt, ctx->dt_bits, ctx->dtmax_bits);
    return SPH_OK;
}

#define SPH_DISPATCH_LANES_TS(FN, R, ctx)          \
    switch ((ctx)->cfg.ngb_lanes) {                \
        case 1: rc = FN<R, 1>(ctx); break;         \
        case 2: rc = FN<R, 2>(ctx); break;         \
        case 4: rc = FN<R, 4>(ctx); break;         \
        case 8: rc = FN<R, 8>(ctx); break;         \
        case 16: rc = FN<R, 16>(ctx); break;       \
        default: rc = FN<R, 32>(ctx); break;       \
    }

}  // namespace

// per-particle steps, dh/dt and the per-cloud minimum into dt_bits (committed
// by k_dt_commit); needs the lists, rho, c and the accelerations of this step
int launch_dt_individual(sph_ctx *ctx) {
    const int n = ctx->n;
    if (n <= 0) return SPH_OK;
    CK(cudaMemsetAsync(ctx->dtmax_bits, 0, sizeof(unsigned long long) * ctx->ncloud, ctx->stream));
    if (ctx->p2_dirty) {
        int r = launch_repack_p2(ctx);
        if (r) return r;
    }
    int rc;
    if (ctx->cfg.precision == SPH_PREC_MIXED) { SPH_DISPATCH_LANES_TS(run_dt_indiv, float, ctx); }
    else { SPH_DISPATCH_LANES_TS(run_dt_indiv, double, ctx); }
    if (rc) return rc;
    return ctx_check_launch(ctx, "dt_individual");
}

int launch_dt_bins(sph_ctx *ctx) {
    const int n = ctx->n;
    if (n <= 0) return SPH_OK;
    k_dt_bins<<<div_up(n, 256), 256, 0, ctx->stream>>>(n, ctx->dt_part, ctx->cloud[ctx->cur],
                                                       ctx->cfg.dt_max, ctx->dtmax_bits,
                                                       ctx->dbin);
    return ctx_check_launch(ctx, "dt_bins");
}
