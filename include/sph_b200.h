/*
 * sph_b200.h -- C ABI of libsphb200.so, the B200 (sm_100a) per-step hot path
 * of a self-gravitating SPH code (Evrard collapse, cooling cloud collapse).
 *
 * The reference (hassanfv/SPH_2) exposes this path in two forms: numba
 * functions over caller-owned NumPy arrays with a row range [nbeg, nend)
 * (MPI_sph/sph_code/libsx.py, shear.py) and CUDA __global__ kernels over
 * caller-owned float* SoA device arrays (Particles_in_BH_Tree_II/Evrard_test/
 * hfvCLibs_v7_hfv_v2.h, bh_tree_iteration_v2.h, ngb_v3.h).  Each entry point
 * below names the reference functions it replaces.
 *
 * Conventions
 *  - Every call returns SPH_OK (0) or a negative SPH_ERR_* code; nothing in
 *    the library exits, aborts, traps or prints.  Data-dependent device loops
 *    are bounded and report through status counters (sph_get_status).
 *  - Work is queued on the context's stream (sph_set_stream); calls return
 *    before the GPU has finished unless they copy data to the host.
 *  - Particle state lives on the device in FP64 (positions, velocities, u,
 *    h, masses).  The context reorders particles along Morton keys at every
 *    sph_sort; sph_get_field / sph_set_field take and give arrays in the
 *    caller's ORIGINAL particle order unless `storage_order` is set.
 *  - Pointers flagged `host` are host memory (pageable or pinned); otherwise
 *    device memory of the context's device.
 *  - One context per host thread at a time.
 */
#ifndef SPH_B200_H
#define SPH_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---- */
#define SPH_OK 0
#define SPH_ERR_ARG (-1)        /* bad argument (null pointer, size, enum)            */
#define SPH_ERR_CUDA (-2)       /* a CUDA runtime call failed (see sph_last_error)     */
#define SPH_ERR_CAPACITY (-3)   /* n or a cloud count above the context's capacity     */
#define SPH_ERR_NOCONV (-4)     /* smoothing-length iteration did not converge         */
#define SPH_ERR_OVERFLOW (-5)   /* neighbour list or traversal stack overflow          */
#define SPH_ERR_NONFINITE (-6)  /* NaN/Inf found in positions or results               */
#define SPH_ERR_STATE (-7)      /* call order violated (e.g. forces before density)    */
#define SPH_ERR_NOMEM (-8)      /* device allocation failed                            */
#define SPH_ERR_IO (-9)         /* file cannot be opened/read/written, or its size
                                   does not match the format                         */

/* ---- enums ---- */
#define SPH_PREC_FP64 0   /* every sum and the gravity walk in FP64                  */
#define SPH_PREC_MIXED 1  /* FP32 walk and SPH sums (the SPH sums with Kahan
                             compensation); FP64 positions, integration, h
                             convergence, reductions                                */
#define SPH_AV_MG83 0     /* Monaghan & Gingold 1983 (libsx.py:185-262)              */
#define SPH_AV_GADGET 1   /* signal-velocity form (shear.py:243-330, hfvCLibs:705)   */
#define SPH_DT_COURANT 0  /* dt = courant min_i min(h/v_sig, sqrt(h/|a|)) per cloud  */
#define SPH_DT_INDIVIDUAL 1 /* dt = min_i of the six per-particle estimates of
                             sph_dt_individual, per cloud                       */

/* fields for sph_get_field / sph_set_field (FP64 unless noted) */
#define SPH_F_X 0
#define SPH_F_Y 1
#define SPH_F_Z 2
#define SPH_F_VX 3
#define SPH_F_VY 4
#define SPH_F_VZ 5
#define SPH_F_M 6
#define SPH_F_H 7
#define SPH_F_U 8
#define SPH_F_RHO 9
#define SPH_F_P 10
#define SPH_F_C 11
#define SPH_F_DIVV 12
#define SPH_F_CURLV 13
#define SPH_F_AX_SPH 14
#define SPH_F_AY_SPH 15
#define SPH_F_AZ_SPH 16
#define SPH_F_AX_GRAV 17
#define SPH_F_AY_GRAV 18
#define SPH_F_AZ_GRAV 19
#define SPH_F_DUDT 20
#define SPH_F_VSIG 21
#define SPH_F_POT 22
#define SPH_F_DUDT_PREV 23
#define SPH_F_U_PREV 24
#define SPH_NFIELDS 25

/* status counters (sph_get_status) */
#define SPH_S_H_NOCONV 0      /* particles whose Newton h iteration hit the cap   */
#define SPH_S_NGB_OVERFLOW 1  /* rows longer than max_ngb (truncated)            */
#define SPH_S_STACK_OVERFLOW 2/* traversal stack overflows (walk or search)      */
#define SPH_S_H_RETRY 3       /* candidate searches repeated for growing h       */
#define SPH_S_COOL_NOCONV 4   /* cooling solves that hit the iteration cap       */
#define SPH_S_MLP_FALLBACK 5  /* surrogate rows sent back to the exact solver    */
#define SPH_S_NONFINITE 6     /* non-finite inputs seen                          */
#define SPH_S_WALK_STACK_MAX 7/* deepest traversal stack seen in the gravity walk */
#define SPH_S_WAIT_TIMEOUT 8  /* bounded device waits that gave up (tensor-core MLP
                                 tiles; their rows go to the exact solver)        */
#define SPH_NSTATUS 9

#define SPH_FLAG_DUDT_FUSED 1  /* du/dt in the force pass (one pass) instead of the
                                  reference order (after the closing kick)          */
#define SPH_FLAG_COOLING 2     /* apply the implicit cooling in sph_step            */
#define SPH_FLAG_COOLING_MLP 4 /* use the MLP surrogate (exact fallback)            */
#define SPH_FLAG_NO_GRAPH 8    /* run sph_step eagerly, without CUDA graph replay   */
#define SPH_FLAG_POTENTIAL 16  /* compute the gravitational potential in the walk   */
#define SPH_FLAG_TIMING 32     /* record CUDA events between the phases of sph_step */
#define SPH_FLAG_COOLING_TABLE 64 /* with SPH_FLAG_COOLING: the grid-file backend
                                  (sph_cooling_table) instead of the implicit solve */
#define SPH_FLAG_MLP_WARP_MMA 256 /* MLP inference on the warp-level mma.sync path
                                  instead of tcgen05.mma with a TMEM accumulator  */
#define SPH_FLAG_STATIC_GRID 128 /* launch the group kernels (walk, searches, h
                                  iteration) with a grid over the groups instead of
                                  a persistent grid draining a work queue        */
#define SPH_FLAG_NO_ROW_REUSE 512 /* search every particle in each h iteration
                                  instead of keeping a candidate row that the
                                  particles' moves since its search leave complete */

typedef struct sph_config {
    int32_t n_max;        /* particle capacity                                    */
    int32_t n_cloud_max;  /* cloud capacity (ensemble); 1 for a single sphere     */
    int32_t precision;    /* SPH_PREC_*                                           */
    int32_t av_mode;      /* SPH_AV_*                                             */
    int32_t balsara;      /* 1: multiply the viscosity by the Balsara factor      */
    int32_t leaf_size;    /* tree bucket size, 1..64                              */
    int32_t ngb_lanes;    /* lanes per particle in neighbour sums: 1, 2, 4, 8, 16, 32 */
    int32_t block_size;   /* threads per block of the neighbour-sum passes: 64..256,
                             a multiple of 32                                   */
    int32_t max_ngb;      /* neighbour-list row capacity                          */
    int32_t h_max_iter;   /* Newton iteration cap                                 */
    int32_t flags;        /* SPH_FLAG_*                                           */
    int32_t walk_blocks;  /* gravity-walk blocks per SM; fewer leave room for the
                             SPH passes running beside the walk in sph_step.
                             0: 4 per SM for the FP32 walk inside sph_step, the
                             occupancy limit otherwise                         */
    double n_ngb;         /* target (4pi/3)(2h)^3 rho / m                         */
    double h_tol;         /* |dh/h| convergence of the Newton iteration           */
    double gamma, alpha, beta, eta; /* EOS and viscosity (libsx.py:22-26)         */
    double G, eps;        /* gravity constant and Plummer softening               */
    double theta;         /* opening angle                                        */
    double courant;       /* dt = courant * min(h/v_sig, sqrt(h/|a|))             */
    double dt_max;        /* upper bound on dt (0: none)                          */
    double dt_fixed;      /* >0: fixed step (reference drivers), no Courant dt    */
    double theta_local;   /* mixed-precision walk: accepted cells farther than
                             R / theta_local from a group's or super-group's
                             centre (R its radius) enter a Taylor expansion at
                             that centre (monopole and quadrupole field and
                             gradient, monopole terms to third order), once
                             per group or super-group; 0: off                 */
    double theta_small;   /* opening angle of the cells of at most small_cell
                             particles (their mass is small, so their
                             truncation error is too); 0: theta for all cells */
    int32_t small_cell;   /* see theta_small; the error it adds follows the
                             cells' mass fraction: 128 was tuned at N = 1M
                             (theta 0.36, theta_small 0.45), scale it with N  */
    int32_t dt_mode;      /* time step of sph_step and sph_prologue when dt_fixed
                             is 0: SPH_DT_COURANT or SPH_DT_INDIVIDUAL         */
    double ext_sigma;     /* > 0: isothermal galaxy potential of this velocity
                             dispersion added to the gravity, a = -2 sigma^2
                             r / |r|^2 about the origin (galaxy_isothermal_
                             potential, hfvCLibs_v7_hfv_v2.h:1215-1235); it is
                             not part of the potential energy of sph_energies */
    int32_t rebuild_every;/* sph_step sorts the particles and builds the tree
                             topology on every rebuild_every-th step; the
                             steps between keep the storage order and the
                             topology and refit the tree (every node's box,
                             moments, h_max and opening radius recomputed
                             from the drifted particles, so every walk and
                             search stays exact for the tree it walks).
                             1 (default): every step, the reference's order.
                             A load, an injection, a restart file read or
                             written, or an explicit sph_sort makes the next
                             step a full rebuild                               */
    int32_t reserved;     /* 0                                                 */
} sph_config;

typedef struct sph_ctx sph_ctx;

/* cooling problem (physical units) for the implicit solve and the surrogate */
typedef struct sph_cooling_params {
    int32_t n_bins;        /* bins of the log-log Lambda(T) table (table has n_bins+1) */
    int32_t max_iter;      /* bisection cap                                           */
    double logT0, logT1;   /* table range, log10 K                                    */
    double mu, gamma, XH;  /* mean molecular weight, adiabatic index, H mass fraction */
    double gamma_heat;     /* heating per H atom, erg/s                               */
    double tol;            /* |du/u| stopping test of the bisection                   */
    double unit_rho, unit_u, unit_t; /* code -> cgs factors                           */
    double mlp_err_tol;    /* surrogate rows with estimated |du/u| above this fall back */
} sph_cooling_params;

/* ---- context ---- */
int sph_default_config(sph_config *cfg);
int sph_ctx_create(const sph_config *cfg, sph_ctx **out);
void sph_ctx_destroy(sph_ctx *ctx);
int sph_set_stream(sph_ctx *ctx, void *cuda_stream);
int sph_sync(sph_ctx *ctx);
const char *sph_last_error(sph_ctx *ctx);
int sph_get_config(sph_ctx *ctx, sph_config *out);
int sph_set_params(sph_ctx *ctx, const sph_config *cfg); /* physics scalars only */
int64_t sph_device_bytes(sph_ctx *ctx);

/* Load n particles (replaces readVectorsFromFile + cudaMemcpy H2D,
 * hfvCLibs_v7_hfv_v2.h:59, EVR.cu:508-556, and the pickle IC of
 * sph_mpi4_v4.py:44-53).  cloud may be NULL (one cloud).  Arrays in host or
 * device memory (host != 0: host). */
int sph_load(sph_ctx *ctx, int32_t n, const int32_t *cloud, const double *x, const double *y,
             const double *z, const double *vx, const double *vy, const double *vz,
             const double *m, const double *h, const double *u, int32_t host);
int32_t sph_count(sph_ctx *ctx);
int32_t sph_cloud_count(sph_ctx *ctx);
int sph_get_field(sph_ctx *ctx, int32_t field, double *out, int32_t host, int32_t storage_order);
int sph_set_field(sph_ctx *ctx, int32_t field, const double *in, int32_t host, int32_t storage_order);
/* nfield fields at once (fields[k] from in[k] / into out[k]): one
 * synchronisation and one rebuild of the particle records per call instead
 * of one per field; same arguments and order conventions as above */
int sph_set_fields(sph_ctx *ctx, int32_t nfield, const int32_t *fields, const double *const *in,
                   int32_t host, int32_t storage_order);
int sph_get_fields(sph_ctx *ctx, int32_t nfield, const int32_t *fields, double *const *out,
                   int32_t host, int32_t storage_order);
/* original id of each stored particle (storage order) */
int sph_get_ids(sph_ctx *ctx, int32_t *out, int32_t host);
int sph_get_status(sph_ctx *ctx, int64_t *out /* SPH_NSTATUS */, int32_t reset);
int sph_get_dt(sph_ctx *ctx, double *dt /* per cloud */);
int sph_set_dt(sph_ctx *ctx, const double *dt /* per cloud */);

/* ---- phases (each queued on the context stream) ---- */

/* Per-cloud bounding box (compute_bounding_box_kernel, bh_tree_iteration_v2.h:
 * 76-145), 63-bit Morton keys and a stable LSD radix sort of the storage order
 * (replaces CountBodies/ComputeOffset/GroupBodies, ngb_v3.h:58-117), then the
 * particle state is permuted into key order. */
int sph_sort(sph_ctx *ctx);
/* keys of the CURRENT storage order (before permutation) and the stable
 * permutation perm (new slot s holds old slot perm[s]), from the last sort */
int sph_get_sort(sph_ctx *ctx, uint64_t *keys, int32_t *perm, int32_t host);

/* Karras radix tree over the sorted keys with FP64 bottom-up mass, centre of
 * mass, quadrupole, box and h_max (replaces reset_arrays_kernel,
 * build_tree_kernel, centre_of_mass_kernel, sort_kernel,
 * bh_tree_iteration_v2.h:29-450). */
int sph_build_tree(sph_ctx *ctx);
/* FP64 node records (16 doubles each: com xyz, mass, Qxx Qyy Qzz Qxy Qxz Qyz,
 * box min xyz, box max xyz), child pairs, particle ranges, opening radii^2 */
int sph_get_tree(sph_ctx *ctx, double *node, int32_t *child, int32_t *first, int32_t *last,
                 double *open_r2, double *hmax, int32_t host);

/* The walk/search groups of the last tree build: maximal tree nodes with at
 * most 32 particles of one cloud, in Morton order (start index, size). */
int sph_get_groups(sph_ctx *ctx, int32_t *ngroup, int32_t *gstart, int32_t *gcount, int32_t host);

/* Newton smoothing-length iteration (replaces smoothing_h_ngb,
 * hfvCLibs_v7_hfv_v2.h:367-455, and h_smooth_fast_mpi, libsx.py:854-902).
 * Needs sph_build_tree. */
int sph_smoothing_h(sph_ctx *ctx);
/* The reference's own smoothing-length iteration (h_smooth_fast_mpi,
 * MPI_sph/sph_code/libsx.py:854-902, with n_target 50, n_tol 5, step_frac
 * 0.003): starting from the current h, h <- h (1 - step_frac) while
 * #{j : |r_ij| < 2h} > n_target + n_tol and h <- h (1 + step_frac) while it is
 * below n_target - n_tol (self included, distances rounded as the reference
 * computes them), so the result is bit-exact with the reference on the same
 * positions.  The reference iterates without bound (it only prints after 100
 * iterations); here a particle stops after max_iter iterations and is
 * counted in SPH_S_H_NOCONV.  n_target + n_tol must not exceed max_ngb.
 * Needs sph_build_tree. */
int sph_smoothing_h_count(sph_ctx *ctx, int32_t n_target, int32_t n_tol, double step_frac,
                          int32_t max_iter);
/* The reference's starting smoothing length (smoothing_length_mpi,
 * MPI_sph/sph_code/libsx.py:777-800 with k = 50): h = half the k-th smallest
 * distance to the particles of its cloud, the particle itself counted at
 * distance 0, the distance rounded as the reference computes it; the
 * candidate search starts from the current h.  k + 1 must not exceed max_ngb.
 * Needs sph_build_tree. */
int sph_smoothing_length_kth(sph_ctx *ctx, int32_t k);
/* Exact neighbour lists |r_ij|^2 <= (h_i+h_j)^2 (replaces ngbDB_new_v2,
 * ngb_v3.h:124-238).  Needs sph_build_tree (h_max is refitted here). */
int sph_neighbours(sph_ctx *ctx);
/* canonical export: CSR over storage order, rows sorted ascending by
 * storage index; off has n+1 entries; lst capacity cap */
int sph_get_neighbours(sph_ctx *ctx, int64_t *off, int32_t *lst, int64_t cap, int32_t host);

/* rho = sum m_j W(r_ij, h_ij) and the EOS epilogue P, c (getDensity_ngb,
 * getPressure_Adiabatic, getCsound_Adiabatic, hfvCLibs_v7_hfv_v2.h:474-612;
 * getDensity_mpi, libsx.py:52-86) */
int sph_density(sph_ctx *ctx);
/* div v, |curl v| (div_curlVel_ngb, hfvCLibs:617-700; div_curlVel_mpi,
 * shear.py:78-142) */
int sph_divcurl(sph_ctx *ctx);
/* pressure + viscous acceleration and signal velocity (acc_sph_ngb,
 * hfvCLibs:705-801; getAcc_sph_shear_mpi, shear.py:243-330;
 * getAcc_sph_mpiXXX, libsx.py:185-262); with SPH_FLAG_DUDT_FUSED also du/dt */
int sph_forces(sph_ctx *ctx);
/* du/dt (get_dU_ngb, hfvCLibs:825-916; get_dU_shear_mpi, shear.py:413-485) */
int sph_dudt(sph_ctx *ctx);
/* Barnes-Hut walk, monopole + quadrupole, Plummer softening (replaces
 * compute_forces_kernel, bh_tree_iteration_v2.h:454-588).  Counts the
 * interactions (sph_get_counters). */
int sph_gravity(sph_ctx *ctx);
/* FP64 direct Plummer sum onto ntarget particles (storage indices) from all
 * particles of their cloud (replaces acc_g, hfvCLibs:532-584, and
 * getAcc_g_smth_mimj_mpi, libsx.py:910-947).  out: ntarget*4 (ax,ay,az,pot). */
int sph_gravity_direct(sph_ctx *ctx, int32_t ntarget, const int32_t *targets, double *out,
                       int32_t host);
/* spline-softened direct sum of libsx.py:910-947 with per-particle eps
 * (eps_ij = (eps_i+eps_j)/2), FP64, out: ntarget*3 */
int sph_gravity_direct_spline(sph_ctx *ctx, const double *eps, int32_t ntarget,
                              const int32_t *targets, double *out, int32_t host);
/* the reference's partial field of rows [nbeg, nend) (getAcc_g_smth_mimj_mpi,
 * libsx.py:910-947): every pair (a, b), a < b in original index with a in
 * the rows, adds its spline-softened attraction to both a and b, so the sum
 * of the fields of a partition of [0, N) is the full field.  eps and out
 * (n x 3, row per particle) in original order, FP64. */
int sph_gravity_direct_spline_rows(sph_ctx *ctx, const double *eps, int32_t nbeg, int32_t nend,
                                   double *out, int32_t host);
/* v += a dt * fac with a = a_sph + a_grav (v_evolve, hfvCLibs:936-949) */
int sph_kick(sph_ctx *ctx, double fac);
/* x += v dt (r_evolveT, hfvCLibs:981-994) */
int sph_drift(sph_ctx *ctx);
/* u = u_prev + dt/2 (dudt + dudt_prev); u_prev = u; dudt_prev = dudt
 * (u_updater, hfvCLibs:921-931; sph_mpi4_v4.py:413-424).  first != 0: the
 * prologue form u += dudt dt (sph_mpi4_v4.py:240-244). */
int sph_update_u(sph_ctx *ctx, int32_t first);
/* Courant step per cloud dt = courant * min_i min(h/v_sig, sqrt(h/|a|))
 * (dt_array_indiv_dt, hfvCLibs:999-1078, over neighbours only); stored as
 * the step of the next sph_step and returned in dt (per cloud) if not NULL */
int sph_cfl_dt(sph_ctx *ctx, double *dt);
/* Individual time steps (replaces dt_array_indiv_dt, hfvCLibs_v7_hfv_v2.h:
 * 999-1078, and the min_finder of EVR.cu:1733): for every particle the
 * smallest of C h / max_j v_sig,ij, C h / (h |div v| + max(c, |v|)(1 + 0.6
 * alpha)), 0.4 sqrt(eps / |a|), 0.4 eps / |v|, sqrt(h / |a_grav|) and
 * sqrt(h / |a|), with v_sig,ij = c_i + c_j - 3 v_ij.r_ij / (|r_ij| + 1e-5)
 * maximised over the particle's neighbour list (the reference loops over all
 * N particles) and C = courant, eps the Plummer softening, a = a_sph +
 * a_grav; dh/dt = h div v / 3 with div v signed.  The per-cloud minimum is
 * stored as the next step (dt_fixed still wins) and returned by sph_get_dt.
 * bin[i] = the smallest k >= 0 with dt_ref / 2^k <= dt[i] (dt_ref = dt_max if
 * set, else the cloud's largest dt[i]; -1 for a particle without a finite
 * positive step).  dt, dhdt and bin (each may be NULL) receive n values in
 * the caller's original order.  Needs the lists, density and accelerations
 * of the current state (sph_prologue or sph_step). */
int sph_dt_individual(sph_ctx *ctx, double *dt, double *dhdt, int32_t *bin, int32_t host);
/* totals: [KE, U, PE, px, py, pz, Lx, Ly, Lz, M] (getKE/getPE, libsx.py:571-620);
 * PE needs SPH_FLAG_POTENTIAL in the last gravity call */
int sph_energies(sph_ctx *ctx, double *out10);
/* interaction counters of the last gravity call: [cells, particles] */
int sph_get_counters(sph_ctx *ctx, int64_t *out2);
/* far cells of the last walk that went through the local expansions
 * (sph_config.theta_local), summed over groups and super-groups (one per
 * cell and group or super-group) */
int sph_get_far_cells(sph_ctx *ctx, int64_t *out);
/* super-groups of the last mixed walk with theta_local > 0 (maximal tree
 * nodes of at most 128 particles, walked once for the far cells their groups
 * share): [far cells through their expansions, super-groups whose node list
 * did not fit (their groups walked from the root)] */
int sph_get_supergroup_stats(sph_ctx *ctx, int64_t *out2);

/* ---- cooling (DoCooling, myPhotoLibsGPU.h:615-686; hcoolingx, hfvCLibs:1240) ---- */
int sph_cooling_setup(sph_ctx *ctx, const sph_cooling_params *p, const double *log_lambda);
/* implicit solve for every particle over dt (code units) */
int sph_cooling_exact(sph_ctx *ctx);
/* MLP surrogate + error estimate + exact fallback */
int sph_cooling_mlp(sph_ctx *ctx);
/* Standalone batched solves on arrays (physical cgs units).  u_new may alias
 * u_old.  iters may be NULL. */
int sph_cool_solve(sph_ctx *ctx, int32_t n, const double *rho, const double *u_old,
                   const double *dt, double *u_new, int32_t *iters, int32_t host);

/* ---- table cooling with ion fractions (hcoolingx, hfvCLibs_v7_hfv_v2.h:
 * 1240-1418; grid file coolHeatGridNew.bin read as in
 * hfvGpuSphBHtree_v3_check_v1_cooling_t3_Evrard.cu:137-179) ---- */
typedef struct sph_cool_table_params {
    double unit_rho, unit_u, unit_t; /* code -> cgs                                  */
    double unit_length;              /* code length in cm                             */
    double kpc_cm;                   /* 3.086e21                                      */
    double XH, mH;                   /* n_H = rho X_H / m_H (0.70, 1.6726e-24)        */
    int32_t z_row;                   /* metallicity row of the grid (the reference: 1) */
    int32_t reserved;                /* 0 */
} sph_cool_table_params;
/* dims6 = N_kpc, N_nH, N_Z, N_T, N_M, N_Time of a grid file, whose size is
 * checked against them (host only, no GPU) */
int sph_cooling_table_dims(const char *path, int32_t *dims6);
/* read the grid file onto the device (replacing an earlier one) */
int sph_cooling_table_load(sph_ctx *ctx, const char *path, const sph_cool_table_params *p);
/* new u of every particle over the current dt from the grid: nearest radius
 * (kpc) and n_H cell, the first u row at or above u and the first time at or
 * above dt, linear in u between that row and the one below; and the N_M ion
 * fractions of that cell.  The step applies it with SPH_FLAG_COOLING |
 * SPH_FLAG_COOLING_TABLE. */
int sph_cooling_table(sph_ctx *ctx);
/* ion fractions of the last table cooling, n rows of N_M floats in original
 * particle order (the snapshot's ionFrac block) */
int sph_get_ion_frac(sph_ctx *ctx, float *out, int32_t host);

/* ---- cooling-surrogate MLP 3->64->64->1 (GELU), BF16 weights ---- */
/* parameters in FP32: W1[3*64] b1[64] W2[64*64] b2[64] W3[64] b3[1] and the
 * input/output normalisation norm[8] = (mean[3], scale[3], y_mean, y_scale) */
#define SPH_MLP_NPARAM (3 * 64 + 64 + 64 * 64 + 64 + 64 + 1)
int sph_mlp_set(sph_ctx *ctx, const float *params, const float *norm, int32_t host);
int sph_mlp_get(sph_ctx *ctx, float *params, float *norm, int32_t host);
/* forward on n rows of normalised inputs X[n*3] -> y[n] (tensor cores) */
int sph_mlp_forward(sph_ctx *ctx, int32_t n, const float *X, float *y, int32_t host);
/* gradient of 0.5*mean((y - t)^2) over n rows -> grad[SPH_MLP_NPARAM], and
 * the loss; forward+backward on tensor cores */
int sph_mlp_grad(sph_ctx *ctx, int32_t n, const float *X, const float *t, float *grad,
                 float *loss, int32_t host);
/* nsteps of Adam (lr; beta1 0.9, beta2 0.999, eps 1e-8) on consecutive
 * minibatches of size batch of the device arrays X[n*3], t[n] (wrapping);
 * writes the loss of the last minibatch to *loss (host) */
int sph_mlp_train(sph_ctx *ctx, int32_t n, const float *X, const float *t, int32_t batch,
                  int32_t nsteps, float lr, float *loss);
/* surrogate cooling on device arrays (cgs): u_new from the MLP where its
 * estimated relative error is within mlp_err_tol, else from the exact solve;
 * fell_back[i] = 1 where the exact solve ran (may be NULL) */
int sph_cool_solve_mlp(sph_ctx *ctx, int32_t n, const double *rho, const double *u_old,
                       const double *dt, double *u_new, int32_t *fell_back);

/* ---- full step ---- */
/* The prologue of the reference loop (sph_mpi4_v4.py:106-265): h, rho, forces,
 * gravity, du/dt, u += du/dt dt, and the first dt. */
int sph_prologue(sph_ctx *ctx);
/* nsteps of kick-drift-(sort, tree, h, lists, rho, div/curl, forces | gravity)
 * -kick-du/dt-u-[cooling]-dt (sph_mpi4_v4.py:278-442; EVR.cu:1139-1782),
 * replayed from a CUDA graph unless SPH_FLAG_NO_GRAPH. */
int sph_step(sph_ctx *ctx, int32_t nsteps);
/* One step with its host transfers, for drivers that exchange particle fields
 * with the host every step (the reference's GPU loop copies x, y, z and the
 * masses out and the tree arrays back in every step, EVR.cu:1462-1482): the
 * nin fields fin[k] are copied in from the host arrays in[k] (as
 * sph_set_fields, caller order), one step runs (as sph_step), and the nout
 * fields fout[k] are copied to the host arrays out[k] (as sph_get_fields,
 * caller order).  The out copies run on a copy stream of the context, each
 * as soon as the step has written the field's last value (positions and
 * masses after the sort, h after the neighbour pass, velocities after the
 * closing kick, the rest at the end), so they overlap the rest of the step.
 * in[k] and out[j] may be the same array.  The first call allocates a staging
 * buffer of max(nin, nout) x n_max doubles and the copy stream.  Returns when
 * the step and every copy are complete. */
int sph_step_io(sph_ctx *ctx, int32_t nin, const int32_t *fin, const double *const *in,
                int32_t nout, const int32_t *fout, double *const *out);

/* internal per-particle arrays for diagnostics, storage order:
 * 0 candidate count (int32), 1 list count (int32), 2 retry flag (int32),
 * 3 candidate radius / 2 (double), 4 h of the packed position record,
 * 5 mass of the packed velocity record (both as double),
 * 6 tree-search flags of the last list build (int32, n + 1: per particle 1 =
 *   its list came from the tree search, not from its candidate row; the last
 *   entry 1 = every list did) */
int sph_debug_copy(sph_ctx *ctx, int32_t which, void *out, int32_t host);

/* ---- measurement ---- */
/* Phase durations of the last sph_step (needs SPH_FLAG_TIMING), in ms:
 * [kick+drift, sort, tree, h, lists, density, div/curl, forces, wait+kick,
 *  du/dt, u(+cooling)+dt, gravity (own stream)]; returns the count (12). */
#define SPH_NPHASE 12
int sph_get_phase_times(sph_ctx *ctx, float *ms);
/* run nsteps of sph_step between two CUDA events on the context's stream and
 * return their device time in ms (the autotuner's clock) */
int sph_time_steps(sph_ctx *ctx, int32_t nsteps, float *ms);
/* kernel nodes in the step graph captured last (0 before the first graph
 * step) */
int sph_graph_kernel_count(sph_ctx *ctx, int32_t *count);
/* kernel nodes of every step graph launched since the last reset (rebuild
 * and refit steps have graphs of their own); reset != 0: start again at 0 */
int sph_graph_kernels_launched(sph_ctx *ctx, int64_t *count, int32_t reset);
/* particles whose candidate row the last h iteration (sph_step or
 * sph_smoothing_h) kept instead of searching again: the distances that they
 * and the particles near them moved since the row's search leave it complete
 * (0 with SPH_FLAG_NO_ROW_REUSE, after a sort, or after the count and k-th
 * iterations) */
int sph_rows_kept(sph_ctx *ctx, int64_t *kept);
/* FP32 FMA throughput of this GPU measured by dependent-chain kernels of
 * scalar and of packed (f32x2) FMAs, the larger of the two, TFLOP/s (2 flops
 * per FMA): the denominator for FP32-bound kernels */
int sph_measure_fp32_peak(sph_ctx *ctx, double *tflops);

/* ---- allocation-free Morton order ---- */
/* No counterpart in the reference.  For callers that must not allocate device
 * memory when they need the particle order -- e.g. code whose device memory is
 * all held by another framework's caching allocator, or that cannot afford the
 * implicit synchronisation of cudaMalloc: 63-bit Morton keys of one cloud
 * (keys[i], input order) and the stable sort permutation (perm[s] = input
 * index of sorted slot s), the same definitions as sph_sort / sph_get_sort.
 * x, y, z, keys and perm are caller-owned device arrays; nothing is allocated.
 * Scratch is a fixed array compiled into the library (6.4 MB, held on
 * every GPU that loads the library until the process exits), so
 * n <= SPH_NOALLOC_MAX_N (SPH_ERR_CAPACITY above it).  All calls share that
 * array: calls that overlap on the GPU race.  The first call on a device looks
 * up the array's device address (cudaGetSymbolAddress); make that first call
 * before any stream capture.  The address is kept until the process exits: after
 * a cudaDeviceReset the library must be reloaded before this entry point is used
 * again.  If a CUDA error from the caller's earlier work is pending on entry,
 * the call returns SPH_ERR_CUDA without launching and leaves that error set.
 * Work is queued on cuda_stream (NULL: the legacy default stream) of the
 * current device. */
#define SPH_NOALLOC_MAX_N 262144
int sph_morton_sort_noalloc(const double *x, const double *y, const double *z, int32_t n,
                            uint64_t *keys, int32_t *perm, void *cuda_stream);

/* ---- outflow injection (outflow_injector2, hfvCLibs_v7_hfv_v2.h:1094-1210) ---- */
typedef struct sph_outflow_params {
    double mdot;        /* injected mass per unit time (M_dot_in)                     */
    double v_in;        /* radial outward speed of the injected particles             */
    double m_particle;  /* mass of each injected particle (mass_sph_high_res)         */
    double u_inject;    /* their specific internal energy (u_for_10K_Temp)            */
    double r_max;       /* radius of the injection sphere about the origin            */
    double h_first;     /* h of the first pair when nothing was injected before       */
    uint64_t seed;      /* the pairs' random numbers; vary it from call to call       */
    int32_t cloud;      /* cloud the pairs join: the last cloud (ncloud - 1)          */
    int32_t reserved;   /* 0 */
} sph_outflow_params;
/* mass = mdot * dt(cloud) + *leftover_mass is spawned as floor(mass / (2 m))
 * pairs at +r and -r (|r| uniform in [0, r_max), isotropic), with velocities
 * +-v_in r/|r|, mass m, u = u_inject and h (and softening) of the particle
 * injected last by an earlier call (h_first before the first one).  The new
 * particles are appended (original ids n, n+1, ...; sph_count grows) and
 * join the next step; *leftover_mass (host, in/out) keeps the remainder and
 * *n_added (host, may be NULL) receives 2 * pairs.  Random numbers come from
 * SplitMix64 keyed by (seed, pair number), not cuRAND: the distribution is
 * the reference's, the values are not.  SPH_ERR_CAPACITY (nothing injected)
 * when n_max would be passed. */
int sph_outflow_inject(sph_ctx *ctx, const sph_outflow_params *p, double *leftover_mass,
                       int32_t *n_added);

/* ---- FP64 restart (replaces the float text dumps the reference restarts
 * from, GPU_sph/With_metal_cooling/Check_Restart_version/hfv_sph_gpu_v5.cu) ----
 * The file holds the particle state in FP64 and in the context's storage
 * order (ids and clouds, x y z vx vy vz m h u du/dt_prev and the largest
 * neighbour h), the last step's accelerations and every cloud's dt.  A context
 * that reads it (capacity permitting) continues exactly as the writing context
 * would have: the next sph_step repeats it bit for bit in the same precision.
 * (With rebuild_every > 1 both the writing and the reading context make that
 * next step a full rebuild.)  Cooling tables and surrogate parameters are not
 * part of it. */
int sph_write_restart(sph_ctx *ctx, const char *path);
int sph_read_restart(sph_ctx *ctx, const char *path);

/* ---- the reference's binary files (host I/O) ---- */
/* IC file of IC_evrard4.cu:245-260 / readVectorsFromFile
 * (hfvCLibs_v7_hfv_v2.h:59-101): int32 N, int32 Typ[N], then float32 x, y, z,
 * vx, vy, vz, u, h, eps, mass, N values each.  sph_ic_count reads and checks
 * the header (file size must equal 4 + 44 N) and needs no GPU.  sph_load_ic
 * replaces the context's particles with the file's (widened to FP64; Typ must
 * be 0, gas, else SPH_ERR_ARG); eps_out (host, n, may be NULL) receives the
 * per-particle softening column.  sph_write_ic writes the context's particles
 * in original order (Typ 0; eps = the given host array, or h as
 * IC_evrard4.cu:224-229 does when eps is NULL). */
int sph_ic_count(const char *path, int32_t *n);
int sph_load_ic(sph_ctx *ctx, const char *path, double *eps_out);
int sph_write_ic(sph_ctx *ctx, const char *path, const double *eps);
/* Snapshot of saveArraysToBinary (hfvCLibs_v7_hfv_v2.h:107-143), as read by
 * Evrard_test/singlex_gpu_data.py:55-72: int32 N, int32 N_ionFrac, int32
 * Typ[N], float32 x, y, z, vx, vy, vz, rho, h, u, mass (N each), float32
 * ionFrac[N_ionFrac], int32 per-particle debug slot[N] (written here as the
 * neighbour count, -1 before the first list build).  Original particle order.
 * ion_frac is host memory and may be NULL when n_ion_frac is 0. */
int sph_write_snapshot(sph_ctx *ctx, const char *path, const float *ion_frac, int32_t n_ion_frac);

/* The same entry points a single GPU runs, for a rank of a multi-GPU job
 * that owns a slice of the ensemble: nothing here talks to other ranks. */

#ifdef __cplusplus
}
#endif
#endif /* SPH_B200_H */
