/*
 * pipeflow_b200.h -- C ABI of the B200 (sm_100a) timestep hot path of the
 * openpipeflow pipe-flow DNS (Fortran 90 reference, openpipeflow 1.12).
 *
 * Every entry point returns an int status: PF_OK (0) or a negative PF_ERR_*
 * code; pf_last_error() gives the message of the calling thread's last
 * failure.  A Fortran ISO_C_BINDING shim maps a non-zero status to
 * `stop <message>`, which is the reference's error behaviour for every
 * failure (e.g. timestep.f90:93,117, meshs.f90:238).
 *
 * Object model (one pf_ctx per pipe == the module state of the reference's
 * modules variables/transform/timestep/velocity for one run):
 *   pf_ctx     parameters.f90 + module state (tim_*, vel_*, matrices)
 *   pf_coll    one `type (coll)` field on the device       (variables.f90:37-40)
 *   pf_phys    one `type (phys)` field on the device       (variables.f90:42-44)
 *   pf_mesh    one set of per-mode `type (mesh)` band matrices (meshs.f90:37-39)
 *   pf_lumesh  one set of per-mode `type (lumesh)` LU factors (meshs.f90:42-45)
 *
 * Host-array layouts follow the reference exactly (Fortran column-major):
 *   coll: re[nh*N + n], im[nh*N + n]        == %Re(n+1, nh), %Im(n+1, nh)
 *   phys: re[(n*Th + t)*Z + z]              == %Re(z, t, n+1)
 *   mesh: M[(nh*N + j)*(2KL+1) + row]       == A(nh)%M(row+1, j+1)
 *   lumesh: M[(nh*N + j)*(3KL+1) + row], ipiv[nh*N + j] (1-based, LAPACK)
 * with the harmonic order of the serial _loop_km macro (parallel.h:47-57):
 * nh = m*(2K-1)+k, m = 0..M-1, k = -(K-1)..K-1, skipping k<0 when m=0.
 *
 * Calls are asynchronous on the context's CUDA stream unless they return a
 * host value (norms, corrector error, CFL, downloads), which synchronise it.
 * A context is not thread-safe; separate contexts may be used concurrently.
 */
#ifndef PIPEFLOW_B200_H
#define PIPEFLOW_B200_H

#ifdef __cplusplus
extern "C" {
#endif

#define PF_OK            0
#define PF_ERR_ARG      -1   /* bad argument / size mismatch                */
#define PF_ERR_CUDA     -2   /* CUDA runtime failure                        */
#define PF_ERR_SINGULAR -3   /* zero pivot in a banded or 4x4 factorisation */
#define PF_ERR_NOMEM    -4   /* device allocation failed / over budget      */
#define PF_ERR_STATE    -5   /* call out of order (e.g. step before matrices) */
#define PF_ERR_CONVERGE -6   /* corrector diverged / too many iterations    */
#define PF_ERR_NODEVICE -7   /* no CUDA device visible                      */
#define PF_ERR_CANCELLED -8  /* a served request was cancelled              */

#define PF_KL 4              /* i_KL, parameters.f90:43 */

/* precision of the transform / nonlinear-product stage */
#define PF_PREC_FP64  0      /* everything FP64 (the reference's arithmetic) */
#define PF_PREC_MIXED 1      /* FP32 FFTs and u x curl(u); FP64 elsewhere    */

/* Runtime replacement of the compile-time parameters (parameters.f90:15-51). */
typedef struct pf_config {
    int    N, K, M, Mp;          /* i_N, i_K, i_M, i_Mp                        */
    double Re, alpha;            /* d_Re, d_alpha                              */
    double dt;                   /* d_timestep (>0 fixed, <0 adaptive)         */
    double implicit;             /* d_implicit (0.51)                          */
    double dterr;                /* d_dterr    (1e-5)                          */
    double courant;              /* d_courant  (0.5)                           */
    double maxdt;                /* d_maxdt    (1e99)                          */
    int    const_flux;           /* b_const_flux                               */
    int    mirrorsym, shiftrefl, shiftrott;   /* b_mirrorsym, ...             */
    const double *r;             /* custom radial mesh (mesh.in, meshs.f90:76-88); NULL = default */
    int    precision;            /* PF_PREC_FP64 or PF_PREC_MIXED              */
} pf_config;

/* Timestep module scalars (timestep.f90:12-21). */
typedef struct pf_tim_state {
    double t, dt, dterr, corr_dt, cfl_dt;
    int    it, step, cfl_dir, new_dt, pcn;
} pf_tim_state;

typedef struct pf_ctx    pf_ctx;
typedef struct pf_coll   pf_coll;
typedef struct pf_phys   pf_phys;
typedef struct pf_mesh   pf_mesh;
typedef struct pf_lumesh pf_lumesh;

/* ---------------------------------------------------------------- context */
const char *pf_last_error(void);
int pf_version(int *major, int *minor);
/* par_precompute + mes_precompute + var_precompute + tra_precompute +
 * tim_precompute + vel_precompute (main.f90:109-114; parameters.f90:59-62;
 * meshs.f90:66-103; variables.f90:60-88; transform.fftw3.f90:35-59;
 * timestep.f90:29-40; velocity.f90:47-55).  device < 0 keeps the current one. */
int pf_ctx_create(const pf_config *cfg, int device, pf_ctx **out);
int pf_ctx_destroy(pf_ctx *ctx);
/* New physical parameters (Re, alpha, dt, implicit, dterr, courant, maxdt,
 * flags) for a context of the same N, K, M, Mp, precision and default mesh:
 * the context starts a fresh run as pf_ctx_create would, reusing its device
 * memory.  pf_vel_matrices must be called again before stepping. */
int pf_ctx_reconfigure(pf_ctx *ctx, const pf_config *cfg);
/* Run the context's work on an external cudaStream_t (NULL = own stream). */
int pf_ctx_set_stream(pf_ctx *ctx, void *cuda_stream);

/* Launch choices of a context's fused timestep.  No counterpart in the
 * reference, whose only tuning is FFTW_PATIENT planning
 * (transform.fftw3.f90:36-57).  Every choice gives the same numbers bit for
 * bit; only the speed differs.  The autotuner (pipeflow.tune) sets them by
 * timing the candidates per pipe shape.  A zero struct is the built-in
 * choice.  Setting them drops the context's captured step graphs. */
#define PF_LD_AUTO     0  /* the built-in choice (streamed factors) */
#define PF_LD_STREAMED 1  /* Helmholtz factors streamed from HBM */
#define PF_LD_REBUILT  2  /* Helmholtz factors rebuilt on chip (factorisations
                             that did not pivot, N >= 10; else streamed) */
#define PF_LD_PAIRED   3  /* streamed factors, modes k and -k paired on one
                             factor stream (pressure and Helmholtz solves) */
#define PF_LD_WARPRING 4  /* streamed Helmholtz factors, one shared-memory ring
                             per mode read by its real and imaginary lanes (the
                             pressure solve does so for every choice but
                             PF_LD_PAIRED) */
typedef struct {
    int ld_solver; /* PF_LD_* */
    int nl_mc;     /* z-pass columns per block (1..M; 0 = built-in) */
    int nl_zc;     /* theta-pass z rows per block (even, 2..32; 0 = built-in) */
    int nl_fused;  /* 1: mixed precision, the transforms of one radial point
                      in one block where that kernel is built and its plane
                      fits (0 = built-in: three passes) */
} pf_tuning;
int pf_ctx_set_tuning(pf_ctx *ctx, const pf_tuning *t);
int pf_ctx_get_tuning(const pf_ctx *ctx, pf_tuning *t);
/* How the fused nonlinear terms run with the current tuning: *passes = 1
 * (mixed precision, one block per radial point: z inverse, theta pass and z
 * forward with the (m, z) plane in shared memory) or 3 (three launches with
 * the plane in HBM). */
int pf_nl_passes(const pf_ctx *ctx, int *passes);
int pf_ctx_sync(pf_ctx *ctx);
/* H = number of harmonics (i_H1+1), Z = 3K, Th = 3M. */
int pf_ctx_dims(const pf_ctx *ctx, int *N, int *H, int *Z, int *Th);
/* Bytes of device memory held by the context (fields, factors, scratch). */
int pf_ctx_device_bytes(const pf_ctx *ctx, unsigned long long *bytes);

/* Radial mesh `mes_D` (meshs.f90:48-58): r(N), dr(KL) bands [(i*N+j)*(2KL+1)+row],
 * radLap band, dr0/dr1 [(i*(KL+1))+j] == dr0(j+1,i), intrdr(N).  Any pointer may be NULL. */
int pf_mes_get(const pf_ctx *ctx, double *r, double *dr, double *radLap,
               double *dr0, double *dr1, double *intrdr);
/* The same mesh computed on the host only (no device needed): mes_precompute
 * + mes_rdom_init (meshs.f90:66-194) for N points; custom_r may be NULL. */
int pf_mes_compute(int N, const double *custom_r, double *r, double *dr,
                   double *radLap, double *dr0, double *dr1, double *intrdr);

/* ----------------------------------------------------------------- fields */
int pf_coll_create(pf_ctx *ctx, pf_coll **out);
int pf_coll_destroy(pf_coll *c);
int pf_coll_upload(pf_coll *c, const double *re, const double *im);
int pf_coll_download(const pf_coll *c, double *re, double *im);
int pf_phys_create(pf_ctx *ctx, pf_phys **out);
int pf_phys_destroy(pf_phys *p);
int pf_phys_upload(pf_phys *p, const double *re);
int pf_phys_download(const pf_phys *p, double *re);

/* --------------------------------------------------------- variables.f90 */
int pf_var_coll_init(pf_coll *a);                                   /* :118-122 */
int pf_var_coll_copy(const pf_coll *in, pf_coll *out);              /* :128-133 */
int pf_var_coll_add(const pf_coll *ac, pf_coll *a);                 /* :139-144 */
int pf_var_coll_sub(const pf_coll *ac, pf_coll *a);                 /* :150-155 */
int pf_var_coll_dmult(double d, pf_coll *a);                        /* :161-166 */
int pf_var_coll_neg(const pf_coll *ac, pf_coll *a);                 /* :172-177 */
/* out = mes_D%dr(p) . in  (p = 1..KL) */
int pf_var_coll_meshmult(int p, const pf_coll *in, pf_coll *out);   /* :378-402 */
int pf_var_coll_curl(const pf_coll *r, const pf_coll *t, const pf_coll *z,
                     pf_coll *or_, pf_coll *ot, pf_coll *oz);       /* :408-436 */
int pf_var_coll_grad(const pf_coll *p, pf_coll *r, pf_coll *t, pf_coll *z); /* :442-459 */
int pf_var_coll_div(const pf_coll *r, const pf_coll *t, const pf_coll *z,
                    pf_coll *dv);                                   /* :465-481 */
int pf_var_coll_shift(double dt, double dz, const pf_coll *a, pf_coll *b); /* :487-528 */
int pf_var_imposesym(int i, pf_coll *r, pf_coll *t, pf_coll *z);    /* :538-618 */
/* E and the spectra Ek(0:K-1), Em(0:M-1) (either may be NULL) */
int pf_var_coll_norm(const pf_coll *a, double *E, double *Ek, double *Em); /* :718-751 */

/* -------------------------------------------------- transform.fftw3.f90 */
/* var_coll2spec + tra_spec2phys (variables.f90:184-197, transform.fftw3.f90:65-102) */
int pf_tra_coll2phys(const pf_coll *c, pf_phys *p);
/* tra_phys2spec + var_spec2coll (transform.fftw3.f90:108-147, variables.f90:281-294) */
int pf_tra_phys2coll(const pf_phys *p, pf_coll *c);

/* No counterpart in the reference.  The coll -> phys transform for callers
 * that cannot allocate device memory (their device memory belongs to another
 * allocator or pool, or they must not allocate inside their own step loop):
 * no pf_ctx, no cudaMalloc/cudaFree.  re/im are the caller's DEVICE arrays in
 * the coll host layout (re[nh*N + n]); phys is the caller's DEVICE output in
 * the phys layout ([(n*3M + t)*3K + z]); the work is queued on cuda_stream
 * (NULL = the legacy default stream).  Scratch is one static device array of
 * PF_NOALLOC_SCRATCH_BYTES per GPU: sizes with N*M*3K*16 + 64 KiB above it,
 * or with 3K or 3M outside {12,15,18,24,36,48,72,96,144,192,288,384}, are
 * rejected with PF_ERR_ARG.  All calls share the scratch, so calls that
 * overlap on the GPU race.  The first call on a device (with that device
 * current) is its set-up: it looks up the scratch address
 * (cudaGetSymbolAddress) and writes the twiddle tables of every built length
 * into the scratch with one synchronous copy; make it before any stream
 * capture.  Later calls only queue two kernels on cuda_stream.  The set-up is
 * kept for the process's life: a cudaDeviceReset on that device makes the
 * entry point unusable there. */
#define PF_NOALLOC_SCRATCH_BYTES (24u * 1024u * 1024u)
int pf_tra_coll2phys_noalloc(int N, int K, int M, const double *re, const double *im,
                             double *phys, void *cuda_stream);

/* ---------------------------------------------------------- timestep.f90 */
int pf_tim_get(const pf_ctx *ctx, pf_tim_state *s);
int pf_tim_set(pf_ctx *ctx, const pf_tim_state *s);
/* A = c1 I + c2 Lap(PM) per mode (timestep.f90:46-60) */
int pf_tim_mesh_init(pf_ctx *ctx, int PM, double c1, double c2, pf_mesh **out);
int pf_mesh_destroy(pf_mesh *A);
int pf_mesh_download(const pf_mesh *A, double *M);
/* Same matrix with axis-parity / wall rows, banded LU with partial pivoting
 * (dgbtrf semantics), skipped for BC=1 at k=m=0 (timestep.f90:67-96) */
int pf_tim_lumesh_init(pf_ctx *ctx, int PM, int BC, double c1, double c2, pf_lumesh **out);
int pf_lumesh_destroy(pf_lumesh *A);
int pf_lumesh_download(const pf_lumesh *A, double *M, int *ipiv);
/* b := A^-1 b per mode, Re and Im (dgbtrs semantics; zero for BC=1,k=m=0)
 * (timestep.f90:102-123) */
int pf_tim_lumesh_invert(int BC, const pf_lumesh *A, pf_coll *b);
/* d = A b + c (timestep.f90:130-154); d may alias b or c */
int pf_tim_meshmult(int S, const pf_mesh *A, const pf_coll *b, const pf_coll *c, pf_coll *d);
int pf_tim_zerobc(pf_coll *a);                                      /* :160-169 */
int pf_tim_nlincorr(const pf_coll *N_, pf_coll *Nn);                /* :174-184 */
int pf_tim_measurecorr(const pf_coll *c1, const pf_coll *c2, const pf_coll *c3); /* :190-207 */
int pf_tim_check_cgce(pf_ctx *ctx);                                 /* :214-253 */
int pf_tim_new_tstep(pf_ctx *ctx);                                  /* :259-278 */

/* ---------------------------------------------------------- velocity.f90 */
/* Module fields: 0..2 vel_ur,vel_ut,vel_uz; 3..5 vel_Nr,vel_Nt,vel_Nz (coll);
 * physical 0..5 vel_r,vel_t,vel_z,vel_curlr,vel_curlt,vel_curlz. */
#define PF_UR 0
#define PF_UT 1
#define PF_UZ 2
#define PF_NR 3
#define PF_NT 4
#define PF_NZ 5
int pf_vel_coll(pf_ctx *ctx, int which, pf_coll **out);
int pf_vel_phys(pf_ctx *ctx, int which, pf_phys **out);
/* Host state in / out: vel_ur, vel_ut, vel_uz in the coll host layout. */
int pf_vel_set_state(pf_ctx *ctx, const double *ur_re, const double *ur_im,
                     const double *ut_re, const double *ut_im,
                     const double *uz_re, const double *uz_im);
int pf_vel_get_state(pf_ctx *ctx, double *ur_re, double *ur_im,
                     double *ut_re, double *ut_im, double *uz_re, double *uz_im);
/* The same copy queued on the context's stream without waiting (the arrays
 * are complete once pf_ctx_sync returns; page-locked arrays let the copies of
 * many contexts overlap).  No separate reference routine: the host side of
 * io.f90's state access, batched. */
int pf_vel_get_state_async(pf_ctx *ctx, double *ur_re, double *ur_im, double *ut_re,
                           double *ut_im, double *uz_re, double *uz_im);
int pf_vel_get_scalars(const pf_ctx *ctx, double *Pr0, double *nu);
int pf_vel_imposesym(pf_ctx *ctx);                                  /* :61-74 */
int pf_vel_matrices(pf_ctx *ctx);                                   /* :120-146 */
int pf_vel_transform(pf_ctx *ctx);                                  /* :304-317 */
int pf_vel_nonlinear(pf_ctx *ctx);                                  /* :323-335 */
/* vel_transform + vel_nonlinear fused (velocity.f90:304-361): N from u in
 * three launches without materialising vel_r..vel_curlz (those module
 * fields are not updated); CFL maxima are kept for pf_vel_maxtstep. */
int pf_vel_transform_nonlinear(pf_ctx *ctx);
int pf_vel_predictor(pf_ctx *ctx);                                  /* :400-410 */
int pf_vel_corrector(pf_ctx *ctx);                                  /* :416-432 */
int pf_vel_maxtstep(pf_ctx *ctx);                                   /* :438-481 */
/* Influence data of vel_adjPPE(0): U(N,nh,6) [(c*H+nh)*N+n] and the inverted
 * 4x4 A(4,4,nh) [nh*16 + j*4 + i] == A(i+1,j+1,nh). */
int pf_vel_influence_download(const pf_ctx *ctx, double *U, double *A);

/* -------------------------------------------------------------- drivers */
/* One pass of the main.f90 loop body (main.f90:20-44): imposesym, transform,
 * nonlinear, [adaptive dt], predictor, corrector iterated until
 * tim_check_cgce says converged.  *ncorr (may be NULL) = corrector passes.
 * Returns PF_ERR_CONVERGE when tim_check_cgce reports divergence. */
int pf_timestep(pf_ctx *ctx, int *ncorr);
/* nsteps passes of steporbit's body (newton.f90:740-762): exactly one
 * corrector per step, no adaptive dt, no shift. */
int pf_steporbit(pf_ctx *ctx, int nsteps);

/* ------------------------------------------------------- orbit vectors */
/* Device side of the Newton-Krylov orbit search (newton.f90).  A vector
 * holds pf_orbit_vec_len = 8 + 6*N*H doubles in device memory: x[0..2] the
 * theta shift, z shift and period (each divided by scaleT), x[3] the
 * continuation parameter, x[4..7] unused, and from x[8] on the scaled state
 * (mode-major, then radial point, then ur/ut/uz Re/Im).  The calls work
 * through the context's velocity fields (vel_ur, vel_ut, vel_uz), as the
 * reference's routines do, and leave them holding the last state handled. */
/* The first call also fixes the alpha of the weights w: rtz2vec computes
 * them once (newton.f90:580-587), so they stay when a continuation in alpha
 * reconfigures the context. */
int pf_orbit_set_scales(pf_ctx *ctx, const double *scaleU, double scaleT); /* newton.f90:272-305 */
int pf_orbit_vec_len(const pf_ctx *ctx, long long *n);                     /* newton.f90:36 */
int pf_orbit_rtz2vec(pf_ctx *ctx, double *v);                              /* newton.f90:567-602 */
int pf_orbit_vec2rtz(pf_ctx *ctx, const double *v);                        /* newton.f90:608-643 */
/* dotprod(n_,a,b) (newton.f90:652-672): n_ = -1 skips x[0..7].  The sum
 * order is fixed, so equal inputs give equal results.  Synchronises. */
int pf_orbit_dotprod(pf_ctx *ctx, int n_, const double *a, const double *b, double *out);
/* getshiftdir(i,n,x,s), i = 1 (theta) or 2 (z) (newton.f90:533-561); s[0..7]
 * are not written. */
int pf_orbit_shiftdir(pf_ctx *ctx, int i, const double *x, double *s);
/* steporbit(ndts,x,y) without parameter continuation or output files
 * (newton.f90:721-831): y[8:] = the state ndts steps on from x, shifted back
 * by (x[0], x[1])*scaleT when ndts != 1; y[0..7] are not written.  With
 * ndts != 1, dt = x[2]*scaleT/ndts, vel_matrices runs first, and time and
 * step count advance; a single step leaves dt, time and step count as they
 * were.  y may equal x.  Returns PF_ERR_CONVERGE as pf_steporbit does. */
int pf_orbit_step(pf_ctx *ctx, int ndts, const double *x, double *y);
/* Perturbation energy and friction diagnostics of io.f90:501-514, 627-639. */
int pf_diag_energy(pf_ctx *ctx, double *E);
int pf_diag_friction(pf_ctx *ctx, double *Ub, double *Uc, double *Ufr);

/* ------------------------------------------------------------ util hook */
/* The plug-in hook of main.f90: var_null(2) after every evaluation of the
 * nonlinear terms, var_null(1) once per step before the predictor
 * (main.f90:23,30,38); pf_timestep calls it when a plug-in is set (orbit
 * steps, like newton.f90's steporbit, do not call it).  The Coriolis and
 * Carreau-Yasuda plug-ins are device work only and run inside the step's
 * CUDA graphs; LES (its update_nu_r reads max nu_t back to the host) and a
 * host callback make pf_timestep run eagerly.  Built-in plug-ins, on the
 * device:
 *   PF_UTIL_CORIOLIS: params Ek0, phi -- Coriolis.f90:13-73 (Mp must be 1)
 *   PF_UTIL_CARREAU_YASUDA: params rho, radius, mu_0, mu_inf, lam_CY, n_CY,
 *     a_CY[, fc1] -- nonnewtonian.f90:32-246; sets one corrector pass per
 *     step (tim_pcn = 1) as the reference does
 *   PF_UTIL_LES: params model (1 Smagorinsky, 2 Vreman), C_s, filter (1, 2,
 *     3), A_plus -- the eddy-viscosity terms of LES.f90:102-339 (get_nu,
 *     update_nu_r with its re-factorisation when the reference viscosity
 *     moves, update_nonlin_terms); one corrector pass per step as there.
 *     Its var_null(1) side (LES.f90:51-56: bisect, profiles, vel_Retau.dat)
 *     is output and is not built.
 * A host callback fn(ctx, flag, user) runs after the built-in at both
 * flags, for plug-ins written against this ABI (adding to vel_Nr/Nt/Nz
 * through pf_vel_coll and pf_var_coll_add).  pf_util runs the hook once, for
 * drivers that step through the module calls themselves. */
#define PF_UTIL_NONE            0
#define PF_UTIL_CORIOLIS        1
#define PF_UTIL_CARREAU_YASUDA  2
#define PF_UTIL_LES             3
typedef void (*pf_util_fn)(pf_ctx *ctx, int flag, void *user);
int pf_util_set(pf_ctx *ctx, int kind, const double *params, int nparams);
int pf_util_set_callback(pf_ctx *ctx, pf_util_fn fn, void *user);
int pf_util(pf_ctx *ctx, int flag);
/* nu at the wall (mean mode), min and max over the grid from the last
 * Carreau-Yasuda or LES evaluation (write_Re_nu, nonnewtonian.f90:302-318;
 * for LES, the eddy viscosity nu_t whose maximum is LES.f90's nu_max);
 * PF_ERR_STATE before the first evaluation */
int pf_util_nu_stats(pf_ctx *ctx, double *nu_wall, double *nu_min, double *nu_max);

/* ------------------------------------------------------------ state files */
/* The netCDF-3 state files of io.f90 (state*.cdf.dat / state.cdf.in):
 * dimensions r, H, ReIm; global attributes t, Re, alpha; variables r, dt,
 * dtcor, dtcfl and Ur, Ut, Uz(ReIm, H, r) with attributes K, M, Mp.  Written
 * and parsed without libnetcdf (the format is the published netCDF classic /
 * 64-bit-offset layout).
 * pf_io_save_state: io_save_state (io.f90:303-378) of the context's state,
 *   mesh, t, dt, corr/CFL dt, Re and alpha to `path`.
 * pf_io_load_state: io_load_state (io.f90:98-226) into the context: radial
 *   interpolation (io_interp_wts/io_interp, io.f90:232-288) when the file's
 *   mesh differs, K/M re-truncation with zero fill, t from the file if
 *   flags has PF_IO_TIME_FROM_FILE (the reference's d_time < 0), dt from the
 *   file for an adaptive-dt run (dt < 0) else the configured dt, and the
 *   file's dtcor/dtcfl if present.  *changes (may be NULL) gets bit 1 if
 *   interpolated, 2 if K, 4 if M, 8 if Mp differed.  New dt needs
 *   pf_vel_matrices before stepping, as in the reference's initialise.
 * pf_state_write / pf_state_read: the same without a context or a GPU, on
 *   host arrays in pf_vel_set_state's layout (H x N, radial index fastest);
 *   r is the N radial points written / to interpolate onto; scalars holds
 *   t, Re, alpha, dt, dtcor, dtcfl (read: NaN where the file has none). */
#define PF_IO_TIME_FROM_FILE 1
int pf_io_save_state(pf_ctx *ctx, const char *path);
int pf_io_load_state(pf_ctx *ctx, const char *path, int flags, int *changes);
int pf_state_write(const char *path, int N, int K, int M, int Mp, const double *r, const double *ur_re,
                   const double *ur_im, const double *ut_re, const double *ut_im, const double *uz_re,
                   const double *uz_im, const double *scalars);
int pf_state_read(const char *path, int N, int K, int M, int Mp, const double *r, double *ur_re, double *ur_im,
                  double *ut_re, double *ut_im, double *uz_re, double *uz_im, double *scalars, int *changes);

/* ----------------------------------------------------------------- batches */
/* Many independent pipes of uneven (N, K, M, Re, alpha, dt) advanced together;
 * one timestep of the batch is a single CUDA graph.  Where every pipe fits
 * the batched kernels (fixed dt, N <= 128, built transform lengths 12 to 384,
 * either precision, mean-mode symmetry only) each stage is one launch over the tiles
 * of all pipes; otherwise the graph holds one kernel chain per pipe.  Each
 * pipe's arithmetic is the lone-pipe path, so results are the same alone and
 * in the batch.  No single reference routine: this drives the main.f90 loop
 * body (main.f90:20-44) or steporbit's (newton.f90:740-762) for every pipe. */
typedef struct pf_batch pf_batch;
int pf_batch_create(int npipes, const pf_config *cfgs, int device, pf_batch **out);
int pf_batch_destroy(pf_batch *b);
/* The context of pipe i (owned by the batch): set its state, read results. */
int pf_batch_pipe(pf_batch *b, int i, pf_ctx **out);
/* vel_matrices for every pipe. */
int pf_batch_matrices(pf_batch *b);
/* nsteps timesteps of every pipe; orbit=0 iterates each pipe's corrector to
 * convergence, orbit=1 takes exactly one corrector pass.  *corr_passes
 * (may be NULL) = corrector passes summed over pipes and steps. */
int pf_batch_step(pf_batch *b, int nsteps, int orbit, long long *corr_passes);
int pf_batch_sync(pf_batch *b);
/* The cudaStream_t the batch's graphs are launched on (for event timing). */
int pf_batch_stream(pf_batch *b, void **stream);
/* Pipelined state I/O of a whole batch.  No single reference routine: the
 * host side of io.f90's state access (what pf_vel_set_state and
 * pf_vel_get_state do per pipe), for every pipe at once and overlapped with
 * stepping.  A state block holds every pipe's state in batch order; pipe i
 * takes 6*N_i*H_i doubles: ur Re, ur Im, ut Re, ut Im, uz Re, uz Im, each
 * H_i x N_i with the radial index fastest (%Re(n,nh)).  There are two input
 * and two output slots on the device and one copy stream per direction:
 *   put_states(s+1); step_io(s); get_states(s)
 * with s alternating 0, 1 uploads the next block and downloads the last one
 * while the step in between computes.  The first use allocates four blocks
 * of device staging.  Host blocks should be page-locked for the copies to
 * overlap.
 * pf_batch_io_bytes: bytes of one state block for the current membership.
 * pf_batch_put_states: queue the upload of `host` into input slot `slot`;
 *   the host block may change once a pf_batch_step_io(slot, nsteps >= 1)
 *   has returned, or after pf_batch_io_sync.
 * pf_batch_step_io: every pipe's velocity from input slot `slot`, nsteps
 *   steps as pf_batch_step, then the states into output slot `slot`;
 *   PF_ERR_STATE if nothing was put into the slot since its last use.
 * pf_batch_get_states: queue the download of output slot `slot` into `host`;
 *   complete after pf_batch_io_wait(slot) or pf_batch_io_sync. */
int pf_batch_io_bytes(pf_batch *b, unsigned long long *bytes);
int pf_batch_put_states(pf_batch *b, int slot, const double *host);
int pf_batch_step_io(pf_batch *b, int slot, int nsteps, int orbit, long long *corr_passes);
int pf_batch_get_states(pf_batch *b, int slot, double *host);
int pf_batch_io_wait(pf_batch *b, int slot);
int pf_batch_io_sync(pf_batch *b);
/* Kernel-category event timing for every pipe (see pf_prof_enable), and the
 * totals summed over the pipes.  Kernel spans of different pipes overlap in
 * time, so per-launch durations here include the sharing of the GPU. */
int pf_batch_prof_enable(pf_batch *b, int mask);
int pf_batch_prof_read(pf_batch *b, int cat, double *ms, unsigned long long *launches);
/* Only the spans of the stage-batched launches (each covers every pipe of the
 * batch), without the per-pipe launches such as one pipe's extra corrector
 * pass: these are the spans whose bytes are the whole batch's. */
int pf_batch_prof_read_staged(pf_batch *b, int cat, double *ms, unsigned long long *launches);
/* Number of pipes, and membership changes.  A batch made with npipes = 0
 * starts empty.  pf_batch_attach adds a context the caller created and still
 * owns (same device; it must outlive its membership); pf_batch_detach removes
 * it.  The batch's launches are rebuilt at the next step. */
int pf_batch_size(pf_batch *b, int *n);
int pf_batch_attach(pf_batch *b, pf_ctx *c);
int pf_batch_detach(pf_batch *b, pf_ctx *c);
/* on = 1 (default): steps replay captured CUDA graphs; on = 0: every step
 * launches its kernels directly (for membership that changes every step). */
int pf_batch_set_graphs(pf_batch *b, int on);
/* Kernels launched so far by the batch (its pipes' and its batched ones). */
int pf_batch_launches(pf_batch *b, unsigned long long *n);
/* *staged = 1 when the batch's graphs launch each stage once for all pipes. */
int pf_batch_staged(pf_batch *b, int *staged);
/* Form of the stage-batched transform stages.  No counterpart in the
 * reference (it runs one state per process).  on = 1: each of the three
 * transform stages (z inverse, theta pass with u x curl(u), z forward) is
 * one persistent launch whose blocks take the tiles of every pipe, of every
 * transform length, from one work list (longest lengths first), where every
 * pipe is in mixed precision with transform lengths from 36 to 192; on = 0 (the
 * default): one launch per stage and transform length, the lengths' launches
 * running concurrently.  The numbers are bitwise the same either way; the
 * autotuner (pipeflow.tune) times both.  A change drops the batch's graphs. */
int pf_batch_set_worklist(pf_batch *b, int on);
int pf_batch_get_worklist(pf_batch *b, int *on);

/* ---------------------------------------------------------------- serving */
/* Requests "advance this state by nsteps timesteps" (time-T maps, e.g. the
 * Newton-Krylov evaluations of newton.f90:399-465 through steporbit,
 * newton.f90:721-787) served with continuous batching: every admitted
 * request's state stays resident in its own context, and all of them advance
 * together in one batch (stage-batched launches).  Between batch steps the
 * server admits queued requests in arrival order while the HBM budget and the
 * slot cap allow (reusing pooled contexts of the same shape) and retires the
 * finished ones.  A request's result equals the lone-pipe result exactly.
 * No single reference routine: the reference runs one state per process. */
typedef struct pf_server pf_server;
/* orbit = 1: steporbit steps (one corrector each); 0: main-loop steps. */
int pf_serve_create(int device, unsigned long long hbm_budget_bytes, int max_active, int orbit,
                    pf_server **out);
int pf_serve_destroy(pf_server *s);
/* Queue a request (cfg->dt > 0, default mesh); the six arrays (reference coll
 * layout, H*N doubles each) are copied. */
int pf_serve_submit(pf_server *s, const pf_config *cfg, int nsteps,
                    const double *ur_re, const double *ur_im, const double *ut_re,
                    const double *ut_im, const double *uz_re, const double *uz_im, long long *id);
/* Admit what fits, advance every admitted request one timestep, retire the
 * finished; *admitted / *finished (may be NULL) count this call's. */
int pf_serve_step(pf_server *s, int *admitted, int *finished);
/* Ids finished since the last call (up to cap). */
int pf_serve_finished(pf_server *s, long long *ids, int cap, int *n);
/* Cancel a queued or running request: it leaves the queue or the batch at
 * once (its context goes back to the pool) and is reported finished; its
 * pf_serve_result returns PF_ERR_CANCELLED.  PF_ERR_STATE if the request has
 * already finished, PF_ERR_ARG for an unknown id.  No reference routine: the
 * reference runs one state per process. */
int pf_serve_cancel(pf_server *s, long long id);
/* Final state of a finished request; the request is forgotten afterwards.
 * A request that failed returns its own error instead, alone: the corrector
 * check's abort (PF_ERR_CONVERGE with tim_check_cgce's message,
 * timestep.f90:222-240), a non-finite corrector error (a NaN or Inf in its
 * state; PF_ERR_CONVERGE), a failed admission, or PF_ERR_CANCELLED.  The
 * other requests of the batch are not affected. */
int pf_serve_result(pf_server *s, long long id, double *ur_re, double *ur_im, double *ut_re,
                    double *ut_im, double *uz_re, double *uz_im);
int pf_serve_stats(pf_server *s, int *queued, int *active, int *pooled, unsigned long long *bytes,
                   long long *steps);
/* The batch the server steps (its stream, launch counter and profiling). */
int pf_serve_batch(pf_server *s, pf_batch **b);

/* ------------------------------------------------------- instrumentation */
/* Kernel categories timed by CUDA events when profiling is on (the reference
 * has only the CPU-time clk_time, main.f90:175-186). */
#define PF_K_ZINV     0   /* z pass spectral -> (m,z) columns              */
#define PF_K_THINV    1   /* theta pass (c2r) -> physical                   */
#define PF_K_THFWD    2   /* theta pass (r2c), fused u x curl(u)            */
#define PF_K_ZFWD     3   /* z pass -> spectral, truncation                 */
#define PF_K_LUSOLVE  4   /* banded solves (the Helmholtz u+, u-, uz ones in
                             the fused step)                                 */
#define PF_K_STENCIL  5   /* meshmult / curl / grad / div / tim_meshmult    */
#define PF_K_EW       6   /* elementwise, symmetry, reductions, transfers   */
#define PF_K_INFL     7   /* influence correction, flux, addHPF             */
#define PF_K_FACTOR   8   /* banded LU factorisation (vel_matrices)          */
#define PF_K_STEP     9   /* fused per-mode step kernels                     */
#define PF_K_PPE     10   /* pressure-Poisson banded solve of the fused step */
#define PF_K_NCAT    11
/* Count of this library's kernel launches on the context since creation. */
int pf_ctx_launches(const pf_ctx *ctx, unsigned long long *n);
/* Event timing for the categories whose bit (1 << PF_K_*) is set in mask;
 * 0 disables.  Each call clears the totals. */
int pf_prof_enable(pf_ctx *ctx, int mask);
/* Total device milliseconds and launches of category `cat` since enabling
 * (synchronises the stream). */
int pf_prof_read(pf_ctx *ctx, int cat, double *ms, unsigned long long *launches);

#ifdef __cplusplus
}
#endif
#endif /* PIPEFLOW_B200_H */
