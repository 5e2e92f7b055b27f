// Internal definitions shared by the pipeflow_b200 translation units.
//
// Device data layout (all FP64 unless noted):
//   coll field  : double2 d[n*Hp + nh]   (complex, harmonic index fastest, row
//                 pitch Hp = H rounded up to 32).  The reference's coll type is
//                 (n fastest); storing the harmonic index fastest makes the
//                 per-radial-point transform tiles contiguous and keeps the
//                 per-mode solves coalesced across modes, so the reference's
//                 coll<->spec transposes (variables.f90:184-370) vanish on the
//                 device.  Host<->device copies reorder once.
//   phys field  : double d[(n*Th + t)*Z + z]  (identical to the reference)
//   LU factors  : double lu[(row*N + col)*Hp + nh], row = LAPACK band row-1
//                 (0..3KL), pivots uint8 piv[col*Hp + nh] = ipiv-col (0..KL)
//   FFT scratch : complex T[((c*N + n)*M + m)*Z + z]
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <algorithm>
#include <string>
#include <vector>
#include "pipeflow_b200.h"

#define KL PF_KL
#define KV (2 * PF_KL)          // LAPACK KV = KU+KL
#define NBAND (2 * PF_KL + 1)   // rows of a mesh band
#define NLU (3 * PF_KL + 1)     // rows of a lumesh band (LDAB)

// ------------------------------------------------------------------ errors
void pf_set_error(const char *fmt, ...);
#define PF_CUDA(call)                                                        \
    do {                                                                     \
        cudaError_t e_ = (call);                                             \
        if (e_ != cudaSuccess) {                                             \
            pf_set_error("%s:%d %s: %s", __FILE__, __LINE__, #call,          \
                         cudaGetErrorString(e_));                            \
            return PF_ERR_CUDA;                                              \
        }                                                                    \
    } while (0)
#define PF_CHECK_LAUNCH() PF_CUDA(cudaGetLastError())
#define PF_TRY(expr)                                                         \
    do {                                                                     \
        int s_ = (expr);                                                     \
        if (s_ != PF_OK) return s_;                                          \
    } while (0)
#define PF_ARG(cond, msg)                                                    \
    do {                                                                     \
        if (!(cond)) {                                                       \
            pf_set_error("%s", msg);                                         \
            return PF_ERR_ARG;                                               \
        }                                                                    \
    } while (0)

// ---------------------------------------------------------------- geometry
struct Geo {
    int N, K, M, Mp, H, Hp, Z, Th;
    double alpha, Re;
};

// harmonic index -> (k, m): inverse of nh = m*(2K-1)+k (parallel.h:27-38)
__host__ __device__ inline void mode_km(int nh, int K, int &k, int &m) {
    if (nh < K) {
        m = 0;
        k = nh;
    } else {
        m = (nh + K - 1) / (2 * K - 1);
        k = nh - m * (2 * K - 1);
    }
}

// Compact index of the modes with k >= 0 (c = m*K + |k|, M*K of them), the
// layout of the factor copies the streamed solves read, and its padded size.
__host__ __device__ inline int mode_compact(int nh, int K) {
    int k = 0, m = 0;
    mode_km(nh, K, k, m);
    return m * K + (k < 0 ? -k : k);
}
inline int pf_compact_modes_padded(const Geo &g) { return (g.M * g.K + 31) / 32 * 32; }

// Radial mesh on the device (meshs.f90:48-55).
struct DevMesh {
    const double *rp;      // r^j, j=-3..3: rp[(j+3)*N + n]
    const double *dr;      // dr(1..KL) bands: dr[((p-1)*NBAND + row)*N + col]
    const double *radLap;  // [row*N + col]
    const double *dr0;     // dr0[i*(KL+1) + j] == dr0(j+1, i)
    const double *dr1;     // dr1[i*(KL+1) + j] == dr1(j+1, i)
    const double *intrdr;  // [n]
    const double *velU;    // 1 - r^2
    const double *velUp;   // -2 r
};

// Host copy of the mesh (same layouts as DevMesh).
struct HostMesh {
    std::vector<double> r, rp, dr, radLap, dr0, dr1, intrdr;
};
int pf_build_mesh(int N, const double *custom_r, HostMesh &hm);

// Entry A(r, c), |r - c| <= KL, 0 <= r, c < N, of the system c1 I + c2 Lap(PM)
// for mode (k, m) with the axis-parity first row dr0(:, 1-S) and the wall row
// dr1(:, BC) (timestep.f90:46-90).  Every product and sum is rounded
// explicitly (no contraction into fma), so every kernel that assembles an
// entry gets the same bits: the factorisation (k_lu_factor) and the fused
// Helmholtz solve that rebuilds its factors on chip.  The matrices of (k, m)
// and (-k, m) are bitwise equal.
__device__ __forceinline__ double lumesh_entry(const DevMesh &dm, int N, int Mp, double alpha, int PM, int BC,
                                               double c1, double c2, int k, int m, int S, int r, int c) {
    if (r == 0) return dm.dr0[(1 - S) * (PF_KL + 1) + c];
    if (r == N - 1) return dm.dr1[BC * (PF_KL + 1) + (c - (N - 1 - PF_KL))];
    double v = __dmul_rn(c2, dm.radLap[(PF_KL + r - c) * N + c]);
    if (r == c) {
        const double r2m = dm.rp[1 * N + c];
        // d = -m^2 Mp^2 / r^2 - alpha^2 k^2, and -1/r^2 - 2 PM m Mp / r^2 for u+-
        const double t1 = __dmul_rn(__dmul_rn(__dmul_rn(__dmul_rn(r2m, (double)Mp), (double)m), (double)Mp), (double)m);
        const double t2 = __dmul_rn(__dmul_rn(__dmul_rn(alpha, (double)k), alpha), (double)k);
        double d = __dsub_rn(-t1, t2);
        if (PM != 0)
            d = __dsub_rn(__dsub_rn(d, r2m),
                          __dmul_rn(__dmul_rn(__dmul_rn(2.0 * PM, (double)Mp), (double)m), r2m));
        v = __dadd_rn(__dadd_rn(v, __dmul_rn(c2, d)), c1);
    }
    return v;
}

// Device scalars of one context.
struct DevScalars {
    double Pr0;                      // vel_Pr0
    double flux_d1;                  // vel_adjustFlux d1
    unsigned long long dterr2_bits;  // max |corr|^2 as ordered bits
    int info;                        // first singular pivot (1-based col), 0 = ok
    int pad;
};

// Mixed-radix FFT plan of length L: radices in application order.
struct FFTPlan {
    int L, nf;
    int f[16];
};
int pf_make_plan(int L, FFTPlan &p);

struct pf_ctx;

struct pf_coll {
    pf_ctx *ctx;
    double2 *d;
};
struct pf_phys {
    pf_ctx *ctx;
    double *d;
};
struct pf_mesh {
    pf_ctx *ctx;
    int PM;
    double c1, c2;
};
struct pf_lumesh {
    pf_ctx *ctx;
    int PM, BC;
    int pivoted;         // host copy: any row interchange in the factorisation
    double *pivd;        // pivot offsets as doubles [col*Hp + nh] (context sets only)
    double c1, c2;
    double *lu;
    unsigned char *piv;
    // context sets only: the factors and pivots (as doubles) of the modes
    // with k >= 0, [(row*N + col)*Hcp + c] and [col*Hcp + c] with
    // c = m*K + |k|.  The matrix of mode (-k, m) is bitwise that of (k, m)
    // (k enters as alpha*k*alpha*k only, timestep.f90:76), so its factors are
    // too; the streamed solves read this copy and fetch half the factor bytes.
    double *luc;
    double *pivdc;
};

struct pf_ctx {
    pf_config cfg;
    Geo g;
    int device;
    cudaStream_t stream;
    bool own_stream;
    HostMesh hm;
    DevMesh dm;
    double *dmesh_mem;  // backing store of dm
    FFTPlan planZ, planT;
    double2 *twZ, *twT;  // exp(+2 pi i t/L), t=0..L-1, FP64
    float2 *twZf, *twTf; // same in FP32 (mixed precision)
    DevScalars *dsc;     // device scalars
    DevScalars *hsc;     // pinned host mirror
    unsigned long long bytes;
    // timestep module (timestep.f90:12-21)
    pf_tim_state tim;
    double lasterr;
    int newdt_i;
    // velocity module (velocity.f90:14-39)
    pf_coll vel[6];      // ur ut uz Nr Nt Nz
    pf_coll prev[6];     // ur_ ut_ uz_ Nr_ Nt_ Nz_
    pf_coll save[3];     // corrector's r,t,z copies
    pf_coll s[8];        // scratch
    pf_phys phys[6];     // vel_r .. vel_curlz
    pf_lumesh LNp, LDp, LDm, LDz;
    pf_mesh Ltp, Ltm, Ltz;
    bool LNp_set, matrices_ready;
    bool custom_mesh;  // built from a caller-supplied radial mesh
    unsigned long long matrices_gen;  // bumped by every vel_matrices and tuning change
    pf_tuning tune;      // launch choices (zero = built-in)
    int last_status;     // corrector check of the last batched step (PF_OK or the abort)
    std::string last_error;  // its message
    double vel_nu;
    double *U;           // influence solutions [(c*N + n)*Hp + nh], c=0..5
    double *Ainv;        // inverted 4x4 [(i*4+j)*Hp + nh] == A(i+1,j+1,nh)
    double *Ui;          // flux influence vector [N]
    double *red;         // reduction scratch (>= 3*N + H doubles)
    double *mpart;       // FP64 mean-mode partial sums [ceil(H/32)][N][3]
    // Newton-Krylov vectors (newton.f90:36-37): scaleU, scaleT, dot partials
    double orbit_scaleU[3], orbit_scaleT;
    double orbit_walpha;  // alpha of the vector weights, fixed when the scales are set
    bool orbit_set;
    double *orbit_red;   // ORBIT_DOT_BLOCKS + 1 doubles
    // util plug-in (var_null hook of main.f90): built-in kind, its
    // parameters, device scratch, host callback, nu diagnostics
    int util_kind;
    double util_par[8];
    double *util_phys;
    int util_nphys;
    double *util_coll;
    int util_ncoll;
    pf_util_fn util_cb;
    void *util_user;
    double *util_diag_d;
    double *util_tab;    // per-radial-point tables of a plug-in (LES filter widths)
    unsigned long long util_evals;  // plug-in evaluations since pf_util_set
    unsigned long long *cflmax;  // 3*N CFL maxima of the last fused transform
    bool cfl_fused;              // cflmax is current (else use vel_r/t/z)
    int *anypiv;         // per LU set: 1 if dgbtf2 swapped any row
    void *T;             // FFT scratch: 6*N*M*Z complex (FP64)
    size_t T_bytes;
    int zinv_mc, zfwd_mc, th_zc;   // tile sizes
    std::vector<void *> allocs;    // everything to free
    // CUDA graphs of the timestep: main[p] = imposesym, nonlinear terms,
    // predictor, nonlinear terms, corrector starting from pointer parity p;
    // corr[q] = nonlinear terms + corrector at parity q
    int parity;                    // vel/prev pointer swap state
    bool use_graphs, graph_warm;
    cudaGraphExec_t g_main[2], g_corr[2];
    unsigned long long g_main_n[2], g_corr_n[2];
    // event pairs recorded inside each graph (profiled categories), and the
    // graphs replayed since the last host synchronisation
    std::vector<std::pair<int, std::pair<cudaEvent_t, cudaEvent_t>>> g_ev[4];
    std::vector<int> g_pending;
    // instrumentation
    unsigned long long launches;
    int prof_mask;
    std::vector<cudaEvent_t> ev_pool;                 // free events
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> ev_open[PF_K_NCAT];
    double prof_ms[PF_K_NCAT];
    unsigned long long prof_n[PF_K_NCAT];
};

// Records a start/stop event pair around the launches in its scope when
// profiling is enabled on the context.  While the stream is being captured
// the records are made external, so the graph gets real event-record nodes
// whose times can be read after each replay.
cudaEvent_t pf_event_get(pf_ctx *ctx);
inline void pf_event_record(cudaEvent_t e, cudaStream_t s) {
    cudaStreamCaptureStatus st = cudaStreamCaptureStatusNone;
    cudaStreamIsCapturing(s, &st);
    if (st == cudaStreamCaptureStatusActive)
        cudaEventRecordWithFlags(e, s, cudaEventRecordExternal);
    else
        cudaEventRecord(e, s);
}
struct ProfScope {
    pf_ctx *ctx;
    int cat;
    cudaEvent_t a;
    ProfScope(pf_ctx *c, int k) : ctx(c), cat(k), a(nullptr) {
        if (ctx->prof_mask & (1 << k)) {
            a = pf_event_get(ctx);
            pf_event_record(a, ctx->stream);
        }
    }
    ~ProfScope() {
        if (a) {
            cudaEvent_t b = pf_event_get(ctx);
            pf_event_record(b, ctx->stream);
            ctx->ev_open[cat].push_back({a, b});
        }
    }
};
#define PF_LAUNCHED(ctx)     \
    do {                     \
        (ctx)->launches++;   \
        PF_CHECK_LAUNCH();   \
    } while (0)

// -------------------------------------------------------------- utilities
int pf_alloc(pf_ctx *ctx, void **p, size_t bytes);
// Raise, never lower, a kernel's dynamic shared-memory limit on the current
// device: a limit lowered for a small launch would no longer cover a larger
// launch of the same kernel that a CUDA graph captured earlier.
int pf_raise_smem(const void *fn, size_t bytes);
int pf_coll_init_storage(pf_ctx *ctx, pf_coll *c);
int pf_phys_init_storage(pf_ctx *ctx, pf_phys *p);
inline double bits_to_double(unsigned long long b) {
    double d;
    std::memcpy(&d, &b, sizeof(d));
    return d;
}
// p[i] for i in 0..2 without indexing the array at run time, so a struct
// of pointers copied into a kernel stays in registers
template <typename T> __device__ __forceinline__ T pick3(T const (&p)[3], int i) {
    return i == 0 ? p[0] : (i == 1 ? p[1] : p[2]);
}

// x / d for 0 <= x < 2^22 and d > 0, given inv = 1.0f / d: a float
// reciprocal estimate corrected by one step (cheaper than a run-time integer
// division inside index loops)
__device__ __forceinline__ int fdiv(int x, int d, float inv) {
    int q = __float2int_rz((float)x * inv);
    const int r = x - q * d;
    if (r < 0) --q;
    else if (r >= d) ++q;
    return q;
}

// partial sums of pf_orbit_dotprod (a fixed count keeps the sum order fixed)
#define ORBIT_DOT_BLOCKS 256

inline unsigned grid1(long long n, int block) {
    return (unsigned)((n + block - 1) / block);
}

// launchers implemented in the .cu files (all on ctx->stream)
enum EwOp {
    EW_ZERO, EW_COPY, EW_ADD, EW_SUB, EW_NEG, EW_DMULT, EW_RT2PM, EW_PM2RT,
    EW_NLINCORR, EW_SUBFROM
};
int pf_launch_ew(pf_ctx *ctx, EwOp op, const double2 *a, const double2 *b,
                 double2 *o1, double2 *o2, double s);
int pf_launch_zerobc(pf_ctx *ctx, double2 *a);
int pf_launch_meshmult_dr(pf_ctx *ctx, int p, const double2 *in, double2 *out);
int pf_launch_curl(pf_ctx *ctx, const double2 *r, const double2 *t, const double2 *z,
                   double2 *or_, double2 *ot, double2 *oz);
int pf_launch_grad(pf_ctx *ctx, const double2 *p, double2 *r, double2 *t, double2 *z);
int pf_launch_div(pf_ctx *ctx, const double2 *r, const double2 *t, const double2 *z,
                  double2 *dv);
int pf_launch_tim_meshmult(pf_ctx *ctx, const pf_mesh *A, const double2 *b,
                           const double2 *c, double2 *d);
int pf_launch_imposesym(pf_ctx *ctx, int i, double2 *r, double2 *t, double2 *z);
int pf_launch_measurecorr(pf_ctx *ctx, const double2 *a0, const double2 *b0,
                          const double2 *a1, const double2 *b1,
                          const double2 *a2, const double2 *b2, bool reset);
int pf_launch_addHPF(pf_ctx *ctx);
int pf_launch_lu_factor(pf_ctx *ctx, pf_lumesh *A);
int pf_launch_lu_solve(pf_ctx *ctx, int BC, const pf_lumesh *A, double2 *b);
int pf_launch_adjppe2(pf_ctx *ctx);
int pf_launch_flux1(pf_ctx *ctx);
int pf_launch_zero_mode0(pf_ctx *ctx);
int pf_vel_matrices_impl(pf_ctx *ctx);
int pf_launch_coll2phys(pf_ctx *ctx, int ncomp, const double2 *const *src,
                        double *const *dst);
int pf_launch_phys2coll(pf_ctx *ctx, int ncomp, const double *const *src,
                        double2 *const *dst, bool cross);
int pf_launch_maxtstep(pf_ctx *ctx, double *dt3);
int pf_norm_host(pf_ctx *ctx, const double2 *a, double *E, double *Ek, double *Em);
bool pf_nl_fused_supported(const pf_ctx *ctx);
int pf_nl_tiles_check(const pf_ctx *ctx, const pf_tuning *t);
bool pf_util_active(const pf_ctx *ctx);
int pf_util_run(pf_ctx *ctx, int flag);

// Batched launches: one launch per stage over the tiles of many pipes.
// Stage timing of such launches (event pairs on the launching stream, made
// external while it is captured) is kept per category in a pf_stage_prof.
struct pf_stage_prof {
    int mask = 0;
    std::vector<cudaEvent_t> pool;  // free events
    struct Open {
        int cat;
        cudaEvent_t a, b;
    };
    std::vector<Open> open;  // recorded pairs not yet read
    double ms[PF_K_NCAT] = {};
    unsigned long long n[PF_K_NCAT] = {};
    cudaEvent_t get() {
        cudaEvent_t e = nullptr;
        if (!pool.empty()) {
            e = pool.back();
            pool.pop_back();
        } else {
            cudaEventCreate(&e);
        }
        return e;
    }
};
struct StageScope {
    pf_stage_prof *p;
    int cat;
    cudaStream_t s;
    cudaEvent_t a;
    StageScope(pf_stage_prof *p_, int k, cudaStream_t s_) : p(p_), cat(k), s(s_), a(nullptr) {
        if (p && (p->mask & (1 << k))) {
            a = p->get();
            pf_event_record(a, s);
        }
    }
    ~StageScope() {
        if (a) {
            cudaEvent_t b = p->get();
            pf_event_record(b, s);
            p->open.push_back({cat, a, b});
        }
    }
};
struct pf_nl_batch;
bool pf_nl_batch_supported(pf_ctx *const *pipes, int n);
int pf_nl_batch_build(pf_ctx *const *pipes, int n, bool worklist, pf_nl_batch **out);
int pf_nl_batch_launch(pf_nl_batch *b, int state, cudaStream_t st, pf_stage_prof *prof, unsigned long long *nk);
void pf_nl_batch_free(pf_nl_batch *b);
struct pf_step_batch;
int pf_step_batch_build(pf_ctx *const *pipes, int n, pf_step_batch **out);
int pf_step_batch_launch(pf_step_batch *b, int state, int corrector, cudaStream_t st, pf_stage_prof *prof,
                         unsigned long long *nk);
void pf_step_batch_free(pf_step_batch *b);
int pf_launch_nl_fused(pf_ctx *ctx);
int pf_vel_step_fused(pf_ctx *ctx, int corrector);
void pf_graphs_reset(pf_ctx *ctx);
int pf_transform_nonlinear(pf_ctx *ctx);
int pf_read_dterr(pf_ctx *ctx);
bool pf_fused_step_ok(const pf_ctx *ctx);
void pf_graph_events_collect(pf_ctx *ctx);  // after a host sync
