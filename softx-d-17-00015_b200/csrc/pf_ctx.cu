// Context, device memory, field handles and host<->device transfer.
#include <cmath>
#include <cstdarg>
#include <cstring>
#include <mutex>
#include <vector>
#include "pf_internal.cuh"

static thread_local char g_err[512] = "";

void pf_set_error(const char *fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
}

extern "C" const char *pf_last_error(void) { return g_err; }

extern "C" int pf_version(int *major, int *minor) {
    if (major) *major = 1;
    if (minor) *minor = 0;
    return PF_OK;
}

int pf_raise_smem(const void *fn, size_t bytes) {
    struct Limit {
        const void *fn;
        int device;
        size_t bytes;
    };
    static std::mutex mu;
    static std::vector<Limit> limits;
    int dev = 0;
    PF_CUDA(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lock(mu);
    Limit *hit = nullptr;
    for (Limit &l : limits)
        if (l.fn == fn && l.device == dev) hit = &l;
    if (hit && hit->bytes >= bytes) return PF_OK;
    PF_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
    if (hit) hit->bytes = bytes;
    else limits.push_back(Limit{fn, dev, bytes});
    return PF_OK;
}

int pf_alloc(pf_ctx *ctx, void **p, size_t bytes) {
    *p = nullptr;
    if (bytes == 0) bytes = 16;
    cudaError_t e = cudaMalloc(p, bytes);
    if (e != cudaSuccess) {
        pf_set_error("cudaMalloc(%zu): %s", bytes, cudaGetErrorString(e));
        return e == cudaErrorMemoryAllocation ? PF_ERR_NOMEM : PF_ERR_CUDA;
    }
    ctx->allocs.push_back(*p);
    ctx->bytes += bytes;
    PF_CUDA(cudaMemsetAsync(*p, 0, bytes, ctx->stream));
    return PF_OK;
}

static size_t coll_bytes(const pf_ctx *ctx) {
    return (size_t)ctx->g.N * ctx->g.Hp * sizeof(double2);
}
static size_t phys_bytes(const pf_ctx *ctx) {
    return (size_t)ctx->g.N * ctx->g.Th * ctx->g.Z * sizeof(double);
}

int pf_coll_init_storage(pf_ctx *ctx, pf_coll *c) {
    c->ctx = ctx;
    return pf_alloc(ctx, (void **)&c->d, coll_bytes(ctx));
}
int pf_phys_init_storage(pf_ctx *ctx, pf_phys *p) {
    p->ctx = ctx;
    return pf_alloc(ctx, (void **)&p->d, phys_bytes(ctx));
}

void pf_events_release(pf_ctx *ctx);

void pf_graphs_reset(pf_ctx *ctx) {
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    for (int p = 0; p < 2; ++p) {
        if (ctx->g_main[p]) cudaGraphExecDestroy(ctx->g_main[p]);
        if (ctx->g_corr[p]) cudaGraphExecDestroy(ctx->g_corr[p]);
        ctx->g_main[p] = ctx->g_corr[p] = nullptr;
    }
    for (int i = 0; i < 4; ++i) {
        for (auto &e : ctx->g_ev[i]) {
            ctx->ev_pool.push_back(e.second.first);
            ctx->ev_pool.push_back(e.second.second);
        }
        ctx->g_ev[i].clear();
    }
    ctx->g_pending.clear();
}

// Accumulate the event pairs of the graphs replayed since the last sync.
void pf_graph_events_collect(pf_ctx *ctx) {
    for (int gi : ctx->g_pending)
        for (auto &e : ctx->g_ev[gi]) {
            float ms = 0.f;
            if (cudaEventElapsedTime(&ms, e.second.first, e.second.second) == cudaSuccess) {
                ctx->prof_ms[e.first] += ms;
                ctx->prof_n[e.first] += 1;
            } else {
                cudaGetLastError();  // an unreadable pair must not surface at a later launch check
            }
        }
    ctx->g_pending.clear();
}

static void free_all(pf_ctx *ctx) {
    pf_graphs_reset(ctx);
    if (ctx->stream) pf_events_release(ctx);
    for (void *p : ctx->allocs) cudaFree(p);
    ctx->allocs.clear();
    if (ctx->hsc) cudaFreeHost(ctx->hsc);
    ctx->hsc = nullptr;
    if (ctx->own_stream && ctx->stream) cudaStreamDestroy(ctx->stream);
    ctx->stream = nullptr;
}

static int upload_twiddles(pf_ctx *ctx, int L, double2 **d64, float2 **d32) {
    std::vector<double2> h(L);
    std::vector<float2> hf(L);
    for (int t = 0; t < L; ++t) {
        // exp(+2 pi i t / L), computed in long double and rounded once
        const long double a = 2.0L * 3.14159265358979323846264338327950288L * (long double)t / (long double)L;
        h[t].x = (double)cosl(a);
        h[t].y = (double)sinl(a);
        hf[t].x = (float)cosl(a);
        hf[t].y = (float)sinl(a);
    }
    PF_TRY(pf_alloc(ctx, (void **)d64, L * sizeof(double2)));
    PF_TRY(pf_alloc(ctx, (void **)d32, L * sizeof(float2)));
    PF_CUDA(cudaMemcpyAsync(*d64, h.data(), L * sizeof(double2), cudaMemcpyHostToDevice, ctx->stream));
    PF_CUDA(cudaMemcpyAsync(*d32, hf.data(), L * sizeof(float2), cudaMemcpyHostToDevice, ctx->stream));
    PF_CUDA(cudaStreamSynchronize(ctx->stream));
    return PF_OK;
}

static int ctx_init(pf_ctx *ctx, const pf_config *cfg, int device) {
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        pf_set_error("no CUDA device visible");
        return PF_ERR_NODEVICE;
    }
    if (device >= 0) PF_CUDA(cudaSetDevice(device));
    PF_CUDA(cudaGetDevice(&ctx->device));
    PF_CUDA(cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking));
    ctx->own_stream = true;
    ctx->cfg = *cfg;
    ctx->cfg.r = nullptr;
    ctx->custom_mesh = cfg->r != nullptr;
    Geo &g = ctx->g;
    g.N = cfg->N;
    g.K = cfg->K;
    g.M = cfg->M;
    g.Mp = cfg->Mp;
    g.H = (2 * cfg->K - 1) * cfg->M - (cfg->K - 1);
    g.Hp = (g.H + 31) / 32 * 32;
    g.Z = 3 * cfg->K;
    g.Th = 3 * cfg->M;
    g.alpha = cfg->alpha;
    g.Re = cfg->Re;
    PF_TRY(pf_make_plan(g.Z, ctx->planZ));
    PF_TRY(pf_make_plan(g.Th, ctx->planT));
    // radial mesh on the host, uploaded once (meshs.f90:66-194)
    PF_TRY(pf_build_mesh(g.N, cfg->r, ctx->hm));
    const int N = g.N;
    const size_t nmesh = 7 * N + KL * NBAND * N + NBAND * N + 2 * (KL + 1) * (KL + 1) + 3 * N;
    PF_TRY(pf_alloc(ctx, (void **)&ctx->dmesh_mem, nmesh * sizeof(double)));
    {
        std::vector<double> h(nmesh);
        size_t o = 0;
        auto put = [&](const std::vector<double> &v) {
            const size_t at = o;
            std::memcpy(&h[o], v.data(), v.size() * sizeof(double));
            o += v.size();
            return ctx->dmesh_mem + at;
        };
        ctx->dm.rp = put(ctx->hm.rp);
        ctx->dm.dr = put(ctx->hm.dr);
        ctx->dm.radLap = put(ctx->hm.radLap);
        ctx->dm.dr0 = put(ctx->hm.dr0);
        ctx->dm.dr1 = put(ctx->hm.dr1);
        ctx->dm.intrdr = put(ctx->hm.intrdr);
        std::vector<double> U(N), Up(N);
        for (int n = 0; n < N; ++n) {  // vel_precompute (velocity.f90:53-54)
            U[n] = 1.0 - ctx->hm.rp[5 * N + n];
            Up[n] = -2.0 * ctx->hm.r[n];
        }
        ctx->dm.velU = put(U);
        ctx->dm.velUp = put(Up);
        PF_CUDA(cudaMemcpyAsync(ctx->dmesh_mem, h.data(), nmesh * sizeof(double),
                                cudaMemcpyHostToDevice, ctx->stream));
    }
    PF_TRY(upload_twiddles(ctx, g.Z, &ctx->twZ, &ctx->twZf));
    PF_TRY(upload_twiddles(ctx, g.Th, &ctx->twT, &ctx->twTf));
    PF_TRY(pf_alloc(ctx, (void **)&ctx->dsc, sizeof(DevScalars)));
    PF_CUDA(cudaMallocHost((void **)&ctx->hsc, sizeof(DevScalars)));
    std::memset(ctx->hsc, 0, sizeof(DevScalars));
    // module fields
    for (int i = 0; i < 6; ++i) {
        PF_TRY(pf_coll_init_storage(ctx, &ctx->vel[i]));
        PF_TRY(pf_coll_init_storage(ctx, &ctx->prev[i]));
        PF_TRY(pf_phys_init_storage(ctx, &ctx->phys[i]));
    }
    for (int i = 0; i < 3; ++i) PF_TRY(pf_coll_init_storage(ctx, &ctx->save[i]));
    for (int i = 0; i < 8; ++i) PF_TRY(pf_coll_init_storage(ctx, &ctx->s[i]));
    PF_TRY(pf_alloc(ctx, (void **)&ctx->U, (size_t)6 * N * g.Hp * sizeof(double)));
    PF_TRY(pf_alloc(ctx, (void **)&ctx->Ainv, (size_t)16 * g.Hp * sizeof(double)));
    PF_TRY(pf_alloc(ctx, (void **)&ctx->Ui, (size_t)N * sizeof(double)));
    PF_TRY(pf_alloc(ctx, (void **)&ctx->red, (size_t)(3 * N + g.Hp + 64) * sizeof(double)));
    PF_TRY(pf_alloc(ctx, (void **)&ctx->orbit_red, (size_t)(ORBIT_DOT_BLOCKS + 1) * sizeof(double)));
    PF_TRY(pf_alloc(ctx, (void **)&ctx->cflmax, (size_t)3 * N * sizeof(unsigned long long)));
    PF_TRY(pf_alloc(ctx, (void **)&ctx->mpart, (size_t)((g.H + 31) / 32) * N * 3 * sizeof(double)));
    PF_TRY(pf_alloc(ctx, (void **)&ctx->anypiv, sizeof(int)));
    // the (m, z) intermediate in FP64; in mixed precision its FP32 copy takes
    // the first 6*N*M*Z float2 and the FP32 curl(u) fields (3*N*Hp float2) follow
    ctx->T_bytes = std::max((size_t)6 * N * g.M * g.Z * sizeof(double2),
                            ((size_t)6 * N * g.M * g.Z + (size_t)3 * N * g.Hp) * sizeof(float2));
    PF_TRY(pf_alloc(ctx, &ctx->T, ctx->T_bytes));
    // LU factor storage for the four matrix sets
    pf_lumesh *L[4] = {&ctx->LNp, &ctx->LDp, &ctx->LDm, &ctx->LDz};
    const int Hcp = pf_compact_modes_padded(g);
    for (pf_lumesh *A : L) {
        A->ctx = ctx;
        PF_TRY(pf_alloc(ctx, (void **)&A->lu, (size_t)NLU * N * g.Hp * sizeof(double)));
        PF_TRY(pf_alloc(ctx, (void **)&A->piv, (size_t)N * g.Hp));
        PF_TRY(pf_alloc(ctx, (void **)&A->pivd, (size_t)N * g.Hp * sizeof(double)));
        PF_TRY(pf_alloc(ctx, (void **)&A->luc, (size_t)NLU * N * Hcp * sizeof(double)));
        PF_TRY(pf_alloc(ctx, (void **)&A->pivdc, (size_t)N * Hcp * sizeof(double)));
    }
    ctx->Ltp.ctx = ctx->Ltm.ctx = ctx->Ltz.ctx = ctx;
    // tim_precompute (timestep.f90:29-40)
    std::memset(&ctx->tim, 0, sizeof(ctx->tim));
    ctx->tim.t = 0.0;
    ctx->tim.dt = cfg->dt;
    // the plug-ins' one corrector pass
    ctx->tim.pcn = (ctx->util_kind == PF_UTIL_CARREAU_YASUDA || ctx->util_kind == PF_UTIL_LES) ? 1 : -1;
    ctx->lasterr = 1e99;
    ctx->newdt_i = 0;
    ctx->vel_nu = 1.0;
    ctx->use_graphs = true;
    PF_CUDA(cudaStreamSynchronize(ctx->stream));
    return PF_OK;
}

extern "C" int pf_ctx_create(const pf_config *cfg, int device, pf_ctx **out) {
    PF_ARG(cfg && out, "pf_ctx_create: null argument");
    *out = nullptr;
    PF_ARG(cfg->N > 2 * KL + 1, "pf_ctx_create: N must exceed 2*KL+1");
    PF_ARG(cfg->K >= 1 && cfg->M >= 1 && cfg->Mp >= 1, "pf_ctx_create: K, M, Mp must be >= 1");
    PF_ARG(cfg->alpha != 0.0, "var_coll_norm: alpha=0");
    PF_ARG(cfg->Re > 0.0, "pf_ctx_create: Re must be > 0");
    PF_ARG(cfg->precision == PF_PREC_FP64 || cfg->precision == PF_PREC_MIXED,
           "pf_ctx_create: unknown precision");
    pf_ctx *ctx = new pf_ctx();
    int s = ctx_init(ctx, cfg, device);
    if (s != PF_OK) {
        free_all(ctx);
        delete ctx;
        return s;
    }
    *out = ctx;
    return PF_OK;
}

// New physical parameters for an existing context of the same shape (N, K,
// M, Mp, precision, default mesh): a fresh run as pf_ctx_create would start
// it, reusing the device memory.  vel_matrices must be called again.
extern "C" int pf_ctx_reconfigure(pf_ctx *ctx, const pf_config *cfg) {
    PF_ARG(ctx && cfg, "pf_ctx_reconfigure: null argument");
    PF_ARG(cfg->N == ctx->cfg.N && cfg->K == ctx->cfg.K && cfg->M == ctx->cfg.M && cfg->Mp == ctx->cfg.Mp &&
               cfg->precision == ctx->cfg.precision && cfg->r == nullptr && !ctx->custom_mesh,
           "pf_ctx_reconfigure: shape, precision or mesh differs");
    PF_ARG(cfg->alpha != 0.0, "var_coll_norm: alpha=0");
    PF_ARG(cfg->Re > 0.0, "pf_ctx_reconfigure: Re must be > 0");
    PF_CUDA(cudaSetDevice(ctx->device));
    PF_CUDA(cudaStreamSynchronize(ctx->stream));
    pf_graphs_reset(ctx);
    ctx->cfg = *cfg;
    ctx->cfg.r = nullptr;
    ctx->g.alpha = cfg->alpha;
    ctx->g.Re = cfg->Re;
    ctx->matrices_ready = false;
    ctx->LNp_set = false;
    ctx->cfl_fused = false;
    // tim_precompute (timestep.f90:29-40)
    std::memset(&ctx->tim, 0, sizeof(ctx->tim));
    ctx->tim.dt = cfg->dt;
    // the plug-ins' one corrector pass
    ctx->tim.pcn = (ctx->util_kind == PF_UTIL_CARREAU_YASUDA || ctx->util_kind == PF_UTIL_LES) ? 1 : -1;
    ctx->lasterr = 1e99;
    ctx->newdt_i = 0;
    ctx->vel_nu = 1.0;
    PF_CUDA(cudaMemsetAsync(ctx->dsc, 0, sizeof(DevScalars), ctx->stream));
    if (ctx->util_kind == PF_UTIL_LES) {  // its filter widths depend on alpha
        double p[8];
        std::memcpy(p, ctx->util_par, sizeof(p));
        PF_TRY(pf_util_set(ctx, PF_UTIL_LES, p, 4));
    }
    return PF_OK;
}

extern "C" int pf_ctx_destroy(pf_ctx *ctx) {
    if (!ctx) return PF_OK;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    free_all(ctx);
    delete ctx;
    return PF_OK;
}

extern "C" int pf_ctx_set_stream(pf_ctx *ctx, void *stream) {
    PF_ARG(ctx, "null ctx");
    PF_CUDA(cudaStreamSynchronize(ctx->stream));
    pf_graphs_reset(ctx);
    if (ctx->own_stream) cudaStreamDestroy(ctx->stream);
    if (stream) {
        ctx->stream = (cudaStream_t)stream;
        ctx->own_stream = false;
    } else {
        PF_CUDA(cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking));
        ctx->own_stream = true;
    }
    return PF_OK;
}

extern "C" int pf_ctx_set_tuning(pf_ctx *ctx, const pf_tuning *t) {
    PF_ARG(ctx && t, "pf_ctx_set_tuning: null argument");
    PF_ARG(t->ld_solver == PF_LD_AUTO || t->ld_solver == PF_LD_STREAMED || t->ld_solver == PF_LD_REBUILT ||
               t->ld_solver == PF_LD_PAIRED || t->ld_solver == PF_LD_WARPRING,
           "pf_ctx_set_tuning: bad ld_solver");
    PF_ARG(t->nl_fused == 0 || t->nl_fused == 1, "pf_ctx_set_tuning: nl_fused is 0 or 1");
    PF_TRY(pf_nl_tiles_check(ctx, t));
    if (std::memcmp(&ctx->tune, t, sizeof(pf_tuning)) == 0) return PF_OK;
    PF_CUDA(cudaStreamSynchronize(ctx->stream));
    ctx->tune = *t;
    pf_graphs_reset(ctx);
    ctx->matrices_gen++;  // batches holding this pipe rebuild their launches
    return PF_OK;
}

extern "C" int pf_ctx_get_tuning(const pf_ctx *ctx, pf_tuning *t) {
    PF_ARG(ctx && t, "pf_ctx_get_tuning: null argument");
    *t = ctx->tune;
    return PF_OK;
}

extern "C" int pf_ctx_sync(pf_ctx *ctx) {
    PF_ARG(ctx, "null ctx");
    PF_CUDA(cudaStreamSynchronize(ctx->stream));
    return PF_OK;
}

extern "C" int pf_ctx_dims(const pf_ctx *ctx, int *N, int *H, int *Z, int *Th) {
    PF_ARG(ctx, "null ctx");
    if (N) *N = ctx->g.N;
    if (H) *H = ctx->g.H;
    if (Z) *Z = ctx->g.Z;
    if (Th) *Th = ctx->g.Th;
    return PF_OK;
}

extern "C" int pf_ctx_device_bytes(const pf_ctx *ctx, unsigned long long *bytes) {
    PF_ARG(ctx && bytes, "null argument");
    *bytes = ctx->bytes;
    return PF_OK;
}

static void mesh_export(const HostMesh &hm, int N, double *r, double *dr, double *radLap, double *dr0,
                        double *dr1, double *intrdr);

extern "C" int pf_mes_get(const pf_ctx *ctx, double *r, double *dr, double *radLap,
                          double *dr0, double *dr1, double *intrdr) {
    PF_ARG(ctx, "null ctx");
    mesh_export(ctx->hm, ctx->g.N, r, dr, radLap, dr0, dr1, intrdr);
    return PF_OK;
}

extern "C" int pf_mes_compute(int N, const double *custom_r, double *r, double *dr, double *radLap,
                              double *dr0, double *dr1, double *intrdr) {
    PF_ARG(N > 2 * KL + 1, "pf_mes_compute: N must exceed 2*KL+1");
    HostMesh hm;
    PF_TRY(pf_build_mesh(N, custom_r, hm));
    mesh_export(hm, N, r, dr, radLap, dr0, dr1, intrdr);
    return PF_OK;
}

static void mesh_export(const HostMesh &hm, int N, double *r, double *dr, double *radLap, double *dr0,
                        double *dr1, double *intrdr) {
    if (r) std::memcpy(r, hm.r.data(), N * sizeof(double));
    if (dr)  // host layout [(i*N + j)*(2KL+1) + row]
        for (int i = 0; i < KL; ++i)
            for (int j = 0; j < N; ++j)
                for (int row = 0; row < NBAND; ++row)
                    dr[((size_t)i * N + j) * NBAND + row] = hm.dr[(i * NBAND + row) * N + j];
    if (radLap)
        for (int j = 0; j < N; ++j)
            for (int row = 0; row < NBAND; ++row)
                radLap[(size_t)j * NBAND + row] = hm.radLap[row * N + j];
    if (dr0) std::memcpy(dr0, hm.dr0.data(), hm.dr0.size() * sizeof(double));
    if (dr1) std::memcpy(dr1, hm.dr1.data(), hm.dr1.size() * sizeof(double));
    if (intrdr) std::memcpy(intrdr, hm.intrdr.data(), N * sizeof(double));
}

// ------------------------------------------------------ host <-> device
// host coll (re[nh*N+n], im[...]) <-> device double2 [n*Hp+nh]
__global__ void k_coll_from_host(const double *__restrict__ re, const double *__restrict__ im,
                                 double2 *__restrict__ out, int N, int H, int Hp) {
    __shared__ double2 tile[32][33];
    const int nh0 = blockIdx.x * 32, n0 = blockIdx.y * 32;
    for (int i = threadIdx.y; i < 32; i += blockDim.y) {
        const int nh = nh0 + i, n = n0 + threadIdx.x;
        if (nh < H && n < N) {
            const size_t at = (size_t)nh * N + n;
            tile[i][threadIdx.x] = make_double2(re[at], im[at]);
        }
    }
    __syncthreads();
    for (int i = threadIdx.y; i < 32; i += blockDim.y) {
        const int n = n0 + i, nh = nh0 + threadIdx.x;
        if (n < N && nh < Hp) out[(size_t)n * Hp + nh] = nh < H ? tile[threadIdx.x][i] : make_double2(0.0, 0.0);
    }
}

__global__ void k_coll_to_host(const double2 *__restrict__ in, double *__restrict__ re,
                               double *__restrict__ im, int N, int H, int Hp) {
    __shared__ double2 tile[32][33];
    const int nh0 = blockIdx.x * 32, n0 = blockIdx.y * 32;
    for (int i = threadIdx.y; i < 32; i += blockDim.y) {
        const int n = n0 + i, nh = nh0 + threadIdx.x;
        if (n < N && nh < H) tile[threadIdx.x][i] = in[(size_t)n * Hp + nh];
    }
    __syncthreads();
    for (int i = threadIdx.y; i < 32; i += blockDim.y) {
        const int nh = nh0 + i, n = n0 + threadIdx.x;
        if (nh < H && n < N) {
            const double2 v = tile[i][threadIdx.x];
            const size_t at = (size_t)nh * N + n;
            re[at] = v.x;
            im[at] = v.y;
        }
    }
}

// Staged copies through a device buffer (pageable or pinned host memory).
static int coll_upload(pf_ctx *ctx, double2 *dst, const double *re, const double *im) {
    const Geo &g = ctx->g;
    const size_t nb = (size_t)g.N * g.H * sizeof(double);
    double *stage = (double *)ctx->s[7].d;  // scratch coll has 2*N*Hp doubles >= 2*N*H
    PF_CUDA(cudaMemcpyAsync(stage, re, nb, cudaMemcpyHostToDevice, ctx->stream));
    PF_CUDA(cudaMemcpyAsync(stage + (size_t)g.N * g.H, im, nb, cudaMemcpyHostToDevice, ctx->stream));
    dim3 grid(grid1(g.Hp, 32), grid1(g.N, 32)), block(32, 8);
    {
        ProfScope ps_(ctx, PF_K_EW);
        k_coll_from_host<<<grid, block, 0, ctx->stream>>>(stage, stage + (size_t)g.N * g.H, dst, g.N, g.H, g.Hp);
    }
    PF_LAUNCHED(ctx);
    return PF_OK;
}

static int coll_download_async(pf_ctx *ctx, const double2 *src, double *re, double *im) {
    const Geo &g = ctx->g;
    const size_t nb = (size_t)g.N * g.H * sizeof(double);
    double *stage = (double *)ctx->s[7].d;  // reused in stream order by the next field
    dim3 grid(grid1(g.Hp, 32), grid1(g.N, 32)), block(32, 8);
    {
        ProfScope ps_(ctx, PF_K_EW);
        k_coll_to_host<<<grid, block, 0, ctx->stream>>>(src, stage, stage + (size_t)g.N * g.H, g.N, g.H, g.Hp);
    }
    PF_LAUNCHED(ctx);
    PF_CUDA(cudaMemcpyAsync(re, stage, nb, cudaMemcpyDeviceToHost, ctx->stream));
    PF_CUDA(cudaMemcpyAsync(im, stage + (size_t)g.N * g.H, nb, cudaMemcpyDeviceToHost, ctx->stream));
    return PF_OK;
}

static int coll_download(pf_ctx *ctx, const double2 *src, double *re, double *im) {
    const Geo &g = ctx->g;
    const size_t nb = (size_t)g.N * g.H * sizeof(double);
    double *stage = (double *)ctx->s[7].d;
    dim3 grid(grid1(g.Hp, 32), grid1(g.N, 32)), block(32, 8);
    {
        ProfScope ps_(ctx, PF_K_EW);
        k_coll_to_host<<<grid, block, 0, ctx->stream>>>(src, stage, stage + (size_t)g.N * g.H, g.N, g.H, g.Hp);
    }
    PF_LAUNCHED(ctx);
    PF_CUDA(cudaMemcpyAsync(re, stage, nb, cudaMemcpyDeviceToHost, ctx->stream));
    PF_CUDA(cudaMemcpyAsync(im, stage + (size_t)g.N * g.H, nb, cudaMemcpyDeviceToHost, ctx->stream));
    PF_CUDA(cudaStreamSynchronize(ctx->stream));
    return PF_OK;
}

extern "C" int pf_coll_create(pf_ctx *ctx, pf_coll **out) {
    PF_ARG(ctx && out, "null argument");
    pf_coll *c = new pf_coll();
    int s = pf_coll_init_storage(ctx, c);
    if (s != PF_OK) {
        delete c;
        return s;
    }
    *out = c;
    return PF_OK;
}

extern "C" int pf_coll_destroy(pf_coll *c) {
    if (!c) return PF_OK;
    pf_ctx *ctx = c->ctx;
    cudaStreamSynchronize(ctx->stream);
    for (size_t i = 0; i < ctx->allocs.size(); ++i)
        if (ctx->allocs[i] == (void *)c->d) {
            cudaFree(c->d);
            ctx->allocs.erase(ctx->allocs.begin() + i);
            ctx->bytes -= (size_t)ctx->g.N * ctx->g.Hp * sizeof(double2);
            break;
        }
    delete c;
    return PF_OK;
}

extern "C" int pf_coll_upload(pf_coll *c, const double *re, const double *im) {
    PF_ARG(c && re && im, "null argument");
    return coll_upload(c->ctx, c->d, re, im);
}

extern "C" int pf_coll_download(const pf_coll *c, double *re, double *im) {
    PF_ARG(c && re && im, "null argument");
    return coll_download(c->ctx, c->d, re, im);
}

extern "C" int pf_phys_create(pf_ctx *ctx, pf_phys **out) {
    PF_ARG(ctx && out, "null argument");
    pf_phys *p = new pf_phys();
    int s = pf_phys_init_storage(ctx, p);
    if (s != PF_OK) {
        delete p;
        return s;
    }
    *out = p;
    return PF_OK;
}

extern "C" int pf_phys_destroy(pf_phys *p) {
    if (!p) return PF_OK;
    pf_ctx *ctx = p->ctx;
    cudaStreamSynchronize(ctx->stream);
    for (size_t i = 0; i < ctx->allocs.size(); ++i)
        if (ctx->allocs[i] == (void *)p->d) {
            cudaFree(p->d);
            ctx->allocs.erase(ctx->allocs.begin() + i);
            ctx->bytes -= (size_t)ctx->g.N * ctx->g.Th * ctx->g.Z * sizeof(double);
            break;
        }
    delete p;
    return PF_OK;
}

extern "C" int pf_phys_upload(pf_phys *p, const double *re) {
    PF_ARG(p && re, "null argument");
    pf_ctx *ctx = p->ctx;
    PF_CUDA(cudaMemcpyAsync(p->d, re, (size_t)ctx->g.N * ctx->g.Th * ctx->g.Z * sizeof(double),
                            cudaMemcpyHostToDevice, ctx->stream));
    PF_CUDA(cudaStreamSynchronize(ctx->stream));
    return PF_OK;
}

extern "C" int pf_phys_download(const pf_phys *p, double *re) {
    PF_ARG(p && re, "null argument");
    pf_ctx *ctx = p->ctx;
    PF_CUDA(cudaMemcpyAsync(re, p->d, (size_t)ctx->g.N * ctx->g.Th * ctx->g.Z * sizeof(double),
                            cudaMemcpyDeviceToHost, ctx->stream));
    PF_CUDA(cudaStreamSynchronize(ctx->stream));
    return PF_OK;
}

extern "C" int pf_vel_coll(pf_ctx *ctx, int which, pf_coll **out) {
    PF_ARG(ctx && out && which >= 0 && which < 6, "pf_vel_coll: bad argument");
    *out = &ctx->vel[which];
    return PF_OK;
}

extern "C" int pf_vel_phys(pf_ctx *ctx, int which, pf_phys **out) {
    PF_ARG(ctx && out && which >= 0 && which < 6, "pf_vel_phys: bad argument");
    *out = &ctx->phys[which];
    return PF_OK;
}

extern "C" int pf_vel_set_state(pf_ctx *ctx, const double *ur_re, const double *ur_im,
                                const double *ut_re, const double *ut_im,
                                const double *uz_re, const double *uz_im) {
    PF_ARG(ctx && ur_re && ur_im && ut_re && ut_im && uz_re && uz_im, "null argument");
    PF_TRY(coll_upload(ctx, ctx->vel[0].d, ur_re, ur_im));
    PF_TRY(coll_upload(ctx, ctx->vel[1].d, ut_re, ut_im));
    PF_TRY(coll_upload(ctx, ctx->vel[2].d, uz_re, uz_im));
    return PF_OK;
}

extern "C" int pf_vel_get_state(pf_ctx *ctx, double *ur_re, double *ur_im, double *ut_re,
                                double *ut_im, double *uz_re, double *uz_im) {
    PF_ARG(ctx && ur_re && ur_im && ut_re && ut_im && uz_re && uz_im, "null argument");
    PF_TRY(coll_download(ctx, ctx->vel[0].d, ur_re, ur_im));
    PF_TRY(coll_download(ctx, ctx->vel[1].d, ut_re, ut_im));
    PF_TRY(coll_download(ctx, ctx->vel[2].d, uz_re, uz_im));
    return PF_OK;
}

// As pf_vel_get_state, without waiting: the copies are queued on the
// context's stream and the host arrays are filled once pf_ctx_sync returns.
// The host arrays should be page-locked for the copies to overlap other work.
extern "C" int pf_vel_get_state_async(pf_ctx *ctx, double *ur_re, double *ur_im, double *ut_re, double *ut_im,
                                      double *uz_re, double *uz_im) {
    PF_ARG(ctx && ur_re && ur_im && ut_re && ut_im && uz_re && uz_im, "null argument");
    PF_TRY(coll_download_async(ctx, ctx->vel[0].d, ur_re, ur_im));
    PF_TRY(coll_download_async(ctx, ctx->vel[1].d, ut_re, ut_im));
    PF_TRY(coll_download_async(ctx, ctx->vel[2].d, uz_re, uz_im));
    return PF_OK;
}

extern "C" int pf_vel_get_scalars(const pf_ctx *ctx, double *Pr0, double *nu) {
    PF_ARG(ctx, "null ctx");
    PF_CUDA(cudaMemcpyAsync(ctx->hsc, ctx->dsc, sizeof(DevScalars), cudaMemcpyDeviceToHost, ctx->stream));
    PF_CUDA(cudaStreamSynchronize(ctx->stream));
    if (Pr0) *Pr0 = ctx->hsc->Pr0;
    if (nu) *nu = ctx->vel_nu;
    return PF_OK;
}

extern "C" int pf_tim_get(const pf_ctx *ctx, pf_tim_state *s) {
    PF_ARG(ctx && s, "null argument");
    *s = ctx->tim;
    return PF_OK;
}

extern "C" int pf_tim_set(pf_ctx *ctx, const pf_tim_state *s) {
    PF_ARG(ctx && s, "null argument");
    ctx->tim = *s;
    return PF_OK;
}

// ------------------------------------------------------- instrumentation
cudaEvent_t pf_event_get(pf_ctx *ctx) {
    if (!ctx->ev_pool.empty()) {
        cudaEvent_t e = ctx->ev_pool.back();
        ctx->ev_pool.pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    cudaEventCreate(&e);
    return e;
}

static void prof_drain(pf_ctx *ctx) {
    cudaStreamSynchronize(ctx->stream);
    for (int c = 0; c < PF_K_NCAT; ++c) {
        for (auto &pr : ctx->ev_open[c]) {
            float ms = 0.f;
            if (cudaEventElapsedTime(&ms, pr.first, pr.second) == cudaSuccess) {
                ctx->prof_ms[c] += ms;
                ctx->prof_n[c] += 1;
            } else {
                cudaGetLastError();
            }
            ctx->ev_pool.push_back(pr.first);
            ctx->ev_pool.push_back(pr.second);
        }
        ctx->ev_open[c].clear();
    }
}

void pf_events_release(pf_ctx *ctx) {
    prof_drain(ctx);
    for (cudaEvent_t e : ctx->ev_pool) cudaEventDestroy(e);
    ctx->ev_pool.clear();
}

extern "C" int pf_ctx_launches(const pf_ctx *ctx, unsigned long long *n) {
    PF_ARG(ctx && n, "null argument");
    *n = ctx->launches;
    return PF_OK;
}

extern "C" int pf_prof_enable(pf_ctx *ctx, int mask) {
    PF_ARG(ctx, "null ctx");
    prof_drain(ctx);
    pf_graph_events_collect(ctx);
    if (mask != ctx->prof_mask) pf_graphs_reset(ctx);  // graphs bake in their event nodes
    for (int c = 0; c < PF_K_NCAT; ++c) {
        ctx->prof_ms[c] = 0.0;
        ctx->prof_n[c] = 0;
    }
    ctx->prof_mask = mask;
    return PF_OK;
}

extern "C" int pf_prof_read(pf_ctx *ctx, int cat, double *ms, unsigned long long *launches) {
    PF_ARG(ctx && cat >= 0 && cat < PF_K_NCAT, "pf_prof_read: bad argument");
    prof_drain(ctx);
    pf_graph_events_collect(ctx);
    if (ms) *ms = ctx->prof_ms[cat];
    if (launches) *launches = ctx->prof_n[cat];
    return PF_OK;
}
