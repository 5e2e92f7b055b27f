// Velocity module and drivers: vel_transform / vel_nonlinear / vel_step /
// predictor / corrector, corrector control and adaptive dt, and the main-loop
// and steporbit step drivers (velocity.f90:61-481; timestep.f90:214-278;
// main.f90:20-44; newton.f90:740-762).
#include <cmath>
#include "pf_internal.cuh"

static int require_matrices(pf_ctx *ctx) {
    if (!ctx->matrices_ready) {
        pf_set_error("vel_matrices has not been called for this context");
        return PF_ERR_STATE;
    }
    return PF_OK;
}

extern "C" int pf_vel_imposesym(pf_ctx *ctx) {
    PF_ARG(ctx, "null ctx");
    double2 *r = ctx->vel[0].d, *t = ctx->vel[1].d, *z = ctx->vel[2].d;
    PF_TRY(pf_launch_imposesym(ctx, 0, r, t, z));
    if (ctx->cfg.mirrorsym) PF_TRY(pf_launch_imposesym(ctx, 1, r, t, z));
    if (ctx->cfg.shiftrefl) PF_TRY(pf_launch_imposesym(ctx, 2, r, t, z));
    if (ctx->cfg.shiftrott) PF_TRY(pf_launch_imposesym(ctx, 3, r, t, z));
    return PF_OK;
}

extern "C" int pf_vel_matrices(pf_ctx *ctx) {
    PF_ARG(ctx, "null ctx");
    return pf_vel_matrices_impl(ctx);
}

// u and curl(u) to physical space (velocity.f90:304-317)
extern "C" int pf_vel_transform(pf_ctx *ctx) {
    PF_ARG(ctx, "null ctx");
    PF_TRY(pf_launch_curl(ctx, ctx->vel[0].d, ctx->vel[1].d, ctx->vel[2].d, ctx->s[0].d, ctx->s[1].d,
                          ctx->s[2].d));
    const double2 *src[6] = {ctx->vel[0].d, ctx->vel[1].d, ctx->vel[2].d, ctx->s[0].d, ctx->s[1].d, ctx->s[2].d};
    double *dst[6];
    for (int i = 0; i < 6; ++i) dst[i] = ctx->phys[i].d;
    ctx->cfl_fused = false;
    return pf_launch_coll2phys(ctx, 6, src, dst);
}

// u x curl(u), forward transforms, background-flow terms (velocity.f90:323-361)
extern "C" int pf_vel_nonlinear(pf_ctx *ctx) {
    PF_ARG(ctx, "null ctx");
    const double *src[6];
    for (int i = 0; i < 6; ++i) src[i] = ctx->phys[i].d;
    double2 *dst[3] = {ctx->vel[3].d, ctx->vel[4].d, ctx->vel[5].d};
    PF_TRY(pf_launch_phys2coll(ctx, 3, src, dst, true));
    return pf_launch_addHPF(ctx);
}

// velocity.f90:367-394
static int vel_step(pf_ctx *ctx) {
    PF_TRY(require_matrices(ctx));
    double2 *ur = ctx->vel[0].d, *ut = ctx->vel[1].d, *uz = ctx->vel[2].d;
    double2 *Nr = ctx->vel[3].d, *Nt = ctx->vel[4].d, *Nz = ctx->vel[5].d;
    double2 *s0 = ctx->s[0].d, *s1 = ctx->s[1].d, *s2 = ctx->s[2].d, *s3 = ctx->s[3].d;
    double2 *s4 = ctx->s[4].d, *s5 = ctx->s[5].d;
    // rhs = A u_ + N
    PF_TRY(pf_launch_ew(ctx, EW_RT2PM, Nr, Nt, s0, s1, 0.0));
    PF_TRY(pf_launch_ew(ctx, EW_RT2PM, ctx->prev[0].d, ctx->prev[1].d, s2, s3, 0.0));
    PF_TRY(pf_launch_tim_meshmult(ctx, &ctx->Ltp, s2, s0, ur));
    PF_TRY(pf_launch_tim_meshmult(ctx, &ctx->Ltm, s3, s1, ut));
    PF_TRY(pf_launch_tim_meshmult(ctx, &ctx->Ltz, ctx->prev[2].d, Nz, uz));
    // vel_adjPPE(1): pressure projection (velocity.f90:227-236)
    PF_TRY(pf_launch_ew(ctx, EW_PM2RT, ur, ut, s0, s1, 0.0));
    PF_TRY(pf_launch_div(ctx, s0, s1, uz, s2));
    PF_TRY(pf_launch_zerobc(ctx, s2));
    PF_TRY(pf_launch_lu_solve(ctx, 1, &ctx->LNp, s2));
    PF_TRY(pf_launch_grad(ctx, s2, s3, s4, s5));
    PF_TRY(pf_launch_ew(ctx, EW_RT2PM, s3, s4, s0, s1, 0.0));
    PF_TRY(pf_launch_ew(ctx, EW_SUB, s0, nullptr, ur, nullptr, 0.0));
    PF_TRY(pf_launch_ew(ctx, EW_SUB, s1, nullptr, ut, nullptr, 0.0));
    PF_TRY(pf_launch_ew(ctx, EW_SUB, s5, nullptr, uz, nullptr, 0.0));
    // invert
    PF_TRY(pf_launch_zerobc(ctx, ur));
    PF_TRY(pf_launch_zerobc(ctx, ut));
    PF_TRY(pf_launch_zerobc(ctx, uz));
    PF_TRY(pf_launch_lu_solve(ctx, 0, &ctx->LDp, ur));
    PF_TRY(pf_launch_lu_solve(ctx, 0, &ctx->LDm, ut));
    PF_TRY(pf_launch_lu_solve(ctx, 0, &ctx->LDz, uz));
    PF_TRY(pf_launch_adjppe2(ctx));
    PF_TRY(pf_launch_ew(ctx, EW_PM2RT, ur, ut, ur, ut, 0.0));
    PF_TRY(pf_launch_flux1(ctx));
    return pf_launch_zero_mode0(ctx);
}

bool pf_fused_step_ok(const pf_ctx *ctx);
static bool fused_step_ok(const pf_ctx *ctx) { return pf_fused_step_ok(ctx); }
bool pf_fused_step_ok(const pf_ctx *ctx) { return ctx->g.N <= 128; }

// velocity.f90:400-410
extern "C" int pf_vel_predictor(pf_ctx *ctx) {
    PF_ARG(ctx, "null ctx");
    PF_TRY(require_matrices(ctx));
    if (fused_step_ok(ctx)) return pf_vel_step_fused(ctx, 0);
    for (int i = 0; i < 6; ++i)
        PF_TRY(pf_launch_ew(ctx, EW_COPY, ctx->vel[i].d, nullptr, ctx->prev[i].d, nullptr, 0.0));
    return vel_step(ctx);
}

// velocity.f90:416-432 (tim_measurecorr folded into one device reduction)
static int vel_corrector_async(pf_ctx *ctx) {
    PF_TRY(require_matrices(ctx));
    if (fused_step_ok(ctx)) return pf_vel_step_fused(ctx, 1);
    for (int i = 0; i < 3; ++i)
        PF_TRY(pf_launch_ew(ctx, EW_COPY, ctx->vel[i].d, nullptr, ctx->save[i].d, nullptr, 0.0));
    for (int i = 3; i < 6; ++i)
        PF_TRY(pf_launch_ew(ctx, EW_NLINCORR, ctx->prev[i].d, nullptr, ctx->vel[i].d, nullptr,
                            ctx->cfg.implicit));
    PF_TRY(vel_step(ctx));
    return pf_launch_measurecorr(ctx, ctx->save[0].d, ctx->vel[0].d, ctx->save[1].d, ctx->vel[1].d,
                                 ctx->save[2].d, ctx->vel[2].d, true);
}

int pf_read_dterr(pf_ctx *ctx);
static int read_dterr(pf_ctx *ctx) { return pf_read_dterr(ctx); }
int pf_read_dterr(pf_ctx *ctx) {
    PF_CUDA(cudaMemcpyAsync(ctx->hsc, ctx->dsc, sizeof(DevScalars), cudaMemcpyDeviceToHost, ctx->stream));
    PF_CUDA(cudaStreamSynchronize(ctx->stream));
    pf_graph_events_collect(ctx);
    const double d2 = bits_to_double(ctx->hsc->dterr2_bits);
    ctx->tim.dterr = std::max(ctx->tim.dterr, std::sqrt(d2));
    return PF_OK;
}

extern "C" int pf_vel_corrector(pf_ctx *ctx) {
    PF_ARG(ctx, "null ctx");
    PF_TRY(vel_corrector_async(ctx));
    return read_dterr(ctx);
}

// vel_transform + vel_nonlinear for the drivers: the fused three-launch
// path when the transform lengths are instantiated, else the materialising one
int pf_transform_nonlinear(pf_ctx *ctx);
static int transform_nonlinear(pf_ctx *ctx) { return pf_transform_nonlinear(ctx); }
int pf_transform_nonlinear(pf_ctx *ctx) {
    if (pf_nl_fused_supported(ctx)) {
        PF_TRY(pf_launch_nl_fused(ctx));
        ctx->cfl_fused = true;
        return PF_OK;
    }
    PF_TRY(pf_vel_transform(ctx));
    return pf_vel_nonlinear(ctx);
}

extern "C" int pf_vel_transform_nonlinear(pf_ctx *ctx) {
    PF_ARG(ctx, "null ctx");
    return pf_transform_nonlinear(ctx);
}

extern "C" int pf_vel_maxtstep(pf_ctx *ctx) {
    PF_ARG(ctx, "null ctx");
    double dt[3];
    PF_TRY(pf_launch_maxtstep(ctx, dt));
    ctx->tim.cfl_dt = std::min(dt[0], std::min(dt[1], dt[2]));
    for (int i = 0; i < 3; ++i)
        if (ctx->tim.cfl_dt == dt[i]) ctx->tim.cfl_dir = i + 1;
    return PF_OK;
}

// timestep.f90:214-253; failures are reported as a status instead of
// forcing the step counter to i_maxtstep-1
extern "C" int pf_tim_check_cgce(pf_ctx *ctx) {
    PF_ARG(ctx, "null ctx");
    pf_tim_state &t = ctx->tim;
    const pf_config &c = ctx->cfg;
    int status = PF_OK;
    if (t.it == 1) {
        t.corr_dt = t.dterr > 0.0 ? t.dt * std::sqrt(c.dterr / t.dterr) : INFINITY;
        ctx->lasterr = 1e99;
    }
    if (t.dt < 1e-9 && t.step > 30) {
        pf_set_error("tim_check_cgce: dt --> 0 !!!?");
        status = PF_ERR_CONVERGE;
        t.it = 0;
    } else if (t.it == t.pcn) {
        t.it = 0;
    } else if (t.it > 10) {
        pf_set_error("tim_check_cgce: too many its!!!");
        status = PF_ERR_CONVERGE;
        t.it = 0;
    } else if (t.dterr > ctx->lasterr) {
        if (t.dterr > 2.0 * c.dterr) {
            pf_set_error("tim_check_cgce: increasing error!!!");
            status = PF_ERR_CONVERGE;
        }
        if (t.dterr < 2.0 * c.dterr) t.corr_dt = t.dt / (10.0 * c.courant);
        t.it = 0;
    } else if (t.dterr > c.dterr) {
        ctx->lasterr = t.dterr;
        t.it = t.it + 1;
    } else {
        t.it = 0;
    }
    t.dterr = 0.0;
    return status;
}

// timestep.f90:259-278
extern "C" int pf_tim_new_tstep(pf_ctx *ctx) {
    PF_ARG(ctx, "null ctx");
    pf_tim_state &t = ctx->tim;
    const pf_config &c = ctx->cfg;
    double dt = std::min(t.dt * 1.11, c.maxdt);
    if (t.step == 0 && t.corr_dt == 0.0) dt = std::min(dt, t.cfl_dt * 0.1);
    if (t.cfl_dt > 0.0) dt = std::min(dt, t.cfl_dt * c.courant);
    if (t.corr_dt > 0.0) dt = std::min(dt, t.corr_dt * 0.95);
    ctx->newdt_i = ctx->newdt_i - 1;
    const int i = ctx->newdt_i;
    t.new_dt = (dt < t.dt * 0.95) || (dt > t.dt * 1.10 && i < 0) || (dt == c.maxdt && t.dt < dt && i < 0);
    if (t.new_dt) {
        if (dt >= t.dt) ctx->newdt_i = 99;
        t.dt = dt;
    }
    return PF_OK;
}

// main.f90:20-44
// Capture `body` on the context stream into an executable graph; the
// context's profiling is paused so no event pairs are recorded, and the
// number of kernels captured is returned in *nk.
// Capture `body` on the context stream into an executable graph.  Event
// pairs of profiled categories become event-record nodes of the graph (kept
// in ctx->g_ev[slot]); *nk returns the number of kernels captured.
template <typename F>
static int capture(pf_ctx *ctx, int slot, cudaGraphExec_t *exec, unsigned long long *nk, F body) {
    const unsigned long long n0 = ctx->launches;
    size_t open0[PF_K_NCAT];
    for (int c = 0; c < PF_K_NCAT; ++c) open0[c] = ctx->ev_open[c].size();
    cudaGraph_t graph = nullptr;
    PF_CUDA(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
    const int s = body();
    const cudaError_t e = cudaStreamEndCapture(ctx->stream, &graph);
    for (int c = 0; c < PF_K_NCAT; ++c) {  // move the captured pairs to the graph's list
        for (size_t i = open0[c]; i < ctx->ev_open[c].size(); ++i) ctx->g_ev[slot].push_back({c, ctx->ev_open[c][i]});
        ctx->ev_open[c].resize(open0[c]);
    }
    if (s != PF_OK) {
        if (graph) cudaGraphDestroy(graph);
        return s;
    }
    if (e != cudaSuccess) {
        pf_set_error("graph capture failed: %s", cudaGetErrorString(e));
        return PF_ERR_CUDA;
    }
    const cudaError_t e2 = cudaGraphInstantiate(exec, graph, 0);
    cudaGraphDestroy(graph);
    if (e2 != cudaSuccess) {
        pf_set_error("graph instantiation failed: %s", cudaGetErrorString(e2));
        return PF_ERR_CUDA;
    }
    *nk = ctx->launches - n0;
    ctx->launches = n0;  // counted again at each replay
    return PF_OK;
}

static int replay(pf_ctx *ctx, int slot, cudaGraphExec_t g, unsigned long long nk) {
    PF_CUDA(cudaGraphLaunch(g, ctx->stream));
    ctx->launches += nk;
    if (!ctx->g_ev[slot].empty()) ctx->g_pending.push_back(slot);
    return PF_OK;
}

// A plug-in whose hook is device work only, queued on the context's stream
// (the Coriolis and Carreau-Yasuda terms), rides in the step graphs; a host
// callback, and LES (it reads max nu_t back to decide on new matrices before
// its terms), keep the step eager.
static bool util_graphable(const pf_ctx *ctx) {
    return ctx->util_cb == nullptr && (ctx->util_kind == PF_UTIL_NONE || ctx->util_kind == PF_UTIL_CORIOLIS ||
                                       ctx->util_kind == PF_UTIL_CARREAU_YASUDA);
}

static bool graphs_ok(const pf_ctx *ctx) {
    return ctx->use_graphs && ctx->cfg.dt > 0.0 && pf_nl_fused_supported(ctx) && fused_step_ok(ctx) &&
           util_graphable(ctx);
}

// vel_transform + vel_nonlinear + var_null(2) of the main loop (main.f90:21-23,
// 36-38): with a plug-in the physical fields vel_r .. vel_curlz are made, as
// the plug-ins read them
static int main_nonlinear(pf_ctx *ctx) {
    if (!pf_util_active(ctx)) return transform_nonlinear(ctx);
    PF_TRY(pf_vel_transform(ctx));
    PF_TRY(pf_vel_nonlinear(ctx));
    return pf_util_run(ctx, 2);
}

// main.f90:20-44.  With a fixed dt and the fused kernels, the pass through
// predictor and first corrector is one graph launch and each further
// corrector pass another; the corrector error is read once per pass.
extern "C" int pf_timestep(pf_ctx *ctx, int *ncorr) {
    PF_ARG(ctx, "null ctx");
    PF_TRY(require_matrices(ctx));
    int nc = 0, status = PF_OK;
    // the first step of a context runs eagerly: it sets every kernel's
    // shared-memory attribute, which must not happen during a capture
    if (graphs_ok(ctx) && ctx->graph_warm) {
        const int p = ctx->parity;
        if (!ctx->g_main[p]) {
            // with a built-in plug-in its var_null(2) terms follow each
            // nonlinear evaluation inside the graph (its var_null(1) does
            // nothing on the device)
            PF_TRY(capture(ctx, p, &ctx->g_main[p], &ctx->g_main_n[p], [&]() {
                PF_TRY(pf_vel_imposesym(ctx));
                PF_TRY(main_nonlinear(ctx));
                PF_TRY(pf_vel_step_fused(ctx, 0));
                PF_TRY(main_nonlinear(ctx));
                return pf_vel_step_fused(ctx, 1);
            }));
            // capture swapped the host pointers; the replay below does it for real
            for (int i = 0; i < 3; ++i) std::swap(ctx->vel[i].d, ctx->prev[i].d);
            ctx->parity = p;
        }
        PF_TRY(replay(ctx, p, ctx->g_main[p], ctx->g_main_n[p]));
        for (int i = 0; i < 3; ++i) std::swap(ctx->vel[i].d, ctx->prev[i].d);
        ctx->parity = p ^ 1;
        ctx->cfl_fused = !pf_util_active(ctx);  // the plug-in path materialises vel_r..vel_z instead
        ctx->tim.it = 1;
        for (;;) {
            PF_TRY(read_dterr(ctx));
            const int s = pf_tim_check_cgce(ctx);
            if (s != PF_OK) status = s;
            ++nc;
            if (ctx->tim.it == 0) break;
            const int q = ctx->parity;
            if (!ctx->g_corr[q])
                PF_TRY(capture(ctx, 2 + q, &ctx->g_corr[q], &ctx->g_corr_n[q], [&]() {
                    PF_TRY(main_nonlinear(ctx));
                    return pf_vel_step_fused(ctx, 1);
                }));
            PF_TRY(replay(ctx, 2 + q, ctx->g_corr[q], ctx->g_corr_n[q]));
        }
    } else {
        PF_TRY(pf_vel_imposesym(ctx));
        PF_TRY(main_nonlinear(ctx));
        if (ctx->cfg.dt < 0.0) {
            PF_TRY(pf_vel_maxtstep(ctx));
            PF_TRY(pf_tim_new_tstep(ctx));
            if (ctx->tim.new_dt) PF_TRY(pf_vel_matrices_impl(ctx));
        }
        if (pf_util_active(ctx)) PF_TRY(pf_util_run(ctx, 1));
        PF_TRY(pf_vel_predictor(ctx));
        ctx->tim.it = 1;
        while (ctx->tim.it != 0) {
            PF_TRY(main_nonlinear(ctx));
            PF_TRY(pf_vel_corrector(ctx));
            const int s = pf_tim_check_cgce(ctx);
            if (s != PF_OK) status = s;
            ++nc;
        }
        ctx->graph_warm = graphs_ok(ctx);
    }
    ctx->tim.t = ctx->tim.t + ctx->tim.dt;
    ctx->tim.step = ctx->tim.step + 1;
    if (ncorr) *ncorr = nc;
    return status;
}

// newton.f90:740-762 (without the periodic shift and output)
extern "C" int pf_steporbit(pf_ctx *ctx, int nsteps) {
    PF_ARG(ctx && nsteps >= 0, "pf_steporbit: bad argument");
    PF_TRY(require_matrices(ctx));
    for (int s = 0; s < nsteps; ++s) {
        PF_TRY(pf_vel_imposesym(ctx));
        PF_TRY(transform_nonlinear(ctx));
        PF_TRY(pf_vel_predictor(ctx));
        PF_TRY(transform_nonlinear(ctx));
        PF_TRY(vel_corrector_async(ctx));
        PF_TRY(pf_vel_imposesym(ctx));
        ctx->tim.t = ctx->tim.t + ctx->tim.dt;
        ctx->tim.step = ctx->tim.step + 1;
    }
    PF_TRY(read_dterr(ctx));
    ctx->tim.it = 1;
    return pf_tim_check_cgce(ctx);
}

extern "C" int pf_diag_energy(pf_ctx *ctx, double *E) {
    PF_ARG(ctx && E, "null argument");
    double e = 0.0, t;
    for (int i = 0; i < 3; ++i) {
        PF_TRY(pf_norm_host(ctx, ctx->vel[i].d, &t, nullptr, nullptr));
        e += t;
    }
    *E = e;
    return PF_OK;
}

// io.f90:627-639
extern "C" int pf_diag_friction(pf_ctx *ctx, double *Ub, double *Uc, double *Ufr) {
    PF_ARG(ctx, "null ctx");
    const Geo &g = ctx->g;
    const int N = g.N;
    std::vector<double2> col(N);
    PF_CUDA(cudaMemcpy2DAsync(col.data(), sizeof(double2), ctx->vel[2].d, g.Hp * sizeof(double2),
                              sizeof(double2), N, cudaMemcpyDeviceToHost, ctx->stream));
    PF_CUDA(cudaMemcpyAsync(ctx->hsc, ctx->dsc, sizeof(DevScalars), cudaMemcpyDeviceToHost, ctx->stream));
    PF_CUDA(cudaStreamSynchronize(ctx->stream));
    const HostMesh &hm = ctx->hm;
    double ub = 0.0;
    for (int n = 0; n < N; ++n) ub += col[n].x * hm.intrdr[n];
    ub = 0.5 + 2.0 * ub;
    if (ctx->cfg.const_flux) ub = ctx->hsc->Pr0;
    double uc = 0.0;
    for (int j = 0; j <= KL; ++j) uc += col[j].x * hm.dr0[0 * (KL + 1) + j];
    uc = 1.0 + uc;
    double uf = 0.0;
    for (int j = 0; j <= KL; ++j) uf += col[N - 1 - KL + j].x * hm.dr1[1 * (KL + 1) + j];
    uf = std::sqrt(std::fabs((uf - 2.0) / g.Re));
    if (Ub) *Ub = ub;
    if (Uc) *Uc = uc;
    if (Ufr) *Ufr = uf;
    return PF_OK;
}
