// Many independent pipes of uneven size advanced together.
//
// Each pipe is a full pf_ctx (its own fields, factors and stream).  One
// timestep of the whole batch is a single CUDA graph, built one of two ways:
//
//  * stage-batched (the usual case: fixed dt, N <= 128, built transform
//    lengths 12 to 384, either precision, no symmetry beyond the mean-mode
//    one; a transform stage takes one launch per length and precision): every stage
//    of the step is ONE launch over the tiles of all pipes (a (pipe, tile) map
//    per stage), so a step of the whole batch is about twenty kernels that
//    each fill the GPU, whatever the mix of sizes;
//  * branch graph (otherwise): on every pipe's stream that pipe's own chain of
//    kernels, as a lone pipe runs it; the chains are independent graph
//    branches and run concurrently.
//
// Both run the same per-tile code as a lone pipe, so every pipe's result is
// bit-identical alone and in the batch.  After the replay one host
// synchronisation reads every pipe's corrector error (gathered into one
// pinned copy); the reference's corrector control (timestep.f90:214-253) is
// then applied per pipe, and the rare pipe that needs another corrector pass
// gets it on its own stream (main.f90:35-41).  In orbit mode every pipe takes
// exactly one corrector pass (newton.f90:740-762).
#include <cmath>
#include "pf_internal.cuh"

struct SymArgs {  // one pipe's velocity in one pointer state
    double2 *u[3];
    int N, Hp;
};

// variables.f90:611-616 (the mean-mode symmetry) for every pipe: block = pipe
__global__ void k_batch_sym0(const SymArgs *__restrict__ s) {
    const SymArgs &a = s[blockIdx.x];
    for (int n = threadIdx.x; n < a.N; n += blockDim.x) {
        const size_t at = (size_t)n * a.Hp;
        a.u[0][at] = make_double2(0.0, 0.0);
        a.u[1][at].y = 0.0;
        a.u[2][at].y = 0.0;
    }
}

// every pipe's device scalars into one array, read back with one copy
__global__ void k_batch_scalars(DevScalars *const *__restrict__ src, DevScalars *__restrict__ dst, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) dst[i] = *src[i];
}

struct BatchIO;
struct pf_batch {
    int n;
    std::vector<pf_ctx *> pipes;
    std::vector<char> owned;   // created (and destroyed) by the batch, or attached by the caller
    int device;
    cudaStream_t master;
    cudaEvent_t fork;
    std::vector<cudaEvent_t> join;
    cudaGraphExec_t g[2][2];   // [orbit][parity of pipe 0]
    unsigned long long gn[2][2];
    bool warm;                 // the per-pipe eager step has run (branch graphs)
    bool use_graphs;           // capture steps into graphs (else launch directly)
    bool worklist;             // transform stages as one work-list launch each
    DevScalars *hsc;           // pinned, one per pipe
    int hsc_cap;
    // event pairs of profiled categories captured into each graph:
    // (pipe, category, start, stop)
    struct Ev {
        int pipe, cat;
        cudaEvent_t a, b;
    };
    std::vector<Ev> gev[2][2];
    std::vector<unsigned long long> gnp[2][2];  // kernels per pipe in each graph
    // graph form, decided when the first graph of a membership is made
    int kind;                        // 0 undecided, 1 stage-batched, 2 per-pipe branches
    std::vector<int> rel0;           // each pipe's pointer parity relative to pipe 0 then
    unsigned long long gen0;         // sum of the pipes' matrices generations then
    // stage-batched launches
    bool fresh;                      // built, no step run yet (the first runs uncaptured)
    pf_nl_batch *nlb;
    pf_step_batch *stb;
    int par0;                        // pipe 0's pointer parity when nlb/stb were built
    SymArgs *d_sym[2];               // [pointer state]
    DevScalars **d_scp;              // each pipe's device scalars
    DevScalars *d_scall;             // gathered scalars
    pf_stage_prof sprof;             // stage timing of the batched launches
    std::vector<pf_stage_prof::Open> sev[2][2];
    unsigned long long launches;     // batched kernels launched (not per pipe)
    struct BatchIO *io;              // pipelined state I/O (made on first use)
};
static void batch_io_free(pf_batch *b);

static void staged_free(pf_batch *b) {
    pf_nl_batch_free(b->nlb);
    pf_step_batch_free(b->stb);
    b->nlb = nullptr;
    b->stb = nullptr;
    for (int s = 0; s < 2; ++s) {
        cudaFree(b->d_sym[s]);
        b->d_sym[s] = nullptr;
    }
    cudaFree(b->d_scp);
    cudaFree(b->d_scall);
    b->d_scp = nullptr;
    b->d_scall = nullptr;
}

static unsigned long long matrices_gen(const pf_batch *b) {
    unsigned long long s = 0;
    for (const pf_ctx *c : b->pipes) s += c->matrices_gen;
    return s;
}

// Destroy the batch graphs and hand their event pairs back to the pipes.
static void batch_graphs_reset(pf_batch *b) {
    if (b->master) cudaStreamSynchronize(b->master);
    for (int o = 0; o < 2; ++o)
        for (int p = 0; p < 2; ++p) {
            if (b->g[o][p]) cudaGraphExecDestroy(b->g[o][p]);
            b->g[o][p] = nullptr;
            for (auto &e : b->gev[o][p]) {
                b->pipes[e.pipe]->ev_pool.push_back(e.a);
                b->pipes[e.pipe]->ev_pool.push_back(e.b);
            }
            b->gev[o][p].clear();
            for (auto &e : b->sev[o][p]) {
                b->sprof.pool.push_back(e.a);
                b->sprof.pool.push_back(e.b);
            }
            b->sev[o][p].clear();
        }
    staged_free(b);
    b->kind = 0;
    b->fresh = false;
    b->warm = false;
}

static void batch_free(pf_batch *b) {
    batch_graphs_reset(b);
    batch_io_free(b);
    for (cudaEvent_t e : b->join) cudaEventDestroy(e);
    if (b->fork) cudaEventDestroy(b->fork);
    if (b->master) cudaStreamDestroy(b->master);
    if (b->hsc) cudaFreeHost(b->hsc);
    for (auto &e : b->sprof.open) {
        b->sprof.pool.push_back(e.a);
        b->sprof.pool.push_back(e.b);
    }
    for (cudaEvent_t e : b->sprof.pool) cudaEventDestroy(e);
    for (int i = 0; i < b->n; ++i)
        if (b->owned[i]) pf_ctx_destroy(b->pipes[i]);
    delete b;
}

// per-pipe host resources for n pipes: join events and the pinned scalars
static int batch_reserve(pf_batch *b, int n) {
    while ((int)b->join.size() < n) {
        cudaEvent_t e = nullptr;
        PF_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        b->join.push_back(e);
    }
    if (n > b->hsc_cap) {
        const int cap = std::max(n, 2 * b->hsc_cap);
        DevScalars *h = nullptr;
        PF_CUDA(cudaMallocHost((void **)&h, cap * sizeof(DevScalars)));
        if (b->hsc) cudaFreeHost(b->hsc);
        b->hsc = h;
        b->hsc_cap = cap;
    }
    return PF_OK;
}

extern "C" int pf_batch_create(int npipes, const pf_config *cfgs, int device, pf_batch **out) {
    PF_ARG(npipes >= 0 && (cfgs || npipes == 0) && out, "pf_batch_create: bad argument");
    *out = nullptr;
    pf_batch *b = new pf_batch();
    b->use_graphs = true;
    if (device >= 0 && cudaSetDevice(device) != cudaSuccess) {
        delete b;
        pf_set_error("pf_batch_create: cannot select device %d", device);
        return PF_ERR_NODEVICE;
    }
    if (cudaGetDevice(&b->device) != cudaSuccess) {
        delete b;
        pf_set_error("pf_batch_create: no CUDA device");
        return PF_ERR_NODEVICE;
    }
    for (int i = 0; i < npipes; ++i) {
        pf_ctx *c = nullptr;
        const int s = pf_ctx_create(&cfgs[i], b->device, &c);
        if (s != PF_OK) {
            batch_free(b);
            return s;
        }
        b->pipes.push_back(c);
        b->owned.push_back(1);
        b->n = (int)b->pipes.size();
    }
    if (cudaStreamCreateWithFlags(&b->master, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming) != cudaSuccess) {
        batch_free(b);
        pf_set_error("pf_batch_create: stream/event allocation failed");
        return PF_ERR_CUDA;
    }
    const int s = batch_reserve(b, std::max(npipes, 1));
    if (s != PF_OK) {
        batch_free(b);
        return s;
    }
    *out = b;
    return PF_OK;
}

extern "C" int pf_batch_destroy(pf_batch *b) {
    if (b) batch_free(b);
    return PF_OK;
}

extern "C" int pf_batch_pipe(pf_batch *b, int i, pf_ctx **out) {
    PF_ARG(b && out && i >= 0 && i < b->n, "pf_batch_pipe: bad argument");
    *out = b->pipes[i];
    return PF_OK;
}

extern "C" int pf_batch_size(pf_batch *b, int *n) {
    PF_ARG(b && n, "pf_batch_size: bad argument");
    *n = b->n;
    return PF_OK;
}

// Add a context the caller owns (it must live on the batch's device and stay
// alive until detached); the next step rebuilds the batch's launches.
extern "C" int pf_batch_attach(pf_batch *b, pf_ctx *c) {
    PF_ARG(b && c, "pf_batch_attach: bad argument");
    PF_ARG(c->device == b->device, "pf_batch_attach: context is on another device");
    for (pf_ctx *q : b->pipes) PF_ARG(q != c, "pf_batch_attach: context already in the batch");
    batch_graphs_reset(b);
    PF_TRY(batch_reserve(b, b->n + 1));
    PF_CUDA(cudaStreamSynchronize(c->stream));  // its own pending work is done before batched launches
    b->pipes.push_back(c);
    b->owned.push_back(0);
    b->n = (int)b->pipes.size();
    return PF_OK;
}

// Remove a context the caller attached (the batch's own pipes stay).
extern "C" int pf_batch_detach(pf_batch *b, pf_ctx *c) {
    PF_ARG(b && c, "pf_batch_detach: bad argument");
    for (int i = 0; i < b->n; ++i)
        if (b->pipes[i] == c) {
            PF_ARG(!b->owned[i], "pf_batch_detach: the batch owns this pipe");
            batch_graphs_reset(b);
            b->pipes.erase(b->pipes.begin() + i);
            b->owned.erase(b->owned.begin() + i);
            b->n = (int)b->pipes.size();
            return PF_OK;
        }
    pf_set_error("pf_batch_detach: context not in the batch");
    return PF_ERR_ARG;
}

// on = 1 (default): steps replay captured graphs; 0: every step launches
// directly (for batches whose membership changes from step to step).
extern "C" int pf_batch_set_graphs(pf_batch *b, int on) {
    PF_ARG(b, "null batch");
    if (!on) batch_graphs_reset(b);
    b->use_graphs = on != 0;
    return PF_OK;
}

// on = 1: in the stage-batched form each transform stage is one persistent
// launch over a work list of every pipe's tiles (where every pipe is in mixed
// precision with transform lengths from 36 to 192); 0 (default): one launch per
// stage and transform length.  Results are bitwise the same either way.
extern "C" int pf_batch_set_worklist(pf_batch *b, int on) {
    PF_ARG(b, "null batch");
    if ((on != 0) != b->worklist) batch_graphs_reset(b);
    b->worklist = on != 0;
    return PF_OK;
}

extern "C" int pf_batch_get_worklist(pf_batch *b, int *on) {
    PF_ARG(b && on, "pf_batch_get_worklist: bad argument");
    *on = b->worklist ? 1 : 0;
    return PF_OK;
}

extern "C" int pf_batch_matrices(pf_batch *b) {
    PF_ARG(b, "null batch");
    batch_graphs_reset(b);
    for (pf_ctx *c : b->pipes) PF_TRY(pf_vel_matrices(c));
    return PF_OK;
}

static bool batch_graphable(const pf_batch *b) {
    for (const pf_ctx *c : b->pipes)
        if (!(c->cfg.dt > 0.0 && c->matrices_ready && pf_nl_fused_supported(c) && pf_fused_step_ok(c)) ||
            pf_util_active(c))
            return false;
    return true;
}

// Whether the stage-batched kernels cover every pipe of the batch.
static bool batch_stageable(const pf_batch *b) {
    for (const pf_ctx *c : b->pipes)
        if (c->cfg.mirrorsym || c->cfg.shiftrefl || c->cfg.shiftrott) return false;
    return pf_nl_batch_supported(b->pipes.data(), b->n);
}

// Per-pipe arguments of the stage-batched kernels for both pointer states.
static int staged_build(pf_batch *b) {
    staged_free(b);
    PF_TRY(pf_nl_batch_build(b->pipes.data(), b->n, b->worklist, &b->nlb));
    PF_TRY(pf_step_batch_build(b->pipes.data(), b->n, &b->stb));
    std::vector<SymArgs> sym(b->n);
    std::vector<DevScalars *> scp(b->n);
    for (int s = 0; s < 2; ++s) {
        for (int i = 0; i < b->n; ++i) {
            const pf_ctx *c = b->pipes[i];
            for (int k = 0; k < 3; ++k) sym[i].u[k] = s ? c->prev[k].d : c->vel[k].d;
            sym[i].N = c->g.N;
            sym[i].Hp = c->g.Hp;
        }
        PF_CUDA(cudaMalloc((void **)&b->d_sym[s], b->n * sizeof(SymArgs)));
        PF_CUDA(cudaMemcpy(b->d_sym[s], sym.data(), b->n * sizeof(SymArgs), cudaMemcpyHostToDevice));
    }
    for (int i = 0; i < b->n; ++i) scp[i] = b->pipes[i]->dsc;
    PF_CUDA(cudaMalloc((void **)&b->d_scp, b->n * sizeof(DevScalars *)));
    PF_CUDA(cudaMemcpy(b->d_scp, scp.data(), b->n * sizeof(DevScalars *), cudaMemcpyHostToDevice));
    PF_CUDA(cudaMalloc((void **)&b->d_scall, b->n * sizeof(DevScalars)));
    b->par0 = b->pipes[0]->parity;
    b->gen0 = matrices_gen(b);
    return PF_OK;
}

// The stage-batched step: imposesym, nonlinear terms, predictor, nonlinear
// terms, corrector (and imposesym in orbit mode) of every pipe, then the
// gathered device scalars to pinned host memory.
static int staged_body(pf_batch *b, int orbit, int par, unsigned long long *nk) {
    const int s0 = par ^ b->par0, s1 = s0 ^ 1;  // pointer state before / after the predictor's swap
    cudaStream_t st = b->master;
    pf_stage_prof *pr = &b->sprof;
    {
        StageScope ss_(pr, PF_K_EW, st);
        k_batch_sym0<<<b->n, 64, 0, st>>>(b->d_sym[s0]);
    }
    PF_CHECK_LAUNCH();
    ++*nk;
    PF_TRY(pf_nl_batch_launch(b->nlb, s0, st, pr, nk));
    PF_TRY(pf_step_batch_launch(b->stb, s1, 0, st, pr, nk));
    PF_TRY(pf_nl_batch_launch(b->nlb, s1, st, pr, nk));
    PF_TRY(pf_step_batch_launch(b->stb, s1, 1, st, pr, nk));
    if (orbit) {
        {
            StageScope ss_(pr, PF_K_EW, st);
            k_batch_sym0<<<b->n, 64, 0, st>>>(b->d_sym[s1]);
        }
        PF_CHECK_LAUNCH();
        ++*nk;
    }
    {
        StageScope ss_(pr, PF_K_EW, st);
        k_batch_scalars<<<grid1(b->n, 128), 128, 0, st>>>(b->d_scp, b->d_scall, b->n);
    }
    PF_CHECK_LAUNCH();
    ++*nk;
    PF_CUDA(cudaMemcpyAsync(b->hsc, b->d_scall, b->n * sizeof(DevScalars), cudaMemcpyDeviceToHost, st));
    return PF_OK;
}

static int staged_capture(pf_batch *b, int orbit, int par, cudaGraphExec_t *exec, unsigned long long *nk) {
    const size_t open0 = b->sprof.open.size();
    cudaGraph_t graph = nullptr;
    *nk = 0;
    PF_CUDA(cudaStreamBeginCapture(b->master, cudaStreamCaptureModeThreadLocal));
    const int s = staged_body(b, orbit, par, nk);
    const cudaError_t e = cudaStreamEndCapture(b->master, &graph);
    for (size_t k = open0; k < b->sprof.open.size(); ++k) b->sev[orbit][par].push_back(b->sprof.open[k]);
    b->sprof.open.resize(open0);
    if (s != PF_OK || e != cudaSuccess) {
        if (graph) cudaGraphDestroy(graph);
        if (s == PF_OK) pf_set_error("batch graph capture failed: %s", cudaGetErrorString(e));
        return s == PF_OK ? PF_ERR_CUDA : s;
    }
    const cudaError_t e2 = cudaGraphInstantiate(exec, graph, 0);
    cudaGraphDestroy(graph);
    if (e2 != cudaSuccess) {
        pf_set_error("batch graph instantiation failed: %s", cudaGetErrorString(e2));
        return PF_ERR_CUDA;
    }
    return PF_OK;
}

// one pipe's body of the batch graph
static int pipe_body(pf_ctx *c, int orbit) {
    PF_TRY(pf_vel_imposesym(c));
    PF_TRY(pf_transform_nonlinear(c));
    PF_TRY(pf_vel_step_fused(c, 0));
    PF_TRY(pf_transform_nonlinear(c));
    PF_TRY(pf_vel_step_fused(c, 1));
    if (orbit) PF_TRY(pf_vel_imposesym(c));
    return PF_OK;
}

static int batch_capture(pf_batch *b, int orbit, int par, cudaGraphExec_t *exec, unsigned long long *nk) {
    std::vector<unsigned long long> n0(b->n);
    for (int i = 0; i < b->n; ++i) n0[i] = b->pipes[i]->launches;
    std::vector<size_t> open0((size_t)b->n * PF_K_NCAT);
    for (int i = 0; i < b->n; ++i)
        for (int c = 0; c < PF_K_NCAT; ++c) open0[(size_t)i * PF_K_NCAT + c] = b->pipes[i]->ev_open[c].size();
    cudaGraph_t graph = nullptr;
    PF_CUDA(cudaStreamBeginCapture(b->master, cudaStreamCaptureModeThreadLocal));
    int s = PF_OK;
    if (cudaEventRecord(b->fork, b->master) != cudaSuccess) s = PF_ERR_CUDA;
    for (int i = 0; i < b->n && s == PF_OK; ++i) {
        pf_ctx *c = b->pipes[i];
        if (cudaStreamWaitEvent(c->stream, b->fork, 0) != cudaSuccess) { s = PF_ERR_CUDA; break; }
        s = pipe_body(c, orbit);
        if (s != PF_OK) break;
        if (cudaMemcpyAsync(&b->hsc[i], c->dsc, sizeof(DevScalars), cudaMemcpyDeviceToHost, c->stream) != cudaSuccess ||
            cudaEventRecord(b->join[i], c->stream) != cudaSuccess ||
            cudaStreamWaitEvent(b->master, b->join[i], 0) != cudaSuccess)
            s = PF_ERR_CUDA;
    }
    const cudaError_t e = cudaStreamEndCapture(b->master, &graph);
    // event pairs recorded during the capture belong to the graph
    for (int i = 0; i < b->n; ++i)
        for (int c = 0; c < PF_K_NCAT; ++c) {
            auto &open = b->pipes[i]->ev_open[c];
            const size_t from = open0[(size_t)i * PF_K_NCAT + c];
            for (size_t k = from; k < open.size(); ++k) b->gev[orbit][par].push_back({i, c, open[k].first, open[k].second});
            open.resize(from);
        }
    // the capture swapped each pipe's host pointers; the replay does it for real
    for (pf_ctx *c : b->pipes)
        for (int i = 0; i < 3; ++i) std::swap(c->vel[i].d, c->prev[i].d);
    for (pf_ctx *c : b->pipes) c->parity ^= 1;
    if (s != PF_OK || e != cudaSuccess) {
        if (graph) cudaGraphDestroy(graph);
        if (s == PF_OK) pf_set_error("batch graph capture failed: %s", cudaGetErrorString(e));
        return s == PF_OK ? PF_ERR_CUDA : s;
    }
    const cudaError_t e2 = cudaGraphInstantiate(exec, graph, 0);
    cudaGraphDestroy(graph);
    if (e2 != cudaSuccess) {
        pf_set_error("batch graph instantiation failed: %s", cudaGetErrorString(e2));
        return PF_ERR_CUDA;
    }
    // kernels per pipe are counted at each replay, not at capture
    b->gnp[orbit][par].assign(b->n, 0);
    *nk = 0;
    for (int i = 0; i < b->n; ++i) {
        b->gnp[orbit][par][i] = b->pipes[i]->launches - n0[i];
        *nk += b->gnp[orbit][par][i];
        b->pipes[i]->launches = n0[i];
    }
    return PF_OK;
}

// The pipes' pointer parities relative to pipe 0.  Every batched step swaps
// every pipe, so they stay fixed unless a pipe is stepped on its own.
static std::vector<int> rel_parity(const pf_batch *b) {
    std::vector<int> r(b->n);
    for (int i = 0; i < b->n; ++i) r[i] = b->pipes[i]->parity ^ b->pipes[0]->parity;
    return r;
}

// Corrector control after a batched step (timestep.f90:214-253, main.f90:35-41)
// from the scalars the step left in b->hsc; returns the passes taken.
static long long batch_after_step(pf_batch *b, int orbit, int *status) {
    long long passes = 0;
    for (int i = 0; i < b->n; ++i) {
        pf_ctx *c = b->pipes[i];
        const double err2 = bits_to_double(b->hsc[i].dterr2_bits);
        c->tim.dterr = std::max(c->tim.dterr, std::sqrt(err2));
        c->tim.it = 1;
        c->last_status = PF_OK;
        c->last_error.clear();
        int s = pf_tim_check_cgce(c);
        if (s != PF_OK) {
            c->last_status = s;
            c->last_error = pf_last_error();
        }
        // the state went non-finite: the max of the corrections' bit patterns
        // is a NaN or Inf pattern (the reference would carry on with NaN)
        if (!std::isfinite(err2) && c->last_status == PF_OK) {
            c->last_status = PF_ERR_CONVERGE;
            c->last_error = "non-finite corrector error: NaN or Inf in the state";
        }
        ++passes;
        if (!orbit) {
            while (c->tim.it != 0) {  // further corrector passes for this pipe only
                int e = pf_transform_nonlinear(c);
                if (e == PF_OK) e = pf_vel_step_fused(c, 1);
                if (e == PF_OK) e = pf_read_dterr(c);
                if (e != PF_OK) {
                    *status = e;
                    c->tim.it = 0;
                    break;
                }
                s = pf_tim_check_cgce(c);
                if (s != PF_OK && c->last_status == PF_OK) {
                    c->last_status = s;
                    c->last_error = pf_last_error();
                }
                ++passes;
            }
            if (s != PF_OK) *status = s;
        } else {
            c->tim.it = 0;
        }
        c->tim.t = c->tim.t + c->tim.dt;
        c->tim.step = c->tim.step + 1;
    }
    return passes;
}

// Read the stage and kernel event pairs of a finished step into the totals.
static void batch_collect_events(pf_batch *b, std::vector<pf_stage_prof::Open> *stage, bool release) {
    for (auto &e : *stage) {
        float ms = 0.f;
        if (cudaEventElapsedTime(&ms, e.a, e.b) == cudaSuccess) {
            b->sprof.ms[e.cat] += ms;
            b->sprof.n[e.cat] += 1;
        } else {
            cudaGetLastError();
        }
        if (release) {
            b->sprof.pool.push_back(e.a);
            b->sprof.pool.push_back(e.b);
        }
    }
    if (release) stage->clear();
}

// Advance every pipe by nsteps timesteps.  orbit=0: the main.f90 step with
// the corrector iterated to convergence per pipe; orbit=1: steporbit's step
// with exactly one corrector.  *corr_passes (may be NULL) returns the total
// number of corrector passes taken over all pipes and steps.
extern "C" int pf_batch_step(pf_batch *b, int nsteps, int orbit, long long *corr_passes) {
    PF_ARG(b && nsteps >= 0, "pf_batch_step: bad argument");
    orbit = orbit ? 1 : 0;
    long long passes = 0;
    int status = PF_OK;
    for (int st = 0; st < nsteps && b->n > 0; ++st) {
        if (!batch_graphable(b)) {  // adaptive dt, very large N, unbuilt lengths: eager per pipe
            for (pf_ctx *c : b->pipes) {
                if (orbit) {
                    PF_TRY(pf_steporbit(c, 1));
                    passes += 1;
                } else {
                    int nc = 0;
                    const int s = pf_timestep(c, &nc);
                    c->last_status = s;
                    c->last_error = s != PF_OK ? pf_last_error() : "";
                    if (s != PF_OK) status = s;
                    passes += nc;
                }
            }
            continue;
        }
        // the graphs and batched arguments bake in each pipe's factor sets,
        // 1/dt and pointer state relative to the other pipes
        if (b->kind != 0 && (matrices_gen(b) != b->gen0 || rel_parity(b) != b->rel0)) batch_graphs_reset(b);
        if (b->kind == 0) {
            b->gen0 = matrices_gen(b);
            b->rel0 = rel_parity(b);
            b->kind = batch_stageable(b) ? 1 : 2;
            if (b->kind == 1) {
                PF_TRY(staged_build(b));
                b->fresh = true;
            }
        }
        const int p = b->pipes[0]->parity;
        // work the caller queued on a pipe's own stream (set_state, uploads)
        // comes before the batch's launches on the master stream
        for (int i = 0; i < b->n; ++i) {
            PF_CUDA(cudaEventRecord(b->join[i], b->pipes[i]->stream));
            PF_CUDA(cudaStreamWaitEvent(b->master, b->join[i], 0));
        }
        if (b->kind == 1 && (b->fresh || !b->use_graphs)) {
            // launched directly: the first step after a build (it also sets
            // the kernels' shared-memory limits outside any capture) and
            // every step of a batch whose membership keeps changing
            unsigned long long nk = 0;
            const size_t open0 = b->sprof.open.size();
            PF_TRY(staged_body(b, orbit, p, &nk));
            b->launches += nk;
            b->fresh = false;
            for (pf_ctx *c : b->pipes) {
                for (int i = 0; i < 3; ++i) std::swap(c->vel[i].d, c->prev[i].d);
                c->parity ^= 1;
                c->cfl_fused = true;
            }
            PF_CUDA(cudaStreamSynchronize(b->master));
            std::vector<pf_stage_prof::Open> mine(b->sprof.open.begin() + open0, b->sprof.open.end());
            b->sprof.open.resize(open0);
            batch_collect_events(b, &mine, true);
            passes += batch_after_step(b, orbit, &status);
            continue;
        }
        if (b->kind == 2 && !b->warm) {
            // eager step per pipe (also sets every kernel attribute before any capture)
            for (pf_ctx *c : b->pipes) {
                if (orbit) {
                    PF_TRY(pf_steporbit(c, 1));
                    passes += 1;
                } else {
                    int nc = 0;
                    const int s = pf_timestep(c, &nc);
                    if (s != PF_OK) status = s;
                    passes += nc;
                }
            }
            b->warm = true;
            b->rel0 = rel_parity(b);
            continue;
        }
        if (!b->g[orbit][p]) {
            if (b->kind == 1) PF_TRY(staged_capture(b, orbit, p, &b->g[orbit][p], &b->gn[orbit][p]));
            else PF_TRY(batch_capture(b, orbit, p, &b->g[orbit][p], &b->gn[orbit][p]));
        }
        PF_CUDA(cudaGraphLaunch(b->g[orbit][p], b->master));
        for (pf_ctx *c : b->pipes) {
            for (int i = 0; i < 3; ++i) std::swap(c->vel[i].d, c->prev[i].d);
            c->parity ^= 1;
            c->cfl_fused = true;
        }
        if (b->kind == 1)
            b->launches += b->gn[orbit][p];
        else
            for (int i = 0; i < b->n; ++i) b->pipes[i]->launches += b->gnp[orbit][p][i];
        PF_CUDA(cudaStreamSynchronize(b->master));
        batch_collect_events(b, &b->sev[orbit][p], false);
        for (auto &e : b->gev[orbit][p]) {  // kernel times of the profiled categories
            float ms = 0.f;
            pf_ctx *c = b->pipes[e.pipe];
            if (cudaEventElapsedTime(&ms, e.a, e.b) == cudaSuccess) {
                c->prof_ms[e.cat] += ms;
                c->prof_n[e.cat] += 1;
            } else {
                cudaGetLastError();
            }
        }
        passes += batch_after_step(b, orbit, &status);
    }
    if (corr_passes) *corr_passes = passes;
    return status;
}

extern "C" int pf_batch_sync(pf_batch *b) {
    PF_ARG(b, "null batch");
    PF_CUDA(cudaStreamSynchronize(b->master));
    for (pf_ctx *c : b->pipes) PF_CUDA(cudaStreamSynchronize(c->stream));
    return PF_OK;
}

// Event timing of the categories in `mask` (1 << PF_K_*) for every pipe of
// the batch, inside the batch graphs; each call clears the totals.
extern "C" int pf_batch_prof_enable(pf_batch *b, int mask) {
    PF_ARG(b, "null batch");
    bool changed = b->sprof.mask != mask;
    for (pf_ctx *c : b->pipes) changed |= (c->prof_mask != mask);
    if (changed) batch_graphs_reset(b);
    for (pf_ctx *c : b->pipes) PF_TRY(pf_prof_enable(c, mask));
    b->sprof.mask = mask;
    for (int c = 0; c < PF_K_NCAT; ++c) {
        b->sprof.ms[c] = 0.0;
        b->sprof.n[c] = 0;
    }
    return PF_OK;
}

// Device milliseconds and launches of category `cat` summed over the pipes.
extern "C" int pf_batch_prof_read(pf_batch *b, int cat, double *ms, unsigned long long *launches) {
    PF_ARG(b && cat >= 0 && cat < PF_K_NCAT, "pf_batch_prof_read: bad argument");
    double t = 0.0;
    unsigned long long n = 0;
    for (pf_ctx *c : b->pipes) {
        double m = 0.0;
        unsigned long long k = 0;
        PF_TRY(pf_prof_read(c, cat, &m, &k));
        t += m;
        n += k;
    }
    if (ms) *ms = t + b->sprof.ms[cat];
    if (launches) *launches = n + b->sprof.n[cat];
    return PF_OK;
}

// Device milliseconds and spans of category `cat` of the stage-batched
// launches alone (every span covers all pipes of the batch).
extern "C" int pf_batch_prof_read_staged(pf_batch *b, int cat, double *ms, unsigned long long *launches) {
    PF_ARG(b && cat >= 0 && cat < PF_K_NCAT, "pf_batch_prof_read_staged: bad argument");
    if (ms) *ms = b->sprof.ms[cat];
    if (launches) *launches = b->sprof.n[cat];
    return PF_OK;
}

// Kernels launched by the batch: the pipes' own plus the batched ones.
extern "C" int pf_batch_launches(pf_batch *b, unsigned long long *n) {
    PF_ARG(b && n, "pf_batch_launches: bad argument");
    unsigned long long t = b->launches;
    for (const pf_ctx *c : b->pipes) t += c->launches;
    *n = t;
    return PF_OK;
}

// 1 when the batch's graphs are stage-batched (one launch per stage over
// every pipe), 0 for per-pipe graph branches or before the first graph.
extern "C" int pf_batch_staged(pf_batch *b, int *staged) {
    PF_ARG(b && staged, "pf_batch_staged: bad argument");
    *staged = b->kind == 1 ? 1 : 0;
    return PF_OK;
}

// The batch's master stream (graph launches are ordered on it).
extern "C" int pf_batch_stream(pf_batch *b, void **stream) {
    PF_ARG(b && stream, "pf_batch_stream: bad argument");
    *stream = (void *)b->master;
    return PF_OK;
}

// ------------------------------------------------------- pipelined state I/O
// A state block holds the velocity states of every pipe of the batch, pipe
// after pipe in batch order; pipe i takes 6*N_i*H_i doubles: ur Re, ur Im,
// ut Re, ut Im, uz Re, uz Im, each H_i x N_i with the radial index fastest
// (the layout of pf_vel_set_state's arrays, that of %Re(n,nh)).  Two input
// and two output slots on the device, and one copy stream per direction, let
// the upload of the next block and the download of the last one run while
// the step in between computes.  No reference routine: the host side of
// io.f90's state access for many pipes, overlapped with stepping.

#define IO_MAX 64  // pipes per pack/unpack launch (kernel parameter space)

struct IoPipe {
    double2 *f[3];
    long long off;  // doubles from the start of the block
    int N, H, Hp;
};
struct IoArgs {
    IoPipe p[IO_MAX];
    int tile0[IO_MAX + 1];  // first 32x32 tile of each pipe (3 fields per pipe)
    int n;
};

// block <-> device fields for up to IO_MAX pipes; one block per 32x32 tile
// (radial points x modes) of one field, transposed through shared memory
template <bool UNPACK>
static __global__ void __launch_bounds__(256) k_batch_io(const __grid_constant__ IoArgs a, double *__restrict__ blk) {
    __shared__ double2 tile[32][33];
    const int b = blockIdx.x;
    int p = 0;
    while (p + 1 < a.n && a.tile0[p + 1] <= b) ++p;
    const IoPipe &q = a.p[p];
    const int N = q.N, H = q.H, Hp = q.Hp;
    const int th = (H + 31) >> 5, tn = (N + 31) >> 5;
    int t = b - a.tile0[p];
    const int c = t / (th * tn);
    t -= c * th * tn;
    const int nh0 = (t % th) * 32, n0 = (t / th) * 32;
    double *re = blk + q.off + (size_t)(2 * c) * H * N;
    double *im = re + (size_t)H * N;
    double2 *f = c == 0 ? q.f[0] : (c == 1 ? q.f[1] : q.f[2]);
    if (UNPACK) {
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
            if (n < N && nh < Hp) f[(size_t)n * Hp + nh] = nh < H ? tile[threadIdx.x][i] : make_double2(0.0, 0.0);
        }
    } else {
        for (int i = threadIdx.y; i < 32; i += blockDim.y) {
            const int n = n0 + i, nh = nh0 + threadIdx.x;
            if (n < N && nh < H) tile[threadIdx.x][i] = f[(size_t)n * Hp + nh];
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
}

struct BatchIO {
    size_t cap;  // doubles per slot
    double *in[2], *out[2];
    cudaStream_t up, down;
    cudaEvent_t in_ready[2], in_free[2], out_ready[2], out_free[2];
    bool filled[2];  // an upload into in[slot] has been queued
};

static void batch_io_free(pf_batch *b) {
    BatchIO *io = b->io;
    if (!io) return;
    if (io->up) cudaStreamSynchronize(io->up);
    if (io->down) cudaStreamSynchronize(io->down);
    if (b->master) cudaStreamSynchronize(b->master);
    for (int s = 0; s < 2; ++s) {
        cudaFree(io->in[s]);
        cudaFree(io->out[s]);
        for (cudaEvent_t e : {io->in_ready[s], io->in_free[s], io->out_ready[s], io->out_free[s]})
            if (e) cudaEventDestroy(e);
    }
    if (io->up) cudaStreamDestroy(io->up);
    if (io->down) cudaStreamDestroy(io->down);
    delete io;
    b->io = nullptr;
}

// doubles of a state block for the current membership
static size_t io_total(const pf_batch *b) {
    size_t t = 0;
    for (const pf_ctx *c : b->pipes) t += (size_t)6 * c->g.N * c->g.H;
    return t;
}

// the I/O state with slots of at least `need` doubles
static int io_ready(pf_batch *b, size_t need, BatchIO **out) {
    if (!b->io) {
        BatchIO *io = new BatchIO();
        b->io = io;
        PF_CUDA(cudaStreamCreateWithFlags(&io->up, cudaStreamNonBlocking));
        PF_CUDA(cudaStreamCreateWithFlags(&io->down, cudaStreamNonBlocking));
        for (int s = 0; s < 2; ++s)
            for (cudaEvent_t *e : {&io->in_ready[s], &io->in_free[s], &io->out_ready[s], &io->out_free[s]})
                PF_CUDA(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
    }
    BatchIO *io = b->io;
    if (need > io->cap) {
        PF_CUDA(cudaStreamSynchronize(io->up));
        PF_CUDA(cudaStreamSynchronize(io->down));
        PF_CUDA(cudaStreamSynchronize(b->master));
        for (int s = 0; s < 2; ++s) {
            cudaFree(io->in[s]);
            cudaFree(io->out[s]);
            io->in[s] = io->out[s] = nullptr;
            io->filled[s] = false;
        }
        io->cap = 0;
        for (int s = 0; s < 2; ++s) {
            if (cudaMalloc((void **)&io->in[s], need * sizeof(double)) != cudaSuccess ||
                cudaMalloc((void **)&io->out[s], need * sizeof(double)) != cudaSuccess) {
                cudaGetLastError();
                pf_set_error("pf_batch state I/O: cannot allocate 4 x %zu bytes of staging", need * sizeof(double));
                return PF_ERR_NOMEM;
            }
        }
        io->cap = need;
    }
    *out = io;
    return PF_OK;
}

// pack (UNPACK=false) or unpack every pipe's fields on the master stream
static int io_launch(pf_batch *b, bool unpack, double *blk) {
    long long off = 0;
    for (int i0 = 0; i0 < b->n; i0 += IO_MAX) {
        IoArgs a{};
        a.n = std::min(IO_MAX, b->n - i0);
        int tiles = 0;
        for (int j = 0; j < a.n; ++j) {
            pf_ctx *c = b->pipes[i0 + j];
            IoPipe &q = a.p[j];
            for (int f = 0; f < 3; ++f) q.f[f] = c->vel[f].d;
            q.off = off;
            q.N = c->g.N;
            q.H = c->g.H;
            q.Hp = c->g.Hp;
            a.tile0[j] = tiles;
            tiles += 3 * ((q.H + 31) / 32) * ((q.N + 31) / 32);
            off += 6LL * q.N * q.H;
        }
        a.tile0[a.n] = tiles;
        if (tiles == 0) continue;
        if (unpack)
            k_batch_io<true><<<tiles, dim3(32, 8), 0, b->master>>>(a, blk);
        else
            k_batch_io<false><<<tiles, dim3(32, 8), 0, b->master>>>(a, blk);
        PF_CHECK_LAUNCH();
        b->launches++;
    }
    return PF_OK;
}

extern "C" int pf_batch_io_bytes(pf_batch *b, unsigned long long *bytes) {
    PF_ARG(b && bytes, "pf_batch_io_bytes: null argument");
    *bytes = (unsigned long long)io_total(b) * sizeof(double);
    return PF_OK;
}

extern "C" int pf_batch_put_states(pf_batch *b, int slot, const double *host) {
    PF_ARG(b && host && (slot == 0 || slot == 1), "pf_batch_put_states: bad argument");
    const size_t total = io_total(b);
    BatchIO *io = nullptr;
    PF_TRY(io_ready(b, std::max<size_t>(total, 1), &io));
    PF_CUDA(cudaStreamWaitEvent(io->up, io->in_free[slot], 0));
    PF_CUDA(cudaMemcpyAsync(io->in[slot], host, total * sizeof(double), cudaMemcpyHostToDevice, io->up));
    PF_CUDA(cudaEventRecord(io->in_ready[slot], io->up));
    io->filled[slot] = true;
    return PF_OK;
}

extern "C" int pf_batch_step_io(pf_batch *b, int slot, int nsteps, int orbit, long long *corr_passes) {
    PF_ARG(b && (slot == 0 || slot == 1) && nsteps >= 0, "pf_batch_step_io: bad argument");
    const size_t total = io_total(b);
    if (!b->io || b->io->cap < total || !b->io->filled[slot]) {
        pf_set_error("pf_batch_step_io: no state block put into slot %d for this membership", slot);
        return PF_ERR_STATE;
    }
    BatchIO *io = b->io;
    // the block's upload, then every pipe's fields from it
    PF_CUDA(cudaStreamWaitEvent(b->master, io->in_ready[slot], 0));
    PF_TRY(io_launch(b, true, io->in[slot]));
    PF_CUDA(cudaEventRecord(io->in_free[slot], b->master));
    io->filled[slot] = false;
    // steps that run per pipe on the pipes' own streams come after it
    PF_CUDA(cudaEventRecord(b->fork, b->master));
    for (pf_ctx *c : b->pipes) PF_CUDA(cudaStreamWaitEvent(c->stream, b->fork, 0));
    const int s = pf_batch_step(b, nsteps, orbit, corr_passes);
    if (s != PF_OK && s != PF_ERR_CONVERGE) return s;
    for (int i = 0; i < b->n; ++i) {
        PF_CUDA(cudaEventRecord(b->join[i], b->pipes[i]->stream));
        PF_CUDA(cudaStreamWaitEvent(b->master, b->join[i], 0));
    }
    // the states into the output slot once its last download has finished
    PF_CUDA(cudaStreamWaitEvent(b->master, io->out_free[slot], 0));
    PF_TRY(io_launch(b, false, io->out[slot]));
    PF_CUDA(cudaEventRecord(io->out_ready[slot], b->master));
    return s;
}

extern "C" int pf_batch_get_states(pf_batch *b, int slot, double *host) {
    PF_ARG(b && host && (slot == 0 || slot == 1), "pf_batch_get_states: bad argument");
    const size_t total = io_total(b);
    if (!b->io || b->io->cap < total) {
        pf_set_error("pf_batch_get_states: no pf_batch_step_io has filled slot %d", slot);
        return PF_ERR_STATE;
    }
    BatchIO *io = b->io;
    PF_CUDA(cudaStreamWaitEvent(io->down, io->out_ready[slot], 0));
    PF_CUDA(cudaMemcpyAsync(host, io->out[slot], total * sizeof(double), cudaMemcpyDeviceToHost, io->down));
    PF_CUDA(cudaEventRecord(io->out_free[slot], io->down));
    return PF_OK;
}

extern "C" int pf_batch_io_wait(pf_batch *b, int slot) {
    PF_ARG(b && (slot == 0 || slot == 1), "pf_batch_io_wait: bad argument");
    if (!b->io) return PF_OK;
    PF_CUDA(cudaEventSynchronize(b->io->out_free[slot]));
    return PF_OK;
}

extern "C" int pf_batch_io_sync(pf_batch *b) {
    PF_ARG(b, "pf_batch_io_sync: null batch");
    if (!b->io) return PF_OK;
    PF_CUDA(cudaStreamSynchronize(b->io->up));
    PF_CUDA(cudaStreamSynchronize(b->master));
    PF_CUDA(cudaStreamSynchronize(b->io->down));
    return PF_OK;
}
