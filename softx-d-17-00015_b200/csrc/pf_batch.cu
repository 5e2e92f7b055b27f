// Many independent pipes of uneven size advanced together.
//
// Each pipe is a full pf_ctx (its own fields, factors and stream).  One
// timestep of the whole batch is a single CUDA graph: a fork event on the
// batch's master stream, then on every pipe's stream that pipe's imposesym,
// nonlinear terms, predictor, nonlinear terms and corrector (the same
// kernels as a lone pipe, so every pipe's result is bit-identical alone and
// in the batch), a copy of the pipe's device scalars to pinned host memory,
// and a join back into the master stream.  The pipes' kernel chains are
// independent graph branches, so the GPU runs them concurrently.
//
// After the replay one host synchronisation reads every pipe's corrector
// error; the reference's corrector control (timestep.f90:214-253) is then
// applied per pipe, and the rare pipe that needs another corrector pass gets
// it on its own stream (main.f90:35-41).  In orbit mode every pipe takes
// exactly one corrector pass (newton.f90:740-762).
#include <cmath>
#include "pf_internal.cuh"

struct pf_batch {
    int n;
    std::vector<pf_ctx *> pipes;
    cudaStream_t master;
    cudaEvent_t fork;
    std::vector<cudaEvent_t> join;
    cudaGraphExec_t g[2][2];   // [orbit][parity]
    unsigned long long gn[2][2];
    int parity;
    bool warm;
    DevScalars *hsc;           // pinned, one per pipe
};

static void batch_free(pf_batch *b) {
    if (b->master) cudaStreamSynchronize(b->master);
    for (int o = 0; o < 2; ++o)
        for (int p = 0; p < 2; ++p)
            if (b->g[o][p]) cudaGraphExecDestroy(b->g[o][p]);
    for (cudaEvent_t e : b->join) cudaEventDestroy(e);
    if (b->fork) cudaEventDestroy(b->fork);
    if (b->master) cudaStreamDestroy(b->master);
    if (b->hsc) cudaFreeHost(b->hsc);
    for (pf_ctx *c : b->pipes) pf_ctx_destroy(c);
    delete b;
}

extern "C" int pf_batch_create(int npipes, const pf_config *cfgs, int device, pf_batch **out) {
    PF_ARG(npipes > 0 && cfgs && out, "pf_batch_create: bad argument");
    *out = nullptr;
    pf_batch *b = new pf_batch();
    b->n = npipes;
    for (int i = 0; i < npipes; ++i) {
        pf_ctx *c = nullptr;
        const int s = pf_ctx_create(&cfgs[i], device, &c);
        if (s != PF_OK) {
            batch_free(b);
            return s;
        }
        b->pipes.push_back(c);
    }
    if (cudaStreamCreateWithFlags(&b->master, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming) != cudaSuccess ||
        cudaMallocHost((void **)&b->hsc, npipes * sizeof(DevScalars)) != cudaSuccess) {
        batch_free(b);
        pf_set_error("pf_batch_create: stream/event/pinned allocation failed");
        return PF_ERR_CUDA;
    }
    b->join.resize(npipes);
    for (int i = 0; i < npipes; ++i) {
        if (cudaEventCreateWithFlags(&b->join[i], cudaEventDisableTiming) != cudaSuccess) {
            batch_free(b);
            pf_set_error("pf_batch_create: event creation failed");
            return PF_ERR_CUDA;
        }
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

extern "C" int pf_batch_matrices(pf_batch *b) {
    PF_ARG(b, "null batch");
    for (pf_ctx *c : b->pipes) PF_TRY(pf_vel_matrices(c));
    for (int o = 0; o < 2; ++o)
        for (int p = 0; p < 2; ++p)
            if (b->g[o][p]) {
                cudaGraphExecDestroy(b->g[o][p]);
                b->g[o][p] = nullptr;
            }
    return PF_OK;
}

static bool batch_graphable(const pf_batch *b) {
    for (const pf_ctx *c : b->pipes)
        if (!(c->cfg.dt > 0.0 && c->matrices_ready && pf_nl_fused_supported(c) && pf_fused_step_ok(c)))
            return false;
    return true;
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

static int batch_capture(pf_batch *b, int orbit, cudaGraphExec_t *exec, unsigned long long *nk) {
    unsigned long long n0 = 0;
    for (pf_ctx *c : b->pipes) n0 += c->launches;
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
    unsigned long long n1 = 0;
    for (pf_ctx *c : b->pipes) n1 += c->launches;
    *nk = n1 - n0;
    for (pf_ctx *c : b->pipes) c->launches = c->launches;  // per-pipe counters keep the capture
    return PF_OK;
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
    for (int st = 0; st < nsteps; ++st) {
        if (!b->warm || !batch_graphable(b)) {
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
            continue;
        }
        const int p = b->pipes[0]->parity;
        for (pf_ctx *c : b->pipes)
            if (c->parity != p) {
                pf_set_error("pf_batch_step: pipes out of step (pointer parity differs)");
                return PF_ERR_STATE;
            }
        if (!b->g[orbit][p]) PF_TRY(batch_capture(b, orbit, &b->g[orbit][p], &b->gn[orbit][p]));
        PF_CUDA(cudaGraphLaunch(b->g[orbit][p], b->master));
        for (pf_ctx *c : b->pipes) {
            for (int i = 0; i < 3; ++i) std::swap(c->vel[i].d, c->prev[i].d);
            c->parity ^= 1;
            c->cfl_fused = true;
            c->launches += b->gn[orbit][p] / b->n;
        }
        PF_CUDA(cudaStreamSynchronize(b->master));
        for (int i = 0; i < b->n; ++i) {
            pf_ctx *c = b->pipes[i];
            c->tim.dterr = std::max(c->tim.dterr, std::sqrt(bits_to_double(b->hsc[i].dterr2_bits)));
            c->tim.it = 1;
            int s = pf_tim_check_cgce(c);
            ++passes;
            if (!orbit) {
                while (c->tim.it != 0) {  // further corrector passes for this pipe only
                    PF_TRY(pf_transform_nonlinear(c));
                    PF_TRY(pf_vel_step_fused(c, 1));
                    PF_TRY(pf_read_dterr(c));
                    s = pf_tim_check_cgce(c);
                    ++passes;
                }
                if (s != PF_OK) status = s;
            } else {
                c->tim.it = 0;
            }
            c->tim.t = c->tim.t + c->tim.dt;
            c->tim.step = c->tim.step + 1;
        }
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
