// Request serving with continuous batching.
//
// A request is "advance this state by nsteps timesteps": a time-T map, the
// evaluation newton.f90's Newton-Krylov search makes over and over
// (steporbit, newton.f90:721-787; a GMRES Krylov vector is a base state plus
// a small perturbation, newton.f90:439-445).  The server keeps every admitted
// request's state resident on the device in its own context and advances all
// of them together in one batch (pf_batch, stage-batched launches).
//
// Between two batch steps the server
//   * admits queued requests in arrival order while the HBM budget and the
//     slot cap allow (a context of the request's shape is taken from the pool
//     of free contexts, or created), uploads the initial state, builds the
//     request's matrices and attaches its context to the batch;
//   * retires the requests that have taken their steps: final state to host
//     memory, context detached and returned to the pool;
//   * fails, alone, a request whose corrector check aborted or whose state
//     went non-finite (NaN or Inf): it leaves the batch without a result and
//     the others carry on unchanged; a cancelled request leaves the same way.
// So requests that arrive while others are on the GPU join the running batch
// as soon as memory and a slot free up, and their work shares every launch
// with the others.  A request's arithmetic is exactly the lone-pipe path, so
// its result is the same alone and in any mix.
#include <deque>
#include <map>
#include "pf_internal.cuh"

namespace {
struct Shape {
    int N, K, M, Mp, precision;
    bool operator<(const Shape &o) const {
        if (N != o.N) return N < o.N;
        if (K != o.K) return K < o.K;
        if (M != o.M) return M < o.M;
        if (Mp != o.Mp) return Mp < o.Mp;
        return precision < o.precision;
    }
    bool operator==(const Shape &o) const { return !(*this < o) && !(o < *this); }
};
Shape shape_of(const pf_config &c) { return Shape{c.N, c.K, c.M, c.Mp, c.precision}; }

struct Request {
    long long id;
    pf_config cfg;
    int nsteps, done;
    size_t nval;                  // H*N doubles per array
    std::vector<double> init;     // 6 arrays: ur re/im, ut re/im, uz re/im (reference layout)
    std::vector<double> result;
    pf_ctx *ctx;
    long long passes;
    int status = PF_OK;  // a failed or cancelled request's error
    std::string error;
};

// Device bytes of a context of this shape before one exists, from the
// allocations a context makes (an estimate for admission; the measured
// figure of the first context of a shape replaces it).
unsigned long long bytes_estimate(const pf_config &c) {
    const unsigned long long N = c.N, H = (2ull * c.K - 1) * c.M - (c.K - 1), Hp = (H + 31) / 32 * 32;
    const unsigned long long Z = 3ull * c.K, Th = 3ull * c.M;
    const unsigned long long coll = N * Hp * 16, phys = N * Z * Th * 8;
    unsigned long long b = 0;
    b += 23 * coll;                            // vel, prev, save, scratch
    b += 6 * phys;                             // physical fields
    b += 6ull * N * c.M * Z * 16;              // transform intermediate
    const unsigned long long Hcp = (1ull * c.M * c.K + 31) / 32 * 32;
    b += 4 * (NLU * N * Hp * 8 + N * Hp + N * Hp * 8);  // four factor sets, pivots
    b += 4 * (NLU * N * Hcp * 8 + N * Hcp * 8);          // their compact (k >= 0) copies
    b += 6 * N * Hp * 8 + 16 * Hp * 8;         // influence vectors and 4x4 inverses
    b += 64 * N * 8 + 4 * (Z + Th) * 16;       // mesh, twiddles, small buffers
    return b;
}
}  // namespace

struct pf_server {
    int device;
    unsigned long long budget;
    int max_active;
    int orbit;
    pf_batch *batch;
    std::deque<Request *> queue;
    std::vector<Request *> active;
    std::map<long long, Request *> finished;  // not yet collected
    std::vector<long long> fresh_done;        // finished since the last pf_serve_finished
    std::multimap<Shape, pf_ctx *> pool;      // free contexts
    std::map<Shape, unsigned long long> known_bytes;
    unsigned long long bytes_in_use;          // active and pooled contexts
    long long next_id;
    long long steps, passes;
};

static unsigned long long ctx_bytes(pf_ctx *c) {
    unsigned long long b = 0;
    pf_ctx_device_bytes(c, &b);
    return b;
}

static void release_ctx(pf_server *s, pf_ctx *c) {
    s->bytes_in_use -= std::min(s->bytes_in_use, ctx_bytes(c));
    pf_ctx_destroy(c);
}

// Make room for `need` bytes by destroying pooled contexts (largest first).
static bool make_room(pf_server *s, unsigned long long need) {
    while (s->bytes_in_use + need > s->budget && !s->pool.empty()) {
        auto victim = s->pool.begin();
        unsigned long long vb = 0;
        for (auto it = s->pool.begin(); it != s->pool.end(); ++it) {
            const unsigned long long b = ctx_bytes(it->second);
            if (b > vb) {
                vb = b;
                victim = it;
            }
        }
        pf_ctx *c = victim->second;
        s->pool.erase(victim);
        release_ctx(s, c);
    }
    return s->bytes_in_use + need <= s->budget;
}

// Admit the head of the queue if it fits; returns 1 admitted, 0 not now.
static int admit_one(pf_server *s, int *status) {
    Request *r = s->queue.front();
    const Shape sh = shape_of(r->cfg);
    pf_ctx *c = nullptr;
    auto it = s->pool.find(sh);
    if (it != s->pool.end()) {
        c = it->second;
        s->pool.erase(it);
        *status = pf_ctx_reconfigure(c, &r->cfg);
    } else {
        auto kb = s->known_bytes.find(sh);
        const unsigned long long need = kb != s->known_bytes.end() ? kb->second : bytes_estimate(r->cfg);
        if (!make_room(s, need)) {
            if (s->active.empty()) {  // it would not fit even alone
                pf_set_error("pf_serve: request %lld needs %llu bytes, over the HBM budget %llu", r->id, need,
                             s->budget);
                *status = PF_ERR_NOMEM;
            }
            return 0;
        }
        *status = pf_ctx_create(&r->cfg, s->device, &c);
        if (*status == PF_OK) {
            const unsigned long long b = ctx_bytes(c);
            s->known_bytes[sh] = b;
            s->bytes_in_use += b;
        }
    }
    if (*status == PF_OK) {
        const double *a = r->init.data();
        const size_t v = r->nval;
        *status = pf_vel_set_state(c, a, a + v, a + 2 * v, a + 3 * v, a + 4 * v, a + 5 * v);
    }
    if (*status == PF_OK) *status = pf_vel_matrices(c);
    if (*status == PF_OK) *status = pf_batch_attach(s->batch, c);
    if (*status != PF_OK) {
        if (c) release_ctx(s, c);
        return 0;
    }
    r->ctx = c;
    r->init.clear();
    r->init.shrink_to_fit();
    s->queue.pop_front();
    s->active.push_back(r);
    return 1;
}

// The request ends without a result: out of the batch, its context back to
// the pool (the next admission overwrites its state and matrices).
static int drop(pf_server *s, Request *r, int status, const std::string &why) {
    if (r->ctx) {
        PF_TRY(pf_batch_detach(s->batch, r->ctx));
        s->pool.insert({shape_of(r->cfg), r->ctx});
        r->ctx = nullptr;
    }
    r->status = status;
    r->error = why;
    s->finished[r->id] = r;
    s->fresh_done.push_back(r->id);
    return PF_OK;
}

static int retire(pf_server *s, Request *r) {
    r->result.resize(6 * r->nval);
    double *a = r->result.data();
    const size_t v = r->nval;
    PF_TRY(pf_batch_detach(s->batch, r->ctx));
    PF_TRY(pf_vel_get_state(r->ctx, a, a + v, a + 2 * v, a + 3 * v, a + 4 * v, a + 5 * v));
    s->pool.insert({shape_of(r->cfg), r->ctx});
    r->ctx = nullptr;
    s->finished[r->id] = r;
    s->fresh_done.push_back(r->id);
    return PF_OK;
}

extern "C" int pf_serve_create(int device, unsigned long long hbm_budget, int max_active, int orbit,
                               pf_server **out) {
    PF_ARG(out && hbm_budget > 0 && max_active > 0, "pf_serve_create: bad argument");
    *out = nullptr;
    pf_server *s = new pf_server();
    s->budget = hbm_budget;
    s->max_active = max_active;
    s->orbit = orbit ? 1 : 0;
    const int st = pf_batch_create(0, nullptr, device, &s->batch);
    if (st != PF_OK) {
        delete s;
        return st;
    }
    PF_CUDA(cudaGetDevice(&s->device));
    pf_batch_set_graphs(s->batch, 0);  // membership changes from step to step
    *out = s;
    return PF_OK;
}

extern "C" int pf_serve_destroy(pf_server *s) {
    if (!s) return PF_OK;
    for (Request *r : s->active) pf_batch_detach(s->batch, r->ctx);
    pf_batch_destroy(s->batch);
    for (Request *r : s->active) {
        pf_ctx_destroy(r->ctx);
        delete r;
    }
    for (Request *r : s->queue) delete r;
    for (auto &f : s->finished) delete f.second;
    for (auto &p : s->pool) pf_ctx_destroy(p.second);
    delete s;
    return PF_OK;
}

// Queue a request: advance the given state (reference coll layout, H*N
// doubles per array) by nsteps timesteps of cfg (fixed dt > 0).
extern "C" int pf_serve_submit(pf_server *s, const pf_config *cfg, int nsteps, const double *ur_re,
                               const double *ur_im, const double *ut_re, const double *ut_im, const double *uz_re,
                               const double *uz_im, long long *id) {
    PF_ARG(s && cfg && id && nsteps > 0, "pf_serve_submit: bad argument");
    PF_ARG(cfg->dt > 0.0, "pf_serve_submit: requests need a fixed dt > 0");
    PF_ARG(cfg->r == nullptr, "pf_serve_submit: requests use the default mesh");
    PF_ARG(ur_re && ur_im && ut_re && ut_im && uz_re && uz_im, "pf_serve_submit: null state");
    Request *r = new Request();
    r->id = s->next_id++;
    r->cfg = *cfg;
    r->nsteps = nsteps;
    r->nval = (size_t)((2 * cfg->K - 1) * cfg->M - (cfg->K - 1)) * cfg->N;
    r->init.resize(6 * r->nval);
    const double *src[6] = {ur_re, ur_im, ut_re, ut_im, uz_re, uz_im};
    for (int k = 0; k < 6; ++k) std::memcpy(&r->init[k * r->nval], src[k], r->nval * sizeof(double));
    s->queue.push_back(r);
    *id = r->id;
    return PF_OK;
}

// Admit what fits, advance every admitted request by one timestep, retire
// the finished ones.  *admitted and *finished (may be NULL) count this call's.
extern "C" int pf_serve_step(pf_server *s, int *admitted, int *finished) {
    PF_ARG(s, "null server");
    int na = 0, nf = 0, status = PF_OK;
    while (!s->queue.empty() && (int)s->active.size() < s->max_active) {
        int st = PF_OK;
        if (!admit_one(s, &st)) {
            if (st != PF_OK) {  // the request cannot run: report it finished with no result
                Request *r = s->queue.front();
                s->queue.pop_front();
                r->status = st;
                r->error = pf_last_error();
                s->finished[r->id] = r;
                s->fresh_done.push_back(r->id);
                status = st;
                continue;
            }
            break;  // head of the queue waits for memory
        }
        ++na;
    }
    if (!s->active.empty()) {
        long long p = 0;
        const int st = pf_batch_step(s->batch, 1, s->orbit, &p);
        // a corrector abort belongs to its own request, reported below
        if (st != PF_OK && st != PF_ERR_CONVERGE) status = st;
        s->passes += p;
        s->steps += 1;
        std::vector<Request *> still;
        for (Request *r : s->active) {
            r->done += 1;
            if (r->ctx->last_status != PF_OK) {
                PF_TRY(drop(s, r, r->ctx->last_status, r->ctx->last_error));
                ++nf;
            } else if (r->done >= r->nsteps) {
                PF_TRY(retire(s, r));
                ++nf;
            } else {
                still.push_back(r);
            }
        }
        s->active.swap(still);
    }
    if (admitted) *admitted = na;
    if (finished) *finished = nf;
    return status;
}

// Ids of the requests finished since the last call (up to cap); *n = count.
extern "C" int pf_serve_finished(pf_server *s, long long *ids, int cap, int *n) {
    PF_ARG(s && n && (ids || cap == 0), "pf_serve_finished: bad argument");
    const int k = std::min<int>(cap, (int)s->fresh_done.size());
    for (int i = 0; i < k; ++i) ids[i] = s->fresh_done[i];
    s->fresh_done.erase(s->fresh_done.begin(), s->fresh_done.begin() + k);
    *n = k;
    return PF_OK;
}

extern "C" int pf_serve_cancel(pf_server *s, long long id) {
    PF_ARG(s, "null server");
    for (auto it = s->queue.begin(); it != s->queue.end(); ++it)
        if ((*it)->id == id) {
            Request *r = *it;
            s->queue.erase(it);
            return drop(s, r, PF_ERR_CANCELLED, "request cancelled");
        }
    for (size_t i = 0; i < s->active.size(); ++i)
        if (s->active[i]->id == id) {
            Request *r = s->active[i];
            s->active.erase(s->active.begin() + i);
            return drop(s, r, PF_ERR_CANCELLED, "request cancelled");
        }
    if (s->finished.count(id)) {
        pf_set_error("pf_serve_cancel: request %lld has already finished", id);
        return PF_ERR_STATE;
    }
    pf_set_error("pf_serve_cancel: no request %lld", id);
    return PF_ERR_ARG;
}

// The final state of a finished request (reference coll layout); the request
// is forgotten afterwards.  PF_ERR_STATE if it has not finished; a request
// that failed or was cancelled returns its own status and message.
extern "C" int pf_serve_result(pf_server *s, long long id, double *ur_re, double *ur_im, double *ut_re,
                               double *ut_im, double *uz_re, double *uz_im) {
    PF_ARG(s, "null server");
    auto it = s->finished.find(id);
    if (it == s->finished.end()) {
        pf_set_error("pf_serve_result: request %lld has not finished", id);
        return PF_ERR_STATE;
    }
    Request *r = it->second;
    s->finished.erase(it);
    if (r->status != PF_OK || r->result.empty()) {
        const int st = r->status != PF_OK ? r->status : PF_ERR_ARG;
        pf_set_error("pf_serve_result: request %lld: %s", id,
                     r->error.empty() ? "could not be admitted" : r->error.c_str());
        delete r;
        return st;
    }
    double *dst[6] = {ur_re, ur_im, ut_re, ut_im, uz_re, uz_im};
    for (int k = 0; k < 6; ++k)
        if (dst[k]) std::memcpy(dst[k], &r->result[k * r->nval], r->nval * sizeof(double));
    delete r;
    return PF_OK;
}

// queued, active, pooled contexts, device bytes held (active + pooled),
// batch steps taken.
extern "C" int pf_serve_stats(pf_server *s, int *queued, int *active, int *pooled, unsigned long long *bytes,
                              long long *steps) {
    PF_ARG(s, "null server");
    if (queued) *queued = (int)s->queue.size();
    if (active) *active = (int)s->active.size();
    if (pooled) *pooled = (int)s->pool.size();
    if (bytes) *bytes = s->bytes_in_use;
    if (steps) *steps = s->steps;
    return PF_OK;
}

// The batch the server steps (its stream and launch counters).
extern "C" int pf_serve_batch(pf_server *s, pf_batch **b) {
    PF_ARG(s && b, "pf_serve_batch: bad argument");
    *b = s->batch;
    return PF_OK;
}
