// Device side of the Newton-Krylov orbit search (newton.f90): the maps
// between the velocity fields and a scaled state vector, the vector dot
// product, the shift directions and steporbit's time-T map with its shift,
// all on vectors held in device memory.  The small dense work of GMRES and
// the hookstep (dgelsy, dgesvd in GMRESm.f90) stays with the caller.
//
// A vector has 8 + 6*N*H doubles (newton.f90:36 with one rank): x[0..7] hold
// the shifts, the period and the continuation parameter; from x[8] on, for
// every mode nh in _loop_km order and every radial point n, the six values
// ur Re, ur Im, ut Re, ut Im, uz Re, uz Im, multiplied by
// s(c) = sqrt|intrdr(n)| * w(nh) * scaleU(c), w = 4 / (4 + alpha|k| + Mp|m|),
// except u_z of the mean mode (k = m = 0), multiplied by sqrt|intrdr(n)|
// alone (newton.f90:567-643).
#include <cmath>
#include "pf_internal.cuh"

struct OrbitScale {
    double s1, s2, s3;
    double walpha;  // alpha in the weights w (rtz2vec keeps its first weights, newton.f90:580-587)
};

// the three multipliers of mode nh at radial point n
__device__ __forceinline__ void orbit_scale(int nh, int n, const double *__restrict__ intrdr, const Geo &g,
                                            const OrbitScale &u, double &a, double &b, double &c) {
    int k, m;
    mode_km(nh, g.K, k, m);
    const double d = sqrt(fabs(intrdr[n]));
    const double w = 4.0 / (4.0 + (u.walpha * abs(k)) + (double)(g.Mp * abs(m)));
    a = d * w * u.s1;
    b = d * w * u.s2;
    c = (k == 0 && m == 0) ? d : d * w * u.s3;
}

// rtz2vec (newton.f90:567-602); thread per (mode, radial point), the radial
// point fastest so the six stores of neighbouring threads are contiguous
static __global__ void k_rtz2vec(const double2 *__restrict__ r, const double2 *__restrict__ t,
                                 const double2 *__restrict__ z, double *__restrict__ v,
                                 const double *__restrict__ intrdr, Geo g, OrbitScale u) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (long long)g.H * g.N) return;
    const int nh = (int)(i / g.N), n = (int)(i - (long long)nh * g.N);
    double a, b, c;
    orbit_scale(nh, n, intrdr, g, u, a, b, c);
    const size_t at = (size_t)n * g.Hp + nh;
    const double2 R = r[at], T = t[at], Z = z[at];
    double *o = v + 8 + i * 6;
    o[0] = R.x * a;
    o[1] = R.y * a;
    o[2] = T.x * b;
    o[3] = T.y * b;
    o[4] = Z.x * c;
    o[5] = Z.y * c;
}

// vec2rtz (newton.f90:608-643)
static __global__ void k_vec2rtz(const double *__restrict__ v, double2 *__restrict__ r, double2 *__restrict__ t,
                                 double2 *__restrict__ z, const double *__restrict__ intrdr, Geo g, OrbitScale u) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (long long)g.H * g.N) return;
    const int nh = (int)(i / g.N), n = (int)(i - (long long)nh * g.N);
    double a, b, c;
    orbit_scale(nh, n, intrdr, g, u, a, b, c);
    const size_t at = (size_t)n * g.Hp + nh;
    const double *o = v + 8 + i * 6;
    r[at] = make_double2(o[0] / a, o[1] / a);
    t[at] = make_double2(o[2] / b, o[3] / b);
    z[at] = make_double2(o[4] / c, o[5] / c);
}

// getshiftdir's mode loop (newton.f90:544-556): every coefficient times
// i*ds, ds = Mp*m (dir 1, theta) or alpha*k (dir 2, z)
static __global__ void k_shiftdir(double2 *r, double2 *t, double2 *z, Geo g, int dir) {
    const int nh = blockIdx.x * blockDim.x + threadIdx.x, n = blockIdx.y;
    if (nh >= g.H) return;
    int k, m;
    mode_km(nh, g.K, k, m);
    const double ds = dir == 1 ? (double)(g.Mp * m) : g.alpha * k;
    const size_t at = (size_t)n * g.Hp + nh;
    double2 x = r[at];
    r[at] = make_double2(-x.y * ds, x.x * ds);
    x = t[at];
    t[at] = make_double2(-x.y * ds, x.x * ds);
    x = z[at];
    z[at] = make_double2(-x.y * ds, x.x * ds);
}

// dot_product(a(n1:nn), b(n1:nn)) (newton.f90:652-672) in two fixed-order
// passes: ORBIT_DOT_BLOCKS grid-strided partial sums, then one block
static __global__ void __launch_bounds__(256) k_dot_partial(const double *__restrict__ a, const double *__restrict__ b,
                                                            long long n0, long long n1, double *__restrict__ part) {
    __shared__ double red[256];
    double s = 0.0;
    for (long long i = n0 + (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n1;
         i += (long long)gridDim.x * blockDim.x)
        s = fma(a[i], b[i], s);
    red[threadIdx.x] = s;
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = red[0];
}

static __global__ void __launch_bounds__(256) k_dot_final(const double *__restrict__ part, int np,
                                                          double *__restrict__ out) {
    __shared__ double red[256];
    double s = 0.0;
    for (int i = threadIdx.x; i < np; i += blockDim.x) s += part[i];
    red[threadIdx.x] = s;
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = red[0];
}

static int orbit_ready(const pf_ctx *ctx) {
    if (!ctx->orbit_set) {
        pf_set_error("pf_orbit_*: call pf_orbit_set_scales first");
        return PF_ERR_STATE;
    }
    return PF_OK;
}

static OrbitScale scales(const pf_ctx *ctx) {
    return OrbitScale{ctx->orbit_scaleU[0], ctx->orbit_scaleU[1], ctx->orbit_scaleU[2], ctx->orbit_walpha};
}

static int rtz2vec(pf_ctx *ctx, double *v) {
    const Geo &g = ctx->g;
    {
        ProfScope ps_(ctx, PF_K_EW);
        k_rtz2vec<<<grid1((long long)g.H * g.N, 256), 256, 0, ctx->stream>>>(
            ctx->vel[0].d, ctx->vel[1].d, ctx->vel[2].d, v, ctx->dm.intrdr, g, scales(ctx));
    }
    PF_LAUNCHED(ctx);
    return PF_OK;
}

static int vec2rtz(pf_ctx *ctx, const double *v) {
    const Geo &g = ctx->g;
    {
        ProfScope ps_(ctx, PF_K_EW);
        k_vec2rtz<<<grid1((long long)g.H * g.N, 256), 256, 0, ctx->stream>>>(
            v, ctx->vel[0].d, ctx->vel[1].d, ctx->vel[2].d, ctx->dm.intrdr, g, scales(ctx));
    }
    PF_LAUNCHED(ctx);
    return PF_OK;
}

extern "C" int pf_orbit_set_scales(pf_ctx *ctx, const double *scaleU, double scaleT) {
    PF_ARG(ctx && scaleU, "pf_orbit_set_scales: null argument");
    PF_ARG(std::isfinite(scaleT) && scaleT != 0.0, "pf_orbit_set_scales: scaleT must be finite and nonzero");
    for (int c = 0; c < 3; ++c)
        PF_ARG(std::isfinite(scaleU[c]) && scaleU[c] != 0.0,
               "pf_orbit_set_scales: scaleU must be finite and nonzero");
    for (int c = 0; c < 3; ++c) ctx->orbit_scaleU[c] = scaleU[c];
    ctx->orbit_scaleT = scaleT;
    if (!ctx->orbit_set) ctx->orbit_walpha = ctx->g.alpha;
    ctx->orbit_set = true;
    return PF_OK;
}

extern "C" int pf_orbit_vec_len(const pf_ctx *ctx, long long *n) {
    PF_ARG(ctx && n, "pf_orbit_vec_len: null argument");
    *n = 8 + 6LL * ctx->g.N * ctx->g.H;
    return PF_OK;
}

extern "C" int pf_orbit_rtz2vec(pf_ctx *ctx, double *v) {
    PF_ARG(ctx && v, "pf_orbit_rtz2vec: null argument");
    PF_TRY(orbit_ready(ctx));
    return rtz2vec(ctx, v);
}

extern "C" int pf_orbit_vec2rtz(pf_ctx *ctx, const double *v) {
    PF_ARG(ctx && v, "pf_orbit_vec2rtz: null argument");
    PF_TRY(orbit_ready(ctx));
    return vec2rtz(ctx, v);
}

extern "C" int pf_orbit_dotprod(pf_ctx *ctx, int n_, const double *a, const double *b, double *out) {
    PF_ARG(ctx && a && b && out, "pf_orbit_dotprod: null argument");
    const long long n = 8 + 6LL * ctx->g.N * ctx->g.H;
    const long long n0 = (n_ == -1) ? 8 : 0;
    double *part = ctx->orbit_red;
    {
        ProfScope ps_(ctx, PF_K_EW);
        k_dot_partial<<<ORBIT_DOT_BLOCKS, 256, 0, ctx->stream>>>(a, b, n0, n, part);
    }
    PF_LAUNCHED(ctx);
    {
        ProfScope ps_(ctx, PF_K_EW);
        k_dot_final<<<1, 256, 0, ctx->stream>>>(part, ORBIT_DOT_BLOCKS, part + ORBIT_DOT_BLOCKS);
    }
    PF_LAUNCHED(ctx);
    PF_CUDA(cudaMemcpyAsync(out, part + ORBIT_DOT_BLOCKS, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    PF_CUDA(cudaStreamSynchronize(ctx->stream));
    return PF_OK;
}

// getshiftdir (newton.f90:533-561): s = rtz2vec(d/d(shift) vec2rtz(x))
extern "C" int pf_orbit_shiftdir(pf_ctx *ctx, int i, const double *x, double *s) {
    PF_ARG(ctx && x && s && (i == 1 || i == 2), "pf_orbit_shiftdir: bad argument");
    PF_TRY(orbit_ready(ctx));
    PF_TRY(vec2rtz(ctx, x));
    const Geo &g = ctx->g;
    {
        ProfScope ps_(ctx, PF_K_EW);
        k_shiftdir<<<dim3(grid1(g.H, 128), g.N), 128, 0, ctx->stream>>>(ctx->vel[0].d, ctx->vel[1].d,
                                                                        ctx->vel[2].d, g, i);
    }
    PF_LAUNCHED(ctx);
    return rtz2vec(ctx, s);
}

// steporbit (newton.f90:721-831) without continuation, output or the
// termination checks: p = x(1:3)*scaleT; state from x; for ndts != 1 a new
// dt = p(3)/ndts and new matrices; ndts steps with one corrector each; for
// ndts != 1 time and step count advance and the state is shifted by
// (-p(1), -p(2)); y(9:) from the state.
extern "C" int pf_orbit_step(pf_ctx *ctx, int ndts, const double *x, double *y) {
    PF_ARG(ctx && x && y && ndts >= 1, "pf_orbit_step: bad argument");
    PF_TRY(orbit_ready(ctx));
    double p[3];
    PF_CUDA(cudaMemcpyAsync(p, x, 3 * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    PF_CUDA(cudaStreamSynchronize(ctx->stream));
    for (int c = 0; c < 3; ++c) p[c] = p[c] * ctx->orbit_scaleT;
    PF_TRY(vec2rtz(ctx, x));
    const double t0 = ctx->tim.t;
    const int step0 = ctx->tim.step;
    if (ndts != 1) {
        PF_ARG(p[2] > 0.0 && std::isfinite(p[2]), "pf_orbit_step: the period x[2]*scaleT must be > 0");
        ctx->tim.dt = p[2] / (double)ndts;
        PF_TRY(pf_vel_matrices(ctx));
    }
    const int s = pf_steporbit(ctx, ndts);
    if (s != PF_OK && s != PF_ERR_CONVERGE) return s;
    if (ndts != 1) {
        for (int c = 0; c < 3; ++c) PF_TRY(pf_var_coll_shift(-p[0], -p[1], &ctx->vel[c], &ctx->vel[c]));
    } else {  // time advances only for ndts != 1 (newton.f90:763-766)
        ctx->tim.t = t0;
        ctx->tim.step = step0;
    }
    PF_TRY(rtz2vec(ctx, y));
    return s;
}
