// Spectral field algebra on the device: elementwise ops, banded radial
// stencils, symmetry projection, shift, norms and corrector-error reduction
// (variables.f90:118-751; timestep.f90:130-207; velocity.f90:80-114,338-361).
#include <cmath>
#include "pf_internal.cuh"

static constexpr int BLK = 256;

// ------------------------------------------------------------- elementwise
__global__ void k_ew(int op, const double2 *__restrict__ a, const double2 *__restrict__ b,
                     double2 *o1, double2 *o2, double s, int N, int H, int Hp) {
    const long long total = (long long)N * Hp;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        const int nh = (int)(i % Hp);
        if (nh >= H) continue;
        switch (op) {
        case EW_ZERO: o1[i] = make_double2(0.0, 0.0); break;
        case EW_COPY: o1[i] = a[i]; break;
        case EW_ADD: { const double2 x = a[i], y = o1[i]; o1[i] = make_double2(y.x + x.x, y.y + x.y); } break;
        case EW_SUB: { const double2 x = a[i], y = o1[i]; o1[i] = make_double2(y.x - x.x, y.y - x.y); } break;
        case EW_SUBFROM: { const double2 x = a[i], y = b[i]; o1[i] = make_double2(x.x - y.x, x.y - y.y); } break;
        case EW_NEG: { const double2 x = a[i]; o1[i] = make_double2(-x.x, -x.y); } break;
        case EW_DMULT: { const double2 y = o1[i]; o1[i] = make_double2(y.x * s, y.y * s); } break;
        case EW_RT2PM: {  // velocity.f90:80-95
            const double2 r = a[i], t = b[i];
            o1[i] = make_double2(r.x - t.y, r.y + t.x);
            o2[i] = make_double2(r.x + t.y, r.y - t.x);
        } break;
        case EW_PM2RT: {  // velocity.f90:98-114
            const double2 p = a[i], m = b[i];
            o1[i] = make_double2(0.5 * (p.x + m.x), 0.5 * (p.y + m.y));
            o2[i] = make_double2(0.5 * (p.y - m.y), -0.5 * (p.x - m.x));
        } break;
        case EW_NLINCORR: {  // timestep.f90:174-184: o1 = s*o1 + (1-s)*a
            const double2 x = a[i], y = o1[i];
            const double d2 = 1.0 - s;
            o1[i] = make_double2(s * y.x + d2 * x.x, s * y.y + d2 * x.y);
        } break;
        }
    }
}

int pf_launch_ew(pf_ctx *ctx, EwOp op, const double2 *a, const double2 *b, double2 *o1,
                 double2 *o2, double s) {
    const Geo &g = ctx->g;
    const long long total = (long long)g.N * g.Hp;
    const unsigned grid = (unsigned)std::min<long long>(grid1(total, BLK), 148LL * 16);
    {
        ProfScope ps_(ctx, PF_K_EW);
        k_ew<<<grid, BLK, 0, ctx->stream>>>((int)op, a, b, o1, o2, s, g.N, g.H, g.Hp);
    }
    PF_LAUNCHED(ctx);
    return PF_OK;
}

__global__ void k_zerobc(double2 *a, int N, int H, int Hp) {
    const int nh = blockIdx.x * blockDim.x + threadIdx.x;
    if (nh >= H) return;
    a[nh] = make_double2(0.0, 0.0);
    a[(size_t)(N - 1) * Hp + nh] = make_double2(0.0, 0.0);
}

int pf_launch_zerobc(pf_ctx *ctx, double2 *a) {
    const Geo &g = ctx->g;
    {
        ProfScope ps_(ctx, PF_K_EW);
        k_zerobc<<<grid1(g.H, BLK), BLK, 0, ctx->stream>>>(a, g.N, g.H, g.Hp);
    }
    PF_LAUNCHED(ctx);
    return PF_OK;
}

// --------------------------------------------------------------- stencils
// out(n) = sum_{j=lo..hi} A(KL+n-j, j) in(j), accumulated in increasing j as
// the column-ordered loop of var_coll_meshmult does (variables.f90:388-397).
__device__ __forceinline__ double2 band_row(const double *__restrict__ band, int N, int Hp,
                                            const double2 *__restrict__ in, int n, int nh) {
    const int lo = max(0, n - KL), hi = min(N - 1, n + KL);
    double2 acc = make_double2(0.0, 0.0);
    for (int j = lo; j <= hi; ++j) {
        const double w = band[(KL + n - j) * N + j];
        const double2 v = in[(size_t)j * Hp + nh];
        acc.x = fma(w, v.x, acc.x);
        acc.y = fma(w, v.y, acc.y);
    }
    return acc;
}

__global__ void k_meshmult_dr(const double *__restrict__ band, const double2 *__restrict__ in,
                              double2 *__restrict__ out, int N, int H, int Hp) {
    const int nh = blockIdx.x * blockDim.x + threadIdx.x, n = blockIdx.y;
    if (nh >= H) return;
    out[(size_t)n * Hp + nh] = band_row(band, N, Hp, in, n, nh);
}

int pf_launch_meshmult_dr(pf_ctx *ctx, int p, const double2 *in, double2 *out) {
    const Geo &g = ctx->g;
    dim3 grid(grid1(g.H, 128), g.N);
    {
        ProfScope ps_(ctx, PF_K_STENCIL);
        k_meshmult_dr<<<grid, 128, 0, ctx->stream>>>(ctx->dm.dr + (size_t)(p - 1) * NBAND * g.N, in, out,
                                                     g.N, g.H, g.Hp);
    }
    PF_LAUNCHED(ctx);
    return PF_OK;
}

// curl (variables.f90:408-436); outputs must not alias inputs
__global__ void k_curl(const double2 *__restrict__ r, const double2 *__restrict__ t,
                       const double2 *__restrict__ z, double2 *__restrict__ or_,
                       double2 *__restrict__ ot, double2 *__restrict__ oz, DevMesh dm, Geo g) {
    const int nh = blockIdx.x * blockDim.x + threadIdx.x, n = blockIdx.y;
    if (nh >= g.H) return;
    int k, m;
    mode_km(nh, g.K, k, m);
    const size_t at = (size_t)n * g.Hp + nh;
    const double rm1 = dm.rp[2 * g.N + n];
    const double m1r1 = rm1 * g.Mp * m;      // ad_m1r1 (variables.f90:80)
    const double k1a1 = g.alpha * k;         // ad_k1a1 (variables.f90:85)
    const double2 c1 = r[at], c2 = t[at], c3 = z[at];
    or_[at] = make_double2(-c3.y * m1r1 + c2.y * k1a1, c3.x * m1r1 - c2.x * k1a1);
    const double2 dz = band_row(dm.dr, g.N, g.Hp, z, n, nh);
    ot[at] = make_double2(-c1.y * k1a1 - dz.x, c1.x * k1a1 - dz.y);
    const double2 dt = band_row(dm.dr, g.N, g.Hp, t, n, nh);
    oz[at] = make_double2(c2.x * rm1 + dt.x + c1.y * m1r1, c2.y * rm1 + dt.y - c1.x * m1r1);
}

int pf_launch_curl(pf_ctx *ctx, const double2 *r, const double2 *t, const double2 *z, double2 *or_,
                   double2 *ot, double2 *oz) {
    const Geo &g = ctx->g;
    dim3 grid(grid1(g.H, 128), g.N);
    {
        ProfScope ps_(ctx, PF_K_STENCIL);
        k_curl<<<grid, 128, 0, ctx->stream>>>(r, t, z, or_, ot, oz, ctx->dm, g);
    }
    PF_LAUNCHED(ctx);
    return PF_OK;
}

// grad (variables.f90:442-459); outputs must not alias the input
__global__ void k_grad(const double2 *__restrict__ p, double2 *__restrict__ r,
                       double2 *__restrict__ t, double2 *__restrict__ z, DevMesh dm, Geo g) {
    const int nh = blockIdx.x * blockDim.x + threadIdx.x, n = blockIdx.y;
    if (nh >= g.H) return;
    int k, m;
    mode_km(nh, g.K, k, m);
    const size_t at = (size_t)n * g.Hp + nh;
    const double m1r1 = dm.rp[2 * g.N + n] * g.Mp * m;
    const double k1a1 = g.alpha * k;
    const double2 c1 = p[at];
    r[at] = band_row(dm.dr, g.N, g.Hp, p, n, nh);
    t[at] = make_double2(-c1.y * m1r1, c1.x * m1r1);
    z[at] = make_double2(-c1.y * k1a1, c1.x * k1a1);
}

int pf_launch_grad(pf_ctx *ctx, const double2 *p, double2 *r, double2 *t, double2 *z) {
    const Geo &g = ctx->g;
    dim3 grid(grid1(g.H, 128), g.N);
    {
        ProfScope ps_(ctx, PF_K_STENCIL);
        k_grad<<<grid, 128, 0, ctx->stream>>>(p, r, t, z, ctx->dm, g);
    }
    PF_LAUNCHED(ctx);
    return PF_OK;
}

// div (variables.f90:465-481); dv must not alias the inputs
__global__ void k_div(const double2 *__restrict__ r, const double2 *__restrict__ t,
                      const double2 *__restrict__ z, double2 *__restrict__ dv, DevMesh dm, Geo g) {
    const int nh = blockIdx.x * blockDim.x + threadIdx.x, n = blockIdx.y;
    if (nh >= g.H) return;
    int k, m;
    mode_km(nh, g.K, k, m);
    const size_t at = (size_t)n * g.Hp + nh;
    const double rm1 = dm.rp[2 * g.N + n];
    const double m1r1 = rm1 * g.Mp * m;
    const double k1a1 = g.alpha * k;
    const double2 c1 = band_row(dm.dr, g.N, g.Hp, r, n, nh);
    const double2 a = r[at], b = t[at], c = z[at];
    dv[at] = make_double2(a.x * rm1 + c1.x - b.y * m1r1 - c.y * k1a1,
                          a.y * rm1 + c1.y + b.x * m1r1 + c.x * k1a1);
}

int pf_launch_div(pf_ctx *ctx, const double2 *r, const double2 *t, const double2 *z, double2 *dv) {
    const Geo &g = ctx->g;
    dim3 grid(grid1(g.H, 128), g.N);
    {
        ProfScope ps_(ctx, PF_K_STENCIL);
        k_div<<<grid, 128, 0, ctx->stream>>>(r, t, z, dv, ctx->dm, g);
    }
    PF_LAUNCHED(ctx);
    return PF_OK;
}

// d = A b + c with A = c1 I + c2 Lap(PM) per mode (timestep.f90:46-60, 130-154).
// The per-mode band is never stored: its off-diagonals are c2*radLap and its
// diagonal (c2*radLap + c2*d) + c1, rebuilt here in registers.
__device__ __forceinline__ double lap_d(const DevMesh &dm, const Geo &g, int PM, int n, int k, int m) {
    const double r2 = dm.rp[1 * g.N + n];
    double d = -(r2 * g.Mp * m * g.Mp * m) - g.alpha * k * g.alpha * k;
    if (PM != 0) d = d - r2 - 2.0 * PM * g.Mp * m * r2;
    return d;
}

__global__ void k_tim_meshmult(int PM, double c1, double c2, const double2 *__restrict__ b,
                               const double2 *__restrict__ c, double2 *__restrict__ d, DevMesh dm, Geo g) {
    const int nh = blockIdx.x * blockDim.x + threadIdx.x, n = blockIdx.y;
    if (nh >= g.H) return;
    int k, m;
    mode_km(nh, g.K, k, m);
    const int lo = max(0, n - KL), hi = min(g.N - 1, n + KL);
    double2 acc = c[(size_t)n * g.Hp + nh];
    for (int j = lo; j <= hi; ++j) {
        double w = c2 * dm.radLap[(KL + n - j) * g.N + j];
        if (j == n) w = (w + c2 * lap_d(dm, g, PM, j, k, m)) + c1;
        const double2 v = b[(size_t)j * g.Hp + nh];
        acc.x = fma(w, v.x, acc.x);
        acc.y = fma(w, v.y, acc.y);
    }
    d[(size_t)n * g.Hp + nh] = acc;
}

int pf_launch_tim_meshmult(pf_ctx *ctx, const pf_mesh *A, const double2 *b, const double2 *c, double2 *d) {
    const Geo &g = ctx->g;
    dim3 grid(grid1(g.H, 128), g.N);
    {
        ProfScope ps_(ctx, PF_K_STENCIL);
        k_tim_meshmult<<<grid, 128, 0, ctx->stream>>>(A->PM, A->c1, A->c2, b, c, d, ctx->dm, g);
    }
    PF_LAUNCHED(ctx);
    return PF_OK;
}

// ------------------------------------------------------------- symmetries
__global__ void k_imposesym0(double2 *r, double2 *t, double2 *z, int N, int Hp) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= N) return;
    const size_t at = (size_t)n * Hp;  // mode nh = 0 (variables.f90:611-616)
    r[at] = make_double2(0.0, 0.0);
    t[at].y = 0.0;
    z[at].y = 0.0;
}

// mirror (i=1) / shift-reflect (i=2): out(nh_) = sign * in(nh) with nh_ = (-k, m)
// (variables.f90:545-597); written out of place to (o0,o1,o2)
__global__ void k_imposesym12(int i, const double2 *__restrict__ r, const double2 *__restrict__ t,
                              const double2 *__restrict__ z, double2 *o0, double2 *o1, double2 *o2, Geo g) {
    const int nh = blockIdx.x * blockDim.x + threadIdx.x, n = blockIdx.y;
    if (nh >= g.H) return;
    int k, m;
    mode_km(nh, g.K, k, m);
    // source mode is (-k, m); for m == 0 the mode maps to itself
    const int src = (m == 0) ? nh : m * (2 * g.K - 1) - k;
    const int ks = (m == 0) ? k : -k;
    double b = -1.0, a = 1.0;
    if (i == 2 && (((ks % 2) + 2) % 2) != 0) a = -1.0;
    if (m == 0) b = 1.0;
    const size_t at = (size_t)n * g.Hp + nh, as = (size_t)n * g.Hp + src;
    const double2 vr = r[as], vt = t[as], vz = z[as];
    const double2 cr = make_double2(vr.x * a, vr.y * a * b);
    const double2 ct = make_double2(-vt.x * a, -vt.y * a * b);
    const double2 cz = make_double2(vz.x * a, vz.y * a * b);
    const double2 ur = r[at], ut = t[at], uz = z[at];
    o0[at] = make_double2((ur.x + cr.x) / 2.0, (ur.y + cr.y) / 2.0);
    o1[at] = make_double2((ut.x + ct.x) / 2.0, (ut.y + ct.y) / 2.0);
    o2[at] = make_double2((uz.x + cz.x) / 2.0, (uz.y + cz.y) / 2.0);
}

// shift-rotate (i=3): zero modes with k+m odd (variables.f90:599-609)
__global__ void k_imposesym3(double2 *r, double2 *t, double2 *z, Geo g) {
    const int nh = blockIdx.x * blockDim.x + threadIdx.x, n = blockIdx.y;
    if (nh >= g.H) return;
    int k, m;
    mode_km(nh, g.K, k, m);
    if ((((k + m) % 2) + 2) % 2 == 0) return;
    const size_t at = (size_t)n * g.Hp + nh;
    r[at] = t[at] = z[at] = make_double2(0.0, 0.0);
}

int pf_launch_imposesym(pf_ctx *ctx, int i, double2 *r, double2 *t, double2 *z) {
    const Geo &g = ctx->g;
    dim3 grid(grid1(g.H, 128), g.N);
    if (i == 1 || i == 2) {
        {
            ProfScope ps_(ctx, PF_K_EW);
            k_imposesym12<<<grid, 128, 0, ctx->stream>>>(i, r, t, z, ctx->s[4].d, ctx->s[5].d, ctx->s[6].d, g);
        }
        PF_LAUNCHED(ctx);
        PF_TRY(pf_launch_ew(ctx, EW_COPY, ctx->s[4].d, nullptr, r, nullptr, 0.0));
        PF_TRY(pf_launch_ew(ctx, EW_COPY, ctx->s[5].d, nullptr, t, nullptr, 0.0));
        PF_TRY(pf_launch_ew(ctx, EW_COPY, ctx->s[6].d, nullptr, z, nullptr, 0.0));
    }
    if (i == 3) {
        {
            ProfScope ps_(ctx, PF_K_EW);
            k_imposesym3<<<grid, 128, 0, ctx->stream>>>(r, t, z, g);
        }
        PF_LAUNCHED(ctx);
    }
    {
        ProfScope ps_(ctx, PF_K_EW);
        k_imposesym0<<<grid1(g.N, 64), 64, 0, ctx->stream>>>(r, t, z, g.N, g.Hp);
    }
    PF_LAUNCHED(ctx);
    return PF_OK;
}

// shift in z and theta (variables.f90:487-528)
__global__ void k_shift(double dt, double dz, const double2 *__restrict__ a, double2 *__restrict__ b, Geo g) {
    const int nh = blockIdx.x * blockDim.x + threadIdx.x, n = blockIdx.y;
    if (nh >= g.H) return;
    int k, m;
    mode_km(nh, g.K, k, m);
    const size_t at = (size_t)n * g.Hp + nh;
    double2 v = a[at];
    if (dz != 0.0) {
        const double ang = dz * k * g.alpha, sk = sin(ang), ck = cos(ang);
        const double dRe = v.x;
        v.x = dRe * ck + v.y * sk;
        v.y = v.y * ck - dRe * sk;
    }
    if (dt != 0.0) {
        const double ang = dt * m * g.Mp, sm = sin(ang), cm = cos(ang);
        const double dRe = v.x;
        v.x = dRe * cm + v.y * sm;
        v.y = v.y * cm - dRe * sm;
    }
    b[at] = v;
}

// ------------------------------------------------------------- reductions
// per-mode energy b(nh) = w * sum_n intrdr(n) |a(n,nh)|^2, halved at k=m=0
// (variables.f90:731-738); binned into Ek/Em on the host in nh order
__global__ void k_norm_modes(const double2 *__restrict__ a, const double *__restrict__ intrdr,
                             double *__restrict__ out, double w, int N, int H, int Hp) {
    const int nh = blockIdx.x * blockDim.x + threadIdx.x;
    if (nh >= H) return;
    double b = 0.0;
    for (int n = 0; n < N; ++n) {
        const double2 v = a[(size_t)n * Hp + nh];
        const double f = w * (v.x * v.x + v.y * v.y);
        b = fma(f, intrdr[n], b);
    }
    if (nh == 0) b = 0.5 * b;
    out[nh] = b;
}

int pf_norm_host(pf_ctx *ctx, const double2 *a, double *E, double *Ek, double *Em) {
    const Geo &g = ctx->g;
    const double PI = 3.1415926535897931;
    const double w = 4.0 * PI * PI / g.alpha;
    {
        ProfScope ps_(ctx, PF_K_EW);
        k_norm_modes<<<grid1(g.H, 128), 128, 0, ctx->stream>>>(a, ctx->dm.intrdr, ctx->red, w, g.N, g.H, g.Hp);
    }
    PF_LAUNCHED(ctx);
    std::vector<double> b(g.H);
    PF_CUDA(cudaMemcpyAsync(b.data(), ctx->red, g.H * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    PF_CUDA(cudaStreamSynchronize(ctx->stream));
    std::vector<double> ek(g.K, 0.0), em(g.M, 0.0);
    for (int nh = 0; nh < g.H; ++nh) {
        int k, m;
        mode_km(nh, g.K, k, m);
        em[m] += b[nh];
        ek[k < 0 ? -k : k] += b[nh];
    }
    double s = 0.0;
    for (int m = 0; m < g.M; ++m) s += em[m];
    if (E) *E = s;
    if (Ek) for (int k = 0; k < g.K; ++k) Ek[k] = ek[k];
    if (Em) for (int m = 0; m < g.M; ++m) Em[m] = em[m];
    return PF_OK;
}

// max over (n, nh) of |a_c - b_c|^2 for three pairs (timestep.f90:190-207,
// with the corrector's difference fused in); non-negative doubles are
// monotone as unsigned 64-bit integers, so atomicMax on the bits is exact.
__global__ void k_measurecorr(const double2 *__restrict__ a0, const double2 *__restrict__ b0,
                              const double2 *__restrict__ a1, const double2 *__restrict__ b1,
                              const double2 *__restrict__ a2, const double2 *__restrict__ b2,
                              unsigned long long *out, int N, int H, int Hp) {
    double mx = 0.0;
    const long long total = (long long)N * Hp;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        if ((int)(i % Hp) >= H) continue;
        const double2 *A[3] = {a0, a1, a2};
        const double2 *B[3] = {b0, b1, b2};
        for (int c = 0; c < 3; ++c) {
            double2 v = A[c][i];
            if (B[c]) {
                const double2 w = B[c][i];
                v.x = v.x - w.x;
                v.y = v.y - w.y;
            }
            mx = fmax(mx, v.x * v.x + v.y * v.y);
        }
    }
    for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    if ((threadIdx.x & 31) == 0) atomicMax(out, (unsigned long long)__double_as_longlong(mx));
}

int pf_launch_measurecorr(pf_ctx *ctx, const double2 *a0, const double2 *b0, const double2 *a1,
                          const double2 *b1, const double2 *a2, const double2 *b2, bool reset) {
    const Geo &g = ctx->g;
    unsigned long long *out = &ctx->dsc->dterr2_bits;
    if (reset) PF_CUDA(cudaMemsetAsync(out, 0, sizeof(unsigned long long), ctx->stream));
    const unsigned grid = (unsigned)std::min<long long>(grid1((long long)g.N * g.Hp, BLK), 148LL * 8);
    {
        ProfScope ps_(ctx, PF_K_EW);
        k_measurecorr<<<grid, BLK, 0, ctx->stream>>>(a0, b0, a1, b1, a2, b2, out, g.N, g.H, g.Hp);
    }
    PF_LAUNCHED(ctx);
    return PF_OK;
}

// Hagen-Poiseuille advection and constant-flux pressure (velocity.f90:338-361)
__global__ void k_addHPF(double2 *Nr, double2 *Nt, double2 *Nz, const double2 *__restrict__ ur,
                         const double2 *__restrict__ ut, const double2 *__restrict__ uz,
                         DevMesh dm, Geo g, int const_flux, DevScalars *sc) {
    const int nh = blockIdx.x * blockDim.x + threadIdx.x, n = blockIdx.y;
    if (nh >= g.H) return;
    int k, m;
    mode_km(nh, g.K, k, m);
    const size_t at = (size_t)n * g.Hp + nh;
    const double a = g.alpha * k * dm.velU[n];
    const double b = -dm.velUp[n];
    const double2 vr = ur[at], vt = ut[at], vz = uz[at];
    double2 x = Nr[at];
    Nr[at] = make_double2(x.x + a * vr.y, x.y - a * vr.x);
    x = Nt[at];
    Nt[at] = make_double2(x.x + a * vt.y, x.y - a * vt.x);
    x = Nz[at];
    double zr = x.x + a * vz.y + b * vr.x;
    const double zi = x.y - a * vz.x + b * vr.y;
    if (const_flux && nh == 0) {
        double p = 0.0;
        for (int j = 0; j <= KL; ++j) p += uz[(size_t)(g.N - 1 - KL + j) * g.Hp].x * dm.dr1[1 * (KL + 1) + j];
        p = p / (-2.0);
        zr = zr + 4.0 * p / g.Re;
        if (n == 0) sc->Pr0 = p;
    }
    Nz[at] = make_double2(zr, zi);
}

int pf_launch_addHPF(pf_ctx *ctx) {
    const Geo &g = ctx->g;
    dim3 grid(grid1(g.H, 128), g.N);
    {
        ProfScope ps_(ctx, PF_K_INFL);
        k_addHPF<<<grid, 128, 0, ctx->stream>>>(ctx->vel[3].d, ctx->vel[4].d, ctx->vel[5].d, ctx->vel[0].d,
                                                ctx->vel[1].d, ctx->vel[2].d, ctx->dm, g,
                                                ctx->cfg.const_flux, ctx->dsc);
    }
    PF_LAUNCHED(ctx);
    return PF_OK;
}

// zero the k=m=0 parts fixed by symmetry after a step (velocity.f90:387-392)
__global__ void k_zero_mode0(double2 *ur, double2 *ut, double2 *uz, int N, int Hp) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= N) return;
    const size_t at = (size_t)n * Hp;
    ur[at] = make_double2(0.0, 0.0);
    ut[at].y = 0.0;
    uz[at].y = 0.0;
}

int pf_launch_zero_mode0(pf_ctx *ctx) {
    {
        ProfScope ps_(ctx, PF_K_INFL);
        k_zero_mode0<<<grid1(ctx->g.N, 64), 64, 0, ctx->stream>>>(ctx->vel[0].d, ctx->vel[1].d, ctx->vel[2].d,
                                                                  ctx->g.N, ctx->g.Hp);
    }
    PF_LAUNCHED(ctx);
    return PF_OK;
}

// ------------------------------------------------------------------ C ABI
#define SAMECTX2(a, b) PF_ARG((a) && (b) && (a)->ctx == (b)->ctx, "fields of different contexts")

extern "C" int pf_var_coll_init(pf_coll *a) {
    PF_ARG(a, "null field");
    return pf_launch_ew(a->ctx, EW_ZERO, nullptr, nullptr, a->d, nullptr, 0.0);
}
extern "C" int pf_var_coll_copy(const pf_coll *in, pf_coll *out) {
    SAMECTX2(in, out);
    if (in->d == out->d) return PF_OK;
    return pf_launch_ew(in->ctx, EW_COPY, in->d, nullptr, out->d, nullptr, 0.0);
}
extern "C" int pf_var_coll_add(const pf_coll *ac, pf_coll *a) {
    SAMECTX2(ac, a);
    return pf_launch_ew(a->ctx, EW_ADD, ac->d, nullptr, a->d, nullptr, 0.0);
}
extern "C" int pf_var_coll_sub(const pf_coll *ac, pf_coll *a) {
    SAMECTX2(ac, a);
    return pf_launch_ew(a->ctx, EW_SUB, ac->d, nullptr, a->d, nullptr, 0.0);
}
extern "C" int pf_var_coll_dmult(double d, pf_coll *a) {
    PF_ARG(a, "null field");
    return pf_launch_ew(a->ctx, EW_DMULT, nullptr, nullptr, a->d, nullptr, d);
}
extern "C" int pf_var_coll_neg(const pf_coll *ac, pf_coll *a) {
    SAMECTX2(ac, a);
    return pf_launch_ew(a->ctx, EW_NEG, ac->d, nullptr, a->d, nullptr, 0.0);
}

// Inputs that alias an output are first copied to scratch, so every routine
// has the reference's copy-in semantics (variables.f90:413-415, 447).
static const double2 *unalias(pf_ctx *ctx, const double2 *in, std::initializer_list<const double2 *> outs,
                              int slot, int *status) {
    *status = PF_OK;
    for (const double2 *o : outs)
        if (o == in) {
            *status = pf_launch_ew(ctx, EW_COPY, in, nullptr, ctx->s[slot].d, nullptr, 0.0);
            return ctx->s[slot].d;
        }
    return in;
}

extern "C" int pf_var_coll_meshmult(int p, const pf_coll *in, pf_coll *out) {
    SAMECTX2(in, out);
    PF_ARG(p >= 1 && p <= KL, "pf_var_coll_meshmult: derivative order must be 1..KL");
    int s;
    const double2 *i0 = unalias(in->ctx, in->d, {out->d}, 0, &s);
    PF_TRY(s);
    return pf_launch_meshmult_dr(in->ctx, p, i0, out->d);
}

extern "C" int pf_var_coll_curl(const pf_coll *r, const pf_coll *t, const pf_coll *z, pf_coll *or_,
                                pf_coll *ot, pf_coll *oz) {
    SAMECTX2(r, t);
    SAMECTX2(z, or_);
    SAMECTX2(ot, oz);
    SAMECTX2(r, oz);
    pf_ctx *ctx = r->ctx;
    int s;
    const double2 *a = unalias(ctx, r->d, {or_->d, ot->d, oz->d}, 0, &s); PF_TRY(s);
    const double2 *b = unalias(ctx, t->d, {or_->d, ot->d, oz->d}, 1, &s); PF_TRY(s);
    const double2 *c = unalias(ctx, z->d, {or_->d, ot->d, oz->d}, 2, &s); PF_TRY(s);
    return pf_launch_curl(ctx, a, b, c, or_->d, ot->d, oz->d);
}

extern "C" int pf_var_coll_grad(const pf_coll *p, pf_coll *r, pf_coll *t, pf_coll *z) {
    SAMECTX2(p, r);
    SAMECTX2(t, z);
    SAMECTX2(p, z);
    int s;
    const double2 *a = unalias(p->ctx, p->d, {r->d, t->d, z->d}, 0, &s); PF_TRY(s);
    return pf_launch_grad(p->ctx, a, r->d, t->d, z->d);
}

extern "C" int pf_var_coll_div(const pf_coll *r, const pf_coll *t, const pf_coll *z, pf_coll *dv) {
    SAMECTX2(r, t);
    SAMECTX2(z, dv);
    SAMECTX2(r, dv);
    pf_ctx *ctx = r->ctx;
    int s;
    const double2 *a = unalias(ctx, r->d, {dv->d}, 0, &s); PF_TRY(s);
    const double2 *b = unalias(ctx, t->d, {dv->d}, 1, &s); PF_TRY(s);
    const double2 *c = unalias(ctx, z->d, {dv->d}, 2, &s); PF_TRY(s);
    return pf_launch_div(ctx, a, b, c, dv->d);
}

extern "C" int pf_var_coll_shift(double dt, double dz, const pf_coll *a, pf_coll *b) {
    SAMECTX2(a, b);
    pf_ctx *ctx = a->ctx;
    const Geo &g = ctx->g;
    dim3 grid(grid1(g.H, 128), g.N);
    {
        ProfScope ps_(ctx, PF_K_EW);
        k_shift<<<grid, 128, 0, ctx->stream>>>(dt, dz, a->d, b->d, g);
    }
    PF_LAUNCHED(ctx);
    return PF_OK;
}

extern "C" int pf_var_imposesym(int i, pf_coll *r, pf_coll *t, pf_coll *z) {
    SAMECTX2(r, t);
    SAMECTX2(t, z);
    PF_ARG(i >= 0 && i <= 3, "pf_var_imposesym: i must be 0..3");
    return pf_launch_imposesym(r->ctx, i, r->d, t->d, z->d);
}

extern "C" int pf_var_coll_norm(const pf_coll *a, double *E, double *Ek, double *Em) {
    PF_ARG(a, "null field");
    return pf_norm_host(a->ctx, a->d, E, Ek, Em);
}

extern "C" int pf_tim_zerobc(pf_coll *a) {
    PF_ARG(a, "null field");
    return pf_launch_zerobc(a->ctx, a->d);
}

extern "C" int pf_tim_nlincorr(const pf_coll *N_, pf_coll *Nn) {
    SAMECTX2(N_, Nn);
    return pf_launch_ew(Nn->ctx, EW_NLINCORR, N_->d, nullptr, Nn->d, nullptr, Nn->ctx->cfg.implicit);
}

extern "C" int pf_tim_measurecorr(const pf_coll *c1, const pf_coll *c2, const pf_coll *c3) {
    SAMECTX2(c1, c2);
    SAMECTX2(c2, c3);
    pf_ctx *ctx = c1->ctx;
    PF_TRY(pf_launch_measurecorr(ctx, c1->d, nullptr, c2->d, nullptr, c3->d, nullptr, true));
    PF_CUDA(cudaMemcpyAsync(ctx->hsc, ctx->dsc, sizeof(DevScalars), cudaMemcpyDeviceToHost, ctx->stream));
    PF_CUDA(cudaStreamSynchronize(ctx->stream));
    const double d2 = bits_to_double(ctx->hsc->dterr2_bits);
    ctx->tim.dterr = std::max(ctx->tim.dterr, std::sqrt(d2));
    return PF_OK;
}

extern "C" int pf_tim_meshmult(int S, const pf_mesh *A, const pf_coll *b, const pf_coll *c, pf_coll *d) {
    (void)S;  // parity hint of the reference; the product is the same for both
    PF_ARG(A && b && c && d, "null argument");
    pf_ctx *ctx = b->ctx;
    int s;
    const double2 *bb = unalias(ctx, b->d, {d->d}, 0, &s); PF_TRY(s);
    const double2 *cc = unalias(ctx, c->d, {d->d}, 1, &s); PF_TRY(s);
    return pf_launch_tim_meshmult(ctx, A, bb, cc, d->d);
}
