// The util plug-in hook: main.f90 calls var_null(2) after every evaluation
// of the nonlinear terms and var_null(1) once per step before the predictor
// (main.f90:23,30,38); a plug-in built in place of var_null adds its own
// terms to vel_N.  Two of the reference's plug-ins run here on the device:
//   Coriolis.f90     : the Coriolis force -1/(4 Ro) Omega x (U + u') of a
//                      pipe rotating about an axis at angle phi to its own,
//                      Ro = Re Ek0 (Coriolis.f90:13-73);
//   nonnewtonian.f90 : Carreau-Yasuda shear-thinning viscosity nu(strain
//                      rate) and the extra stress terms it gives
//                      (nonnewtonian.f90:32-246);
//   LES.f90          : Smagorinsky or Vreman eddy viscosity nu_t with van
//                      Driest wall damping, the reference viscosity nu_r it
//                      keeps near 1.1 (1 + Re max nu_t), and the
//                      variable-viscosity terms (LES.f90:102-339).
// A host callback can be registered as well, for plug-ins written against
// the C ABI (they run on the context's stream between the same calls).
#include <cmath>
#include "pf_internal.cuh"

// ------------------------------------------------------------------ Coriolis
// N = d1 (Omega x (U + u')), Omega = (sin(phi) cos(th), -sin(phi) sin(th),
// cos(phi)), on the physical grid (Coriolis.f90:40-68)
static __global__ void k_coriolis(const double *__restrict__ vr, const double *__restrict__ vt,
                                  const double *__restrict__ vz, double *__restrict__ nr, double *__restrict__ nt,
                                  double *__restrict__ nz, const double *__restrict__ velU, Geo g, double d1,
                                  double sphi, double cphi) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const size_t per_n = (size_t)g.Th * g.Z;
    if (i >= per_n * g.N) return;
    const int n = (int)(i / per_n);
    const int m = (int)((i - (size_t)n * per_n) / g.Z);
    const double a = 2.0 * 3.1415926535897931 / (double)g.Th * m;
    const double Or = sphi * cos(a), Ot = -sphi * sin(a), Oz = cphi;
    const double w = vz[i] + velU[n];
    nr[i] = d1 * (Ot * w - Oz * vt[i]);
    nt[i] = d1 * (Oz * vr[i] - Or * w);
    nz[i] = d1 * (Or * vt[i] - Ot * vr[i]);
}

// ------------------------------------------------------------ non-Newtonian
// velocity gradient rows A(2,j) = (1/r)(d/dth u_j + ...) and A(3,j) = d/dz u_j
// in spectral space (nonnewtonian.f90:134-157)
static __global__ void k_nn_grad_rows(const double2 *__restrict__ ur, const double2 *__restrict__ ut,
                                      const double2 *__restrict__ uz, double2 *__restrict__ c1,
                                      double2 *__restrict__ c2, double2 *__restrict__ c3, DevMesh dm, Geo g,
                                      int row) {
    const int nh = blockIdx.x * blockDim.x + threadIdx.x, n = blockIdx.y;
    if (nh >= g.H) return;
    int k, m;
    mode_km(nh, g.K, k, m);
    const size_t at = (size_t)n * g.Hp + nh;
    const double2 a = ur[at], b = ut[at], c = uz[at];
    if (row == 2) {
        const double m_ = (double)(m * g.Mp), rm1 = dm.rp[2 * g.N + n];
        c1[at] = make_double2(rm1 * (-a.y * m_ - b.x), rm1 * (a.x * m_ - b.y));
        c2[at] = make_double2(rm1 * (-b.y * m_ + a.x), rm1 * (b.x * m_ + a.y));
        c3[at] = make_double2(rm1 * (-c.y * m_), rm1 * (c.x * m_));
    } else {
        const double d1 = g.alpha * k;
        c1[at] = make_double2(-a.y * d1, a.x * d1);
        c2[at] = make_double2(-b.y * d1, b.x * d1);
        c3[at] = make_double2(-c.y * d1, c.x * d1);
    }
}

// S = (A + A^T)/2 in place in A[9] (row-major 3x3 of phys fields), strain
// rate (2 S_ij S_ij)^(1/2) and the Carreau-Yasuda nu (nonnewtonian.f90:158-176)
struct Phys9 {
    double *a[9];
};
static __global__ void k_nn_strain(Phys9 A, double *__restrict__ nu, size_t np, double lam, double d1, double aCY,
                                   double d2) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= np) return;
    const double s12 = 0.5 * (A.a[1][i] + A.a[3][i]);
    const double s13 = 0.5 * (A.a[2][i] + A.a[6][i]);
    const double s23 = 0.5 * (A.a[5][i] + A.a[7][i]);
    A.a[1][i] = s12;
    A.a[3][i] = s12;
    A.a[2][i] = s13;
    A.a[6][i] = s13;
    A.a[5][i] = s23;
    A.a[7][i] = s23;
    const double s11 = A.a[0][i], s22 = A.a[4][i], s33 = A.a[8][i];
    double sr = s11 * s11 + s22 * s22 + s33 * s33 + 2.0 * (s12 * s12 + s13 * s13 + s23 * s23);
    sr = sqrt(2.0 * sr);
    nu[i] = d1 + (1.0 - d1) * pow(1.0 + pow(lam * sr, aCY), d2);
}

// N' = (1/Re)[(nu - nu_r)(-curl curl u) + 2 grad(nu).S + (nu_r - 1)(-4 z)]
// (nonnewtonian.f90:218-229), into q in place
static __global__ void k_nn_terms(Phys9 S, const double *__restrict__ nu, const double *__restrict__ g0,
                                  const double *__restrict__ g1, const double *__restrict__ g2, double *q0, double *q1,
                                  double *q2, size_t np, double velnu, double rRe) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= np) return;
    const double nu_ = nu[i] - velnu;
    const double g[3] = {g0[i], g1[i], g2[i]};
    double *q[3] = {q0, q1, q2};
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        double v = nu_ * (-q[c][i]);
#pragma unroll
        for (int j = 0; j < 3; ++j) v = v + g[j] * S.a[j * 3 + c][i] * 2.0;
        if (c == 2) v = v + (velnu - 1.0) * (-4.0);
        q[c][i] = v / rRe;
    }
}

// ----------------------------------------------------------------- LES
// Per radial point: r, Delta (Smagorinsky filter width), the squared
// azimuthal width of Vreman's filter; filled on the host by pf_util_set.
enum { LES_R = 0, LES_DELTA = 1, LES_DTH2 = 2, LES_DR2 = 3, LES_NT = 4 };

// nu_t on the grid from the gradient tensor A (LES.f90:195-274), then
// S = (A + A^T)/2 in place; u_tau from the wall derivative of the mean axial
// perturbation (LES.f90:164-171)
static __global__ void k_les_nu(Phys9 A, double *__restrict__ nu, Geo g, const double *__restrict__ tab,
                                const double2 *__restrict__ uz, const double *__restrict__ dr1, int model,
                                double Cs, double Aplus, double dz2) {
    const size_t per_n = (size_t)g.Th * g.Z;
    const size_t np = per_n * g.N;
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= np) return;
    const int n = (int)(i / per_n), N = g.N;
    double d1 = 0.0;
    for (int j = 0; j <= KL; ++j) d1 += uz[(size_t)(N - 1 - KL + j) * g.Hp].x * dr1[1 * (KL + 1) + j];
    const double u_tau = sqrt(fabs((d1 - 2.0) / g.Re));
    const double y_plus = g.Re * u_tau * (1.0 - tab[LES_R * N + n]);
    const double yA = Aplus > 0.0 ? y_plus / Aplus : 0.0;
    const double vanDr = Aplus > 0.0 ? 1.0 - exp(-(yA * yA)) : 0.0;  // van Driest (LES.f90:215, 267)
    double a[9];
#pragma unroll
    for (int q = 0; q < 9; ++q) a[q] = A.a[q][i];
    const double s12 = 0.5 * (a[1] + a[3]), s13 = 0.5 * (a[2] + a[6]), s23 = 0.5 * (a[5] + a[7]);
    double v;
    if (model == 1) {  // Smagorinsky: vanDr (C_s Delta)^2 |S|
        double sr = a[0] * a[0] + a[4] * a[4] + a[8] * a[8] + 2.0 * (s12 * s12 + s13 * s13 + s23 * s23);
        sr = sqrt(2.0 * sr);
        const double cd = Cs * tab[LES_DELTA * N + n];
        v = (vanDr * (cd * cd)) * sr;
    } else {  // Vreman
        double AA = 0.0;
#pragma unroll
        for (int q = 0; q < 9; ++q) AA = AA + a[q] * a[q];
        const double dm2[3] = {tab[LES_DR2 * N + n], tab[LES_DTH2 * N + n], dz2};
        double B[9];
#pragma unroll
        for (int p = 0; p < 3; ++p)
#pragma unroll
            for (int q = 0; q < 3; ++q) {
                double b = 0.0;
#pragma unroll
                for (int m = 0; m < 3; ++m) b = b + dm2[m] * a[m * 3 + p] * a[m * 3 + q];
                B[p * 3 + q] = b;
            }
        double P = B[0] * B[4] - B[1] * B[1] + B[0] * B[8] - B[2] * B[2] + B[4] * B[8] - B[5] * B[5];
        if (AA < 1e-12) P = 0.0;
        P = fmax(P, 0.0);
        AA = fmax(AA, 1e-12);
        v = Cs * sqrt(P / AA);
        if (Aplus > 0.0) {
            double w = 0.03 / Cs;
            w = w + (1.0 - w) * vanDr;
            v = w * v;
        }
    }
    nu[i] = v;
    A.a[1][i] = s12;
    A.a[3][i] = s12;
    A.a[2][i] = s13;
    A.a[6][i] = s13;
    A.a[5][i] = s23;
    A.a[7][i] = s23;
}

// N' = (1/Re)(Re nu_t + 1 - nu_r)(-curl curl u) + nu_t (-4 z) + 2 grad(nu_t).S
// (LES.f90:318-329), into q in place
static __global__ void k_les_terms(Phys9 S, const double *__restrict__ nu, const double *__restrict__ g0,
                                   const double *__restrict__ g1, const double *__restrict__ g2, double *q0,
                                   double *q1, double *q2, size_t np, double velnu, double Re) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= np) return;
    const double nut = nu[i];
    const double nu_ = Re * nut + (1.0 - velnu);
    const double g[3] = {g0[i], g1[i], g2[i]};
    double *q[3] = {q0, q1, q2};
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        double v = (1.0 / Re) * nu_ * (-q[c][i]);
        if (c == 2) v = v + nut * (-4.0);
#pragma unroll
        for (int j = 0; j < 3; ++j) v = v + g[j] * S.a[j * 3 + c][i] * 2.0;
        q[c][i] = v;
    }
}

// uz(:, mode 0) += U (the laminar profile), the total velocity the strain
// rate is formed from (nonnewtonian.f90:126-129)
static __global__ void k_add_laminar(double2 *uz, const double *__restrict__ velU, Geo g) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= g.N) return;
    uz[(size_t)n * g.Hp].x += velU[n];
}

static __global__ void k_minmax(const double *__restrict__ a, size_t n, unsigned long long *mx,
                                unsigned long long *mn_neg) {
    // nu > 0: ordered bit patterns of non-negative doubles compare as integers
    unsigned long long hi = 0, lo = 0;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const double v = fabs(a[i]);
        const unsigned long long b = (unsigned long long)__double_as_longlong(v);
        hi = b > hi ? b : hi;
        const unsigned long long c = ~b;  // max of ~b is the min of b
        lo = c > lo ? c : lo;
    }
    atomicMax(mx, hi);
    atomicMax(mn_neg, lo);
}

bool pf_util_active(const pf_ctx *ctx) { return ctx->util_kind != PF_UTIL_NONE || ctx->util_cb != nullptr; }

static size_t phys_elems(const pf_ctx *ctx) { return (size_t)ctx->g.N * ctx->g.Th * ctx->g.Z; }
static size_t coll_elems(const pf_ctx *ctx) { return (size_t)ctx->g.N * ctx->g.Hp; }

static int ensure_scratch(pf_ctx *ctx, int nphys, int ncoll) {
    if (ctx->util_nphys < nphys) {
        PF_TRY(pf_alloc(ctx, (void **)&ctx->util_phys, (size_t)nphys * phys_elems(ctx) * sizeof(double)));
        ctx->util_nphys = nphys;
    }
    if (ctx->util_ncoll < ncoll) {
        const size_t bytes = (size_t)ncoll * coll_elems(ctx) * sizeof(double2);
        PF_TRY(pf_alloc(ctx, (void **)&ctx->util_coll, bytes));
        PF_CUDA(cudaMemsetAsync(ctx->util_coll, 0, bytes, ctx->stream));  // padding modes stay zero
        ctx->util_ncoll = ncoll;
    }
    return PF_OK;
}

static int add_to_N(pf_ctx *ctx, double2 *const *c) {
    for (int i = 0; i < 3; ++i) PF_TRY(pf_launch_ew(ctx, EW_ADD, c[i], nullptr, ctx->vel[3 + i].d, nullptr, 0.0));
    return PF_OK;
}

static int coriolis(pf_ctx *ctx) {
    const Geo &g = ctx->g;
    const size_t np = phys_elems(ctx);
    double *ph = ctx->util_phys;
    const double Ro = g.Re * ctx->util_par[0];  // Ro = Re_0 Ek_0
    const double d1 = -1.0 / (4.0 * Ro);
    {
        ProfScope ps_(ctx, PF_K_EW);
        k_coriolis<<<grid1(np, 256), 256, 0, ctx->stream>>>(ctx->phys[0].d, ctx->phys[1].d, ctx->phys[2].d, ph,
                                                             ph + np, ph + 2 * np, ctx->dm.velU, g, d1,
                                                             std::sin(ctx->util_par[1]), std::cos(ctx->util_par[1]));
    }
    PF_LAUNCHED(ctx);
    double2 *cc = (double2 *)ctx->util_coll;
    const size_t ce = coll_elems(ctx);
    const double *src[3] = {ph, ph + np, ph + 2 * np};
    double2 *dst[3] = {cc, cc + ce, cc + 2 * ce};
    PF_TRY(pf_launch_phys2coll(ctx, 3, src, dst, false));
    return add_to_N(ctx, dst);
}

// get_nu + update_nonlin_terms (nonnewtonian.f90:111-247)
static int nonnewtonian(pf_ctx *ctx) {
    const Geo &g = ctx->g;
    const size_t np = phys_elems(ctx), ce = coll_elems(ctx);
    double *ph = ctx->util_phys;
    double2 *cc = (double2 *)ctx->util_coll;
    double2 *u[3] = {cc, cc + ce, cc + 2 * ce};           // ur, ut, uz (total)
    double2 *c[3] = {cc + 3 * ce, cc + 4 * ce, cc + 5 * ce};  // scratch
    double2 *nuc = cc + 6 * ce;
    double2 *w[3] = {cc + 7 * ce, cc + 8 * ce, cc + 9 * ce};  // curl u
    Phys9 A;
    for (int i = 0; i < 9; ++i) A.a[i] = ph + (size_t)i * np;
    double *nu = ph + 9 * np;
    double *gp[3] = {ph + 10 * np, ph + 11 * np, ph + 12 * np};
    double *q[3] = {ph + 13 * np, ph + 14 * np, ph + 15 * np};
    dim3 grid(grid1(g.H, 128), g.N);
    // vec{u} = (ur, ut, uz + U)
    for (int i = 0; i < 3; ++i) PF_TRY(pf_launch_ew(ctx, EW_COPY, ctx->vel[i].d, nullptr, u[i], nullptr, 0.0));
    {
        ProfScope ps_(ctx, PF_K_EW);
        k_add_laminar<<<grid1(g.N, 128), 128, 0, ctx->stream>>>(u[2], ctx->dm.velU, g);
    }
    PF_LAUNCHED(ctx);
    // A(1,j) = d/dr u_j
    for (int i = 0; i < 3; ++i) PF_TRY(pf_launch_meshmult_dr(ctx, 1, u[i], c[i]));
    {
        const double2 *s[3] = {c[0], c[1], c[2]};
        double *d[3] = {A.a[0], A.a[1], A.a[2]};
        PF_TRY(pf_launch_coll2phys(ctx, 3, s, d));
    }
    for (int row = 2; row <= 3; ++row) {
        {
            ProfScope ps_(ctx, PF_K_STENCIL);
            k_nn_grad_rows<<<grid, 128, 0, ctx->stream>>>(u[0], u[1], u[2], c[0], c[1], c[2], ctx->dm, g, row);
        }
        PF_LAUNCHED(ctx);
        const double2 *s[3] = {c[0], c[1], c[2]};
        double *d[3] = {A.a[(row - 1) * 3], A.a[(row - 1) * 3 + 1], A.a[(row - 1) * 3 + 2]};
        PF_TRY(pf_launch_coll2phys(ctx, 3, s, d));
    }
    // S, strain rate, nu; nu to spectral
    const double rho = ctx->util_par[0], radius = ctx->util_par[1], mu0 = ctx->util_par[2], muinf = ctx->util_par[3];
    const double lamCY = ctx->util_par[4], nCY = ctx->util_par[5], aCY = ctx->util_par[6];
    const double lam = g.Re * lamCY * mu0 / (rho * radius * radius);
    {
        ProfScope ps_(ctx, PF_K_EW);
        k_nn_strain<<<grid1(np, 256), 256, 0, ctx->stream>>>(A, nu, np, lam, muinf / mu0, aCY, -nCY / aCY);
    }
    PF_LAUNCHED(ctx);
    {
        const double *s[1] = {nu};
        double2 *d[1] = {nuc};
        PF_TRY(pf_launch_phys2coll(ctx, 1, s, d, false));
    }
    // diagnostics of write_Re_nu: nu at the wall (mean mode), min and max over the grid
    {
        unsigned long long *mm = (unsigned long long *)ctx->red;
        PF_CUDA(cudaMemsetAsync(mm, 0, 2 * sizeof(unsigned long long), ctx->stream));
        {
            ProfScope ps_(ctx, PF_K_EW);
            k_minmax<<<148, 256, 0, ctx->stream>>>(nu, np, mm, mm + 1);
        }
        PF_LAUNCHED(ctx);
        PF_CUDA(cudaMemcpyAsync(ctx->util_diag_d, mm, 2 * sizeof(unsigned long long), cudaMemcpyDeviceToDevice,
                                ctx->stream));
        PF_CUDA(cudaMemcpyAsync(ctx->util_diag_d + 2, nuc + (size_t)(g.N - 1) * g.Hp, sizeof(double),
                                cudaMemcpyDeviceToDevice, ctx->stream));
    }
    // grad(nu) and curl(curl(u)) on the grid
    PF_TRY(pf_launch_grad(ctx, nuc, c[0], c[1], c[2]));
    {
        const double2 *s[3] = {c[0], c[1], c[2]};
        PF_TRY(pf_launch_coll2phys(ctx, 3, s, gp));
    }
    PF_TRY(pf_launch_curl(ctx, u[0], u[1], u[2], w[0], w[1], w[2]));
    PF_TRY(pf_launch_curl(ctx, w[0], w[1], w[2], c[0], c[1], c[2]));
    {
        const double2 *s[3] = {c[0], c[1], c[2]};
        PF_TRY(pf_launch_coll2phys(ctx, 3, s, q));
    }
    {
        ProfScope ps_(ctx, PF_K_EW);
        k_nn_terms<<<grid1(np, 256), 256, 0, ctx->stream>>>(A, nu, gp[0], gp[1], gp[2], q[0], q[1], q[2], np,
                                                             ctx->vel_nu, g.Re);
    }
    PF_LAUNCHED(ctx);
    {
        const double *s[3] = {q[0], q[1], q[2]};
        PF_TRY(pf_launch_phys2coll(ctx, 3, s, c, false));
    }
    return add_to_N(ctx, c);
}

// The velocity gradient tensor A(i, j) on the grid from the total velocity
// u = u' + U (LES.f90:109-150, nonnewtonian.f90:119-157): A(1,j) = d/dr u_j,
// A(2,j), A(3,j) the azimuthal and axial rows.  u, c: 3 coll fields each.
static int velocity_gradient(pf_ctx *ctx, double2 *const *u, double2 *const *c, const Phys9 &A) {
    const Geo &g = ctx->g;
    for (int i = 0; i < 3; ++i) PF_TRY(pf_launch_ew(ctx, EW_COPY, ctx->vel[i].d, nullptr, u[i], nullptr, 0.0));
    {
        ProfScope ps_(ctx, PF_K_EW);
        k_add_laminar<<<grid1(g.N, 128), 128, 0, ctx->stream>>>(u[2], ctx->dm.velU, g);
    }
    PF_LAUNCHED(ctx);
    for (int i = 0; i < 3; ++i) PF_TRY(pf_launch_meshmult_dr(ctx, 1, u[i], c[i]));
    {
        const double2 *s[3] = {c[0], c[1], c[2]};
        double *d[3] = {A.a[0], A.a[1], A.a[2]};
        PF_TRY(pf_launch_coll2phys(ctx, 3, s, d));
    }
    const dim3 grid(grid1(g.H, 128), g.N);
    for (int row = 2; row <= 3; ++row) {
        {
            ProfScope ps_(ctx, PF_K_STENCIL);
            k_nn_grad_rows<<<grid, 128, 0, ctx->stream>>>(u[0], u[1], u[2], c[0], c[1], c[2], ctx->dm, g, row);
        }
        PF_LAUNCHED(ctx);
        const double2 *s[3] = {c[0], c[1], c[2]};
        double *d[3] = {A.a[(row - 1) * 3], A.a[(row - 1) * 3 + 1], A.a[(row - 1) * 3 + 2]};
        PF_TRY(pf_launch_coll2phys(ctx, 3, s, d));
    }
    return PF_OK;
}

// get_nu, update_nu_r, update_nonlin_terms of LES.f90 (util(2), :58-62)
static int les(pf_ctx *ctx) {
    const Geo &g = ctx->g;
    const size_t np = phys_elems(ctx), ce = coll_elems(ctx);
    double *ph = ctx->util_phys;
    double2 *cc = (double2 *)ctx->util_coll;
    double2 *u[3] = {cc, cc + ce, cc + 2 * ce};
    double2 *c[3] = {cc + 3 * ce, cc + 4 * ce, cc + 5 * ce};
    double2 *nuc = cc + 6 * ce;
    double2 *w[3] = {cc + 7 * ce, cc + 8 * ce, cc + 9 * ce};
    Phys9 A;
    for (int i = 0; i < 9; ++i) A.a[i] = ph + (size_t)i * np;
    double *nu = ph + 9 * np;
    double *gp[3] = {ph + 10 * np, ph + 11 * np, ph + 12 * np};
    double *q[3] = {ph + 13 * np, ph + 14 * np, ph + 15 * np};
    const int model = (int)ctx->util_par[0];
    const double Cs = ctx->util_par[1], Aplus = ctx->util_par[3];
    const double dz = ctx->util_par[5];
    PF_TRY(velocity_gradient(ctx, u, c, A));
    {
        ProfScope ps_(ctx, PF_K_EW);
        k_les_nu<<<grid1(np, 256), 256, 0, ctx->stream>>>(A, nu, g, ctx->util_tab, ctx->vel[2].d, ctx->dm.dr1, model,
                                                          Cs, Aplus, dz * dz);
    }
    PF_LAUNCHED(ctx);
    {
        const double *s[1] = {nu};
        double2 *d[1] = {nuc};
        PF_TRY(pf_launch_phys2coll(ctx, 1, s, d, false));
    }
    // max nu_t (LES.f90:183-188), and nu_t at the wall for the statistics
    unsigned long long *mm = (unsigned long long *)ctx->red;
    PF_CUDA(cudaMemsetAsync(mm, 0, 2 * sizeof(unsigned long long), ctx->stream));
    {
        ProfScope ps_(ctx, PF_K_EW);
        k_minmax<<<148, 256, 0, ctx->stream>>>(nu, np, mm, mm + 1);
    }
    PF_LAUNCHED(ctx);
    PF_CUDA(cudaMemcpyAsync(ctx->util_diag_d, mm, 2 * sizeof(unsigned long long), cudaMemcpyDeviceToDevice,
                            ctx->stream));
    PF_CUDA(cudaMemcpyAsync(ctx->util_diag_d + 2, nuc + (size_t)(g.N - 1) * g.Hp, sizeof(double),
                            cudaMemcpyDeviceToDevice, ctx->stream));
    if (ctx->tim.it == 0) {
        // update_nu_r (LES.f90:280-290): nu_r near 1.1 (1 + Re max nu_t);
        // a move beyond 7% re-factorises the matrices before the terms use it
        unsigned long long mx = 0;
        PF_CUDA(cudaMemcpyAsync(&mx, mm, sizeof(mx), cudaMemcpyDeviceToHost, ctx->stream));
        PF_CUDA(cudaStreamSynchronize(ctx->stream));
        double nu_max;
        std::memcpy(&nu_max, &mx, sizeof(double));
        double d1 = 1.0 + g.Re * nu_max;
        d1 = 1.10 * d1;
        if (ctx->vel_nu < 0.93 * d1 || ctx->vel_nu > 1.07 * d1) {
            ctx->vel_nu = d1;
            PF_TRY(pf_vel_matrices_impl(ctx));
        }
    }
    // grad(nu_t) and curl(curl(u)) on the grid, the terms, back to spectral
    PF_TRY(pf_launch_grad(ctx, nuc, c[0], c[1], c[2]));
    {
        const double2 *s[3] = {c[0], c[1], c[2]};
        PF_TRY(pf_launch_coll2phys(ctx, 3, s, gp));
    }
    PF_TRY(pf_launch_curl(ctx, u[0], u[1], u[2], w[0], w[1], w[2]));
    PF_TRY(pf_launch_curl(ctx, w[0], w[1], w[2], c[0], c[1], c[2]));
    {
        const double2 *s[3] = {c[0], c[1], c[2]};
        PF_TRY(pf_launch_coll2phys(ctx, 3, s, q));
    }
    {
        ProfScope ps_(ctx, PF_K_EW);
        k_les_terms<<<grid1(np, 256), 256, 0, ctx->stream>>>(A, nu, gp[0], gp[1], gp[2], q[0], q[1], q[2], np,
                                                              ctx->vel_nu, g.Re);
    }
    PF_LAUNCHED(ctx);
    {
        const double *s[3] = {q[0], q[1], q[2]};
        PF_TRY(pf_launch_phys2coll(ctx, 3, s, c, false));
    }
    return add_to_N(ctx, c);
}

// Filter widths per radial point (init_params_model, LES.f90:80-90, and the
// widths of Smagorinsky and Vreman, :205-212, :240-246), in d_PI's digits
static int les_tables(pf_ctx *ctx, int filter) {
    const Geo &g = ctx->g;
    const int N = g.N;
    const double PI = 3.1415926535897931;
    const double Rdth = (2.0 * PI / (double)(g.Mp * g.Th)) * (3.0 / 2.0);
    const double dz = (2.0 * PI / (g.alpha * g.Z)) * (3.0 / 2.0);
    const std::vector<double> &r = ctx->hm.r;
    std::vector<double> Dr(N), tab((size_t)LES_NT * N);
    Dr[0] = (r[1] - 0.0) / 2.0;
    for (int n = 1; n < N - 1; ++n) Dr[n] = (r[n + 1] - r[n - 1]) / 2.0;
    Dr[N - 1] = 1.0 - r[N - 2];
    for (int n = 0; n < N; ++n) {
        tab[LES_R * N + n] = r[n];
        double D;
        if (filter == 1) D = std::pow(Dr[n] * Rdth * dz, 1.0 / 3.0);
        else if (filter == 2) D = std::pow(Dr[n] * r[n] * Rdth * dz, 1.0 / 3.0);
        else D = std::sqrt((Dr[n] * Dr[n] + (r[n] * Rdth) * (r[n] * Rdth) + dz * dz) / 3.0);
        tab[LES_DELTA * N + n] = D;
        // Vreman's azimuthal width: R dth (filter 1), r R dth (2); with
        // filter 3 the reference sets none and keeps the last radial width
        const double dth = filter == 1 ? Rdth : (filter == 2 ? r[n] * Rdth : Dr[N - 1]);
        tab[LES_DTH2 * N + n] = dth * dth;
        tab[LES_DR2 * N + n] = Dr[n] * Dr[n];
    }
    if (!ctx->util_tab) PF_TRY(pf_alloc(ctx, (void **)&ctx->util_tab, (size_t)LES_NT * 128 * sizeof(double)));
    PF_CUDA(cudaMemcpy(ctx->util_tab, tab.data(), tab.size() * sizeof(double), cudaMemcpyHostToDevice));
    ctx->util_par[5] = dz;
    return PF_OK;
}

int pf_util_run(pf_ctx *ctx, int flag) {
    if (flag == 2) {
        if (ctx->util_kind == PF_UTIL_CORIOLIS) PF_TRY(coriolis(ctx));
        else if (ctx->util_kind == PF_UTIL_CARREAU_YASUDA) {
            PF_TRY(nonnewtonian(ctx));
            ++ctx->util_evals;
        } else if (ctx->util_kind == PF_UTIL_LES) {
            PF_TRY(les(ctx));
            ++ctx->util_evals;
        }
    }
    if (ctx->util_cb) ctx->util_cb(ctx, flag, ctx->util_user);
    return PF_OK;
}

extern "C" int pf_util_set(pf_ctx *ctx, int kind, const double *params, int nparams) {
    PF_ARG(ctx, "pf_util_set: null ctx");
    switch (kind) {
    case PF_UTIL_NONE:
        break;
    case PF_UTIL_CORIOLIS:
        PF_ARG(params && nparams >= 2, "pf_util_set: Coriolis needs Ek0, phi");
        PF_ARG(params[0] != 0.0, "pf_util_set: Ek0 must be nonzero");
        if (ctx->g.Mp != 1) {
            pf_set_error("add_coriolis: i_Mp/=1");
            return PF_ERR_ARG;
        }
        PF_TRY(ensure_scratch(ctx, 3, 3));
        break;
    case PF_UTIL_CARREAU_YASUDA:
        PF_ARG(params && nparams >= 7, "pf_util_set: Carreau-Yasuda needs rho, radius, mu_0, mu_inf, lam, n, a");
        PF_ARG(params[0] > 0.0 && params[1] > 0.0 && params[2] > 0.0 && params[6] != 0.0,
               "pf_util_set: rho, radius, mu_0 must be > 0 and a nonzero");
        PF_TRY(ensure_scratch(ctx, 16, 10));
        if (!ctx->util_diag_d) {
            PF_TRY(pf_alloc(ctx, (void **)&ctx->util_diag_d, 4 * sizeof(double)));
            PF_CUDA(cudaMemsetAsync(ctx->util_diag_d, 0, 4 * sizeof(double), ctx->stream));
        }
        ctx->tim.pcn = 1;  // one corrector pass per step (nonnewtonian.f90:66-67)
        ctx->tim.it = 0;
        break;
    case PF_UTIL_LES:
        PF_ARG(params && nparams >= 4, "pf_util_set: LES needs model, C_s, filter, A_plus");
        PF_ARG(params[0] == 1.0 || params[0] == 2.0, "pf_util_set: LES model must be 1 (Smagorinsky) or 2 (Vreman)");
        PF_ARG(params[2] == 1.0 || params[2] == 2.0 || params[2] == 3.0, "pf_util_set: LES filter must be 1, 2 or 3");
        PF_ARG(params[1] > 0.0, "pf_util_set: LES C_s must be > 0");
        PF_ARG(params[0] == 2.0 || params[3] > 0.0, "pf_util_set: Smagorinsky needs A_plus > 0 (van Driest)");
        PF_ARG(ctx->g.N <= 128, "pf_util_set: LES supports N <= 128");
        PF_TRY(ensure_scratch(ctx, 16, 10));
        if (!ctx->util_diag_d) {
            PF_TRY(pf_alloc(ctx, (void **)&ctx->util_diag_d, 4 * sizeof(double)));
            PF_CUDA(cudaMemsetAsync(ctx->util_diag_d, 0, 4 * sizeof(double), ctx->stream));
        }
        ctx->tim.pcn = 1;  // one corrector pass per step (LES.f90:74-75)
        ctx->tim.it = 0;
        break;
    default:
        pf_set_error("pf_util_set: unknown plug-in %d", kind);
        return PF_ERR_ARG;
    }
    for (int i = 0; i < 8; ++i) ctx->util_par[i] = (params && i < nparams) ? params[i] : 0.0;
    if (kind == PF_UTIL_LES) PF_TRY(les_tables(ctx, (int)params[2]));
    ctx->util_kind = kind;
    ctx->util_evals = 0;
    pf_graphs_reset(ctx);
    return PF_OK;
}

extern "C" int pf_util_set_callback(pf_ctx *ctx, pf_util_fn fn, void *user) {
    PF_ARG(ctx, "pf_util_set_callback: null ctx");
    ctx->util_cb = fn;
    ctx->util_user = user;
    pf_graphs_reset(ctx);
    return PF_OK;
}

extern "C" int pf_util(pf_ctx *ctx, int flag) {
    PF_ARG(ctx && (flag == 1 || flag == 2), "pf_util: flag must be 1 or 2");
    return pf_util_run(ctx, flag);
}

extern "C" int pf_util_nu_stats(pf_ctx *ctx, double *nu_wall, double *nu_min, double *nu_max) {
    PF_ARG(ctx, "pf_util_nu_stats: null ctx");
    if ((ctx->util_kind != PF_UTIL_CARREAU_YASUDA && ctx->util_kind != PF_UTIL_LES) || !ctx->util_evals) {
        pf_set_error("pf_util_nu_stats: no Carreau-Yasuda or LES evaluation yet");
        return PF_ERR_STATE;
    }
    double h[3];
    PF_CUDA(cudaMemcpyAsync(h, ctx->util_diag_d, 3 * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    PF_CUDA(cudaStreamSynchronize(ctx->stream));
    unsigned long long mx, mn;
    std::memcpy(&mx, &h[0], 8);
    std::memcpy(&mn, &h[1], 8);
    mn = ~mn;
    if (nu_max) std::memcpy(nu_max, &mx, 8);
    if (nu_min) std::memcpy(nu_min, &mn, 8);
    if (nu_wall) *nu_wall = h[2];
    return PF_OK;
}
