// Per-Fourier-mode banded Helmholtz / pressure-Poisson systems on the device:
// matrix assembly with axis-parity and wall rows, banded LU with partial
// pivoting (LAPACK dgbtrf == dgbtf2 for KL=4 < block size), banded solves
// (dgbtrs), the influence-matrix precompute and correction, and the
// constant-flux adjustment (timestep.f90:46-123; velocity.f90:120-298).
//
// Storage: lu[(row*N + col)*Hp + nh] with `row` the 0-based LAPACK band row
// (diagonal at row KV), so one thread per mode reads column-major bands and
// consecutive modes are consecutive in memory.
#include <cmath>
#include "pf_internal.cuh"

#define LU(row, col) lu[((size_t)(row) * N + (col)) * Hp + nh]

// Assemble A = c1 I + c2 Lap(PM) with the axis-parity first row and the wall
// row, then factor in place (timestep.f90:75-93; dgbtf2).
__global__ void k_lu_factor(double *__restrict__ lu, unsigned char *__restrict__ piv, DevMesh dm, Geo g,
                            int PM, int BC, double c1, double c2, int *info, int *anypiv) {
    const int nh = blockIdx.x * blockDim.x + threadIdx.x;
    if (nh >= g.H) return;
    const int N = g.N, Hp = g.Hp;
    int k, m;
    mode_km(nh, g.K, k, m);
    const int S = (m * g.Mp + abs(PM)) % 2;  // axis parity (timestep.f90:82)
    for (int col = 0; col < N; ++col) {
        for (int row = 0; row < KL; ++row) LU(row, col) = 0.0;
        for (int r2 = 0; r2 < NBAND; ++r2) {  // A(col + r2 - KL, col)
            const int row = col + r2 - KL;
            LU(KL + r2, col) = (row >= 0 && row < N)
                                   ? lumesh_entry(dm, N, g.Mp, g.alpha, PM, BC, c1, c2, k, m, S, row, col)
                                   : __dmul_rn(c2, dm.radLap[r2 * N + col]);
        }
    }
    if (BC == 1 && k == 0 && m == 0) return;  // singular Neumann mean mode: skipped
    // dgbtf2: A(r,c) lives at band row KV + r - c
    int ju = 0;
    for (int j = 0; j < N; ++j) {
        const int km = min(KL, N - 1 - j);
        int jp = 0;
        double amax = fabs(LU(KV, j));
        for (int i = 1; i <= km; ++i) {
            const double a = fabs(LU(KV + i, j));
            if (a > amax) {
                amax = a;
                jp = i;
            }
        }
        piv[(size_t)j * Hp + nh] = (unsigned char)jp;
        if (jp != 0) atomicOr(anypiv, 1);
        if (LU(KV + jp, j) != 0.0) {
            ju = max(ju, min(j + KL + jp, N - 1));
            if (jp != 0)
                for (int c = j; c <= ju; ++c) {
                    const double t = LU(KV + jp - (c - j), c);
                    LU(KV + jp - (c - j), c) = LU(KV - (c - j), c);
                    LU(KV - (c - j), c) = t;
                }
            if (km > 0) {
                const double rp = 1.0 / LU(KV, j);
                for (int i = 1; i <= km; ++i) LU(KV + i, j) *= rp;
                for (int c = j + 1; c <= ju; ++c) {
                    const double y = -LU(KV - (c - j), c);  // -A(j, c)
                    for (int i = 1; i <= km; ++i)
                        LU(KV + i - (c - j), c) = fma(LU(KV + i, j), y, LU(KV + i - (c - j), c));
                }
            }
        } else {
            atomicCAS(info, 0, j + 1);
        }
    }
}

// One banded solve (dgbtrs 'N' with one right-hand side): forward sweep with
// the row interchanges and unit-lower multipliers, then the upper-triangular
// band back substitution (dtbsv).  b(n) is at b[n*stride]; the active part of
// the vector is held in a register window.
__device__ __forceinline__ void lu_solve_one(const double *__restrict__ lu, const unsigned char *__restrict__ piv,
                                             int N, int Hp, int nh, double *b, size_t stride) {
    double w[KL + 1];
#pragma unroll
    for (int i = 0; i <= KL; ++i) w[i] = (i < N) ? b[(size_t)i * stride] : 0.0;
    for (int j = 0; j < N; ++j) {
        if (j < N - 1) {
            const int p = piv[(size_t)j * Hp + nh];
#pragma unroll
            for (int i = 1; i <= KL; ++i)
                if (p == i) {
                    const double t = w[0];
                    w[0] = w[i];
                    w[i] = t;
                }
            const double bj = w[0];
#pragma unroll
            for (int i = 1; i <= KL; ++i)
                if (j + i < N) w[i] = fma(-LU(KV + i, j), bj, w[i]);
        }
        b[(size_t)j * stride] = w[0];
#pragma unroll
        for (int i = 0; i < KL; ++i) w[i] = w[i + 1];
        w[KL] = (j + KL + 1 < N) ? b[(size_t)(j + KL + 1) * stride] : 0.0;
    }
    double v[KV + 1];
#pragma unroll
    for (int i = 0; i <= KV; ++i) v[i] = (N - 1 - i >= 0) ? b[(size_t)(N - 1 - i) * stride] : 0.0;
    for (int j = N - 1; j >= 0; --j) {
        double x = v[0];
        if (x != 0.0) {
            x = x / LU(KV, j);
#pragma unroll
            for (int i = 1; i <= KV; ++i)
                if (j - i >= 0) v[i] = fma(-x, LU(KV - i, j), v[i]);
        }
        b[(size_t)j * stride] = x;
#pragma unroll
        for (int i = 0; i < KV; ++i) v[i] = v[i + 1];
        v[KV] = (j - KV - 1 >= 0) ? b[(size_t)(j - KV - 1) * stride] : 0.0;
    }
}

// thread = (mode, re/im); timestep.f90:109-121
__global__ void k_lu_solve(const double *__restrict__ lu, const unsigned char *__restrict__ piv,
                           double2 *b, int N, int H, int Hp, int BC) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int nh = t >> 1, part = t & 1;
    if (nh >= H) return;
    double *bp = reinterpret_cast<double *>(b) + 2 * (size_t)nh + part;
    const size_t stride = 2 * (size_t)Hp;
    if (BC == 1 && nh == 0) {
        for (int n = 0; n < N; ++n) bp[n * stride] = 0.0;
        return;
    }
    lu_solve_one(lu, piv, N, Hp, nh, bp, stride);
}

int pf_launch_lu_factor(pf_ctx *ctx, pf_lumesh *A) {
    const Geo &g = ctx->g;
    PF_CUDA(cudaMemsetAsync(&ctx->dsc->info, 0, sizeof(int), ctx->stream));
    PF_CUDA(cudaMemsetAsync(ctx->anypiv, 0, sizeof(int), ctx->stream));
    {
        ProfScope ps_(ctx, PF_K_FACTOR);
        k_lu_factor<<<grid1(g.H, 64), 64, 0, ctx->stream>>>(A->lu, A->piv, ctx->dm, g, A->PM, A->BC, A->c1, A->c2,
                                                             &ctx->dsc->info, ctx->anypiv);
    }
    PF_LAUNCHED(ctx);
    int info = 0;
    PF_CUDA(cudaMemcpyAsync(&info, &ctx->dsc->info, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    PF_CUDA(cudaMemcpyAsync(&A->pivoted, ctx->anypiv, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    PF_CUDA(cudaStreamSynchronize(ctx->stream));
    if (info != 0) {
        pf_set_error("tim_lumesh_init: zero pivot in column %d", info);
        return PF_ERR_SINGULAR;
    }
    return PF_OK;
}

int pf_launch_lu_solve(pf_ctx *ctx, int BC, const pf_lumesh *A, double2 *b) {
    const Geo &g = ctx->g;
    {
        ProfScope ps_(ctx, PF_K_LUSOLVE);
        k_lu_solve<<<grid1(2LL * g.H, 128), 128, 0, ctx->stream>>>(A->lu, A->piv, b, g.N, g.H, g.Hp, BC);
    }
    PF_LAUNCHED(ctx);
    return PF_OK;
}

// ------------------------------------------------- influence matrices
// Boundary residuals of (u+, u-, uz) at r=1 (velocity.f90:262-298).
__device__ __forceinline__ void eval_bc(const double2 *__restrict__ up, const double2 *__restrict__ um,
                                        const double2 *__restrict__ uz, const DevMesh &dm, const Geo &g,
                                        int nh, int k, int m, double BRe[4], double BIm[4]) {
    const int N = g.N;
    const size_t at = (size_t)(N - 1) * g.Hp + nh;
    const double2 p = up[at], q = um[at], z = uz[at];
    const double urRe = 0.5 * (p.x + q.x), urIm = 0.5 * (p.y + q.y);
    const double utRe = 0.5 * (p.y - q.y), utIm = -0.5 * (p.x - q.x);
    double drRe = 0.0, drIm = 0.0;
    for (int j = 0; j <= KL; ++j) {
        const size_t a = (size_t)(N - 1 - KL + j) * g.Hp + nh;
        const double w = dm.dr1[1 * (KL + 1) + j];
        drRe += w * (up[a].x + um[a].x);
        drIm += w * (up[a].y + um[a].y);
    }
    drRe = 0.5 * drRe;
    drIm = 0.5 * drIm;
    const double d = dm.rp[2 * N + (N - 1)];
    const double m_ = (double)(m * g.Mp), a_ = g.alpha * k;
    BRe[0] = p.x; BIm[0] = p.y;
    BRe[1] = q.x; BIm[1] = q.y;
    BRe[2] = -z.y; BIm[2] = z.x;
    BRe[3] = urRe * d + drRe - d * m_ * utIm - a_ * z.y;
    BIm[3] = urIm * d + drIm + d * m_ * utRe + a_ * z.x;
}

// Column j of A (velocity.f90:219-220) and the stored solution U(:,:,c).
__global__ void k_ppe0_column(int j, const double2 *up, const double2 *um, const double2 *uz, double *Ainv,
                              double *U, DevMesh dm, Geo g) {
    const int nh = blockIdx.x * blockDim.x + threadIdx.x;
    if (nh >= g.H) return;
    int k, m;
    mode_km(nh, g.K, k, m);
    double BRe[4], BIm[4];
    if (nh != 0) {
        eval_bc(up, um, uz, dm, g, nh, k, m, BRe, BIm);
        for (int i = 0; i < 4; ++i) Ainv[(size_t)(i * 4 + j) * g.Hp + nh] = BRe[i];
    }
    const int N = g.N;
    for (int n = 0; n < N; ++n) {
        const size_t at = (size_t)n * g.Hp + nh;
        if (j == 0) U[(size_t)(0 * N + n) * g.Hp + nh] = up[at].x;
        if (j == 1) U[(size_t)(1 * N + n) * g.Hp + nh] = um[at].x;
        if (j == 2) U[(size_t)(2 * N + n) * g.Hp + nh] = uz[at].y;
        if (j == 3) {
            U[(size_t)(3 * N + n) * g.Hp + nh] = up[at].x;
            U[(size_t)(4 * N + n) * g.Hp + nh] = um[at].x;
            U[(size_t)(5 * N + n) * g.Hp + nh] = uz[at].y;
        }
    }
}

// Replace each mode's 4x4 A by its inverse (mes_mat_invert, meshs.f90:231-243),
// Gauss-Jordan with partial pivoting; k=m=0 skipped (velocity.f90:222-225).
__global__ void k_invert4(double *Ainv, int H, int Hp, int *info) {
    const int nh = blockIdx.x * blockDim.x + threadIdx.x;
    if (nh >= H || nh == 0) return;
    double a[4][4], b[4][4];
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) {
            a[i][j] = Ainv[(size_t)(i * 4 + j) * Hp + nh];
            b[i][j] = (i == j) ? 1.0 : 0.0;
        }
    for (int c = 0; c < 4; ++c) {
        int p = c;
        for (int r = c + 1; r < 4; ++r)
            if (fabs(a[r][c]) > fabs(a[p][c])) p = r;
        if (a[p][c] == 0.0) {
            atomicCAS(info, 0, -(nh + 1));
            return;
        }
        if (p != c)
            for (int q = 0; q < 4; ++q) {
                double t = a[p][q]; a[p][q] = a[c][q]; a[c][q] = t;
                t = b[p][q]; b[p][q] = b[c][q]; b[c][q] = t;
            }
        const double inv = 1.0 / a[c][c];
        for (int q = 0; q < 4; ++q) {
            a[c][q] *= inv;
            b[c][q] *= inv;
        }
        for (int r = 0; r < 4; ++r) {
            if (r == c) continue;
            const double f = a[r][c];
            for (int q = 0; q < 4; ++q) {
                a[r][q] -= f * a[c][q];
                b[r][q] -= f * b[c][q];
            }
        }
    }
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) Ainv[(size_t)(i * 4 + j) * Hp + nh] = b[i][j];
}

// vel_adjPPE(2): u += sum_j a_j U_j with a = -A^-1 B (velocity.f90:238-256).
__global__ void k_adjppe2(double2 *ur, double2 *ut, double2 *uz, const double *__restrict__ Ainv,
                          const double *__restrict__ U, DevMesh dm, Geo g) {
    const int nh = blockIdx.x * blockDim.x + threadIdx.x;
    if (nh >= g.H || nh == 0) return;
    int k, m;
    mode_km(nh, g.K, k, m);
    double BRe[4], BIm[4], aR[4], aI[4];
    eval_bc(ur, ut, uz, dm, g, nh, k, m, BRe, BIm);
    for (int i = 0; i < 4; ++i) {
        double sr = 0.0, si = 0.0;
        for (int j = 0; j < 4; ++j) {
            const double a = Ainv[(size_t)(i * 4 + j) * g.Hp + nh];
            sr += a * BRe[j];
            si += a * BIm[j];
        }
        aR[i] = -sr;
        aI[i] = -si;
    }
    const int N = g.N;
    for (int n = 0; n < N; ++n) {
        const size_t at = (size_t)n * g.Hp + nh;
        const double U1 = U[(size_t)(0 * N + n) * g.Hp + nh], U2 = U[(size_t)(1 * N + n) * g.Hp + nh];
        const double U3 = U[(size_t)(2 * N + n) * g.Hp + nh], U4 = U[(size_t)(3 * N + n) * g.Hp + nh];
        const double U5 = U[(size_t)(4 * N + n) * g.Hp + nh], U6 = U[(size_t)(5 * N + n) * g.Hp + nh];
        double2 r = ur[at], t = ut[at], z = uz[at];
        r.x = r.x + aR[0] * U1; r.y = r.y + aI[0] * U1;
        t.x = t.x + aR[1] * U2; t.y = t.y + aI[1] * U2;
        z.x = z.x - aI[2] * U3; z.y = z.y + aR[2] * U3;
        r.x = r.x + aR[3] * U4; r.y = r.y + aI[3] * U4;
        t.x = t.x + aR[3] * U5; t.y = t.y + aI[3] * U5;
        z.x = z.x - aI[3] * U6; z.y = z.y + aR[3] * U6;
        ur[at] = r; ut[at] = t; uz[at] = z;
    }
}

int pf_launch_adjppe2(pf_ctx *ctx) {
    const Geo &g = ctx->g;
    {
        ProfScope ps_(ctx, PF_K_INFL);
        k_adjppe2<<<grid1(g.H, 64), 64, 0, ctx->stream>>>(ctx->vel[0].d, ctx->vel[1].d, ctx->vel[2].d, ctx->Ainv,
                                                           ctx->U, ctx->dm, g);
    }
    PF_LAUNCHED(ctx);
    return PF_OK;
}

// ------------------------------------------------------- constant flux
// F=0: Ui = LDz(0)^-1 [0,1,..,1,0], d1 = 2 int Ui r dr (velocity.f90:160-168)
__global__ void k_flux0(const double *lu, const unsigned char *piv, double *Ui, DevMesh dm, Geo g,
                        DevScalars *sc) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const int N = g.N;
    for (int n = 0; n < N; ++n) Ui[n] = (n == 0 || n == N - 1) ? 0.0 : 1.0;
    lu_solve_one(lu, piv, N, g.Hp, 0, Ui, 1);
    double d1 = 0.0;
    for (int n = 0; n < N; ++n) d1 += Ui[n] * dm.intrdr[n];
    sc->flux_d1 = 2.0 * d1;
}

// F=1: remove the mean-flux excess and update Pr0 (velocity.f90:170-175)
__global__ void k_flux1(double2 *uz, const double *__restrict__ Ui, DevMesh dm, Geo g, DevScalars *sc) {
    __shared__ double part[32];
    const int N = g.N;
    double s = 0.0;
    for (int n = threadIdx.x; n < N; n += blockDim.x) s += uz[(size_t)n * g.Hp].x * dm.intrdr[n];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < (int)(blockDim.x + 31) / 32; ++w) t += part[w];
        part[0] = t;
    }
    __syncthreads();
    const double d2 = 2.0 * part[0];
    const double d3 = -d2 / sc->flux_d1;
    for (int n = threadIdx.x; n < N; n += blockDim.x) {
        double2 v = uz[(size_t)n * g.Hp];
        v.x = v.x + d3 * Ui[n];
        uz[(size_t)n * g.Hp] = v;
    }
    if (threadIdx.x == 0) sc->Pr0 = sc->Pr0 + d3 * g.Re / 4.0;
}

int pf_launch_flux1(pf_ctx *ctx) {
    if (!ctx->cfg.const_flux) return PF_OK;
    {
        ProfScope ps_(ctx, PF_K_INFL);
        k_flux1<<<1, 256, 0, ctx->stream>>>(ctx->vel[2].d, ctx->Ui, ctx->dm, ctx->g, ctx->dsc);
    }
    PF_LAUNCHED(ctx);
    return PF_OK;
}

// ---------------------------------------------------------- vel_matrices
__global__ void k_piv_to_double(const unsigned char *__restrict__ piv, double *__restrict__ pivd, size_t n) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        pivd[i] = (double)piv[i];
}

// The compact copy of a factor set: the band and pivots of the modes with
// k >= 0 only, at c = m*K + k (padding columns zero).
__global__ void k_lu_compact(const double *__restrict__ lu, const double *__restrict__ pivd, double *__restrict__ luc,
                             double *__restrict__ pivdc, int N, int Hp, int Hcp, int K, int M) {
    const size_t rows = (size_t)NLU * N + N;  // band entries, then the pivot row of each column
    const size_t total = rows * Hcp;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
        const size_t r = i / Hcp;
        const int c = (int)(i - r * Hcp);
        double v = 0.0;
        if (c < M * K) {
            const int m = c / K, k = c - m * K;
            const int nh = m == 0 ? k : m * (2 * K - 1) + k;
            v = r < (size_t)NLU * N ? lu[r * Hp + nh] : pivd[(r - (size_t)NLU * N) * Hp + nh];
        }
        if (r < (size_t)NLU * N) luc[r * Hcp + c] = v;
        else pivdc[(r - (size_t)NLU * N) * Hcp + c] = v;
    }
}

static int lumesh_init(pf_ctx *ctx, pf_lumesh *A, int PM, int BC, double c1, double c2) {
    A->PM = PM;
    A->BC = BC;
    A->c1 = c1;
    A->c2 = c2;
    PF_TRY(pf_launch_lu_factor(ctx, A));
    if (A->pivd) {  // pivots as doubles, staged by the fused solves with 8-byte copies
        const Geo &g = ctx->g;
        const size_t np = (size_t)g.N * g.Hp;
        {
            ProfScope ps_(ctx, PF_K_FACTOR);
            k_piv_to_double<<<grid1(np, 256), 256, 0, ctx->stream>>>(A->piv, A->pivd, np);
        }
        PF_LAUNCHED(ctx);
        if (A->luc) {
            const int Hcp = pf_compact_modes_padded(g);
            const size_t nc = ((size_t)NLU * g.N + g.N) * Hcp;
            {
                ProfScope ps_(ctx, PF_K_FACTOR);
                k_lu_compact<<<grid1(nc, 256), 256, 0, ctx->stream>>>(A->lu, A->pivd, A->luc, A->pivdc, g.N, g.Hp, Hcp,
                                                                      g.K, g.M);
            }
            PF_LAUNCHED(ctx);
        }
    }
    return PF_OK;
}

// velocity.f90:120-146 including vel_adjustFlux(0) and vel_adjPPE(0)
int pf_vel_matrices_impl(pf_ctx *ctx) {
    const Geo &g = ctx->g;
    pf_graphs_reset(ctx);  // the graphs bake in 1/dt and the factor sets
    const pf_config &cfg = ctx->cfg;
    if (!ctx->LNp_set) {
        PF_TRY(lumesh_init(ctx, &ctx->LNp, 0, 1, 0.0, 1.0));
        ctx->LNp_set = true;
    }
    double d1 = 1.0 / ctx->tim.dt;
    double d2 = -cfg.implicit * ctx->vel_nu / cfg.Re;
    PF_TRY(lumesh_init(ctx, &ctx->LDp, 1, 0, d1, d2));
    PF_TRY(lumesh_init(ctx, &ctx->LDm, -1, 0, d1, d2));
    PF_TRY(lumesh_init(ctx, &ctx->LDz, 0, 0, d1, d2));
    d1 = 1.0 / ctx->tim.dt;
    d2 = (1.0 - cfg.implicit) * ctx->vel_nu / cfg.Re;
    ctx->Ltp = {ctx, 1, d1, d2};
    ctx->Ltm = {ctx, -1, d1, d2};
    ctx->Ltz = {ctx, 0, d1, d2};
    // vel_adjustFlux(0)
    if (cfg.const_flux) {
        {
            ProfScope ps_(ctx, PF_K_FACTOR);
            k_flux0<<<1, 32, 0, ctx->stream>>>(ctx->LDz.lu, ctx->LDz.piv, ctx->Ui, ctx->dm, g, ctx->dsc);
        }
        PF_LAUNCHED(ctx);
        PF_CUDA(cudaMemcpyAsync(ctx->hsc, ctx->dsc, sizeof(DevScalars), cudaMemcpyDeviceToHost, ctx->stream));
        PF_CUDA(cudaStreamSynchronize(ctx->stream));
        if (ctx->hsc->flux_d1 == 0.0) {
            pf_set_error("vel_adjustFlux: err 2");
            return PF_ERR_SINGULAR;
        }
    }
    // vel_adjPPE(0): unit wall-value solutions (velocity.f90:194-221)
    double2 *c1 = ctx->s[0].d, *c2 = ctx->s[1].d, *c3 = ctx->s[2].d, *c4 = ctx->s[3].d;
    const size_t wall = (size_t)(g.N - 1) * g.Hp;
    std::vector<double2> row(g.Hp);
    for (int j = 0; j < 4; ++j) {
        for (double2 *c : {c1, c2, c3, c4}) PF_TRY(pf_launch_ew(ctx, EW_ZERO, nullptr, nullptr, c, nullptr, 0.0));
        double2 v = make_double2(0.0, 0.0);
        if (j == 0 || j == 1) v.x = 1.0;
        if (j == 2) v.y = 1.0;
        if (j == 3) v.x = -1.0;
        for (int nh = 0; nh < g.Hp; ++nh) row[nh] = nh < g.H ? v : make_double2(0.0, 0.0);
        double2 *target = (j == 1) ? c2 : (j == 2) ? c3 : (j == 3) ? c4 : c1;
        PF_CUDA(cudaMemcpyAsync(target + wall, row.data(), g.Hp * sizeof(double2), cudaMemcpyHostToDevice,
                                ctx->stream));
        if (j == 0) PF_TRY(pf_launch_lu_solve(ctx, 0, &ctx->LDp, c1));
        if (j == 1) PF_TRY(pf_launch_lu_solve(ctx, 0, &ctx->LDm, c2));
        if (j == 2) PF_TRY(pf_launch_lu_solve(ctx, 0, &ctx->LDz, c3));
        if (j == 3) {
            PF_TRY(pf_launch_lu_solve(ctx, 1, &ctx->LNp, c4));
            PF_TRY(pf_launch_grad(ctx, c4, c1, c2, c3));
            PF_TRY(pf_launch_ew(ctx, EW_RT2PM, c1, c2, c1, c2, 0.0));
        }
        {
            ProfScope ps_(ctx, PF_K_FACTOR);
            k_ppe0_column<<<grid1(g.H, 64), 64, 0, ctx->stream>>>(j, c1, c2, c3, ctx->Ainv, ctx->U, ctx->dm, g);
        }
        PF_LAUNCHED(ctx);
        PF_CUDA(cudaStreamSynchronize(ctx->stream));  // `row` is reused
    }
    PF_CUDA(cudaMemsetAsync(&ctx->dsc->info, 0, sizeof(int), ctx->stream));
    {
        ProfScope ps_(ctx, PF_K_FACTOR);
        k_invert4<<<grid1(g.H, 64), 64, 0, ctx->stream>>>(ctx->Ainv, g.H, g.Hp, &ctx->dsc->info);
    }
    PF_LAUNCHED(ctx);
    int info = 0;
    PF_CUDA(cudaMemcpyAsync(&info, &ctx->dsc->info, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    PF_CUDA(cudaStreamSynchronize(ctx->stream));
    if (info != 0) {
        pf_set_error("matrix inversion error 1 (influence matrix of mode %d)", -info - 1);
        return PF_ERR_SINGULAR;
    }
    ctx->matrices_ready = true;
    ctx->matrices_gen++;
    return PF_OK;
}

// ------------------------------------------------------------------ C ABI
extern "C" int pf_tim_mesh_init(pf_ctx *ctx, int PM, double c1, double c2, pf_mesh **out) {
    PF_ARG(ctx && out && PM >= -1 && PM <= 1, "pf_tim_mesh_init: bad argument");
    *out = new pf_mesh{ctx, PM, c1, c2};
    return PF_OK;
}

extern "C" int pf_mesh_destroy(pf_mesh *A) {
    delete A;
    return PF_OK;
}

// host layout M[(nh*N + j)*(2KL+1) + row] == A(nh)%M(row+1, j+1)
extern "C" int pf_mesh_download(const pf_mesh *A, double *M) {
    PF_ARG(A && M, "null argument");
    const pf_ctx *ctx = A->ctx;
    const Geo &g = ctx->g;
    const int N = g.N;
    const HostMesh &hm = ctx->hm;
    for (int nh = 0; nh < g.H; ++nh) {
        int k, m;
        mode_km(nh, g.K, k, m);
        for (int j = 0; j < N; ++j)
            for (int row = 0; row < NBAND; ++row) {
                double v = A->c2 * hm.radLap[row * N + j];
                if (row == KL) {
                    const double r2 = hm.rp[1 * N + j];
                    double d = -(r2 * g.Mp * m * g.Mp * m) - g.alpha * k * g.alpha * k;
                    if (A->PM != 0) d = d - r2 - 2.0 * A->PM * g.Mp * m * r2;
                    v = v + A->c2 * d + A->c1;
                }
                M[((size_t)nh * N + j) * NBAND + row] = v;
            }
    }
    return PF_OK;
}

extern "C" int pf_tim_lumesh_init(pf_ctx *ctx, int PM, int BC, double c1, double c2, pf_lumesh **out) {
    PF_ARG(ctx && out && PM >= -1 && PM <= 1 && (BC == 0 || BC == 1), "pf_tim_lumesh_init: bad argument");
    *out = nullptr;
    pf_lumesh *A = new pf_lumesh();
    A->ctx = ctx;
    const Geo &g = ctx->g;
    int s = pf_alloc(ctx, (void **)&A->lu, (size_t)NLU * g.N * g.Hp * sizeof(double));
    if (s == PF_OK) s = pf_alloc(ctx, (void **)&A->piv, (size_t)g.N * g.Hp);
    if (s == PF_OK) s = lumesh_init(ctx, A, PM, BC, c1, c2);
    if (s != PF_OK) {
        pf_lumesh_destroy(A);
        return s;
    }
    *out = A;
    return PF_OK;
}

extern "C" int pf_lumesh_destroy(pf_lumesh *A) {
    if (!A) return PF_OK;
    pf_ctx *ctx = A->ctx;
    cudaStreamSynchronize(ctx->stream);
    for (void *p : {(void *)A->lu, (void *)A->piv}) {
        for (size_t i = 0; i < ctx->allocs.size(); ++i)
            if (ctx->allocs[i] == p) {
                cudaFree(p);
                ctx->allocs.erase(ctx->allocs.begin() + i);
                break;
            }
    }
    ctx->bytes -= (size_t)NLU * ctx->g.N * ctx->g.Hp * sizeof(double) + (size_t)ctx->g.N * ctx->g.Hp;
    delete A;
    return PF_OK;
}

// host layout M[(nh*N + j)*(3KL+1) + row] == A(nh)%M(row+1, j+1), ipiv 1-based
extern "C" int pf_lumesh_download(const pf_lumesh *A, double *M, int *ipiv) {
    PF_ARG(A && M && ipiv, "null argument");
    pf_ctx *ctx = A->ctx;
    const Geo &g = ctx->g;
    std::vector<double> lu((size_t)NLU * g.N * g.Hp);
    std::vector<unsigned char> pv((size_t)g.N * g.Hp);
    PF_CUDA(cudaMemcpyAsync(lu.data(), A->lu, lu.size() * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    PF_CUDA(cudaMemcpyAsync(pv.data(), A->piv, pv.size(), cudaMemcpyDeviceToHost, ctx->stream));
    PF_CUDA(cudaStreamSynchronize(ctx->stream));
    for (int nh = 0; nh < g.H; ++nh)
        for (int j = 0; j < g.N; ++j) {
            for (int row = 0; row < NLU; ++row)
                M[((size_t)nh * g.N + j) * NLU + row] = lu[((size_t)row * g.N + j) * g.Hp + nh];
            ipiv[(size_t)nh * g.N + j] = j + 1 + pv[(size_t)j * g.Hp + nh];
        }
    return PF_OK;
}

extern "C" int pf_tim_lumesh_invert(int BC, const pf_lumesh *A, pf_coll *b) {
    PF_ARG(A && b && A->ctx == b->ctx && (BC == 0 || BC == 1), "pf_tim_lumesh_invert: bad argument");
    return pf_launch_lu_solve(b->ctx, BC, A, b->d);
}

extern "C" int pf_vel_influence_download(const pf_ctx *ctx, double *U, double *A) {
    PF_ARG(ctx, "null ctx");
    PF_ARG(ctx->matrices_ready, "pf_vel_influence_download: call pf_vel_matrices first");
    const Geo &g = ctx->g;
    const int N = g.N;
    std::vector<double> u((size_t)6 * N * g.Hp), a((size_t)16 * g.Hp);
    PF_CUDA(cudaMemcpyAsync(u.data(), ctx->U, u.size() * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    PF_CUDA(cudaMemcpyAsync(a.data(), ctx->Ainv, a.size() * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    PF_CUDA(cudaStreamSynchronize(ctx->stream));
    if (U)
        for (int c = 0; c < 6; ++c)
            for (int nh = 0; nh < g.H; ++nh)
                for (int n = 0; n < N; ++n)
                    U[((size_t)c * g.H + nh) * N + n] = u[((size_t)c * N + n) * g.Hp + nh];
    if (A)
        for (int nh = 0; nh < g.H; ++nh)
            for (int i = 0; i < 4; ++i)
                for (int j = 0; j < 4; ++j) A[(size_t)nh * 16 + j * 4 + i] = a[(size_t)(i * 4 + j) * g.Hp + nh];
    return PF_OK;
}
