// Fused vel_step (velocity.f90:367-394) in four launches:
//   S1 k_step_rhs  : tile of 32 modes x all radial points: optional
//                    nlincorr (timestep.f90:174-184) or N_ := N copy,
//                    rhs = Lt u_ + N in the u+-/uz variables (velocity.f90:369-373,
//                    tim_meshmult with the per-mode band rebuilt in registers),
//                    then the PPE right-hand side div(pm2rt(rhs)) with zero
//                    boundary rows (velocity.f90:228-230)
//   S2 k_solve_pnp : pressure Poisson solve with LNp (pivoting band LU,
//                    BC=1, mean mode zeroed; timestep.f90:102-123)
//   S4 k_solve_ld  : the u+, u-, uz Helmholtz solves (LDp, LDm, LDz, which
//                    never pivot); the projection rhs - rt2pm(grad p) with
//                    zero boundary rows (velocity.f90:232-236, 376-378) is
//                    formed in the solve's load stage
//   S5 k_step_final: influence-matrix correction (velocity.f90:238-256),
//                    pm2rt, constant-flux adjustment for k=m=0
//                    (velocity.f90:170-175), mean-mode symmetry zeros, and the
//                    corrector error max |u_old - u_new|^2 (timestep.f90:190-207)
// Scratch: v (3 coll) holds rhs then the solutions, p (1 coll) the pressure.
// One thread per (mode, part) or (mode, system, part) runs each banded
// solve; the factor columns of the next two steps are loaded ahead.
#include <cmath>
#include "pf_internal.cuh"

static constexpr int TM = 32;  // modes per tile
static constexpr int TR = 8;   // radial row groups per tile

struct StepArgs {
    const double2 *u_[3];  // previous state (ur_, ut_, uz_)
    double2 *Nl[3];        // vel_N (read; rewritten by nlincorr)
    double2 *N_[3];        // saved N_ (read in the corrector, written in the predictor)
    double2 *v[3];         // scratch: rhs / solutions in u+, u-, uz
    double2 *p;            // scratch: pressure
    double2 *u[3];         // vel_u (read as u_old by the corrector, written)
    const double *lnp, *ldp, *ldm, *ldz;
    const unsigned char *pivp;
    const double *U, *Ainv, *Ui;
    DevMesh dm;
    Geo g;
    double c1, c2;         // Lt coefficients: 1/dt and (1-implicit) nu/Re
    double implicit;
    int mode;              // 0 predictor, 1 corrector
    int const_flux;
    DevScalars *sc;
};

__device__ __forceinline__ double lap_diag(const DevMesh &dm, const Geo &g, int PM, int n, int k, int m) {
    const double r2 = dm.rp[1 * g.N + n];
    double d = -(r2 * g.Mp * m * g.Mp * m) - g.alpha * k * g.alpha * k;
    if (PM != 0) d = d - r2 - 2.0 * PM * g.Mp * m * r2;
    return d;
}

// ------------------------------------------------------------------- S1
__global__ void __launch_bounds__(TM *TR) k_step_rhs(StepArgs a) {
    extern __shared__ double2 rsm[];  // [N][TM]: radial component of pm2rt(rhs)
    const Geo &g = a.g;
    const int N = g.N, Hp = g.Hp;
    const int tx = threadIdx.x % TM, ty = threadIdx.x / TM;
    const int nh = blockIdx.x * TM + tx;
    const bool live = nh < g.H;
    int k = 0, m = 0;
    if (live) mode_km(nh, g.K, k, m);
    const double c1 = a.c1, c2 = a.c2;
    constexpr int RMAX = 16;  // rows per thread (N <= TR*RMAX)
    double2 tkeep[RMAX], zkeep[RMAX];
    int rr = 0;
    for (int n = ty; n < N; n += TR, ++rr) {
        double2 vp = make_double2(0, 0), vm = vp, vz = vp;
        if (live) {
            const size_t at = (size_t)n * Hp + nh;
            double2 Nr = a.Nl[0][at], Nt = a.Nl[1][at], Nz = a.Nl[2][at];
            if (a.mode == 1) {  // N = c N + (1-c) N_
                const double d1 = a.implicit, d2 = 1.0 - a.implicit;
                const double2 Pr = a.N_[0][at], Pt = a.N_[1][at], Pz = a.N_[2][at];
                Nr = make_double2(d1 * Nr.x + d2 * Pr.x, d1 * Nr.y + d2 * Pr.y);
                Nt = make_double2(d1 * Nt.x + d2 * Pt.x, d1 * Nt.y + d2 * Pt.y);
                Nz = make_double2(d1 * Nz.x + d2 * Pz.x, d1 * Nz.y + d2 * Pz.y);
                a.Nl[0][at] = Nr;
                a.Nl[1][at] = Nt;
                a.Nl[2][at] = Nz;
            } else {  // N_ := N
                a.N_[0][at] = Nr;
                a.N_[1][at] = Nt;
                a.N_[2][at] = Nz;
            }
            // rhs = Lt u_ + N, accumulated from N in increasing column order
            vp = make_double2(Nr.x - Nt.y, Nr.y + Nt.x);
            vm = make_double2(Nr.x + Nt.y, Nr.y - Nt.x);
            vz = Nz;
            const int lo = max(0, n - KL), hi = min(N - 1, n + KL);
            for (int j = lo; j <= hi; ++j) {
                const size_t aj = (size_t)j * Hp + nh;
                const double2 r = a.u_[0][aj], t = a.u_[1][aj], z = a.u_[2][aj];
                const double off = c2 * a.dm.radLap[(KL + n - j) * N + j];
                double wp = off, wm = off, wz = off;
                if (j == n) {
                    wp = (off + c2 * lap_diag(a.dm, g, 1, j, k, m)) + c1;
                    wm = (off + c2 * lap_diag(a.dm, g, -1, j, k, m)) + c1;
                    wz = (off + c2 * lap_diag(a.dm, g, 0, j, k, m)) + c1;
                }
                vp.x = fma(wp, r.x - t.y, vp.x);
                vp.y = fma(wp, r.y + t.x, vp.y);
                vm.x = fma(wm, r.x + t.y, vm.x);
                vm.y = fma(wm, r.y - t.x, vm.y);
                vz.x = fma(wz, z.x, vz.x);
                vz.y = fma(wz, z.y, vz.y);
            }
            a.v[0][at] = vp;
            a.v[1][at] = vm;
            a.v[2][at] = vz;
        }
        // pm2rt (velocity.f90:98-114)
        rsm[n * TM + tx] = make_double2(0.5 * (vp.x + vm.x), 0.5 * (vp.y + vm.y));
        tkeep[rr] = make_double2(0.5 * (vp.y - vm.y), -0.5 * (vp.x - vm.x));
        zkeep[rr] = vz;
    }
    __syncthreads();
    if (!live) return;
    const double kal = g.alpha * k;
    rr = 0;
    for (int n = ty; n < N; n += TR, ++rr) {
        double2 dv = make_double2(0, 0);
        if (n != 0 && n != N - 1) {  // tim_zerobc
            const double rm1 = a.dm.rp[2 * N + n];
            const double m1r1 = rm1 * g.Mp * m;
            double2 dr = make_double2(0, 0);
            const int lo = max(0, n - KL), hi = min(N - 1, n + KL);
            for (int j = lo; j <= hi; ++j) {
                const double w = a.dm.dr[(KL + n - j) * N + j];
                const double2 x = rsm[j * TM + tx];
                dr.x = fma(w, x.x, dr.x);
                dr.y = fma(w, x.y, dr.y);
            }
            const double2 r = rsm[n * TM + tx], t = tkeep[rr], z = zkeep[rr];
            dv.x = r.x * rm1 + dr.x - t.y * m1r1 - z.y * kal;   // variables.f90:472-477
            dv.y = r.y * rm1 + dr.y + t.x * m1r1 + z.x * kal;
        }
        a.p[(size_t)n * Hp + nh] = dv;
    }
}

// --------------------------------------------------- banded solves (S2, S4)
// Forward sweep of dgbtrs with the next two factor columns in flight, then
// the dtbsv back substitution.  PIV selects the pivoting layout (U with
// KL+KU superdiagonals) or the pivot-free one (KU superdiagonals).
template <bool PIV, typename Rhs>
__device__ __forceinline__ void solve_chain(const double *__restrict__ lu, const unsigned char *__restrict__ piv,
                                            int N, int Hp, int nh, const Rhs &rhs, double *out, size_t ostride) {
    constexpr int KU = PIV ? KV : KL;
#define LUQ(row, col) lu[((size_t)(row) * N + (col)) * Hp + nh]
    double w[KL + 1];
#pragma unroll
    for (int i = 0; i <= KL; ++i) w[i] = rhs(i);
    double Lc[KL], Ln[KL];
    int pc = 0, pn = 0;
#pragma unroll
    for (int i = 0; i < KL; ++i) {
        Lc[i] = LUQ(KV + 1 + i, 0);
        Ln[i] = (N > 1) ? LUQ(KV + 1 + i, 1) : 0.0;
    }
    if (PIV) {
        pc = piv[nh];
        pn = (N > 1) ? piv[(size_t)Hp + nh] : 0;
    }
    for (int j = 0; j < N; ++j) {
        double Lf[KL];
        int pf = 0;
        const bool more = j + 2 < N - 1;
#pragma unroll
        for (int i = 0; i < KL; ++i) Lf[i] = more ? LUQ(KV + 1 + i, j + 2) : 0.0;
        if (PIV && more) pf = piv[(size_t)(j + 2) * Hp + nh];
        const double ahead = (j + KL + 1 < N) ? rhs(j + KL + 1) : 0.0;
        if (j < N - 1) {
            if (PIV) {
#pragma unroll
                for (int i = 1; i <= KL; ++i)
                    if (pc == i) {
                        const double t = w[0];
                        w[0] = w[i];
                        w[i] = t;
                    }
            }
            const double bj = w[0];
#pragma unroll
            for (int i = 1; i <= KL; ++i)
                if (j + i < N) w[i] = fma(-Lc[i - 1], bj, w[i]);
        }
        out[(size_t)j * ostride] = w[0];
#pragma unroll
        for (int i = 0; i < KL; ++i) w[i] = w[i + 1];
        w[KL] = ahead;
#pragma unroll
        for (int i = 0; i < KL; ++i) {
            Lc[i] = Ln[i];
            Ln[i] = Lf[i];
        }
        pc = pn;
        pn = pf;
    }
    // back substitution (dtbsv 'U','N','N' with K = KU superdiagonals)
    double v[KU + 1];
#pragma unroll
    for (int i = 0; i <= KU; ++i) v[i] = (N - 1 - i >= 0) ? out[(size_t)(N - 1 - i) * ostride] : 0.0;
    double Uc[KU + 1], Un[KU + 1];
#pragma unroll
    for (int i = 0; i <= KU; ++i) {
        Uc[i] = LUQ(KV - i, N - 1);
        Un[i] = (N > 1) ? LUQ(KV - i, N - 2) : 0.0;
    }
    for (int j = N - 1; j >= 0; --j) {
        double Uf[KU + 1];
#pragma unroll
        for (int i = 0; i <= KU; ++i) Uf[i] = (j - 2 >= 0) ? LUQ(KV - i, j - 2) : 0.0;
        const double ahead = (j - KU - 1 >= 0) ? out[(size_t)(j - KU - 1) * ostride] : 0.0;
        double x = v[0];
        if (x != 0.0) {
            x = x / Uc[0];
#pragma unroll
            for (int i = 1; i <= KU; ++i)
                if (j - i >= 0) v[i] = fma(-x, Uc[i], v[i]);
        }
        out[(size_t)j * ostride] = x;
#pragma unroll
        for (int i = 0; i < KU; ++i) v[i] = v[i + 1];
        v[KU] = ahead;
#pragma unroll
        for (int i = 0; i <= KU; ++i) {
            Uc[i] = Un[i];
            Un[i] = Uf[i];
        }
    }
#undef LUQ
}

struct RhsPlain {
    const double *b;
    size_t stride;
    __device__ __forceinline__ double operator()(int n) const { return b[(size_t)n * stride]; }
};

// S2: thread = (mode, re/im)
__global__ void k_solve_pnp(StepArgs a) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int nh = t >> 1, part = t & 1;
    const Geo &g = a.g;
    if (nh >= g.H) return;
    double *bp = reinterpret_cast<double *>(a.p) + 2 * (size_t)nh + part;
    const size_t stride = 2 * (size_t)g.Hp;
    if (nh == 0) {  // BC=1 at k=m=0: zero (timestep.f90:110-113)
        for (int n = 0; n < g.N; ++n) bp[n * stride] = 0.0;
        return;
    }
    solve_chain<true>(a.lnp, a.pivp, g.N, g.Hp, nh, RhsPlain{bp, stride}, bp, stride);
}

// S4 rhs: v - rt2pm(grad p) (or v_z - i alpha k p), zero at n=0 and n=N-1
struct RhsProj {
    const double2 *v, *p;
    const double *dr, *rm1;
    int N, Hp, nh, sys, part;
    double m1, kal;  // m*Mp, alpha*k
    __device__ __forceinline__ double operator()(int n) const {
        if (n == 0 || n == N - 1) return 0.0;
        const size_t at = (size_t)n * Hp + nh;
        const double2 pv = p[at];
        const double2 vv = v[at];
        if (sys == 2) {  // uz: g = (-alpha k p.im, alpha k p.re)
            return part == 0 ? vv.x - (-pv.y * kal) : vv.y - (pv.x * kal);
        }
        double2 dr2 = make_double2(0, 0);
        const int lo = max(0, n - KL), hi = min(N - 1, n + KL);
        for (int j = lo; j <= hi; ++j) {
            const double w = dr[(KL + n - j) * N + j];
            const double2 x = p[(size_t)j * Hp + nh];
            dr2.x = fma(w, x.x, dr2.x);
            dr2.y = fma(w, x.y, dr2.y);
        }
        const double m1r1 = rm1[n] * m1;
        // grad: r = dr p, t = (-p.im m/r, p.re m/r); rt2pm(r, t)
        const double tRe = -pv.y * m1r1, tIm = pv.x * m1r1;
        if (sys == 0) return part == 0 ? vv.x - (dr2.x - tIm) : vv.y - (dr2.y + tRe);
        return part == 0 ? vv.x - (dr2.x + tIm) : vv.y - (dr2.y - tRe);
    }
};

// S4: warp = one (system, re/im) for 32 consecutive modes, so factor loads
// are contiguous across the warp; LD factors are pivot-free
__global__ void __launch_bounds__(192) k_solve_ld(StepArgs a) {
    const Geo &g = a.g;
    const int w = threadIdx.x >> 5;
    const int nh = blockIdx.x * 32 + (threadIdx.x & 31);
    const int sys = w >> 1, part = w & 1;
    if (nh >= g.H) return;
    int k, m;
    mode_km(nh, g.K, k, m);
    RhsProj rhs{a.v[sys], a.p, a.dm.dr, a.dm.rp + 2 * g.N, g.N, g.Hp, nh, sys, part,
                (double)(m * g.Mp), g.alpha * k};
    double *out = reinterpret_cast<double *>(a.v[sys]) + 2 * (size_t)nh + part;
    const double *lu = sys == 0 ? a.ldp : sys == 1 ? a.ldm : a.ldz;
    solve_chain<false>(lu, nullptr, g.N, g.Hp, nh, rhs, out, 2 * (size_t)g.Hp);
}

// ------------------------------------------------------------------- S5
__device__ __forceinline__ double sq(double2 a) { return a.x * a.x + a.y * a.y; }

__global__ void __launch_bounds__(TM *TR) k_step_final(StepArgs a) {
    __shared__ double coef[TM][8];        // aR(1..4), aI(1..4) per mode
    __shared__ double red[TM * TR];
    __shared__ double m0buf[3][2][128];    // mode 0 after pm2rt (N <= 128)
    const Geo &g = a.g;
    const int N = g.N, Hp = g.Hp;
    const int tx = threadIdx.x % TM, ty = threadIdx.x / TM;
    const int nh = blockIdx.x * TM + tx;
    const bool live = nh < g.H;
    int k = 0, m = 0;
    if (live) mode_km(nh, g.K, k, m);
    if (ty == 0 && live) {
        double aR[4] = {0, 0, 0, 0}, aI[4] = {0, 0, 0, 0};
        if (nh != 0) {  // vel_evalBC + a = -A^-1 B (velocity.f90:239-243, 262-298)
            const size_t at = (size_t)(N - 1) * Hp + nh;
            const double2 pw = a.v[0][at], qw = a.v[1][at], zw = a.v[2][at];
            const double urRe = 0.5 * (pw.x + qw.x), urIm = 0.5 * (pw.y + qw.y);
            const double utRe = 0.5 * (pw.y - qw.y), utIm = -0.5 * (pw.x - qw.x);
            double drRe = 0.0, drIm = 0.0;
            for (int j = 0; j <= KL; ++j) {
                const size_t aj = (size_t)(N - 1 - KL + j) * Hp + nh;
                const double w = a.dm.dr1[1 * (KL + 1) + j];
                const double2 x = a.v[0][aj], y = a.v[1][aj];
                drRe += w * (x.x + y.x);
                drIm += w * (x.y + y.y);
            }
            drRe = 0.5 * drRe;
            drIm = 0.5 * drIm;
            const double d = a.dm.rp[2 * N + (N - 1)];
            const double m_ = (double)(m * g.Mp), a_ = g.alpha * k;
            const double BRe[4] = {pw.x, qw.x, -zw.y, urRe * d + drRe - d * m_ * utIm - a_ * zw.y};
            const double BIm[4] = {pw.y, qw.y, zw.x, urIm * d + drIm + d * m_ * utRe + a_ * zw.x};
            for (int i = 0; i < 4; ++i) {
                double sr = 0.0, si = 0.0;
                for (int j = 0; j < 4; ++j) {
                    const double A = a.Ainv[(size_t)(i * 4 + j) * Hp + nh];
                    sr += A * BRe[j];
                    si += A * BIm[j];
                }
                aR[i] = -sr;
                aI[i] = -si;
            }
        }
        for (int i = 0; i < 4; ++i) {
            coef[tx][i] = aR[i];
            coef[tx][4 + i] = aI[i];
        }
    }
    __syncthreads();
    double err = 0.0;
    if (live) {
        const double *cf = coef[tx];
        for (int n = ty; n < N; n += TR) {
            const size_t at = (size_t)n * Hp + nh;
            double2 r = a.v[0][at], t = a.v[1][at], z = a.v[2][at];
            if (nh != 0) {
                const double U1 = a.U[(size_t)(0 * N + n) * Hp + nh], U2 = a.U[(size_t)(1 * N + n) * Hp + nh];
                const double U3 = a.U[(size_t)(2 * N + n) * Hp + nh], U4 = a.U[(size_t)(3 * N + n) * Hp + nh];
                const double U5 = a.U[(size_t)(4 * N + n) * Hp + nh], U6 = a.U[(size_t)(5 * N + n) * Hp + nh];
                r.x = r.x + cf[0] * U1; r.y = r.y + cf[4] * U1;
                t.x = t.x + cf[1] * U2; t.y = t.y + cf[5] * U2;
                z.x = z.x - cf[6] * U3; z.y = z.y + cf[2] * U3;
                r.x = r.x + cf[3] * U4; r.y = r.y + cf[7] * U4;
                t.x = t.x + cf[3] * U5; t.y = t.y + cf[7] * U5;
                z.x = z.x - cf[7] * U6; z.y = z.y + cf[3] * U6;
            }
            // pm2rt
            const double2 ur = make_double2(0.5 * (r.x + t.x), 0.5 * (r.y + t.y));
            const double2 ut = make_double2(0.5 * (r.y - t.y), -0.5 * (r.x - t.x));
            if (nh == 0) {
                m0buf[0][0][n] = ur.x; m0buf[0][1][n] = ur.y;
                m0buf[1][0][n] = ut.x; m0buf[1][1][n] = ut.y;
                m0buf[2][0][n] = z.x;  m0buf[2][1][n] = z.y;
                continue;
            }
            if (a.mode == 1) {
                const double2 o0 = a.u[0][at], o1 = a.u[1][at], o2 = a.u[2][at];
                err = fmax(err, sq(make_double2(o0.x - ur.x, o0.y - ur.y)));
                err = fmax(err, sq(make_double2(o1.x - ut.x, o1.y - ut.y)));
                err = fmax(err, sq(make_double2(o2.x - z.x, o2.y - z.y)));
            }
            a.u[0][at] = ur;
            a.u[1][at] = ut;
            a.u[2][at] = z;
        }
    }
    if (blockIdx.x == 0) {  // mode 0: flux adjustment and symmetry zeros
        __syncthreads();
        double s = 0.0;
        for (int n = threadIdx.x; n < N; n += blockDim.x) s += m0buf[2][0][n] * a.dm.intrdr[n];
        red[threadIdx.x] = s;
        __syncthreads();
        if (threadIdx.x == 0) {
            double tsum = 0.0;
            for (int i = 0; i < (int)blockDim.x; ++i) tsum += red[i];
            red[0] = tsum;
        }
        __syncthreads();
        double d3 = 0.0;
        if (a.const_flux) d3 = -(2.0 * red[0]) / a.sc->flux_d1;
        for (int n = threadIdx.x; n < N; n += blockDim.x) {
            const size_t at = (size_t)n * Hp;
            const double2 ur = make_double2(0.0, 0.0);
            const double2 ut = make_double2(m0buf[1][0][n], 0.0);
            double zr = m0buf[2][0][n];
            if (a.const_flux) zr = zr + d3 * a.Ui[n];
            const double2 uz = make_double2(zr, 0.0);
            if (a.mode == 1) {
                const double2 o0 = a.u[0][at], o1 = a.u[1][at], o2 = a.u[2][at];
                err = fmax(err, sq(make_double2(o0.x - ur.x, o0.y - ur.y)));
                err = fmax(err, sq(make_double2(o1.x - ut.x, o1.y - ut.y)));
                err = fmax(err, sq(make_double2(o2.x - uz.x, o2.y - uz.y)));
            }
            a.u[0][at] = ur;
            a.u[1][at] = ut;
            a.u[2][at] = uz;
        }
        if (threadIdx.x == 0 && a.const_flux) a.sc->Pr0 = a.sc->Pr0 + d3 * g.Re / 4.0;
    }
    if (a.mode == 1) {
        for (int o = 16; o > 0; o >>= 1) err = fmax(err, __shfl_xor_sync(0xffffffffu, err, o));
        if ((threadIdx.x & 31) == 0)
            atomicMax(&a.sc->dterr2_bits, (unsigned long long)__double_as_longlong(err));
    }
}

// ------------------------------------------------------------------ host
// One predictor (corrector=0) or corrector (corrector=1) vel_step.  The
// predictor's u_ := u copy is a pointer swap of vel[0..2] and prev[0..2].
int pf_vel_step_fused(pf_ctx *ctx, int corrector) {
    const Geo &g = ctx->g;
    if (g.N > TR * 16 || g.N > 128) {
        pf_set_error("fused step supports N <= 128");
        return PF_ERR_ARG;
    }
    if (ctx->LDp.pivoted || ctx->LDm.pivoted || ctx->LDz.pivoted) {
        pf_set_error("fused step: Helmholtz factors pivoted");
        return PF_ERR_STATE;
    }
    if (!corrector)
        for (int i = 0; i < 3; ++i) std::swap(ctx->vel[i].d, ctx->prev[i].d);
    StepArgs a;
    for (int i = 0; i < 3; ++i) {
        a.u_[i] = ctx->prev[i].d;
        a.Nl[i] = ctx->vel[3 + i].d;
        a.N_[i] = ctx->prev[3 + i].d;
        a.v[i] = ctx->s[i].d;
        a.u[i] = ctx->vel[i].d;
    }
    a.p = ctx->s[3].d;
    a.lnp = ctx->LNp.lu;
    a.pivp = ctx->LNp.piv;
    a.ldp = ctx->LDp.lu;
    a.ldm = ctx->LDm.lu;
    a.ldz = ctx->LDz.lu;
    a.U = ctx->U;
    a.Ainv = ctx->Ainv;
    a.Ui = ctx->Ui;
    a.dm = ctx->dm;
    a.g = g;
    a.c1 = ctx->Ltz.c1;
    a.c2 = ctx->Ltz.c2;
    a.implicit = ctx->cfg.implicit;
    a.mode = corrector;
    a.const_flux = ctx->cfg.const_flux;
    a.sc = ctx->dsc;
    const unsigned tiles = grid1(g.H, TM);
    {
        ProfScope ps_(ctx, PF_K_STEP);
        k_step_rhs<<<tiles, TM * TR, (size_t)g.N * TM * sizeof(double2), ctx->stream>>>(a);
    }
    PF_LAUNCHED(ctx);
    {
        ProfScope ps_(ctx, PF_K_LUSOLVE);
        k_solve_pnp<<<grid1(2LL * g.H, 128), 128, 0, ctx->stream>>>(a);
    }
    PF_LAUNCHED(ctx);
    {
        ProfScope ps_(ctx, PF_K_LUSOLVE);
        k_solve_ld<<<grid1(g.H, 32), 192, 0, ctx->stream>>>(a);
    }
    PF_LAUNCHED(ctx);
    if (corrector) PF_CUDA(cudaMemsetAsync(&ctx->dsc->dterr2_bits, 0, sizeof(unsigned long long), ctx->stream));
    {
        ProfScope ps_(ctx, PF_K_INFL);
        k_step_final<<<tiles, TM * TR, 0, ctx->stream>>>(a);
    }
    PF_LAUNCHED(ctx);
    return PF_OK;
}
