// Fused vel_step (velocity.f90:367-394) in five launches:
//   S1 k_step_rhs  : tile of 16 modes x all radial points: optional
//                    nlincorr (timestep.f90:174-184) or N_ := N copy,
//                    rhs = Lt u_ + N in the u+-/uz variables (velocity.f90:369-373,
//                    tim_meshmult with the per-mode band rebuilt in registers),
//                    then the PPE right-hand side div(pm2rt(rhs)) with zero
//                    boundary rows (velocity.f90:228-230)
//   S2 k_solve_pnpw: pressure Poisson solve with LNp (pivoting band LU,
//                    BC=1, mean mode zeroed; timestep.f90:102-123), the
//                    factor ring of a mode shared by its re and im lanes
//   S3 k_step_proj : the projection rhs - rt2pm(grad p) with zero boundary
//                    rows (velocity.f90:232-236, 376-378)
//   S4 k_solve_ld  : the u+, u-, uz Helmholtz solves (LDp, LDm, LDz; the
//                    pivot-free sweep unless that factorisation pivoted)
//   S5 k_step_final: influence-matrix correction (velocity.f90:238-256),
//                    pm2rt, constant-flux adjustment for k=m=0
//                    (velocity.f90:170-175), mean-mode symmetry zeros, and the
//                    corrector error max |u_old - u_new|^2 (timestep.f90:190-207)
// Scratch: v (3 coll) holds rhs then the solutions, prhs/p the pressure
// right-hand side and solution, rl (3 coll) the Helmholtz right-hand sides.
#include <cmath>
#include "pf_internal.cuh"

static constexpr int TM = 32;  // modes per tile
static constexpr int TR = 8;   // radial row groups per tile

struct StepArgs {
    const double2 *u_[3];  // previous state (ur_, ut_, uz_)
    double2 *Nl[3];        // vel_N (read; rewritten by nlincorr)
    double2 *N_[3];        // saved N_ (read in the corrector, written in the predictor)
    double2 *v[3];         // scratch: rhs / solutions in u+, u-, uz
    double2 *prhs;         // scratch: pressure right-hand side
    double2 *p;            // scratch: pressure
    double2 *rl[3];        // scratch: Helmholtz right-hand sides
    double2 *u[3];         // vel_u (read as u_old by the corrector, written)
    const double *lnp, *ldp, *ldm, *ldz;
    const double *pivd;    // LNp pivots as doubles [col*Hp + nh]
    const double *pivld[3];  // LDp/LDm/LDz pivots as doubles
    int ldpiv[3];          // 1 if that Helmholtz factorisation pivoted
    // compact copies (modes k >= 0, c = m*K + |k|, stride Hcp) the streamed
    // pressure and Helmholtz solves read: LNp, LDp, LDm, LDz and their pivots
    const double *lnpc, *ldc[3];
    const double *pivdc, *pivldc[3];
    int Hcp;
    double ldc1, ldc2;     // Helmholtz coefficients (LDp/LDm/LDz: 1/dt, -implicit nu/Re)
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
// Block = 16 modes x 16 radial row groups; each thread owns RPT rows
// n = ty + 16 r (RPT = 4 for N <= 64, 8 for N <= 128), so the values it
// keeps between the two phases stay in registers.  Pointers are held as
// __restrict__ locals so loads of later rows can be issued before the stores
// of earlier ones.
static constexpr int HM = 16;  // modes per S1 block
static constexpr int HR = 16;  // row groups per S1 block

template <int RPT>
__device__ __forceinline__ void step_rhs_body(const StepArgs &a, int hb) {
    extern __shared__ double2 rsm[];  // [N][HM]: radial component of pm2rt(rhs)
    const Geo &g = a.g;
    const int N = g.N;
    const size_t Hp = g.Hp;
    const int tx = threadIdx.x % HM, ty = threadIdx.x / HM;
    const int nh = hb * HM + tx;
    // the corrector's error max (timestep.f90:190-207) restarts here; S5
    // accumulates it after every block of this launch has finished
    if (a.mode == 1 && hb == 0 && threadIdx.x == 0) a.sc->dterr2_bits = 0ull;
    const bool live = nh < g.H;
    const int nhc = live ? nh : 0;
    int k = 0, m = 0;
    if (live) mode_km(nh, g.K, k, m);
    const double c1 = a.c1, c2 = a.c2;
    const double2 *__restrict__ ur_ = a.u_[0] + nhc;
    const double2 *__restrict__ ut_ = a.u_[1] + nhc;
    const double2 *__restrict__ uz_ = a.u_[2] + nhc;
    double2 *__restrict__ N0 = a.Nl[0] + nhc;
    double2 *__restrict__ N1 = a.Nl[1] + nhc;
    double2 *__restrict__ N2 = a.Nl[2] + nhc;
    double2 *__restrict__ P0 = a.N_[0] + nhc;
    double2 *__restrict__ P1 = a.N_[1] + nhc;
    double2 *__restrict__ P2 = a.N_[2] + nhc;
    double2 *__restrict__ v0 = a.v[0] + nhc;
    double2 *__restrict__ v1 = a.v[1] + nhc;
    double2 *__restrict__ v2 = a.v[2] + nhc;
    double2 *__restrict__ prhs = a.prhs + nhc;
    const double *__restrict__ radLap = a.dm.radLap;
    const double *__restrict__ drb = a.dm.dr;
    const double *__restrict__ rp = a.dm.rp;
    double2 tkeep[RPT], zkeep[RPT];
#pragma unroll
    for (int r = 0; r < RPT; ++r) {
        const int n = ty + HR * r;
        double2 vp = make_double2(0, 0), vm = vp, vz = vp;
        if (live && n < N) {
            const size_t at = (size_t)n * Hp;
            // read once (and in the corrector overwritten): stream past L1
            double2 Nr = __ldcs(N0 + at), Nt = __ldcs(N1 + at), Nz = __ldcs(N2 + at);
            if (a.mode == 1) {  // N = c N + (1-c) N_
                const double d1 = a.implicit, d2 = 1.0 - a.implicit;
                const double2 Pr = __ldcs(P0 + at), Pt = __ldcs(P1 + at), Pz = __ldcs(P2 + at);
                Nr = make_double2(d1 * Nr.x + d2 * Pr.x, d1 * Nr.y + d2 * Pr.y);
                Nt = make_double2(d1 * Nt.x + d2 * Pt.x, d1 * Nt.y + d2 * Pt.y);
                Nz = make_double2(d1 * Nz.x + d2 * Pz.x, d1 * Nz.y + d2 * Pz.y);
                N0[at] = Nr;
                N1[at] = Nt;
                N2[at] = Nz;
            } else {  // N_ := N
                P0[at] = Nr;
                P1[at] = Nt;
                P2[at] = Nz;
            }
            // rhs = Lt u_ + N, accumulated from N in increasing column order
            vp = make_double2(Nr.x - Nt.y, Nr.y + Nt.x);
            vm = make_double2(Nr.x + Nt.y, Nr.y - Nt.x);
            vz = Nz;
            const int lo = max(0, n - KL), hi = min(N - 1, n + KL);
            for (int j = lo; j <= hi; ++j) {
                const size_t aj = (size_t)j * Hp;
                const double2 rr = ur_[aj], t = ut_[aj], z = uz_[aj];
                const double off = c2 * radLap[(KL + n - j) * N + j];
                double wp = off, wm = off, wz = off;
                if (j == n) {
                    wp = (off + c2 * lap_diag(a.dm, g, 1, j, k, m)) + c1;
                    wm = (off + c2 * lap_diag(a.dm, g, -1, j, k, m)) + c1;
                    wz = (off + c2 * lap_diag(a.dm, g, 0, j, k, m)) + c1;
                }
                vp.x = fma(wp, rr.x - t.y, vp.x);
                vp.y = fma(wp, rr.y + t.x, vp.y);
                vm.x = fma(wm, rr.x + t.y, vm.x);
                vm.y = fma(wm, rr.y - t.x, vm.y);
                vz.x = fma(wz, z.x, vz.x);
                vz.y = fma(wz, z.y, vz.y);
            }
            v0[at] = vp;
            v1[at] = vm;
            v2[at] = vz;
        }
        // pm2rt (velocity.f90:98-114)
        if (n < N) rsm[n * HM + tx] = make_double2(0.5 * (vp.x + vm.x), 0.5 * (vp.y + vm.y));
        tkeep[r] = make_double2(0.5 * (vp.y - vm.y), -0.5 * (vp.x - vm.x));
        zkeep[r] = vz;
    }
    __syncthreads();
    if (!live) return;
    const double kal = g.alpha * k;
#pragma unroll
    for (int r = 0; r < RPT; ++r) {
        const int n = ty + HR * r;
        if (n >= N) break;
        double2 dv = make_double2(0, 0);
        if (n != 0 && n != N - 1) {  // tim_zerobc
            const double rm1 = rp[2 * N + n];
            const double m1r1 = rm1 * g.Mp * m;
            double2 dr = make_double2(0, 0);
            const int lo = max(0, n - KL), hi = min(N - 1, n + KL);
            for (int j = lo; j <= hi; ++j) {
                const double w = drb[(KL + n - j) * N + j];
                const double2 x = rsm[j * HM + tx];
                dr.x = fma(w, x.x, dr.x);
                dr.y = fma(w, x.y, dr.y);
            }
            const double2 rr = rsm[n * HM + tx], t = tkeep[r], z = zkeep[r];
            dv.x = rr.x * rm1 + dr.x - t.y * m1r1 - z.y * kal;  // variables.f90:472-477
            dv.y = rr.y * rm1 + dr.y + t.x * m1r1 + z.x * kal;
        }
        prhs[(size_t)n * Hp] = dv;
    }
}

// --------------------------------------------------- banded solves (S2, S4)
// One thread per (mode, system, re/im) chain.  The factor values of a
// column and the right-hand side entering the elimination window are staged
// D columns ahead into a per-thread shared-memory ring with cp.async (8-byte
// copies, one commit group per column), so each step of the sequential
// sweep reads shared memory instead of waiting on DRAM.  The ring is laid out
// [slot][value][thread] so consecutive threads hit consecutive banks.  Six
// columns ahead, with the register budgets the launch bounds below set (four
// Helmholtz blocks and eight pressure blocks per SM), measured fastest: deeper
// rings or register queues cost more in resident warps than they hide.
static constexpr int RING = 6;

__device__ __forceinline__ void cp_async8(double *smem, const double *gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N> __device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

__device__ __forceinline__ void cp_async8s(unsigned saddr, const double *gmem) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(saddr), "l"(gmem) : "memory");
}

// dgbtrs ('N', one right-hand side) followed by dtbsv: rhs(n) = rhs[n*rs],
// solution to out[n*os] (out must not alias rhs).  PIV: LAPACK band with
// KL+KU superdiagonals in U and pivots pivd[col*Hp+nh] (as doubles); else
// the pivot-free band with KU = KL.  The ring is strided by the block's TS
// threads; the column loop is unrolled by RING so every ring slot is a
// constant shared-memory offset, and the global addresses step by one
// column per iteration instead of being recomputed.
template <bool PIV, int TS>
__device__ __forceinline__ void solve_async(const double *__restrict__ lu, const double *__restrict__ pivd, int N,
                                            int Hp, int nh, const double *__restrict__ rhs, size_t rs, double *out,
                                            size_t os, double *ring) {
    constexpr int KU = PIV ? KV : KL;
    constexpr int SWF = KL + 1 + (PIV ? 1 : 0);  // forward slot: L column, rhs ahead, pivot
    constexpr int SWB = KU + 1;                  // backward slot: U column
    constexpr int SW = SWF > SWB ? SWF : SWB;
    constexpr unsigned QB = 8u * TS, SB = 8u * TS * SW;  // bytes between values / slots
    const size_t rowst = (size_t)N * Hp;                 // doubles between band rows
    const unsigned sbase = (unsigned)__cvta_generic_to_shared(ring);
#define RSLOT(s, q) ring[((s) * SW + (q)) * TS]
    // forward: column j needs L(KV+1+i, j), i < KL, rhs(j+KL+1) and its pivot
    const double *Lj = lu + (size_t)(KV + 1) * rowst + nh;
    const double *Pj = PIV ? pivd + nh : nullptr;
    const double *Rj = rhs + (size_t)(KL + 1) * rs;
    int jj = 0;  // next column to stage
    auto issue_fwd = [&](int s) {
        if (jj < N) {
            if (jj < N - 1) {
#pragma unroll
                for (int i = 0; i < KL; ++i) cp_async8s(sbase + s * SB + i * QB, Lj + i * rowst);
                if (PIV) cp_async8s(sbase + s * SB + (KL + 1) * QB, Pj);
            }
            if (jj + KL + 1 < N) cp_async8s(sbase + s * SB + KL * QB, Rj);
        }
        cp_async_commit();
        ++jj;
        Lj += Hp;
        if (PIV) Pj += Hp;
        Rj += rs;
    };
    double w[KL + 1];
#pragma unroll
    for (int i = 0; i <= KL; ++i) w[i] = (i < N) ? rhs[(size_t)i * rs] : 0.0;
#pragma unroll
    for (int s = 0; s < RING; ++s) issue_fwd(s);
    double *Oj = out;
    for (int j0 = 0; j0 < N; j0 += RING) {
#pragma unroll
        for (int s = 0; s < RING; ++s) {
            const int j = j0 + s;
            if (j < N) {
                cp_async_wait<RING - 1>();
                const double ahead = (j + KL + 1 < N) ? RSLOT(s, KL) : 0.0;
                if (j < N - 1) {
                    if (PIV) {
                        const int p = (int)RSLOT(s, KL + 1);
#pragma unroll
                        for (int i = 1; i <= KL; ++i)
                            if (p == i) {
                                const double t = w[0];
                                w[0] = w[i];
                                w[i] = t;
                            }
                    }
                    const double bj = w[0];
#pragma unroll
                    for (int i = 1; i <= KL; ++i)
                        if (j + i < N) w[i] = fma(-RSLOT(s, i - 1), bj, w[i]);
                }
                *Oj = w[0];
                Oj += os;
#pragma unroll
                for (int i = 0; i < KL; ++i) w[i] = w[i + 1];
                w[KL] = ahead;
                issue_fwd(s);
            }
        }
    }
    cp_async_wait<0>();
    // back substitution: column j needs U(KV-i, j), i <= KU; y (this thread's
    // forward output) is read through a four-deep register queue, with
    // streaming loads: each value is read once and then overwritten
    const double *Uj = lu + (size_t)KV * rowst + (size_t)(N - 1) * Hp + nh;
    int tt = 0;  // next step to stage (step t handles column N-1-t)
    auto issue_bwd = [&](int s) {
        if (tt < N) {
#pragma unroll
            for (int i = 0; i <= KU; ++i) cp_async8s(sbase + s * SB + i * QB, Uj - i * rowst);
        }
        cp_async_commit();
        ++tt;
        Uj -= Hp;
    };
#pragma unroll
    for (int s = 0; s < RING; ++s) issue_bwd(s);
    double v[KU + 1];
#pragma unroll
    for (int i = 0; i <= KU; ++i) v[i] = (N - 1 - i >= 0) ? __ldcs(out + (size_t)(N - 1 - i) * os) : 0.0;
    constexpr int QY = 4;
    double yq[QY];
#pragma unroll
    for (int q = 0; q < QY; ++q) {
        const int r = N - 1 - KU - 1 - q;
        yq[q] = (r >= 0) ? __ldcs(out + (size_t)r * os) : 0.0;
    }
    double *Xj = out + (size_t)(N - 1) * os;
    for (int t0 = 0; t0 < N; t0 += RING) {
#pragma unroll
        for (int s = 0; s < RING; ++s) {
            const int t = t0 + s;
            if (t < N) {
                const int j = N - 1 - t;
                cp_async_wait<RING - 1>();
                const double ahead = yq[0];
#pragma unroll
                for (int q = 0; q < QY - 1; ++q) yq[q] = yq[q + 1];
                {
                    const int r = j - KU - 1 - QY;
                    yq[QY - 1] = (r >= 0) ? __ldcs(out + (size_t)r * os) : 0.0;
                }
                double x = v[0];
                if (x != 0.0) {
                    x = x / RSLOT(s, 0);
#pragma unroll
                    for (int i = 1; i <= KU; ++i)
                        if (j - i >= 0) v[i] = fma(-x, RSLOT(s, i), v[i]);
                }
                *Xj = x;
                Xj -= os;
#pragma unroll
                for (int i = 0; i < KU; ++i) v[i] = v[i + 1];
                v[KU] = (j - KU - 1 >= 0) ? ahead : 0.0;
                issue_bwd(s);
            }
        }
    }
    cp_async_wait<0>();
#undef RSLOT
}

// The same solve with the factor ring of a mode shared by its real and
// imaginary chains, which sit in one warp: lanes 0-15 are the real parts of
// 16 modes, lanes 16-31 their imaginary parts.  Each factor value of a
// column is copied once (the two lanes of a mode split the values), both
// read it from shared memory after a __syncwarp; each lane stages its own
// right-hand-side value.  A slot is refilled only after the next
// __syncwarp, once both lanes have read it, so RING-1 columns are in
// flight.  Every arithmetic operation is solve_async's, so the solutions are
// bitwise the same.  `mask` holds the lanes that run (a mode's two lanes are
// both in it or both out); all of them take the same number of steps.
// Warp ring: RING slots of [FV values][16 modes] + [32 lanes] doubles.
template <bool PIV> __host__ __device__ constexpr int rw_fv() {
    return (KL + (PIV ? 1 : 0)) > ((PIV ? KV : KL) + 1) ? (KL + (PIV ? 1 : 0)) : ((PIV ? KV : KL) + 1);
}
template <bool PIV> __host__ __device__ constexpr int rw_slot() { return rw_fv<PIV>() * 16 + 32; }

template <bool PIV>
__device__ __forceinline__ void solve_async_rw(const double *__restrict__ lu, const double *__restrict__ pivd, int N,
                                               int Hp, int nh, const double *__restrict__ rhs, size_t rs, double *out,
                                               size_t os, double *wring, unsigned mask) {
    constexpr int KU = PIV ? KV : KL;
    constexpr int FQ = KL + (PIV ? 1 : 0);  // forward values: L(KV+1+i, j), i < KL, then the pivot
    constexpr int BQ = KU + 1;              // backward values: U(KV-i, j), i <= KU
    constexpr int SLOT = rw_slot<PIV>(), RQ = rw_fv<PIV>() * 16;
    const int lane = threadIdx.x & 31, ml = lane & 15, part = lane >> 4;
    const size_t rowst = (size_t)N * Hp;
    const unsigned sbase = (unsigned)__cvta_generic_to_shared(wring);
#define WSLOT(s, q) wring[(s) * SLOT + (q) * 16 + ml]
#define WRHS(s) wring[(s) * SLOT + RQ + lane]
    const double *Lj = lu + (size_t)(KV + 1) * rowst + nh;
    const double *Pj = PIV ? pivd + nh : nullptr;
    const double *Rj = rhs + (size_t)(KL + 1) * rs;
    int jj = 0;
    auto issue_fwd = [&](int s) {
        if (jj < N) {
            if (jj < N - 1) {
#pragma unroll
                for (int q = 0; q < FQ; ++q) {
                    if ((q & 1) != part) continue;
                    const unsigned d = sbase + (unsigned)(((s) * SLOT + q * 16 + ml) * 8);
                    if (q < KL) cp_async8s(d, Lj + q * rowst);
                    else cp_async8s(d, Pj);
                }
            }
            if (jj + KL + 1 < N) cp_async8s(sbase + (unsigned)(((s) * SLOT + RQ + lane) * 8), Rj);
        }
        cp_async_commit();
        ++jj;
        Lj += Hp;
        if (PIV) Pj += Hp;
        Rj += rs;
    };
    double w[KL + 1];
#pragma unroll
    for (int i = 0; i <= KL; ++i) w[i] = (i < N) ? rhs[(size_t)i * rs] : 0.0;
#pragma unroll
    for (int s = 0; s < RING - 1; ++s) issue_fwd(s);
    double *Oj = out;
    for (int j0 = 0; j0 < N; j0 += RING) {
#pragma unroll
        for (int s = 0; s < RING; ++s) {
            const int j = j0 + s;
            if (j < N) {
                cp_async_wait<RING - 2>();
                __syncwarp(mask);
                const double ahead = (j + KL + 1 < N) ? WRHS(s) : 0.0;
                if (j < N - 1) {
                    if (PIV) {
                        const int p = (int)WSLOT(s, KL);
#pragma unroll
                        for (int i = 1; i <= KL; ++i)
                            if (p == i) {
                                const double t = w[0];
                                w[0] = w[i];
                                w[i] = t;
                            }
                    }
                    const double bj = w[0];
#pragma unroll
                    for (int i = 1; i <= KL; ++i)
                        if (j + i < N) w[i] = fma(-WSLOT(s, i - 1), bj, w[i]);
                }
                *Oj = w[0];
                Oj += os;
#pragma unroll
                for (int i = 0; i < KL; ++i) w[i] = w[i + 1];
                w[KL] = ahead;
                issue_fwd((s + RING - 1) % RING);  // the slot both lanes finished at j-1
            }
        }
    }
    cp_async_wait<0>();
    __syncwarp(mask);  // the partner has read the last forward slots
    const double *Uj = lu + (size_t)KV * rowst + (size_t)(N - 1) * Hp + nh;
    int tt = 0;
    auto issue_bwd = [&](int s) {
        if (tt < N) {
#pragma unroll
            for (int q = 0; q < BQ; ++q)
                if ((q & 1) == part) cp_async8s(sbase + (unsigned)(((s) * SLOT + q * 16 + ml) * 8), Uj - q * rowst);
        }
        cp_async_commit();
        ++tt;
        Uj -= Hp;
    };
#pragma unroll
    for (int s = 0; s < RING - 1; ++s) issue_bwd(s);
    double v[KU + 1];
#pragma unroll
    for (int i = 0; i <= KU; ++i) v[i] = (N - 1 - i >= 0) ? __ldcs(out + (size_t)(N - 1 - i) * os) : 0.0;
    constexpr int QY = 4;
    double yq[QY];
#pragma unroll
    for (int q = 0; q < QY; ++q) {
        const int r = N - 1 - KU - 1 - q;
        yq[q] = (r >= 0) ? __ldcs(out + (size_t)r * os) : 0.0;
    }
    double *Xj = out + (size_t)(N - 1) * os;
    for (int t0 = 0; t0 < N; t0 += RING) {
#pragma unroll
        for (int s = 0; s < RING; ++s) {
            const int t = t0 + s;
            if (t < N) {
                const int j = N - 1 - t;
                cp_async_wait<RING - 2>();
                __syncwarp(mask);
                const double ahead = yq[0];
#pragma unroll
                for (int q = 0; q < QY - 1; ++q) yq[q] = yq[q + 1];
                {
                    const int r = j - KU - 1 - QY;
                    yq[QY - 1] = (r >= 0) ? __ldcs(out + (size_t)r * os) : 0.0;
                }
                double x = v[0];
                if (x != 0.0) {
                    x = x / WSLOT(s, 0);
#pragma unroll
                    for (int i = 1; i <= KU; ++i)
                        if (j - i >= 0) v[i] = fma(-x, WSLOT(s, i), v[i]);
                }
                *Xj = x;
                Xj -= os;
#pragma unroll
                for (int i = 0; i < KU; ++i) v[i] = v[i + 1];
                v[KU] = (j - KU - 1 >= 0) ? ahead : 0.0;
                issue_bwd((s + RING - 1) % RING);
            }
        }
    }
    cp_async_wait<0>();
#undef WSLOT
#undef WRHS
}

// The same banded solve for two right-hand sides through one factor
// stream: modes (k, m) and (-k, m) have the same matrix (bitwise, see
// lumesh_entry) and therefore the same factors and pivots, so one thread
// solves the real (or imaginary) parts of both and every factor value is
// fetched once for the two.  rhsB/outB belong to the mirror mode; with
// twin false the second chain is idle.  Each chain's operations are those of
// solve_async, so the solutions are bitwise the same.
template <bool PIV, int TS>
__device__ __forceinline__ void solve_async2(const double *__restrict__ lu, const double *__restrict__ pivd, int N,
                                             int Hp, int nh, const double *__restrict__ rhsA,
                                             const double *__restrict__ rhsB, size_t rs, double *outA, double *outB,
                                             size_t os, bool twin, double *ring) {
    constexpr int KU = PIV ? KV : KL;
    constexpr int SWF = KL + 2 + (PIV ? 1 : 0);  // forward slot: L column, two rhs ahead, pivot
    constexpr int SWB = KU + 1;                  // backward slot: U column
    constexpr int SW = SWF > SWB ? SWF : SWB;
    constexpr unsigned QB = 8u * TS, SB = 8u * TS * SW;
    const size_t rowst = (size_t)N * Hp;
    const unsigned sbase = (unsigned)__cvta_generic_to_shared(ring);
#define RSLOT(s, q) ring[((s) * SW + (q)) * TS]
    const double *Lj = lu + (size_t)(KV + 1) * rowst + nh;
    const double *Pj = PIV ? pivd + nh : nullptr;
    const double *RAj = rhsA + (size_t)(KL + 1) * rs;
    const double *RBj = rhsB + (size_t)(KL + 1) * rs;
    int jj = 0;
    auto issue_fwd = [&](int s) {
        if (jj < N) {
            if (jj < N - 1) {
#pragma unroll
                for (int i = 0; i < KL; ++i) cp_async8s(sbase + s * SB + i * QB, Lj + i * rowst);
                if (PIV) cp_async8s(sbase + s * SB + (KL + 2) * QB, Pj);
            }
            if (jj + KL + 1 < N) {
                cp_async8s(sbase + s * SB + KL * QB, RAj);
                if (twin) cp_async8s(sbase + s * SB + (KL + 1) * QB, RBj);
            }
        }
        cp_async_commit();
        ++jj;
        Lj += Hp;
        if (PIV) Pj += Hp;
        RAj += rs;
        RBj += rs;
    };
    double wa[KL + 1], wb[KL + 1];
#pragma unroll
    for (int i = 0; i <= KL; ++i) {
        wa[i] = (i < N) ? rhsA[(size_t)i * rs] : 0.0;
        wb[i] = (i < N && twin) ? rhsB[(size_t)i * rs] : 0.0;
    }
#pragma unroll
    for (int s = 0; s < RING; ++s) issue_fwd(s);
    double *OAj = outA, *OBj = outB;
    for (int j0 = 0; j0 < N; j0 += RING) {
#pragma unroll
        for (int s = 0; s < RING; ++s) {
            const int j = j0 + s;
            if (j < N) {
                cp_async_wait<RING - 1>();
                const double aheadA = (j + KL + 1 < N) ? RSLOT(s, KL) : 0.0;
                const double aheadB = (j + KL + 1 < N && twin) ? RSLOT(s, KL + 1) : 0.0;
                if (j < N - 1) {
                    if (PIV) {
                        const int p = (int)RSLOT(s, KL + 2);
#pragma unroll
                        for (int i = 1; i <= KL; ++i)
                            if (p == i) {
                                const double t = wa[0];
                                wa[0] = wa[i];
                                wa[i] = t;
                                const double u = wb[0];
                                wb[0] = wb[i];
                                wb[i] = u;
                            }
                    }
                    const double bja = wa[0], bjb = wb[0];
#pragma unroll
                    for (int i = 1; i <= KL; ++i)
                        if (j + i < N) {
                            const double L = RSLOT(s, i - 1);
                            wa[i] = fma(-L, bja, wa[i]);
                            wb[i] = fma(-L, bjb, wb[i]);
                        }
                }
                *OAj = wa[0];
                if (twin) *OBj = wb[0];
                OAj += os;
                OBj += os;
#pragma unroll
                for (int i = 0; i < KL; ++i) {
                    wa[i] = wa[i + 1];
                    wb[i] = wb[i + 1];
                }
                wa[KL] = aheadA;
                wb[KL] = aheadB;
                issue_fwd(s);
            }
        }
    }
    cp_async_wait<0>();
    // back substitution with the U columns shared by the two chains
    const double *Uj = lu + (size_t)KV * rowst + (size_t)(N - 1) * Hp + nh;
    int tt = 0;
    auto issue_bwd = [&](int s) {
        if (tt < N) {
#pragma unroll
            for (int i = 0; i <= KU; ++i) cp_async8s(sbase + s * SB + i * QB, Uj - i * rowst);
        }
        cp_async_commit();
        ++tt;
        Uj -= Hp;
    };
#pragma unroll
    for (int s = 0; s < RING; ++s) issue_bwd(s);
    double va[KU + 1], vb[KU + 1];
#pragma unroll
    for (int i = 0; i <= KU; ++i) {
        va[i] = (N - 1 - i >= 0) ? __ldcs(outA + (size_t)(N - 1 - i) * os) : 0.0;
        vb[i] = (N - 1 - i >= 0 && twin) ? __ldcs(outB + (size_t)(N - 1 - i) * os) : 0.0;
    }
    constexpr int QY = 4;
    double ya[QY], yb[QY];
#pragma unroll
    for (int q = 0; q < QY; ++q) {
        const int r = N - 1 - KU - 1 - q;
        ya[q] = (r >= 0) ? __ldcs(outA + (size_t)r * os) : 0.0;
        yb[q] = (r >= 0 && twin) ? __ldcs(outB + (size_t)r * os) : 0.0;
    }
    double *XAj = outA + (size_t)(N - 1) * os, *XBj = outB + (size_t)(N - 1) * os;
    for (int t0 = 0; t0 < N; t0 += RING) {
#pragma unroll
        for (int s = 0; s < RING; ++s) {
            const int t = t0 + s;
            if (t < N) {
                const int j = N - 1 - t;
                cp_async_wait<RING - 1>();
                const double aheadA = ya[0], aheadB = yb[0];
#pragma unroll
                for (int q = 0; q < QY - 1; ++q) {
                    ya[q] = ya[q + 1];
                    yb[q] = yb[q + 1];
                }
                {
                    const int r = j - KU - 1 - QY;
                    ya[QY - 1] = (r >= 0) ? __ldcs(outA + (size_t)r * os) : 0.0;
                    yb[QY - 1] = (r >= 0 && twin) ? __ldcs(outB + (size_t)r * os) : 0.0;
                }
                double xa = va[0], xb = vb[0];
                if (xa != 0.0) {
                    xa = xa / RSLOT(s, 0);
#pragma unroll
                    for (int i = 1; i <= KU; ++i)
                        if (j - i >= 0) va[i] = fma(-xa, RSLOT(s, i), va[i]);
                }
                if (xb != 0.0) {
                    xb = xb / RSLOT(s, 0);
#pragma unroll
                    for (int i = 1; i <= KU; ++i)
                        if (j - i >= 0) vb[i] = fma(-xb, RSLOT(s, i), vb[i]);
                }
                *XAj = xa;
                if (twin) *XBj = xb;
                XAj -= os;
                XBj -= os;
#pragma unroll
                for (int i = 0; i < KU; ++i) {
                    va[i] = va[i + 1];
                    vb[i] = vb[i + 1];
                }
                va[KU] = (j - KU - 1 >= 0) ? aheadA : 0.0;
                vb[KU] = (j - KU - 1 >= 0) ? aheadB : 0.0;
                issue_bwd(s);
            }
        }
    }
    cp_async_wait<0>();
#undef RSLOT
}

// items of the paired solves: item = m*K + k (k >= 0); the primary mode
// (k, m) and, for m >= 1 and k >= 1, its mirror (-k, m)
__device__ __forceinline__ bool pair_item(const Geo &g, int item, int &nh, int &nh2) {
    if (item >= g.M * g.K) return false;
    const int m = item / g.K, k = item - m * g.K;
    const int base = m * (2 * g.K - 1);
    nh = m == 0 ? k : base + k;
    nh2 = (m > 0 && k > 0) ? base - k : -1;
    return true;
}
__host__ __device__ inline int pair_tiles(const Geo &g) { return (g.M * g.K + 31) / 32; }

// S2 with the mirror modes paired: warp = (re or im) of 32 items
__device__ __forceinline__ void solve_pnp2_body(const StepArgs &a, int bx) {
    extern __shared__ double ring2p[];
    const Geo &g = a.g;
    const int part = threadIdx.x >> 5;
    int nh, nh2;
    if (!pair_item(g, bx * 32 + (threadIdx.x & 31), nh, nh2)) return;
    const size_t st = 2 * (size_t)g.Hp;
    const bool twin = nh2 >= 0;
    const int nhb = twin ? nh2 : nh;
    double *outA = reinterpret_cast<double *>(a.p) + 2 * (size_t)nh + part;
    double *outB = reinterpret_cast<double *>(a.p) + 2 * (size_t)nhb + part;
    const double *rhsA = reinterpret_cast<const double *>(a.prhs) + 2 * (size_t)nh + part;
    const double *rhsB = reinterpret_cast<const double *>(a.prhs) + 2 * (size_t)nhb + part;
    if (nh == 0) {  // BC=1 at k=m=0: zero (timestep.f90:110-113); no mirror
        for (int n = 0; n < g.N; ++n) outA[n * st] = 0.0;
        return;
    }
    solve_async2<true, 64>(a.lnp, a.pivd, g.N, g.Hp, nh, rhsA, rhsB, st, outA, outB, st, twin, ring2p + threadIdx.x);
}

// S4 with the mirror modes paired: warp = one (system, re/im) of 32 items
__device__ __forceinline__ void solve_ld2_body(const StepArgs &a, int bx) {
    extern __shared__ double ring4p[];
    const Geo &g = a.g;
    const int w = threadIdx.x >> 5;
    const int sys = w >> 1, part = w & 1;
    int nh, nh2;
    if (!pair_item(g, bx * 32 + (threadIdx.x & 31), nh, nh2)) return;
    const size_t st = 2 * (size_t)g.Hp;
    const bool twin = nh2 >= 0;
    const int nhb = twin ? nh2 : nh;
    const double *rl = reinterpret_cast<const double *>(pick3(a.rl, sys));
    double *v = reinterpret_cast<double *>(pick3(a.v, sys));
    const double *lu = sys == 0 ? a.ldp : sys == 1 ? a.ldm : a.ldz;
    if (pick3(a.ldpiv, sys))
        solve_async2<true, 192>(lu, pick3(a.pivld, sys), g.N, g.Hp, nh, rl + 2 * (size_t)nh + part,
                                rl + 2 * (size_t)nhb + part, st, v + 2 * (size_t)nh + part, v + 2 * (size_t)nhb + part,
                                st, twin, ring4p + threadIdx.x);
    else
        solve_async2<false, 192>(lu, nullptr, g.N, g.Hp, nh, rl + 2 * (size_t)nh + part, rl + 2 * (size_t)nhb + part,
                                 st, v + 2 * (size_t)nh + part, v + 2 * (size_t)nhb + part, st, twin,
                                 ring4p + threadIdx.x);
}

// S2 with the factor ring of a mode shared by its real and imaginary lanes:
// warp = 16 consecutive modes x (re, im)
__device__ __forceinline__ void solve_pnpw_body(const StepArgs &a, int bx) {
    extern __shared__ double ring2w[];
    const Geo &g = a.g;
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31, part = lane >> 4;
    const int nh = bx * 32 + w * 16 + (lane & 15);
    const size_t st = 2 * (size_t)g.Hp;
    double *out = reinterpret_cast<double *>(a.p) + 2 * (size_t)nh + part;
    const bool live = nh < g.H && nh != 0;
    const unsigned mask = __ballot_sync(0xffffffffu, live);
    if (nh == 0) {  // BC=1 at k=m=0: zero (timestep.f90:110-113)
        for (int n = 0; n < g.N; ++n) out[n * st] = 0.0;
        return;
    }
    if (!live) return;
    const double *rhs = reinterpret_cast<const double *>(a.prhs) + 2 * (size_t)nh + part;
    // factors of the compact copy: mode (-k, m) reads those of (k, m)
    solve_async_rw<true>(a.lnpc, a.pivdc, g.N, a.Hcp, mode_compact(nh, g.K), rhs, st, out, st,
                         ring2w + (size_t)w * RING * rw_slot<true>(), mask);
}

// S4 with the shared rings: warp = one system of 16 consecutive modes x (re,
// im); WIDE rings hold the pivoting band (launches of pipes any of whose
// Helmholtz factorisations pivoted), narrow ones the pivot-free band
template <bool WIDE>
__device__ __forceinline__ void solve_ldw_body(const StepArgs &a, int bx) {
    extern __shared__ double ring4w[];
    const Geo &g = a.g;
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31, part = lane >> 4;
    const int sys = w >> 1;
    const int nh = bx * 32 + (w & 1) * 16 + (lane & 15);
    const bool live = nh < g.H;
    const unsigned mask = __ballot_sync(0xffffffffu, live);
    if (!live) return;
    const size_t st = 2 * (size_t)g.Hp;
    const double *rhs = reinterpret_cast<const double *>(pick3(a.rl, sys)) + 2 * (size_t)nh + part;
    double *out = reinterpret_cast<double *>(pick3(a.v, sys)) + 2 * (size_t)nh + part;
    const double *lu = sys == 0 ? a.ldp : sys == 1 ? a.ldm : a.ldz;
    double *wr = ring4w + (size_t)w * RING * rw_slot<WIDE>();
    if constexpr (WIDE) {
        if (pick3(a.ldpiv, sys)) {
            solve_async_rw<true>(lu, pick3(a.pivld, sys), g.N, g.Hp, nh, rhs, st, out, st, wr, mask);
            return;
        }
    }
    solve_async_rw<false>(lu, nullptr, g.N, g.Hp, nh, rhs, st, out, st, wr, mask);
}

// S3: rhs - rt2pm(grad p) (velocity.f90:232-236) with zero boundary rows
// (velocity.f90:376-378), one thread per (mode, PR consecutive rows)
static constexpr int PR = 4;  // S3 rows per thread

__device__ __forceinline__ void step_proj_body(const StepArgs &a, int bx, int by) {
    const Geo &g = a.g;
    const int nh = bx * blockDim.x + threadIdx.x, n0 = by * PR;
    const int N = g.N;
    if (nh >= g.H) return;
    const size_t Hp = g.Hp;
    const double2 *__restrict__ p = a.p + nh;
    const double2 *__restrict__ v0 = a.v[0] + nh;
    const double2 *__restrict__ v1 = a.v[1] + nh;
    const double2 *__restrict__ v2 = a.v[2] + nh;
    double2 *__restrict__ r0 = a.rl[0] + nh;
    double2 *__restrict__ r1 = a.rl[1] + nh;
    double2 *__restrict__ r2 = a.rl[2] + nh;
    const double *__restrict__ drb = a.dm.dr;
    int k, m;
    mode_km(nh, g.K, k, m);
    const double kal = g.alpha * k;
    // the pressure rows this thread's band products touch, loaded once
    double2 pw[PR + 2 * KL];
#pragma unroll
    for (int i = 0; i < PR + 2 * KL; ++i) {
        const int j = n0 - KL + i;
        pw[i] = (j >= 0 && j < N) ? p[(size_t)j * Hp] : make_double2(0.0, 0.0);
    }
#pragma unroll
    for (int q = 0; q < PR; ++q) {
        const int n = n0 + q;
        if (n >= N) break;
        const size_t at = (size_t)n * Hp;
        if (n == 0 || n == N - 1) {
            r0[at] = r1[at] = r2[at] = make_double2(0.0, 0.0);
            continue;
        }
        double2 dr2 = make_double2(0, 0);
        const int lo = max(0, n - KL), hi = min(N - 1, n + KL);
#pragma unroll
        for (int d = -KL; d <= KL; ++d) {
            const int j = n + d;
            if (j < lo || j > hi) continue;
            const double w = drb[(KL + n - j) * N + j];
            const double2 x = pw[q + KL + d];
            dr2.x = fma(w, x.x, dr2.x);
            dr2.y = fma(w, x.y, dr2.y);
        }
        const double2 pv = pw[q + KL];
        const double m1r1 = a.dm.rp[2 * N + n] * g.Mp * m;
        // grad p = (dr p, i m/r p, i alpha k p); rt2pm of its (r, theta) parts
        const double tRe = -pv.y * m1r1, tIm = pv.x * m1r1;
        const double2 vp = v0[at], vm = v1[at], vz = v2[at];
        r0[at] = make_double2(vp.x - (dr2.x - tIm), vp.y - (dr2.y + tRe));
        r1[at] = make_double2(vm.x - (dr2.x + tIm), vm.y - (dr2.y - tRe));
        r2[at] = make_double2(vz.x - (-pv.y * kal), vz.y - (pv.x * kal));
    }
}

// S4: warp = one (system, re/im) of 32 consecutive modes; the pivot-free
// sweep is used for the systems whose factorisation did not pivot
__device__ __forceinline__ void solve_ld_body(const StepArgs &a, int bx) {
    extern __shared__ double ring4[];
    const Geo &g = a.g;
    const int w = threadIdx.x >> 5;
    const int nh = bx * 32 + (threadIdx.x & 31);
    const int sys = w >> 1, part = w & 1;
    if (nh >= g.H) return;
    const size_t st = 2 * (size_t)g.Hp;
    const double *rhs = reinterpret_cast<const double *>(pick3(a.rl, sys)) + 2 * (size_t)nh + part;
    double *out = reinterpret_cast<double *>(pick3(a.v, sys)) + 2 * (size_t)nh + part;
    // factors of the compact copy: mode (-k, m) reads those of (k, m), so a
    // warp's factor loads cover about half as many distinct columns
    const double *lu = pick3(a.ldc, sys);
    const int c = mode_compact(nh, g.K);
    if (pick3(a.ldpiv, sys))  // pivoting band (low Re, small dt or very clustered meshes)
        solve_async<true, 192>(lu, pick3(a.pivldc, sys), g.N, a.Hcp, c, rhs, st, out, st, ring4 + threadIdx.x);
    else
        solve_async<false, 192>(lu, nullptr, g.N, a.Hcp, c, rhs, st, out, st, ring4 + threadIdx.x);
}

// ------------------------- S4 with the factors rebuilt on chip (no pivoting)
// For a pipe none of whose Helmholtz factorisations pivoted.  One thread per
// (system, k >= 0, m): it assembles the band of its mode (lumesh_entry, the
// bits k_lu_factor assembles) and eliminates it column by column in a 5 x 5
// register window in dgbtf2's order of operations, while the unit-lower
// sweep of dgbtrs runs on four right-hand sides at once: the real and
// imaginary parts of mode (k, m) and of its mirror (-k, m), whose matrix is
// the same.  The rows U(j, j..j+3) of the upper factor go to shared memory
// for the back substitution (dtbsv); U(j, j+4) is never updated by the
// elimination, so it is reassembled instead of stored.  Every factor value
// and every solve operation is the one k_lu_factor + solve_async perform, so
// the solutions are bitwise those of the streamed-factor path, but the
// factors never touch HBM: the launch moves the right-hand sides in and the
// solutions out (plus the forward results, written and read back once).
//
// Shared memory per thread: U rows 4*N doubles and a ring of LDR_D
// right-hand-side rows (two modes, double2) staged ahead by cp.async.
static constexpr int LDR_BT = 32;  // items per block
static constexpr int LDR_D = 8;    // right-hand-side rows in flight per item

__device__ __forceinline__ void cp_async16s(unsigned saddr, const void *gmem) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(saddr), "l"(gmem) : "memory");
}

static __host__ __device__ inline size_t ldr_smem(int N) {
    return (size_t)LDR_BT * (4 * (size_t)N * sizeof(double) + (size_t)LDR_D * 2 * sizeof(double2));
}
// tiles of one pipe: 3 systems x ceil(M*K / LDR_BT)
static __host__ __device__ inline int ldr_tiles(const Geo &g) { return 3 * ((g.M * g.K + LDR_BT - 1) / LDR_BT); }

__device__ __forceinline__ void solve_ld_rebuild_body(const StepArgs &a, int tile) {
    extern __shared__ __align__(16) double ldr_sm[];
    const Geo &g = a.g;
    const int N = g.N, K = g.K;
    const int nitem = g.M * K;
    const int per = (nitem + LDR_BT - 1) / LDR_BT;
    const int sys = tile / per;
    const int item = (tile - sys * per) * LDR_BT + (int)threadIdx.x;
    if (item >= nitem) return;  // no block barrier below
    const int m = item / K, k = item - m * K;
    const int base = m * (2 * K - 1);
    const bool twin = m > 0 && k > 0;
    const int nh = m == 0 ? k : base + k;
    const int nh2 = twin ? base - k : nh;
    const int PM = sys == 0 ? 1 : (sys == 1 ? -1 : 0);
    const int S = (m * g.Mp + abs(PM)) % 2;
    const double c1 = a.ldc1, c2 = a.ldc2;
    const DevMesh &dm = a.dm;
    const size_t Hp = g.Hp;
    const double2 *__restrict__ rhs = pick3(a.rl, sys);
    double2 *__restrict__ out = pick3(a.v, sys);
    double *ur = ldr_sm + threadIdx.x;  // U(j, j+c) at ur[(j*4 + c) * LDR_BT]
    double2 *ring = reinterpret_cast<double2 *>(ldr_sm + (size_t)4 * N * LDR_BT) + threadIdx.x;
    const unsigned rbase = (unsigned)__cvta_generic_to_shared(ring);
    constexpr unsigned RSTEP = 16u * LDR_BT;  // bytes between ring entries
    auto A = [&](int r, int c) { return lumesh_entry(dm, N, g.Mp, g.alpha, PM, 0, c1, c2, k, m, S, r, c); };
    // right-hand-side rows enter in order 0, 1, 2, ...; row r sits in slot r % LDR_D
    int rin = 0;
    auto issue = [&](void) {
        if (rin < N) {
            const unsigned sa = rbase + (unsigned)((rin % LDR_D) * 2) * RSTEP;
            cp_async16s(sa, rhs + (size_t)rin * Hp + nh);
            cp_async16s(sa + RSTEP, rhs + (size_t)rin * Hp + nh2);
        }
        cp_async_commit();
        ++rin;
    };
#pragma unroll
    for (int q = 0; q < LDR_D; ++q) issue();
    cp_async_wait<LDR_D - 5>();  // rows 0..4
    // forward window: W[i][c] = A(j+i, j+c) as eliminated so far, held in
    // physical slot [(i+j)%5][(c+j)%5]; right-hand sides w[q][(i+j)%5]
    double W[5][5];
    double2 w0[5], w1[5];
#pragma unroll
    for (int i = 0; i < 5; ++i) {
#pragma unroll
        for (int c = 0; c < 5; ++c) W[i][c] = (i < N && c < N) ? A(i, c) : 0.0;
        const bool in = i < N;
        w0[i] = in ? ring[(size_t)((i % LDR_D) * 2) * LDR_BT] : make_double2(0.0, 0.0);
        w1[i] = in ? ring[(size_t)((i % LDR_D) * 2 + 1) * LDR_BT] : make_double2(0.0, 0.0);
    }
#pragma unroll
    for (int q = 0; q < 5; ++q) issue();
    double2 *Yj = out;  // forward results y(j) of mode nh, then of nh2 at +(nh2-nh)
    const ptrdiff_t d2 = (ptrdiff_t)nh2 - (ptrdiff_t)nh;
    Yj += nh;
    for (int j0 = 0; j0 < N; j0 += 5) {
#pragma unroll
        for (int s = 0; s < 5; ++s) {
            const int j = j0 + s;
            if (j < N) {
                const int km = min(KL, N - 1 - j);
                // column j of L and row j of U (dgbtf2, no interchange)
                double L[5];
                const double piv = W[s % 5][s % 5];
#pragma unroll
                for (int c = 0; c < 4; ++c) ur[(size_t)(j * 4 + c) * LDR_BT] = W[s % 5][(c + s) % 5];
                if (km > 0) {
                    const double rp = 1.0 / piv;
#pragma unroll
                    for (int i = 1; i <= KL; ++i) L[i] = (i <= km) ? W[(i + s) % 5][s % 5] * rp : 0.0;
#pragma unroll
                    for (int c = 1; c <= KL; ++c) {
                        if (c > km) break;
                        const double y = -W[s % 5][(c + s) % 5];
#pragma unroll
                        for (int i = 1; i <= KL; ++i)
                            if (i <= km) W[(i + s) % 5][(c + s) % 5] = fma(L[i], y, W[(i + s) % 5][(c + s) % 5]);
                    }
                    // dgbtrs forward sweep on the four right-hand sides
                    const double2 b0 = w0[s % 5], b1 = w1[s % 5];
#pragma unroll
                    for (int i = 1; i <= KL; ++i)
                        if (i <= km) {
                            double2 &x0 = w0[(i + s) % 5], &x1 = w1[(i + s) % 5];
                            x0.x = fma(-L[i], b0.x, x0.x);
                            x0.y = fma(-L[i], b0.y, x0.y);
                            x1.x = fma(-L[i], b1.x, x1.x);
                            x1.y = fma(-L[i], b1.y, x1.y);
                        }
                }
                Yj[0] = w0[s % 5];
                if (twin) Yj[d2] = w1[s % 5];
                Yj += Hp;
                // the row entering the right-hand-side window: j + 5
                cp_async_wait<LDR_D - 1>();
                const bool more = j + 5 < N;
                const int sl = ((j + 5) % LDR_D) * 2;
                w0[s % 5] = more ? ring[(size_t)sl * LDR_BT] : make_double2(0.0, 0.0);
                w1[s % 5] = more ? ring[(size_t)(sl + 1) * LDR_BT] : make_double2(0.0, 0.0);
                issue();
                // the window moves one row down and one column right: row j+5
                // and column j+5 enter with their assembled values
#pragma unroll
                for (int c = 0; c < 5; ++c) W[s % 5][(c + s) % 5] = (more && c >= 1) ? A(j + 5, j + c) : 0.0;
                if (more) W[s % 5][s % 5] = A(j + 5, j + 5);
#pragma unroll
                for (int i = 1; i < 5; ++i) W[(i + s) % 5][s % 5] = more ? A(j + i, j + 5) : 0.0;
            }
        }
    }
    cp_async_wait<0>();
    // back substitution (dtbsv) on the four right-hand sides; y(j) is read
    // back through a register queue QY rows ahead
    constexpr int QY = 4;
    const double2 *Yr = out + nh;
    double2 v0[5], v1[5], q0[QY], q1[QY];
#pragma unroll
    for (int i = 0; i < 5; ++i) {
        const int r = N - 1 - i;
        v0[i] = r >= 0 ? __ldcg(Yr + (size_t)r * Hp) : make_double2(0.0, 0.0);
        v1[i] = (r >= 0 && twin) ? __ldcg(Yr + (size_t)r * Hp + d2) : make_double2(0.0, 0.0);
    }
#pragma unroll
    for (int q = 0; q < QY; ++q) {
        const int r = N - 1 - 5 - q;
        q0[q] = r >= 0 ? __ldcg(Yr + (size_t)r * Hp) : make_double2(0.0, 0.0);
        q1[q] = (r >= 0 && twin) ? __ldcg(Yr + (size_t)r * Hp + d2) : make_double2(0.0, 0.0);
    }
    double2 *Xj = out + nh + (size_t)(N - 1) * Hp;
    for (int t0 = 0; t0 < N; t0 += 5) {
#pragma unroll
        for (int s = 0; s < 5; ++s) {
            const int t = t0 + s;
            if (t < N) {
                const int j = N - 1 - t;
                // U(j-i, j), i = 0..4
                double Uc[5];
#pragma unroll
                for (int i = 0; i < 4; ++i) Uc[i] = (j - i >= 0) ? ur[(size_t)((j - i) * 4 + i) * LDR_BT] : 0.0;
                Uc[4] = (j - 4 >= 0) ? A(j - 4, j) : 0.0;
                double2 x0 = v0[s % 5], x1 = v1[s % 5];
                // dtbsv skips a column whose right-hand side is exactly zero
                const bool n0x = x0.x != 0.0, n0y = x0.y != 0.0, n1x = x1.x != 0.0, n1y = x1.y != 0.0;
                const double u = Uc[0];
                if (n0x) x0.x = x0.x / u;
                if (n0y) x0.y = x0.y / u;
                if (n1x) x1.x = x1.x / u;
                if (n1y) x1.y = x1.y / u;
#pragma unroll
                for (int i = 1; i <= KL; ++i)
                    if (j - i >= 0) {
                        double2 &a0 = v0[(i + s) % 5], &a1 = v1[(i + s) % 5];
                        if (n0x) a0.x = fma(-x0.x, Uc[i], a0.x);
                        if (n0y) a0.y = fma(-x0.y, Uc[i], a0.y);
                        if (n1x) a1.x = fma(-x1.x, Uc[i], a1.x);
                        if (n1y) a1.y = fma(-x1.y, Uc[i], a1.y);
                    }
                Xj[0] = x0;
                if (twin) Xj[d2] = x1;
                Xj -= Hp;
                const bool more = j - 5 >= 0;
                v0[s % 5] = more ? q0[0] : make_double2(0.0, 0.0);
                v1[s % 5] = more ? q1[0] : make_double2(0.0, 0.0);
#pragma unroll
                for (int q = 0; q < QY - 1; ++q) {
                    q0[q] = q0[q + 1];
                    q1[q] = q1[q + 1];
                }
                const int r = j - 5 - QY;
                q0[QY - 1] = r >= 0 ? __ldcg(Yr + (size_t)r * Hp) : make_double2(0.0, 0.0);
                q1[QY - 1] = (r >= 0 && twin) ? __ldcg(Yr + (size_t)r * Hp + d2) : make_double2(0.0, 0.0);
            }
        }
    }
}

// ------------------------------------------------------------------- S5
__device__ __forceinline__ double sq(double2 a) { return a.x * a.x + a.y * a.y; }
// max that keeps a NaN (fmax drops it): a state gone non-finite shows as a
// NaN corrector error instead of a converged one
__device__ __forceinline__ double nanmax(double a, double b) { return (b > a || b != b) ? b : a; }

__device__ __forceinline__ void step_final_body(const StepArgs &a, int bx) {
    __shared__ double coef[TM][8];        // aR(1..4), aI(1..4) per mode
    __shared__ double red[TM * TR];
    __shared__ double m0buf[3][2][128];    // mode 0 after pm2rt (N <= 128)
    const Geo &g = a.g;
    const int N = g.N, Hp = g.Hp;
    const int tx = threadIdx.x % TM, ty = threadIdx.x / TM;
    const int nh = bx * TM + tx;
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
        const double2 *__restrict__ v0 = a.v[0] + nh;
        const double2 *__restrict__ v1 = a.v[1] + nh;
        const double2 *__restrict__ v2 = a.v[2] + nh;
        const double *__restrict__ Uc = a.U + nh;
        double2 *__restrict__ u0 = a.u[0] + nh;
        double2 *__restrict__ u1 = a.u[1] + nh;
        double2 *__restrict__ u2 = a.u[2] + nh;
        const size_t NH = (size_t)N * Hp;
        // rows are taken two at a time and every load of both rows is issued
        // before either row's stores, so two rows' memory latencies overlap
        constexpr int RB = 2;
        for (int n0 = ty; n0 < N; n0 += RB * TR) {
            double2 r[RB], t[RB], z[RB], o[RB][3];
            double Uv[RB][6];
#pragma unroll
            for (int q = 0; q < RB; ++q) {
                const int n = n0 + q * TR;
                if (n >= N) break;
                const size_t at = (size_t)n * Hp;
                r[q] = v0[at];
                t[q] = v1[at];
                z[q] = v2[at];
                if (nh != 0) {
#pragma unroll
                    for (int i = 0; i < 6; ++i) Uv[q][i] = Uc[i * NH + at];
                }
                if (a.mode == 1 && nh != 0) {  // read once, overwritten below: stream past L1
                    o[q][0] = __ldcs(u0 + at);
                    o[q][1] = __ldcs(u1 + at);
                    o[q][2] = __ldcs(u2 + at);
                }
            }
#pragma unroll
            for (int q = 0; q < RB; ++q) {
                const int n = n0 + q * TR;
                if (n >= N) break;
                const size_t at = (size_t)n * Hp;
                double2 rr = r[q], tt = t[q], zz = z[q];
                if (nh != 0) {
                    const double U1 = Uv[q][0], U2 = Uv[q][1], U3 = Uv[q][2];
                    const double U4 = Uv[q][3], U5 = Uv[q][4], U6 = Uv[q][5];
                    rr.x = rr.x + cf[0] * U1; rr.y = rr.y + cf[4] * U1;
                    tt.x = tt.x + cf[1] * U2; tt.y = tt.y + cf[5] * U2;
                    zz.x = zz.x - cf[6] * U3; zz.y = zz.y + cf[2] * U3;
                    rr.x = rr.x + cf[3] * U4; rr.y = rr.y + cf[7] * U4;
                    tt.x = tt.x + cf[3] * U5; tt.y = tt.y + cf[7] * U5;
                    zz.x = zz.x - cf[7] * U6; zz.y = zz.y + cf[3] * U6;
                }
                // pm2rt
                const double2 ur = make_double2(0.5 * (rr.x + tt.x), 0.5 * (rr.y + tt.y));
                const double2 ut = make_double2(0.5 * (rr.y - tt.y), -0.5 * (rr.x - tt.x));
                if (nh == 0) {
                    m0buf[0][0][n] = ur.x; m0buf[0][1][n] = ur.y;
                    m0buf[1][0][n] = ut.x; m0buf[1][1][n] = ut.y;
                    m0buf[2][0][n] = zz.x; m0buf[2][1][n] = zz.y;
                    continue;
                }
                if (a.mode == 1) {
                    err = nanmax(err, sq(make_double2(o[q][0].x - ur.x, o[q][0].y - ur.y)));
                    err = nanmax(err, sq(make_double2(o[q][1].x - ut.x, o[q][1].y - ut.y)));
                    err = nanmax(err, sq(make_double2(o[q][2].x - zz.x, o[q][2].y - zz.y)));
                }
                u0[at] = ur;
                u1[at] = ut;
                u2[at] = zz;
            }
        }
    }
    if (bx == 0) {  // mode 0: flux adjustment and symmetry zeros
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
                err = nanmax(err, sq(make_double2(o0.x - ur.x, o0.y - ur.y)));
                err = nanmax(err, sq(make_double2(o1.x - ut.x, o1.y - ut.y)));
                err = nanmax(err, sq(make_double2(o2.x - uz.x, o2.y - uz.y)));
            }
            a.u[0][at] = ur;
            a.u[1][at] = ut;
            a.u[2][at] = uz;
        }
        if (threadIdx.x == 0 && a.const_flux) a.sc->Pr0 = a.sc->Pr0 + d3 * g.Re / 4.0;
    }
    if (a.mode == 1) {  // one atomic per block: warp maxima, then the block's
        __shared__ double wmax[TM * TR / 32];
        for (int o = 16; o > 0; o >>= 1) err = nanmax(err, __shfl_xor_sync(0xffffffffu, err, o));
        if ((threadIdx.x & 31) == 0) wmax[threadIdx.x >> 5] = err;
        __syncthreads();
        if (threadIdx.x == 0) {
            double e = wmax[0];
            for (int i = 1; i < TM * TR / 32; ++i) e = nanmax(e, wmax[i]);
            atomicMax(&a.sc->dterr2_bits, (unsigned long long)__double_as_longlong(e));
        }
    }
}

// ------------------------------------------------------------- kernels
// Lone pipe: one launch per stage over that pipe's tiles.  Batch: one launch
// per stage over the tiles of every pipe, blk[b] = (pipe, tile of that pipe).
template <int RPT>
__global__ void __launch_bounds__(HM *HR, 3) k_step_rhs(StepArgs a) { step_rhs_body<RPT>(a, blockIdx.x); }
__global__ void k_step_proj(StepArgs a) { step_proj_body(a, blockIdx.x, blockIdx.y); }
__global__ void __launch_bounds__(192, 4) k_solve_ld(StepArgs a) { solve_ld_body(a, blockIdx.x); }
__global__ void __launch_bounds__(LDR_BT) k_solve_ldr(StepArgs a) { solve_ld_rebuild_body(a, blockIdx.x); }
__global__ void __launch_bounds__(64, 8) k_solve_pnp2(StepArgs a) { solve_pnp2_body(a, blockIdx.x); }
__global__ void __launch_bounds__(192, 3) k_solve_ld2(StepArgs a) { solve_ld2_body(a, blockIdx.x); }
template <bool WIDE>
__global__ void __launch_bounds__(192, 4) k_solve_ldw(StepArgs a) { solve_ldw_body<WIDE>(a, blockIdx.x); }
__global__ void __launch_bounds__(64, 8) k_solve_pnpw(StepArgs a) { solve_pnpw_body(a, blockIdx.x); }
__global__ void __launch_bounds__(TM *TR) k_step_final(StepArgs a) { step_final_body(a, blockIdx.x); }

#define PF_BATCH1(NAME, BODY, BOUNDS)                                                          \
    __global__ void BOUNDS NAME(const StepArgs *__restrict__ args, const int2 *__restrict__ blk) { \
        const int2 pb = blk[blockIdx.x];                                                       \
        const StepArgs a = args[pb.x]; /* by value: stores cannot alias it */                  \
        BODY(a, pb.y);                                                                         \
    }
PF_BATCH1(k_solve_ld_batch, solve_ld_body, __launch_bounds__(192, 4))
PF_BATCH1(k_solve_ldr_batch, solve_ld_rebuild_body, __launch_bounds__(LDR_BT))
PF_BATCH1(k_solve_pnp2_batch, solve_pnp2_body, __launch_bounds__(64, 8))
PF_BATCH1(k_solve_ld2_batch, solve_ld2_body, __launch_bounds__(192, 3))
PF_BATCH1(k_solve_pnpw_batch, solve_pnpw_body, __launch_bounds__(64, 8))
PF_BATCH1(k_solve_ldw_batch0, solve_ldw_body<false>, __launch_bounds__(192, 4))
PF_BATCH1(k_solve_ldw_batch1, solve_ldw_body<true>, __launch_bounds__(192, 4))
PF_BATCH1(k_step_final_batch, step_final_body, __launch_bounds__(TM *TR))
#undef PF_BATCH1

// four blocks per SM in the batch (64 registers; the spilled bytes cost less
// than the extra warps gain: 4.80 -> 4.73 ms per 64-pipe batch step)
template <int RPT>
__global__ void __launch_bounds__(HM *HR, 4) k_step_rhs_batch(const StepArgs *__restrict__ args,
                                                             const int2 *__restrict__ blk) {
    const int2 pb = blk[blockIdx.x];
    const StepArgs a = args[pb.x];  // by value: stores cannot alias it
    step_rhs_body<RPT>(a, pb.y);
}

__global__ void __launch_bounds__(128) k_step_proj_batch(const StepArgs *__restrict__ args, const int2 *__restrict__ blk) {
    const int2 pb = blk[blockIdx.x];
    const StepArgs a = args[pb.x];
    const int gx = (a.g.H + 127) / 128;
    step_proj_body(a, pb.y % gx, pb.y / gx);
}

// ------------------------------------------------------------------ host
static StepArgs make_step_args(const pf_ctx *ctx, int corrector) {
    StepArgs a;
    for (int i = 0; i < 3; ++i) {
        a.u_[i] = ctx->prev[i].d;
        a.Nl[i] = ctx->vel[3 + i].d;
        a.N_[i] = ctx->prev[3 + i].d;
        a.v[i] = ctx->s[i].d;
        a.u[i] = ctx->vel[i].d;
    }
    a.prhs = ctx->s[3].d;
    a.p = ctx->s[4].d;
    a.rl[0] = ctx->s[5].d;
    a.rl[1] = ctx->s[6].d;
    a.rl[2] = ctx->s[3].d;  // free once the pressure is solved
    a.lnp = ctx->LNp.lu;
    a.pivd = ctx->LNp.pivd;
    const pf_lumesh *ld[3] = {&ctx->LDp, &ctx->LDm, &ctx->LDz};
    for (int i = 0; i < 3; ++i) {
        a.pivld[i] = ld[i]->pivd;
        a.ldpiv[i] = ld[i]->pivoted;
        a.ldc[i] = ld[i]->luc;
        a.pivldc[i] = ld[i]->pivdc;
    }
    a.lnpc = ctx->LNp.luc;
    a.pivdc = ctx->LNp.pivdc;
    a.Hcp = pf_compact_modes_padded(ctx->g);
    a.ldc1 = ctx->LDp.c1;
    a.ldc2 = ctx->LDp.c2;
    a.ldp = ctx->LDp.lu;
    a.ldm = ctx->LDm.lu;
    a.ldz = ctx->LDz.lu;
    a.U = ctx->U;
    a.Ainv = ctx->Ainv;
    a.Ui = ctx->Ui;
    a.dm = ctx->dm;
    a.g = ctx->g;
    a.c1 = ctx->Ltz.c1;
    a.c2 = ctx->Ltz.c2;
    a.implicit = ctx->cfg.implicit;
    a.mode = corrector;
    a.const_flux = ctx->cfg.const_flux;
    a.sc = ctx->dsc;
    return a;
}

static bool any_ld_pivoted(const pf_ctx *ctx) {
    return ctx->LDp.pivoted || ctx->LDm.pivoted || ctx->LDz.pivoted;
}

// The Helmholtz solves rebuild their factors on chip when the tuning asks
// for it (PF_LD_REBUILT), no factorisation pivoted and N >= 2 KL + 2; the
// built-in choice streams them.
static bool ld_rebuild(const pf_ctx *ctx) {
    return !any_ld_pivoted(ctx) && ctx->g.N >= 2 * KL + 2 && ctx->tune.ld_solver == PF_LD_REBUILT;
}

// The streamed solves with modes k and -k paired on one factor stream
// (pressure and Helmholtz); PF_LD_AUTO takes the built-in choice.
static constexpr int LD_BUILTIN = PF_LD_STREAMED;
static int ld_choice(const pf_ctx *ctx) {
    return ctx->tune.ld_solver == PF_LD_AUTO ? LD_BUILTIN : ctx->tune.ld_solver;
}
static bool ld_paired(const pf_ctx *ctx) { return ld_choice(ctx) == PF_LD_PAIRED; }
// The streamed solves with the factor ring of a mode shared by its real and
// imaginary lanes (pressure and Helmholtz)
static bool ld_warpring(const pf_ctx *ctx) { return ld_choice(ctx) == PF_LD_WARPRING; }
static size_t ldw_smem(bool wide) {
    return (size_t)(192 / 32) * RING * (wide ? rw_slot<true>() : rw_slot<false>()) * sizeof(double);
}
static size_t pnpw_smem() { return (size_t)(64 / 32) * RING * rw_slot<true>() * sizeof(double); }
static size_t ld2_smem(bool piv) { return (size_t)192 * RING * (piv ? KV + 1 : KL + 2) * sizeof(double); }
static size_t pnp_smem() { return (size_t)64 * RING * (KV + 1) * sizeof(double); }

static size_t rhs_smem(int N) { return (size_t)N * HM * sizeof(double2); }

static int step_attrs() {
    static bool attrs_set = false;
    if (!attrs_set) {
        const int ld = (int)(192 * RING * (KV + 1) * sizeof(double));
        const int pnp = (int)(64 * RING * (KV + 1) * sizeof(double));
        PF_CUDA(cudaFuncSetAttribute(k_solve_ld, cudaFuncAttributeMaxDynamicSharedMemorySize, ld));
        PF_CUDA(cudaFuncSetAttribute(k_solve_ld_batch, cudaFuncAttributeMaxDynamicSharedMemorySize, ld));
        const int ldr = (int)ldr_smem(HR * 8);
        PF_CUDA(cudaFuncSetAttribute(k_solve_ldr, cudaFuncAttributeMaxDynamicSharedMemorySize, ldr));
        PF_CUDA(cudaFuncSetAttribute(k_solve_ldr_batch, cudaFuncAttributeMaxDynamicSharedMemorySize, ldr));
        PF_CUDA(cudaFuncSetAttribute(k_solve_ld2, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ld2_smem(true)));
        PF_CUDA(cudaFuncSetAttribute(k_solve_ld2_batch, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)ld2_smem(true)));
        PF_CUDA(cudaFuncSetAttribute(k_solve_pnp2, cudaFuncAttributeMaxDynamicSharedMemorySize, pnp));
        PF_CUDA(cudaFuncSetAttribute(k_solve_pnp2_batch, cudaFuncAttributeMaxDynamicSharedMemorySize, pnp));
        const int ldw = (int)ldw_smem(true), pnpw = (int)pnpw_smem();
        PF_CUDA(cudaFuncSetAttribute(k_solve_ldw<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, ldw));
        PF_CUDA(cudaFuncSetAttribute(k_solve_ldw<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, ldw));
        PF_CUDA(cudaFuncSetAttribute(k_solve_ldw_batch0, cudaFuncAttributeMaxDynamicSharedMemorySize, ldw));
        PF_CUDA(cudaFuncSetAttribute(k_solve_ldw_batch1, cudaFuncAttributeMaxDynamicSharedMemorySize, ldw));
        PF_CUDA(cudaFuncSetAttribute(k_solve_pnpw, cudaFuncAttributeMaxDynamicSharedMemorySize, pnpw));
        PF_CUDA(cudaFuncSetAttribute(k_solve_pnpw_batch, cudaFuncAttributeMaxDynamicSharedMemorySize, pnpw));
        const int rhs = (int)rhs_smem(128);
        PF_CUDA(cudaFuncSetAttribute(k_step_rhs<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, rhs));
        PF_CUDA(cudaFuncSetAttribute(k_step_rhs<8>, cudaFuncAttributeMaxDynamicSharedMemorySize, rhs));
        PF_CUDA(cudaFuncSetAttribute(k_step_rhs_batch<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, rhs));
        PF_CUDA(cudaFuncSetAttribute(k_step_rhs_batch<8>, cudaFuncAttributeMaxDynamicSharedMemorySize, rhs));
        attrs_set = true;
    }
    return PF_OK;
}

static bool pf_fused_step_geo_ok(const Geo &g) { return g.N <= HR * 8; }

// One predictor (corrector=0) or corrector (corrector=1) vel_step.  The
// predictor's u_ := u copy is a pointer swap of vel[0..2] and prev[0..2].
int pf_vel_step_fused(pf_ctx *ctx, int corrector) {
    const Geo &g = ctx->g;
    if (!pf_fused_step_geo_ok(g)) {
        pf_set_error("fused step supports N <= 128");
        return PF_ERR_ARG;
    }
    if (!corrector) {
        for (int i = 0; i < 3; ++i) std::swap(ctx->vel[i].d, ctx->prev[i].d);
        ctx->parity ^= 1;
    }
    const StepArgs a = make_step_args(ctx, corrector);
    const int ldsw = any_ld_pivoted(ctx) ? KV + 1 : KL + 1;  // ring slot width of the Helmholtz solves
    const unsigned tiles = grid1(g.H, TM);
    PF_TRY(step_attrs());
    {
        ProfScope ps_(ctx, PF_K_STEP);
        if (g.N <= HR * 4)
            k_step_rhs<4><<<grid1(g.H, HM), HM * HR, rhs_smem(g.N), ctx->stream>>>(a);
        else
            k_step_rhs<8><<<grid1(g.H, HM), HM * HR, rhs_smem(g.N), ctx->stream>>>(a);
    }
    PF_LAUNCHED(ctx);
    {
        ProfScope ps_(ctx, PF_K_PPE);
        if (ld_paired(ctx))
            k_solve_pnp2<<<pair_tiles(g), 64, pnp_smem(), ctx->stream>>>(a);
        else  // every other choice: the shared-ring pressure solve (10% faster than a ring per lane)
            k_solve_pnpw<<<tiles, 64, pnpw_smem(), ctx->stream>>>(a);
    }
    PF_LAUNCHED(ctx);
    {
        ProfScope ps_(ctx, PF_K_STEP);
        k_step_proj<<<dim3(grid1(g.H, 128), grid1(g.N, PR)), 128, 0, ctx->stream>>>(a);
    }
    PF_LAUNCHED(ctx);
    {
        ProfScope ps_(ctx, PF_K_LUSOLVE);
        if (ld_rebuild(ctx))
            k_solve_ldr<<<ldr_tiles(g), LDR_BT, ldr_smem(g.N), ctx->stream>>>(a);
        else if (ld_paired(ctx))
            k_solve_ld2<<<pair_tiles(g), 192, ld2_smem(any_ld_pivoted(ctx)), ctx->stream>>>(a);
        else if (ld_warpring(ctx) && any_ld_pivoted(ctx))
            k_solve_ldw<true><<<tiles, 192, ldw_smem(true), ctx->stream>>>(a);
        else if (ld_warpring(ctx))
            k_solve_ldw<false><<<tiles, 192, ldw_smem(false), ctx->stream>>>(a);
        else
            k_solve_ld<<<tiles, 192, (size_t)192 * RING * ldsw * sizeof(double), ctx->stream>>>(a);
    }
    PF_LAUNCHED(ctx);
    {
        ProfScope ps_(ctx, PF_K_INFL);
        k_step_final<<<tiles, TM * TR, 0, ctx->stream>>>(a);
    }
    PF_LAUNCHED(ctx);
    return PF_OK;
}

// ---------------------------------------------------------------- batched
// Step arguments of every pipe for both pointer parities and both modes,
// and the tile maps of the five stages.
struct pf_step_batch {
    int n;
    StepArgs *d_args[2][2];  // [pointer state after the predictor's swap][mode]
    int2 *tile, *proj, *half;  // (pipe, tile) maps: 32-mode tiles, 128-mode x row tiles, 16-mode tiles
    int ntile, nproj, nhalf;
    int2 *ldmap[2];            // 32-mode tiles of the pipes whose Helmholtz factors [0] never / [1] pivot
    int nld[2];
    int2 *ldrmap;              // tiles of the pipes whose Helmholtz factors are rebuilt on chip
    int nldr, ldrN;            // their count and largest N
    int2 *pmap;                // 32-item pair tiles of the pipes whose solves pair modes k and -k
    int np2;
    int2 *ld2map[2];           // the same tiles split by whether any Helmholtz factorisation [1] pivoted
    int nld2[2];
    int2 *pwmap;               // 32-mode tiles of the other pipes (pressure solve, a ring per mode)
    int npw;
    int2 *ldwmap[2];           // the same tiles split by whether any Helmholtz factorisation [1] pivoted
    int nldw[2];
    int maxN;
    bool anypiv;
};

void pf_step_batch_free(pf_step_batch *b) {
    if (!b) return;
    for (int s = 0; s < 2; ++s)
        for (int m = 0; m < 2; ++m) cudaFree(b->d_args[s][m]);
    cudaFree(b->tile);
    cudaFree(b->half);
    cudaFree(b->ldmap[0]);
    cudaFree(b->ldmap[1]);
    cudaFree(b->ldrmap);
    cudaFree(b->pmap);
    cudaFree(b->ld2map[0]);
    cudaFree(b->ld2map[1]);
    cudaFree(b->pwmap);
    cudaFree(b->ldwmap[0]);
    cudaFree(b->ldwmap[1]);
    cudaFree(b->proj);
    delete b;
}

// state 0: the pointers as the pipes hold them now; state 1: vel/prev swapped
int pf_step_batch_build(pf_ctx *const *pipes, int n, pf_step_batch **out) {
    *out = nullptr;
    pf_step_batch *b = new pf_step_batch();
    b->n = n;
    b->maxN = 0;
    b->anypiv = false;
    std::vector<StepArgs> h(n);
    std::vector<int2> tile, proj, half, ldm[2], ldr, pm, ld2m[2], pwm, ldwm[2];
    b->ldrN = 0;
    for (int i = 0; i < n; ++i) {
        const Geo &g = pipes[i]->g;
        if (!pf_fused_step_geo_ok(g)) {
            pf_step_batch_free(b);
            pf_set_error("batched step supports N <= 128");
            return PF_ERR_ARG;
        }
        b->maxN = std::max(b->maxN, g.N);
        b->anypiv |= any_ld_pivoted(pipes[i]);
        for (int t = 0; t < (int)grid1(g.H, TM); ++t) tile.push_back(make_int2(i, t));
        if (ld_paired(pipes[i])) {
            for (int t = 0; t < pair_tiles(g); ++t) pm.push_back(make_int2(i, t));
        } else {
            for (int t = 0; t < (int)grid1(g.H, TM); ++t) pwm.push_back(make_int2(i, t));
        }
        if (ld_paired(pipes[i])) {
            for (int t = 0; t < pair_tiles(g); ++t) ld2m[any_ld_pivoted(pipes[i]) ? 1 : 0].push_back(make_int2(i, t));
        } else if (ld_warpring(pipes[i])) {
            for (int t = 0; t < (int)grid1(g.H, TM); ++t) ldwm[any_ld_pivoted(pipes[i]) ? 1 : 0].push_back(make_int2(i, t));
        } else if (ld_rebuild(pipes[i])) {
            for (int t = 0; t < ldr_tiles(g); ++t) ldr.push_back(make_int2(i, t));
            b->ldrN = std::max(b->ldrN, g.N);
        } else {
            for (int t = 0; t < (int)grid1(g.H, TM); ++t) ldm[any_ld_pivoted(pipes[i]) ? 1 : 0].push_back(make_int2(i, t));
        }
        for (int t = 0; t < (int)grid1(g.H, HM); ++t) half.push_back(make_int2(i, t));
        for (int t = 0; t < (int)(grid1(g.H, 128) * grid1(g.N, PR)); ++t) proj.push_back(make_int2(i, t));
    }
    for (int s = 0; s < 2; ++s)
        for (int m = 0; m < 2; ++m) {
            for (int i = 0; i < n; ++i) {
                pf_ctx *c = pipes[i];
                if (s) for (int k = 0; k < 3; ++k) std::swap(c->vel[k].d, c->prev[k].d);
                h[i] = make_step_args(c, m);
                if (s) for (int k = 0; k < 3; ++k) std::swap(c->vel[k].d, c->prev[k].d);
            }
            if (cudaMalloc((void **)&b->d_args[s][m], n * sizeof(StepArgs)) != cudaSuccess ||
                cudaMemcpy(b->d_args[s][m], h.data(), n * sizeof(StepArgs), cudaMemcpyHostToDevice) != cudaSuccess) {
                pf_step_batch_free(b);
                pf_set_error("batched step: argument upload failed");
                return PF_ERR_CUDA;
            }
        }
    b->ntile = (int)tile.size();
    b->nhalf = (int)half.size();
    for (int q = 0; q < 2; ++q) {
        b->nld[q] = (int)ldm[q].size();
        if (cudaMalloc((void **)&b->ldmap[q], std::max<size_t>(1, ldm[q].size()) * sizeof(int2)) != cudaSuccess ||
            (!ldm[q].empty() && cudaMemcpy(b->ldmap[q], ldm[q].data(), ldm[q].size() * sizeof(int2),
                                           cudaMemcpyHostToDevice) != cudaSuccess)) {
            pf_step_batch_free(b);
            pf_set_error("batched step: tile map upload failed");
            return PF_ERR_CUDA;
        }
    }
    auto upload_map = [&](int2 **d, const std::vector<int2> &h, int *count) {
        *count = (int)h.size();
        return cudaMalloc((void **)d, std::max<size_t>(1, h.size()) * sizeof(int2)) == cudaSuccess &&
               (h.empty() || cudaMemcpy(*d, h.data(), h.size() * sizeof(int2), cudaMemcpyHostToDevice) == cudaSuccess);
    };
    if (!upload_map(&b->ldrmap, ldr, &b->nldr) || !upload_map(&b->pmap, pm, &b->np2) ||
        !upload_map(&b->ld2map[0], ld2m[0], &b->nld2[0]) || !upload_map(&b->ld2map[1], ld2m[1], &b->nld2[1]) ||
        !upload_map(&b->pwmap, pwm, &b->npw) ||
        !upload_map(&b->ldwmap[0], ldwm[0], &b->nldw[0]) || !upload_map(&b->ldwmap[1], ldwm[1], &b->nldw[1])) {
        pf_step_batch_free(b);
        pf_set_error("batched step: tile map upload failed");
        return PF_ERR_CUDA;
    }
    if (cudaMalloc((void **)&b->half, half.size() * sizeof(int2)) != cudaSuccess ||
        cudaMemcpy(b->half, half.data(), half.size() * sizeof(int2), cudaMemcpyHostToDevice) != cudaSuccess) {
        pf_step_batch_free(b);
        pf_set_error("batched step: tile map upload failed");
        return PF_ERR_CUDA;
    }
    b->nproj = (int)proj.size();
    if (cudaMalloc((void **)&b->tile, tile.size() * sizeof(int2)) != cudaSuccess ||
        cudaMalloc((void **)&b->proj, proj.size() * sizeof(int2)) != cudaSuccess ||
        cudaMemcpy(b->tile, tile.data(), tile.size() * sizeof(int2), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(b->proj, proj.data(), proj.size() * sizeof(int2), cudaMemcpyHostToDevice) != cudaSuccess) {
        pf_step_batch_free(b);
        pf_set_error("batched step: tile map upload failed");
        return PF_ERR_CUDA;
    }
    *out = b;
    return PF_OK;
}

// One predictor or corrector vel_step of every pipe in five launches; the
// caller tracks the pointer state (the predictor's swap is the caller's).
int pf_step_batch_launch(pf_step_batch *b, int state, int corrector, cudaStream_t st, pf_stage_prof *prof,
                         unsigned long long *nk) {
    PF_TRY(step_attrs());
    const StepArgs *a = b->d_args[state][corrector ? 1 : 0];
    {
        StageScope ss_(prof, PF_K_STEP, st);
        if (b->maxN <= HR * 4)
            k_step_rhs_batch<4><<<b->nhalf, HM * HR, rhs_smem(b->maxN), st>>>(a, b->half);
        else
            k_step_rhs_batch<8><<<b->nhalf, HM * HR, rhs_smem(b->maxN), st>>>(a, b->half);
    }
    PF_CHECK_LAUNCH();
    {
        StageScope ss_(prof, PF_K_PPE, st);
        if (b->np2 > 0) k_solve_pnp2_batch<<<b->np2, 64, pnp_smem(), st>>>(a, b->pmap);
        if (b->npw > 0) k_solve_pnpw_batch<<<b->npw, 64, pnpw_smem(), st>>>(a, b->pwmap);
    }
    PF_CHECK_LAUNCH();
    {
        StageScope ss_(prof, PF_K_STEP, st);
        k_step_proj_batch<<<b->nproj, 128, 0, st>>>(a, b->proj);
    }
    PF_CHECK_LAUNCH();
    {
        StageScope ss_(prof, PF_K_LUSOLVE, st);
        // pipes whose Helmholtz factors never pivot take the narrow ring (more
        // blocks per SM), the others the wide one
        for (int q = 0; q < 2; ++q)
            if (b->nld[q] > 0)
                k_solve_ld_batch<<<b->nld[q], 192, (size_t)192 * RING * (q ? KV + 1 : KL + 1) * sizeof(double), st>>>(
                    a, b->ldmap[q]);
        if (b->nldr > 0) k_solve_ldr_batch<<<b->nldr, LDR_BT, ldr_smem(b->ldrN), st>>>(a, b->ldrmap);
        for (int q = 0; q < 2; ++q)
            if (b->nld2[q] > 0) k_solve_ld2_batch<<<b->nld2[q], 192, ld2_smem(q == 1), st>>>(a, b->ld2map[q]);
        if (b->nldw[0] > 0) k_solve_ldw_batch0<<<b->nldw[0], 192, ldw_smem(false), st>>>(a, b->ldwmap[0]);
        if (b->nldw[1] > 0) k_solve_ldw_batch1<<<b->nldw[1], 192, ldw_smem(true), st>>>(a, b->ldwmap[1]);
    }
    PF_CHECK_LAUNCH();
    {
        StageScope ss_(prof, PF_K_INFL, st);
        k_step_final_batch<<<b->ntile, TM * TR, 0, st>>>(a, b->tile);
    }
    PF_CHECK_LAUNCH();
    *nk += 3 + (b->np2 > 0) + (b->npw > 0) + (b->nld[0] > 0) + (b->nld[1] > 0) + (b->nldr > 0) +
           (b->nld2[0] > 0) + (b->nld2[1] > 0) + (b->nldw[0] > 0) + (b->nldw[1] > 0);
    return PF_OK;
}
