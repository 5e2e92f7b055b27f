// Fused nonlinear term: vel_transform + vel_nonlinear (velocity.f90:304-361)
// without materialising the six physical fields.
//
//   k_nl_zinv  : per (m-chunk, n, component): u or curl(u) (var_coll_curl,
//                variables.f90:408-436, computed in the load stage), zero-pad
//                k to 3K, Hermitian fill of m=0, c2c along z (sign +1)
//   k_nl_theta : per (z-chunk, n): c2r along theta for the six components
//                (two real rows per complex FFT), u x curl(u), scale by
//                1/(9KM), r2c along theta, CFL maxima of velocity.f90:459-467
//   k_nl_zfwd  : per (m-chunk, n, component): c2c along z (sign -1),
//                truncation to |k|<K, plus the Hagen-Poiseuille and
//                constant-flux terms of vel_addHPF (velocity.f90:338-361)
//
// The (m, z) intermediate T[((c*N + n)*M + m)*Z + z] is the only scratch;
// the compute type C is double2 (FP64) or float2 (mixed precision).
#include <cmath>
#include "pf_internal.cuh"
#include "pf_fftcore.cuh"

static constexpr int NL_THREADS = 256;

struct NLArgs {
    const double2 *u[3];
    double2 *N[3];
    DevMesh dm;
    Geo g;
    int const_flux;
    DevScalars *sc;
    unsigned long long *cfl;  // 3*N maxima as ordered bits
};

template <typename C> __device__ __forceinline__ C to_c(double2 v);
template <> __device__ __forceinline__ double2 to_c<double2>(double2 v) { return v; }
template <> __device__ __forceinline__ float2 to_c<float2>(double2 v) { return make_float2((float)v.x, (float)v.y); }

__device__ __forceinline__ double2 band_row_d(const double *__restrict__ band, int N, int Hp,
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

// component `comp` of (u_r, u_t, u_z, curl_r, curl_t, curl_z) at (n, nh)
__device__ __forceinline__ double2 nl_input(const NLArgs &a, int comp, int n, int nh, int k, int m) {
    const Geo &g = a.g;
    const size_t at = (size_t)n * g.Hp + nh;
    if (comp < 3) return a.u[comp][at];
    const double rm1 = a.dm.rp[2 * g.N + n];
    const double m1r1 = rm1 * g.Mp * m;
    const double k1a1 = g.alpha * k;
    if (comp == 3) {
        const double2 c2 = a.u[1][at], c3 = a.u[2][at];
        return make_double2(-c3.y * m1r1 + c2.y * k1a1, c3.x * m1r1 - c2.x * k1a1);
    }
    if (comp == 4) {
        const double2 c1 = a.u[0][at];
        const double2 dz = band_row_d(a.dm.dr, g.N, g.Hp, a.u[2], n, nh);
        return make_double2(-c1.y * k1a1 - dz.x, c1.x * k1a1 - dz.y);
    }
    const double2 c1 = a.u[0][at], c2 = a.u[1][at];
    const double2 dt = band_row_d(a.dm.dr, g.N, g.Hp, a.u[1], n, nh);
    return make_double2(c2.x * rm1 + dt.x + c1.y * m1r1, c2.y * rm1 + dt.y - c1.x * m1r1);
}

template <int ZL, typename C>
__global__ void __launch_bounds__(NL_THREADS) k_nl_zinv(NLArgs a, C *__restrict__ T, const C *__restrict__ twz, int MC) {
    extern __shared__ __align__(16) unsigned char smraw[];
    using FR = FFTRows<ZL, C>;
    constexpr int RS = FR::pitch;
    C *rows = reinterpret_cast<C *>(smraw);
    C *tw = rows + (FR::smem_elems(MC) - 2 * ZL), *tw2 = tw + ZL;
    const Geo &g = a.g;
    const int K = g.K;
    const int comp = blockIdx.z, n = blockIdx.y, m0 = blockIdx.x * MC;
    const int mc = min(MC, g.M - m0);
    fft4_tables<ZL>(tw, tw2, twz);
    for (int idx = threadIdx.x; idx < mc * ZL; idx += blockDim.x) {
        const int c = idx / ZL, j = idx - c * ZL;
        const int m = m0 + c;
        double2 v = make_double2(0.0, 0.0);
        if (m == 0) {
            if (j < K) v = nl_input(a, comp, n, j, j, 0);
            else if (j >= 2 * K + 1) {
                v = nl_input(a, comp, n, ZL - j, ZL - j, 0);
                v.y = -v.y;
            }
        } else {
            const int kk = j < K ? j : (j >= 2 * K + 1 ? j - ZL : K);
            if (kk < K) v = nl_input(a, comp, n, m * (2 * K - 1) + kk, kk, m);
        }
        rows[c * RS + j] = to_c<C>(v);
    }
    __syncthreads();
    FR::template run<+1>(rows, mc, tw, tw2);
    C *out = T + ((size_t)(comp * g.N + n) * g.M + m0) * ZL;
    for (int idx = threadIdx.x; idx < mc * ZL; idx += blockDim.x) {
        const int c = idx / ZL, j = idx - c * ZL;
        out[idx] = rows[c * RS + j];
    }
}

__device__ __forceinline__ void atomic_max_pos(unsigned long long *p, double v) {
    atomicMax(p, (unsigned long long)__double_as_longlong(v));
}

template <int TL, typename C>
__global__ void __launch_bounds__(NL_THREADS) k_nl_theta(NLArgs a, C *__restrict__ T, const C *__restrict__ twt,
                                                         int ZC, typename CTraits<C>::R scale) {
    using R = typename CTraits<C>::R;
    extern __shared__ __align__(16) unsigned char smraw[];
    using FR = FFTRows<TL, C>;
    constexpr int RS = FR::pitch;
    const Geo &g = a.g;
    const int M = g.M, Z = g.Z, np = ZC / 2;
    const int rowsA = 3 * ZC;  // six components x ZC/2 packed pairs
    C *bufA = reinterpret_cast<C *>(smraw);
    C *bufB = bufA + (FR::smem_elems(rowsA) - 2 * TL);
    C *tw = bufB + (FR::smem_elems(rowsA / 2) - 2 * TL), *tw2 = tw + TL;
    const int n = blockIdx.y, z0 = blockIdx.x * ZC;
    fft4_tables<TL>(tw, tw2, twt);
    for (int i = threadIdx.x; i < rowsA * RS; i += blockDim.x) bufA[i] = CTraits<C>::make(0, 0);
    __syncthreads();
    // Hermitian-extend the M retained theta modes of two z rows into one
    // complex row: X = a + i b (c2r ignores the DC imaginary parts)
    for (int idx = threadIdx.x; idx < 6 * M * np; idx += blockDim.x) {
        const int zp = idx % np, rest = idx / np;
        const int m = rest % M, comp = rest / M;
        const int za = z0 + 2 * zp, zb = za + 1;
        const C *col = T + ((size_t)(comp * g.N + n) * M + m) * Z;
        const C va = (za < Z) ? col[za] : CTraits<C>::make(0, 0);
        const C vb = (zb < Z) ? col[zb] : CTraits<C>::make(0, 0);
        C *X = bufA + (comp * np + zp) * RS;
        if (m == 0) {
            X[0] = CTraits<C>::make(va.x, vb.x);
        } else {
            X[m] = CTraits<C>::make(va.x - vb.y, va.y + vb.x);
            X[TL - m] = CTraits<C>::make(va.x + vb.y, -va.y + vb.x);
        }
    }
    __syncthreads();
    FR::template run<+1>(bufA, rowsA, tw, tw2);
    const C *phys = bufA;
    C *prod = bufB;
    // u x curl(u) (velocity.f90:325-329), scaled for the forward transform
    const R base = (R)(1.0 - a.dm.rp[4 * g.N + n] * a.dm.rp[4 * g.N + n]);
    R mr = 0, mt = 0, mz = 0;
    for (int idx = threadIdx.x; idx < np * TL; idx += blockDim.x) {
        const int zp = idx / TL, t = idx - zp * TL;
        C u[6];
#pragma unroll
        for (int c = 0; c < 6; ++c) u[c] = phys[(c * np + zp) * RS + t];
        // .x holds row za, .y row zb
        const C pr = CTraits<C>::make((u[1].x * u[5].x - u[2].x * u[4].x) * scale,
                                      (u[1].y * u[5].y - u[2].y * u[4].y) * scale);
        const C pt = CTraits<C>::make((u[2].x * u[3].x - u[0].x * u[5].x) * scale,
                                      (u[2].y * u[3].y - u[0].y * u[5].y) * scale);
        const C pz = CTraits<C>::make((u[0].x * u[4].x - u[1].x * u[3].x) * scale,
                                      (u[0].y * u[4].y - u[1].y * u[3].y) * scale);
        prod[(0 * np + zp) * RS + t] = pr;
        prod[(1 * np + zp) * RS + t] = pt;
        prod[(2 * np + zp) * RS + t] = pz;
        const bool hasb = z0 + 2 * zp + 1 < Z;
        mr = fmax(mr, fmax(fabs(u[0].x), hasb ? fabs(u[0].y) : (R)0));
        mt = fmax(mt, fmax(fabs(u[1].x), hasb ? fabs(u[1].y) : (R)0));
        mz = fmax(mz, fmax(fabs(u[2].x + base), hasb ? fabs(u[2].y + base) : (R)0));
    }
    if (a.cfl) {
        for (int o = 16; o > 0; o >>= 1) {
            mr = fmax(mr, __shfl_xor_sync(0xffffffffu, mr, o));
            mt = fmax(mt, __shfl_xor_sync(0xffffffffu, mt, o));
            mz = fmax(mz, __shfl_xor_sync(0xffffffffu, mz, o));
        }
        if ((threadIdx.x & 31) == 0) {
            atomic_max_pos(&a.cfl[3 * n + 0], (double)mr);
            atomic_max_pos(&a.cfl[3 * n + 1], (double)mt);
            atomic_max_pos(&a.cfl[3 * n + 2], (double)mz);
        }
    }
    __syncthreads();
    FR::template run<-1>(prod, 3 * np, tw, tw2);
    // separate the two packed real transforms and keep m < M
    for (int idx = threadIdx.x; idx < 3 * M * np; idx += blockDim.x) {
        const int zp = idx % np, rest = idx / np;
        const int m = rest % M, comp = rest / M;
        const C *X = prod + (comp * np + zp) * RS;
        const C A = X[m], B = X[(TL - m) % TL];
        const C va = CTraits<C>::make((R)0.5 * (A.x + B.x), (R)0.5 * (A.y - B.y));
        const C vb = CTraits<C>::make((R)0.5 * (A.y + B.y), (R)-0.5 * (A.x - B.x));
        C *col = T + ((size_t)(comp * g.N + n) * M + m) * Z;
        const int za = z0 + 2 * zp, zb = za + 1;
        if (za < Z) col[za] = va;
        if (zb < Z) col[zb] = vb;
    }
}

template <int ZL, typename C>
__global__ void __launch_bounds__(NL_THREADS) k_nl_zfwd(NLArgs a, const C *__restrict__ T, const C *__restrict__ twz,
                                                        int MC) {
    extern __shared__ __align__(16) unsigned char smraw[];
    using FR = FFTRows<ZL, C>;
    constexpr int RS = FR::pitch;
    C *rows = reinterpret_cast<C *>(smraw);
    C *tw = rows + (FR::smem_elems(MC) - 2 * ZL), *tw2 = tw + ZL;
    const Geo &g = a.g;
    const int K = g.K;
    const int comp = blockIdx.z, n = blockIdx.y, m0 = blockIdx.x * MC;
    const int mc = min(MC, g.M - m0);
    fft4_tables<ZL>(tw, tw2, twz);
    const C *in = T + ((size_t)(comp * g.N + n) * g.M + m0) * ZL;
    for (int idx = threadIdx.x; idx < mc * ZL; idx += blockDim.x) {
        const int c = idx / ZL, j = idx - c * ZL;
        rows[c * RS + j] = in[idx];
    }
    __syncthreads();
    FR::template run<-1>(rows, mc, tw, tw2);
    const C *res = rows;
    const double U = a.dm.velU[n], b = -a.dm.velUp[n];
    double Pr0 = 0.0;
    if (comp == 2 && a.const_flux) {
        for (int j = 0; j <= KL; ++j) Pr0 += a.u[2][(size_t)(g.N - 1 - KL + j) * g.Hp].x * a.dm.dr1[1 * (KL + 1) + j];
        Pr0 = Pr0 / (-2.0);
        if (n == 0 && m0 == 0 && threadIdx.x == 0) a.sc->Pr0 = Pr0;
    }
    double2 *f = a.N[comp] + (size_t)n * g.Hp;
    for (int idx = threadIdx.x; idx < mc * (2 * K - 1); idx += blockDim.x) {
        const int c = idx / (2 * K - 1), kk = idx - c * (2 * K - 1) - (K - 1);
        const int m = m0 + c;
        if (m == 0 && kk < 0) continue;
        const int nh = m * (2 * K - 1) + kk;
        const C x = res[c * RS + (kk >= 0 ? kk : ZL + kk)];
        const size_t at = (size_t)n * g.Hp + nh;
        const double av = g.alpha * kk * U;
        double2 o = make_double2((double)x.x, (double)x.y);
        if (comp == 2) {
            const double2 vz = a.u[2][at], vr = a.u[0][at];
            o.x = o.x + av * vz.y + b * vr.x;
            o.y = o.y - av * vz.x + b * vr.y;
            if (nh == 0 && a.const_flux) o.x = o.x + 4.0 * Pr0 / g.Re;
        } else {
            const double2 v = a.u[comp][at];
            o.x = o.x + av * v.y;
            o.y = o.y - av * v.x;
        }
        f[nh] = o;
    }
}

// ------------------------------------------------------------ dispatch
#define PF_NL_LENGTHS(X) X(12) X(15) X(18) X(24) X(36) X(48) X(72) X(96) X(144) X(192) X(288) X(384)

static bool nl_length_ok(int L) {
    switch (L) {
#define PF_CASE(L) case L:
        PF_NL_LENGTHS(PF_CASE)
#undef PF_CASE
        return true;
    default:
        return false;
    }
}

bool pf_nl_fused_supported(const pf_ctx *ctx) { return nl_length_ok(ctx->g.Z) && nl_length_ok(ctx->g.Th); }

// shared-memory elements of B transform rows (plus tables) for a built length
template <typename C> static int rows_elems(int L, int B) {
    switch (L) {
#define PF_CASE(L) \
    case L:        \
        return FFTRows<L, C>::smem_elems(B);
        PF_NL_LENGTHS(PF_CASE)
#undef PF_CASE
    default:
        return 2 * B * L + 2 * L;
    }
}

template <typename C>
static int launch_nl(pf_ctx *ctx, const NLArgs &a, const C *twz, const C *twt) {
    const Geo &g = ctx->g;
    C *T = reinterpret_cast<C *>(ctx->T);
    const size_t cs = sizeof(C);
    int MC = g.M;
    while (MC > 1 && (size_t)rows_elems<C>(g.Z, MC) * cs > 64 * 1024) --MC;
    const size_t zsm = (size_t)rows_elems<C>(g.Z, MC) * cs;
    int ZC = 8;
    while (ZC > 2 && (size_t)(rows_elems<C>(g.Th, 3 * ZC) + rows_elems<C>(g.Th, 3 * ZC / 2)) * cs > 64 * 1024) ZC -= 2;
    const size_t tsm = (size_t)(rows_elems<C>(g.Th, 3 * ZC) + rows_elems<C>(g.Th, 3 * ZC / 2)) * cs;
    const dim3 gz((g.M + MC - 1) / MC, g.N, 6), gt((g.Z + ZC - 1) / ZC, g.N), gf((g.M + MC - 1) / MC, g.N, 3);
    const typename CTraits<C>::R scale = (typename CTraits<C>::R)(1.0 / (double)(g.Z * g.Th));
    switch (g.Z) {
#define PF_CASE(L)                                                                                   \
    case L: {                                                                                        \
        static size_t set_ = 0;                                                                      \
        if (zsm > set_) {                                                                              \
            PF_CUDA(cudaFuncSetAttribute(k_nl_zinv<L, C>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)zsm)); \
            set_ = zsm;                                                                               \
        }                                                                                            \
        ProfScope ps_(ctx, PF_K_ZINV);                                                               \
        k_nl_zinv<L, C><<<gz, NL_THREADS, zsm, ctx->stream>>>(a, T, twz, MC);                        \
    } break;
        PF_NL_LENGTHS(PF_CASE)
#undef PF_CASE
    default:
        pf_set_error("fused transform: unsupported Z=%d", g.Z);
        return PF_ERR_ARG;
    }
    PF_LAUNCHED(ctx);
    if (a.cfl) PF_CUDA(cudaMemsetAsync(a.cfl, 0, 3 * g.N * sizeof(unsigned long long), ctx->stream));
    switch (g.Th) {
#define PF_CASE(L)                                                                                    \
    case L: {                                                                                         \
        static size_t set_ = 0;                                                                      \
        if (tsm > set_) {                                                                              \
            PF_CUDA(cudaFuncSetAttribute(k_nl_theta<L, C>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tsm)); \
            set_ = tsm;                                                                               \
        }                                                                                            \
        ProfScope ps_(ctx, PF_K_THFWD);                                                               \
        k_nl_theta<L, C><<<gt, NL_THREADS, tsm, ctx->stream>>>(a, T, twt, ZC, scale);                 \
    } break;
        PF_NL_LENGTHS(PF_CASE)
#undef PF_CASE
    default:
        pf_set_error("fused transform: unsupported Th=%d", g.Th);
        return PF_ERR_ARG;
    }
    PF_LAUNCHED(ctx);
    switch (g.Z) {
#define PF_CASE(L)                                                                                   \
    case L: {                                                                                        \
        static size_t set_ = 0;                                                                      \
        if (zsm > set_) {                                                                              \
            PF_CUDA(cudaFuncSetAttribute(k_nl_zfwd<L, C>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)zsm)); \
            set_ = zsm;                                                                               \
        }                                                                                            \
        ProfScope ps_(ctx, PF_K_ZFWD);                                                               \
        k_nl_zfwd<L, C><<<gf, NL_THREADS, zsm, ctx->stream>>>(a, T, twz, MC);                        \
    } break;
        PF_NL_LENGTHS(PF_CASE)
#undef PF_CASE
    default:
        return PF_ERR_ARG;
    }
    PF_LAUNCHED(ctx);
    return PF_OK;
}

__global__ void k_nl_mean64(NLArgs a);

// vel_transform + vel_nonlinear in three launches; CFL maxima per radial
// point are left in ctx->cflmax.
int pf_launch_nl_fused(pf_ctx *ctx) {
    NLArgs a;
    for (int i = 0; i < 3; ++i) {
        a.u[i] = ctx->vel[i].d;
        a.N[i] = ctx->vel[3 + i].d;
    }
    a.dm = ctx->dm;
    a.g = ctx->g;
    a.const_flux = ctx->cfg.const_flux;
    a.sc = ctx->dsc;
    a.cfl = ctx->cflmax;
    if (ctx->cfg.precision == PF_PREC_MIXED) {
        PF_TRY(launch_nl<float2>(ctx, a, ctx->twZf, ctx->twTf));
        {
            ProfScope ps_(ctx, PF_K_ZFWD);
            k_nl_mean64<<<ctx->g.N, 256, 0, ctx->stream>>>(a);
        }
        PF_LAUNCHED(ctx);
        return PF_OK;
    }
    return launch_nl<double2>(ctx, a, ctx->twZ, ctx->twT);
}

// ------------------------------------------------- FP64 mean mode (mixed)
// With FP32 transforms the k=m=0 coefficient of u x curl(u) is replaced by
// its exact FP64 value.  On the 3/2-dealiased grid no product of retained
// modes aliases onto (0,0), so the grid mean equals the spectral sum
//   mean(f g) = Re f00 Re g00 + 2 sum_{k>=1} Re(f_k0 conj g_k0)
//             + 2 sum_{m>=1, all k} Re(f_km conj g_km)
// (the c2r transform ignores Im f00).  One block per radial point.
__global__ void k_nl_mean64(NLArgs a) {
    const Geo &g = a.g;
    const int n = blockIdx.x;
    double s[3] = {0.0, 0.0, 0.0};
    for (int nh = threadIdx.x; nh < g.H; nh += blockDim.x) {
        int k, m;
        mode_km(nh, g.K, k, m);
        double2 u[6];
        for (int c = 0; c < 6; ++c) u[c] = nl_input(a, c, n, nh, k, m);
        const double w = (nh == 0) ? 1.0 : 2.0;
        auto dot = [&](double2 f, double2 h) { return nh == 0 ? f.x * h.x : f.x * h.x + f.y * h.y; };
        s[0] += w * (dot(u[1], u[5]) - dot(u[2], u[4]));
        s[1] += w * (dot(u[2], u[3]) - dot(u[0], u[5]));
        s[2] += w * (dot(u[0], u[4]) - dot(u[1], u[3]));
    }
    __shared__ double red[3][32];
    for (int c = 0; c < 3; ++c) {
        double v = s[c];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if ((threadIdx.x & 31) == 0) red[c][threadIdx.x >> 5] = v;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double t[3] = {0.0, 0.0, 0.0};
        for (int c = 0; c < 3; ++c)
            for (int i = 0; i < (int)(blockDim.x >> 5); ++i) t[c] += red[c][i];
        const size_t at = (size_t)n * g.Hp;  // nh = 0
        // vel_addHPF at k=m=0: a = 0; N_z += -U' u_r (u_r(0,0) is zero after
        // imposesym but kept for fidelity) and the constant-flux pressure
        const double2 ur = a.u[0][at];
        double zr = t[2] + (-a.dm.velUp[n]) * ur.x;
        if (a.const_flux) {
            double Pr0 = 0.0;
            for (int j = 0; j <= KL; ++j) Pr0 += a.u[2][(size_t)(g.N - 1 - KL + j) * g.Hp].x * a.dm.dr1[1 * (KL + 1) + j];
            Pr0 = Pr0 / (-2.0);
            zr = zr + 4.0 * Pr0 / g.Re;
        }
        a.N[0][at] = make_double2(t[0], 0.0);
        a.N[1][at] = make_double2(t[1], 0.0);
        a.N[2][at] = make_double2(zr, (-a.dm.velUp[n]) * ur.y);
    }
}
