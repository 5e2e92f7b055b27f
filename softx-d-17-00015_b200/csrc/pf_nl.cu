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
#include <functional>
#include "pf_internal.cuh"
#include "pf_fftcore.cuh"

static constexpr int NL_THREADS = 256;
static constexpr int MEAN_THREADS = 256;  // FP64 mean-mode partial sums (mixed precision)

struct NLArgs {
    const double2 *u[3];
    double2 *N[3];
    DevMesh dm;
    Geo g;
    int const_flux;
    DevScalars *sc;
    unsigned long long *cfl;  // 3*N maxima as ordered bits
    void *T;                  // (m, z) intermediate, compute type
    const void *twz, *twt;    // twiddle tables, compute type
    int MC, ZC;               // z-pass columns and theta-pass rows per block
    double *mpart;            // FP64 mean-mode partial sums [ceil(H/32)][N][3]
    float2 *curlf;            // mixed precision: curl(u) in FP32, [(c*N + n)*Hp + nh], made by the
                              // mean-mode pass before the z pass reads it (null in FP64)
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
    if (comp < 3) return pick3(a.u, comp)[at];
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
__device__ __forceinline__ void nl_zinv_body(const NLArgs &a, int bx, int by, int bz) {
    extern __shared__ __align__(16) unsigned char smraw[];
    C *__restrict__ T = reinterpret_cast<C *>(a.T);
    const C *__restrict__ twz = reinterpret_cast<const C *>(a.twz);
    const int MC = a.MC;
    if (a.cfl && bx == 0 && by == 0 && bz == 0)  // reset the CFL maxima the theta pass raises
        for (int i = threadIdx.x; i < 3 * a.g.N; i += blockDim.x) a.cfl[i] = 0ull;
    using FR = FFTRows<ZL, C>;
    constexpr int RS = FR::pitch;
    C *rows = reinterpret_cast<C *>(smraw);
    C *tw = rows + (FR::smem_elems(MC) - 2 * ZL), *tw2 = tw + ZL;
    const Geo &g = a.g;
    const int K = g.K;
    const int comp = bz, n = by, m0 = bx * MC;
    const int mc = min(MC, g.M - m0);
    fft4_tables<ZL>(tw, tw2, twz);
    // FP32 transforms (mixed precision): u, or the curl(u) the mean-mode pass
    // formed once; FP64: u, or curl(u) from 9-row stencils here
    const float2 *__restrict__ cf = (a.curlf && comp >= 3) ? a.curlf + (size_t)((comp - 3) * g.N + n) * g.Hp : nullptr;
    const double2 *__restrict__ uc = comp < 3 ? pick3(a.u, comp) + (size_t)n * g.Hp : nullptr;
    auto input = [&](int nh, int k, int m) -> C {
        if constexpr (sizeof(C) == 8) {
            return comp >= 3 ? cf[nh] : to_c<C>(uc[nh]);
        } else {
            return to_c<C>(nl_input(a, comp, n, nh, k, m));
        }
    };
#pragma unroll 4
    for (int idx = threadIdx.x; idx < mc * ZL; idx += blockDim.x) {
        const int c = idx / ZL, j = idx - c * ZL;
        const int m = m0 + c;
        C v = CTraits<C>::make(0, 0);
        if (m == 0) {
            if (j < K) v = input(j, j, 0);
            else if (j >= 2 * K + 1) {
                v = input(ZL - j, ZL - j, 0);
                v.y = -v.y;
            }
        } else {
            const int kk = j < K ? j : (j >= 2 * K + 1 ? j - ZL : K);
            if (kk < K) v = input(m * (2 * K - 1) + kk, kk, m);
        }
        rows[c * RS + j] = v;
    }
    __syncthreads();
    FR::template run<+1>(rows, mc, tw, tw2);
    C *out = T + ((size_t)(comp * g.N + n) * g.M + m0) * ZL;
    if constexpr (sizeof(C) == 8 && ZL % 2 == 0) {
        // FP32, even length: two z values per 16-byte store (every column
        // of the intermediate starts on a 16-byte boundary)
        for (int idx = threadIdx.x; idx < mc * ZL / 2; idx += blockDim.x) {
            const int c = (2 * idx) / ZL, j = 2 * idx - c * ZL;
            const C x0 = rows[c * RS + j], x1 = rows[c * RS + j + 1];
            reinterpret_cast<float4 *>(out)[idx] = make_float4(x0.x, x0.y, x1.x, x1.y);
        }
    } else {
        for (int idx = threadIdx.x; idx < mc * ZL; idx += blockDim.x) {
            const int c = idx / ZL, j = idx - c * ZL;
            out[idx] = rows[c * RS + j];
        }
    }
}

__device__ __forceinline__ void atomic_max_pos(unsigned long long *p, double v) {
    atomicMax(p, (unsigned long long)__double_as_longlong(v));
}

// u x curl(u) (velocity.f90:325-329) of two packed physical rows (.x row za,
// .y row zb), scaled for the forward transform; u = (u_r, u_t, u_z, curl)
template <typename C, typename R>
__device__ __forceinline__ void cross_scaled(const C (&u)[6], R scale, C &pr, C &pt, C &pz) {
    pr = CTraits<C>::make((u[1].x * u[5].x - u[2].x * u[4].x) * scale, (u[1].y * u[5].y - u[2].y * u[4].y) * scale);
    pt = CTraits<C>::make((u[2].x * u[3].x - u[0].x * u[5].x) * scale, (u[2].y * u[3].y - u[0].y * u[5].y) * scale);
    pz = CTraits<C>::make((u[0].x * u[4].x - u[1].x * u[3].x) * scale, (u[0].y * u[4].y - u[1].y * u[3].y) * scale);
}

// the z-forward epilogue at one kept mode: the transformed product x plus
// vel_addHPF's terms (velocity.f90:338-361); v = u_comp, vr = u_r there
__device__ __forceinline__ double2 hpf_out(double2 o, int comp, double av, double b, double2 v, double2 vr,
                                           bool pr0, double Pr0, double Re) {
    if (comp == 2) {
        o.x = o.x + av * v.y + b * vr.x;
        o.y = o.y - av * v.x + b * vr.y;
        if (pr0) o.x = o.x + 4.0 * Pr0 / Re;
    } else {
        o.x = o.x + av * v.y;
        o.y = o.y - av * v.x;
    }
    return o;
}

// Whether the z-row pair (za, zb = za + 1) of an (m, z) column moves as one
// 16-byte access: FP32 values, an even Z (every column then starts on a
// 16-byte boundary and za, a tile start plus twice the pair index, is even)
// and both rows inside the column.
template <typename C> __device__ __forceinline__ bool pair16(int Z, int zb) {
    return sizeof(C) == 8 && (Z & 1) == 0 && zb < Z;
}

template <int TL, typename C>
__device__ __forceinline__ void nl_theta_body(const NLArgs &a, int bx, int by) {
    using R = typename CTraits<C>::R;
    extern __shared__ __align__(16) unsigned char smraw[];
    C *__restrict__ T = reinterpret_cast<C *>(a.T);
    const C *__restrict__ twt = reinterpret_cast<const C *>(a.twt);
    const int ZC = a.ZC;
    const R scale = (R)(1.0 / (double)(a.g.Z * a.g.Th));  // transform.fftw3.f90:114
    using FR = FFTRows<TL, C>;
    constexpr int RS = FR::pitch;
    const Geo &g = a.g;
    const int M = g.M, Z = g.Z, np = ZC / 2;
    const int rowsA = 3 * ZC;  // six components x ZC/2 packed pairs
    C *bufA = reinterpret_cast<C *>(smraw);
    // the products overwrite the first three components' rows in place
    C *tw = bufA + (FR::smem_elems(rowsA) - 2 * TL), *tw2 = tw + TL;
    const int n = by, z0 = bx * ZC;
    fft4_tables<TL>(tw, tw2, twt);
    // Hermitian-extend the M retained theta modes of two z rows into one
    // complex row: X = a + i b (c2r ignores the DC imaginary parts).  With
    // TL = 3M every entry is written once: X[m] and X[TL-m] by mode m's
    // thread, which also clears X[M+m] of the zero band (and m = 0 X[2M])
    const float inp = 1.0f / np, inM = 1.0f / M;
#pragma unroll 4
    for (int idx = threadIdx.x; idx < 6 * M * np; idx += blockDim.x) {
        const int rest = fdiv(idx, np, inp), zp = idx - rest * np;
        const int comp = fdiv(rest, M, inM), m = rest - comp * M;
        const int za = z0 + 2 * zp, zb = za + 1;
        const C *col = T + ((size_t)(comp * g.N + n) * M + m) * Z;
        C va, vb;
        if (pair16<C>(Z, zb)) {  // both rows in one 16-byte load (FP32, even Z: za even, col 16-byte aligned)
            const float4 q = *reinterpret_cast<const float4 *>(col + za);
            va = CTraits<C>::make(q.x, q.y);
            vb = CTraits<C>::make(q.z, q.w);
        } else {
            va = (za < Z) ? col[za] : CTraits<C>::make(0, 0);
            vb = (zb < Z) ? col[zb] : CTraits<C>::make(0, 0);
        }
        C *X = bufA + (comp * np + zp) * RS;
        X[M + m] = CTraits<C>::make(0, 0);
        if (m == 0) {
            X[0] = CTraits<C>::make(va.x, vb.x);
            X[2 * M] = CTraits<C>::make(0, 0);
        } else {
            X[m] = CTraits<C>::make(va.x - vb.y, va.y + vb.x);
            X[TL - m] = CTraits<C>::make(va.x + vb.y, -va.y + vb.x);
        }
    }
    __syncthreads();
    FR::template run<+1>(bufA, rowsA, tw, tw2);
    const C *phys = bufA;
    C *prod = bufA;  // row (c*np + zp) of component c < 3: read above, then rewritten by the same thread
    // u x curl(u) (velocity.f90:325-329), scaled for the forward transform
    const R base = (R)(1.0 - a.dm.rp[4 * g.N + n] * a.dm.rp[4 * g.N + n]);
    R mr = 0, mt = 0, mz = 0;
    for (int idx = threadIdx.x; idx < np * TL; idx += blockDim.x) {
        const int zp = idx / TL, t = idx - zp * TL;
        C u[6];
#pragma unroll
        for (int c = 0; c < 6; ++c) u[c] = phys[(c * np + zp) * RS + t];
        // .x holds row za, .y row zb
        C pr, pt, pz;
        cross_scaled(u, scale, pr, pt, pz);
        prod[(0 * np + zp) * RS + t] = pr;
        prod[(1 * np + zp) * RS + t] = pt;
        prod[(2 * np + zp) * RS + t] = pz;
        // grid points only: a pair past Z (the last tile's padding) is no point
        if (z0 + 2 * zp < Z) {
            const bool hasb = z0 + 2 * zp + 1 < Z;
            mr = fmax(mr, fmax(fabs(u[0].x), hasb ? fabs(u[0].y) : (R)0));
            mt = fmax(mt, fmax(fabs(u[1].x), hasb ? fabs(u[1].y) : (R)0));
            mz = fmax(mz, fmax(fabs(u[2].x + base), hasb ? fabs(u[2].y + base) : (R)0));
        }
    }
    __shared__ double cflw[3][NL_THREADS / 32];  // warp maxima; three atomics per block
    if (a.cfl) {
        for (int o = 16; o > 0; o >>= 1) {
            mr = fmax(mr, __shfl_xor_sync(0xffffffffu, mr, o));
            mt = fmax(mt, __shfl_xor_sync(0xffffffffu, mt, o));
            mz = fmax(mz, __shfl_xor_sync(0xffffffffu, mz, o));
        }
        if ((threadIdx.x & 31) == 0) {
            cflw[0][threadIdx.x >> 5] = (double)mr;
            cflw[1][threadIdx.x >> 5] = (double)mt;
            cflw[2][threadIdx.x >> 5] = (double)mz;
        }
    }
    __syncthreads();
    if (a.cfl && threadIdx.x < 3) {
        double v = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) v = fmax(v, cflw[threadIdx.x][w]);
        atomic_max_pos(&a.cfl[3 * n + threadIdx.x], v);
    }
    FR::template run<-1>(prod, 3 * np, tw, tw2);
    // separate the two packed real transforms and keep m < M
    for (int idx = threadIdx.x; idx < 3 * M * np; idx += blockDim.x) {
        const int rest = fdiv(idx, np, inp), zp = idx - rest * np;
        const int comp = fdiv(rest, M, inM), m = rest - comp * M;
        const C *X = prod + (comp * np + zp) * RS;
        const C A = X[m], B = X[(TL - m) % TL];
        const C va = CTraits<C>::make((R)0.5 * (A.x + B.x), (R)0.5 * (A.y - B.y));
        const C vb = CTraits<C>::make((R)0.5 * (A.y + B.y), (R)-0.5 * (A.x - B.x));
        C *col = T + ((size_t)(comp * g.N + n) * M + m) * Z;
        const int za = z0 + 2 * zp, zb = za + 1;
        if (pair16<C>(Z, zb)) {
            *reinterpret_cast<float4 *>(col + za) = make_float4(va.x, va.y, vb.x, vb.y);
        } else {
            if (za < Z) col[za] = va;
            if (zb < Z) col[zb] = vb;
        }
    }
}

template <int ZL, typename C>
__device__ __forceinline__ void nl_zfwd_body(const NLArgs &a, int bx, int by, int bz) {
    extern __shared__ __align__(16) unsigned char smraw[];
    const C *__restrict__ T = reinterpret_cast<const C *>(a.T);
    const C *__restrict__ twz = reinterpret_cast<const C *>(a.twz);
    const int MC = a.MC;
    using FR = FFTRows<ZL, C>;
    constexpr int RS = FR::pitch;
    C *rows = reinterpret_cast<C *>(smraw);
    C *tw = rows + (FR::smem_elems(MC) - 2 * ZL), *tw2 = tw + ZL;
    const Geo &g = a.g;
    const int K = g.K;
    const int comp = bz, n = by, m0 = bx * MC;
    const int mc = min(MC, g.M - m0);
    fft4_tables<ZL>(tw, tw2, twz);
    const C *in = T + ((size_t)(comp * g.N + n) * g.M + m0) * ZL;
    if constexpr (sizeof(C) == 8 && ZL % 2 == 0) {  // FP32, even length: 16-byte loads
        for (int idx = threadIdx.x; idx < mc * ZL / 2; idx += blockDim.x) {
            const int c = (2 * idx) / ZL, j = 2 * idx - c * ZL;
            const float4 q = reinterpret_cast<const float4 *>(in)[idx];
            rows[c * RS + j] = CTraits<C>::make(q.x, q.y);
            rows[c * RS + j + 1] = CTraits<C>::make(q.z, q.w);
        }
    } else {
        for (int idx = threadIdx.x; idx < mc * ZL; idx += blockDim.x) {
            const int c = idx / ZL, j = idx - c * ZL;
            rows[c * RS + j] = in[idx];
        }
    }
    __syncthreads();
    FR::template run<-1>(rows, mc, tw, tw2);
    const C *res = rows;
    const double U = a.dm.velU[n], b = -a.dm.velUp[n];
    // the constant-flux pressure Pr0 enters at k = m = 0 only: the first
    // m-chunk of the axial component needs it (vel_addHPF, velocity.f90:355-359)
    double Pr0 = 0.0;
    if (comp == 2 && a.const_flux && m0 == 0) {
        for (int j = 0; j <= KL; ++j) Pr0 += a.u[2][(size_t)(g.N - 1 - KL + j) * g.Hp].x * a.dm.dr1[1 * (KL + 1) + j];
        Pr0 = Pr0 / (-2.0);
        if (n == 0 && threadIdx.x == 0) a.sc->Pr0 = Pr0;
    }
    double2 *__restrict__ f = pick3(a.N, comp) + (size_t)n * g.Hp;
    const double2 *__restrict__ uc = pick3(a.u, comp) + (size_t)n * g.Hp;
    const double2 *__restrict__ ur0 = a.u[0] + (size_t)n * g.Hp;
    const float ik = 1.0f / (2 * K - 1);
#pragma unroll 4
    for (int idx = threadIdx.x; idx < mc * (2 * K - 1); idx += blockDim.x) {
        const int c = fdiv(idx, 2 * K - 1, ik), kk = idx - c * (2 * K - 1) - (K - 1);
        const int m = m0 + c;
        if (m == 0 && kk < 0) continue;
        const int nh = m * (2 * K - 1) + kk;
        const C x = res[c * RS + (kk >= 0 ? kk : ZL + kk)];
        const double av = g.alpha * kk * U;
        const double2 vr = comp == 2 ? ur0[nh] : make_double2(0.0, 0.0);
        f[nh] = hpf_out(make_double2((double)x.x, (double)x.y), comp, av, b, uc[nh], vr, nh == 0 && a.const_flux,
                        Pr0, g.Re);
    }
}

// ------------------------------------------- one radial point in one block
// Mixed precision (FP32 transforms): the z inverse, theta pass and z forward
// of one radial point n run in one block with the (m, z) plane of all six
// components held in shared memory, so the intermediate never leaves the
// SM.  The arithmetic is the three-pass kernels' own (the same row FFTs on
// the same data, the same product and epilogue), so the results are bitwise
// theirs; only where the data waits between the passes differs.
//   plane P[(c*M + m)*PZ + z]  six components x M rows of the z transform
//   rows  Q[(c*np + zp)*PT + t] the theta rows of one chunk of ZC z rows
// The block sees every z of its radial point, so it stores the CFL maxima
// of n outright (no reset, no atomics).
static constexpr int FUSED_THREADS = 512;

// theta-row pitch: the four-step pitch made odd, so the gather's column
// writes of consecutive z-row pairs fall in distinct banks
__host__ __device__ constexpr int fused_tpitch(int L) { return fft4_pitch(L) | 1; }

template <int ZL, int TL>
__host__ __device__ constexpr size_t fused_smem(int M, int ZC) {
    return ((size_t)6 * M * fft4_pitch(ZL) + (size_t)3 * ZC * fused_tpitch(TL) + 2 * ZL + 2 * TL) * sizeof(float2);
}

template <int ZL, int TL>
__device__ __forceinline__ void nl_fused_body(const NLArgs &a, int n) {
    extern __shared__ __align__(16) unsigned char smraw[];
    constexpr int PZ = fft4_pitch(ZL), PT = fused_tpitch(TL);
    const Geo &g = a.g;
    const int K = g.K, M = g.M, Z = ZL;
    const int ZC = a.ZC, np = ZC / 2;
    float2 *P = reinterpret_cast<float2 *>(smraw);
    float2 *Q = P + 6 * M * PZ;
    float2 *twz = Q + 3 * ZC * PT, *twz2 = twz + ZL, *twt = twz2 + ZL, *twt2 = twt + TL;
    fft4_tables<ZL>(twz, twz2, reinterpret_cast<const float2 *>(a.twz));
    fft4_tables<TL>(twt, twt2, reinterpret_cast<const float2 *>(a.twt));
    const size_t Hp = g.Hp, fs = (size_t)g.N * Hp;
    // z inverse input: u, or the FP32 curl(u) of the mean-mode pass,
    // zero-padded to ZL with the Hermitian fill of m = 0 (as k_nl_zinv)
    const float inZ = 1.0f / ZL, inM = 1.0f / M;
#pragma unroll 4
    for (int idx = threadIdx.x; idx < 6 * M * ZL; idx += blockDim.x) {
        const int r = fdiv(idx, ZL, inZ), j = idx - r * ZL;
        const int comp = fdiv(r, M, inM), m = r - comp * M;
        int nh = -1;
        bool conj = false;
        if (m == 0) {
            if (j < K) nh = j;
            else if (j >= 2 * K + 1) nh = ZL - j, conj = true;
        } else {
            const int kk = j < K ? j : (j >= 2 * K + 1 ? j - ZL : K);
            if (kk < K) nh = m * (2 * K - 1) + kk;
        }
        float2 v = make_float2(0.f, 0.f);
        if (nh >= 0) {
            const size_t at = (size_t)n * Hp + nh;
            v = comp < 3 ? to_c<float2>(pick3(a.u, comp)[at]) : a.curlf[(comp - 3) * fs + at];
            if (conj) v.y = -v.y;
        }
        P[r * PZ + j] = v;
    }
    __syncthreads();
    fft4_rows<ZL, +1>(P, 6 * M, PZ, twz, twz2);
    // theta pass, ZC z rows at a time (as k_nl_theta)
    const float scale = (float)(1.0 / (double)(g.Z * g.Th));
    const float base = (float)(1.0 - a.dm.rp[4 * g.N + n] * a.dm.rp[4 * g.N + n]);
    float mr = 0, mt = 0, mz = 0;
    const float inp = 1.0f / np, inT = 1.0f / TL;
    for (int z0 = 0; z0 < Z; z0 += ZC) {
        // the Hermitian extension of M theta modes of two z rows as one
        // complex row, written entry by entry (zeros included)
        for (int idx = threadIdx.x; idx < 6 * np * TL; idx += blockDim.x) {
            const int rest = fdiv(idx, np, inp), zp = idx - rest * np;
            const int comp = fdiv(rest, TL, inT), t = rest - comp * TL;
            const int za = z0 + 2 * zp, zb = za + 1;
            const int m = t < M ? t : (t > TL - M ? TL - t : -1);
            float2 x = make_float2(0.f, 0.f);
            if (m >= 0) {
                const float2 *row = P + (comp * M + m) * PZ;
                const float2 va = za < Z ? row[za] : make_float2(0.f, 0.f);
                const float2 vb = zb < Z ? row[zb] : make_float2(0.f, 0.f);
                if (m == 0) x = make_float2(va.x, vb.x);
                else if (t == m) x = make_float2(va.x - vb.y, va.y + vb.x);
                else x = make_float2(va.x + vb.y, -va.y + vb.x);
            }
            Q[(comp * np + zp) * PT + t] = x;
        }
        __syncthreads();
        fft4_rows<TL, +1>(Q, 6 * np, PT, twt, twt2);
        // u x curl(u) (velocity.f90:325-329) in place over the first three
        // components' rows, scaled for the forward transform
        for (int idx = threadIdx.x; idx < np * TL; idx += blockDim.x) {
            const int zp = fdiv(idx, TL, inT), t = idx - zp * TL;
            float2 u[6];
#pragma unroll
            for (int c = 0; c < 6; ++c) u[c] = Q[(c * np + zp) * PT + t];
            float2 pr, pt, pz;
            cross_scaled(u, scale, pr, pt, pz);
            Q[(0 * np + zp) * PT + t] = pr;
            Q[(1 * np + zp) * PT + t] = pt;
            Q[(2 * np + zp) * PT + t] = pz;
            const int za = z0 + 2 * zp;
            if (za < Z) {
                const bool hasb = za + 1 < Z;
                mr = fmaxf(mr, fmaxf(fabsf(u[0].x), hasb ? fabsf(u[0].y) : 0.f));
                mt = fmaxf(mt, fmaxf(fabsf(u[1].x), hasb ? fabsf(u[1].y) : 0.f));
                mz = fmaxf(mz, fmaxf(fabsf(u[2].x + base), hasb ? fabsf(u[2].y + base) : 0.f));
            }
        }
        __syncthreads();
        fft4_rows<TL, -1>(Q, 3 * np, PT, twt, twt2);
        // separate the two packed real transforms, keep m < M, back into the
        // plane rows of the first three components
        for (int idx = threadIdx.x; idx < 3 * M * np; idx += blockDim.x) {
            const int rest = fdiv(idx, np, inp), zp = idx - rest * np;
            const int comp = fdiv(rest, M, inM), m = rest - comp * M;
            const float2 *X = Q + (comp * np + zp) * PT;
            const float2 A = X[m], B = X[(TL - m) % TL];
            const int za = z0 + 2 * zp, zb = za + 1;
            float2 *row = P + (comp * M + m) * PZ;
            if (za < Z) row[za] = make_float2(0.5f * (A.x + B.x), 0.5f * (A.y - B.y));
            if (zb < Z) row[zb] = make_float2(0.5f * (A.y + B.y), -0.5f * (A.x - B.x));
        }
        __syncthreads();
    }
    __shared__ float cflw[3][FUSED_THREADS / 32];
    if (a.cfl) {
        for (int o = 16; o > 0; o >>= 1) {
            mr = fmaxf(mr, __shfl_xor_sync(0xffffffffu, mr, o));
            mt = fmaxf(mt, __shfl_xor_sync(0xffffffffu, mt, o));
            mz = fmaxf(mz, __shfl_xor_sync(0xffffffffu, mz, o));
        }
        if ((threadIdx.x & 31) == 0) {
            cflw[0][threadIdx.x >> 5] = mr;
            cflw[1][threadIdx.x >> 5] = mt;
            cflw[2][threadIdx.x >> 5] = mz;
        }
    }
    fft4_rows<ZL, -1>(P, 3 * M, PZ, twz, twz2);  // synchronises first: cflw is complete after it
    if (a.cfl && threadIdx.x < 3) {
        float v = 0.f;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) v = fmaxf(v, cflw[threadIdx.x][w]);
        a.cfl[3 * n + threadIdx.x] = (unsigned long long)__double_as_longlong((double)v);
    }
    // truncation to |k| < K and vel_addHPF (as k_nl_zfwd)
    const double U = a.dm.velU[n], b = -a.dm.velUp[n];
    double Pr0 = 0.0;
    if (a.const_flux) {
        for (int j = 0; j <= KL; ++j) Pr0 += a.u[2][(size_t)(g.N - 1 - KL + j) * Hp].x * a.dm.dr1[1 * (KL + 1) + j];
        Pr0 = Pr0 / (-2.0);
        if (n == 0 && threadIdx.x == 0) a.sc->Pr0 = Pr0;
    }
    const double2 *__restrict__ ur0 = a.u[0] + (size_t)n * Hp;
    const float ik = 1.0f / (2 * K - 1), inMH = 1.0f / (M * (2 * K - 1));
#pragma unroll 4
    for (int idx = threadIdx.x; idx < 3 * M * (2 * K - 1); idx += blockDim.x) {
        const int comp = fdiv(idx, M * (2 * K - 1), inMH), rest = idx - comp * M * (2 * K - 1);
        const int m = fdiv(rest, 2 * K - 1, ik), kk = rest - m * (2 * K - 1) - (K - 1);
        if (m == 0 && kk < 0) continue;
        const int nh = m * (2 * K - 1) + kk;
        const float2 x = P[(comp * M + m) * PZ + (kk >= 0 ? kk : ZL + kk)];
        const double av = g.alpha * kk * U;
        const double2 vr = comp == 2 ? ur0[nh] : make_double2(0.0, 0.0);
        pick3(a.N, comp)[(size_t)n * Hp + nh] =
            hpf_out(make_double2((double)x.x, (double)x.y), comp, av, b, pick3(a.u, comp)[(size_t)n * Hp + nh], vr,
                    nh == 0 && a.const_flux, Pr0, g.Re);
    }
}

// Resident blocks per SM the transform kernels are compiled for.  In FP32,
// up to length 192, the register caps these imply cost a few spilled bytes
// and the extra warps
// hide the passes' barrier and shared-memory latency (measured: 4.94 ms ->
// 4.73 ms per 64-pipe mixed batch step).  In FP64, for transform lengths
// of 144 and more, three blocks (80 registers) are the best trade (the
// single N=64 K=128 M=48 pipe: 1.258 -> 1.21 ms per step); shorter FP64
// rows keep the compiler's own register choice (0: no minimum).
template <typename C, int L> struct NLOcc {
    static constexpr int zinv = L >= 144 ? 3 : 0, theta = L >= 144 ? 3 : 0, zfwd = L >= 144 ? 3 : 0;
};
template <int L> struct NLOcc<float2, L> {
    static constexpr int zinv = L <= 192 ? 5 : 0, theta = L <= 192 ? 6 : 0, zfwd = L <= 192 ? 5 : 0;
};

template <int ZL, typename C>
__global__ void __launch_bounds__(NL_THREADS, (NLOcc<C, ZL>::zinv)) k_nl_zinv(NLArgs a) {
    nl_zinv_body<ZL, C>(a, blockIdx.x, blockIdx.y, blockIdx.z);
}
template <int TL, typename C>
__global__ void __launch_bounds__(NL_THREADS, (NLOcc<C, TL>::theta)) k_nl_theta(NLArgs a) {
    nl_theta_body<TL, C>(a, blockIdx.x, blockIdx.y);
}
template <int ZL, typename C>
__global__ void __launch_bounds__(NL_THREADS, (NLOcc<C, ZL>::zfwd)) k_nl_zfwd(NLArgs a) {
    nl_zfwd_body<ZL, C>(a, blockIdx.x, blockIdx.y, blockIdx.z);
}
template <int ZL, int TL>
__global__ void __launch_bounds__(FUSED_THREADS, 1) k_nl_fused(NLArgs a) {
    nl_fused_body<ZL, TL>(a, blockIdx.x);
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
static bool fused_plan(const Geo &g, const pf_tuning &tu, bool mixed, int *ZC, size_t *smem);

extern "C" int pf_nl_passes(const pf_ctx *ctx, int *passes) {
    PF_ARG(ctx && passes, "pf_nl_passes: null argument");
    int zc = 0;
    size_t sm = 0;
    *passes = fused_plan(ctx->g, ctx->tune, ctx->cfg.precision == PF_PREC_MIXED, &zc, &sm) ? 1 : 3;
    return PF_OK;
}

// (Z, Th) pairs the one-block-per-radial-point kernel is built for: the
// batched mix's shapes whose six-component plane fits in shared memory,
// config-1, and the small test shapes
#define PF_NL_FUSED_PAIRS(X) \
    X(12, 12) X(18, 15) X(15, 18) X(72, 48) X(48, 36) X(48, 72) X(48, 96) X(96, 36) X(96, 72) X(96, 96) X(192, 36)

static size_t fused_smem_of(int Z, int Th, int M, int ZC) {
#define PF_CASE(ZL, TL) \
    if (Z == ZL && Th == TL) return fused_smem<ZL, TL>(M, ZC);
    PF_NL_FUSED_PAIRS(PF_CASE)
#undef PF_CASE
    return 0;
}
static constexpr size_t FUSED_MAX_SMEM = 224 * 1024;  // below the 227 KB per block, with the static maxima

// Whether a pipe's transforms run as one block per radial point, and the
// theta chunk and shared memory they take there: a tuning that asks for it,
// mixed precision, a built (Z, Th) pair and a plane that fits.  The built-in
// choice is the three passes: on the 64-pipe mix the one-block kernel took
// 1.23 ms per evaluation against 1.01 ms (one 16-warp block per SM at
// 86-128 registers; the three passes keep many more warps resident, and the
// stages are bound by latency and barriers, not by the plane's HBM traffic).
static bool fused_plan(const Geo &g, const pf_tuning &tu, bool mixed, int *ZC, size_t *smem) {
    if (!mixed || !tu.nl_fused || fused_smem_of(g.Z, g.Th, g.M, 2) == 0) return false;
    int zc = tu.nl_zc > 0 ? tu.nl_zc : 16;
    while (zc > 2 && fused_smem_of(g.Z, g.Th, g.M, zc) > FUSED_MAX_SMEM) zc -= 2;
    const size_t sm = fused_smem_of(g.Z, g.Th, g.M, zc);
    if (sm > FUSED_MAX_SMEM) return false;
    *ZC = zc;
    *smem = sm;
    return true;
}

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

// tiles and shared memory of one pipe's three launches
template <typename C> struct NLTiles {
    int MC, ZC;
    size_t zsm, tsm;
};
static constexpr size_t NL_TILE_MAX_SMEM = 100 * 1024;  // largest tile a tuning may choose

template <typename C> static size_t theta_smem(int Th, int ZC) { return (size_t)rows_elems<C>(Th, 3 * ZC) * sizeof(C); }

// Tiles of the three transform passes: the tuning's choice where it set one,
// else the built-in rule.
template <typename C> static NLTiles<C> nl_tiles(const Geo &g, const pf_tuning &tu) {
    const size_t cs = sizeof(C);
    NLTiles<C> t;
    // built-in: FP32 z-pass tiles up to 32 KB and theta tiles of up to 16 z
    // rows (measured 4.73 -> 4.59 ms per 64-pipe batch step with the kernels'
    // five-to-six-block launch bounds); FP64: up to 64 KB and 8 rows
    const bool f32 = cs == 8;
    if (tu.nl_mc > 0) {
        t.MC = std::min(tu.nl_mc, g.M);
    } else {
        t.MC = g.M;
        while (t.MC > 1 && (size_t)rows_elems<C>(g.Z, t.MC) * cs > (f32 ? 32 : 64) * 1024) --t.MC;
    }
    t.zsm = (size_t)rows_elems<C>(g.Z, t.MC) * cs;
    if (tu.nl_zc > 0) {
        t.ZC = tu.nl_zc;
    } else {
        t.ZC = f32 ? 16 : 8;
        while (t.ZC > 2 && theta_smem<C>(g.Th, t.ZC) > 64 * 1024) t.ZC -= 2;
    }
    t.tsm = theta_smem<C>(g.Th, t.ZC);
    return t;
}

// A tuning's tiles must be even-rowed and fit the shared-memory cap.
int pf_nl_tiles_check(const pf_ctx *ctx, const pf_tuning *tu) {
    PF_ARG(tu->nl_mc >= 0 && tu->nl_zc >= 0 && tu->nl_zc <= 32 && tu->nl_zc % 2 == 0,
           "pf_ctx_set_tuning: nl_mc >= 0, nl_zc even in 0..32");
    if (!pf_nl_fused_supported(ctx)) return PF_OK;
    const bool mixed = ctx->cfg.precision == PF_PREC_MIXED;
    const size_t zsm = mixed ? nl_tiles<float2>(ctx->g, *tu).zsm : nl_tiles<double2>(ctx->g, *tu).zsm;
    const size_t tsm = mixed ? nl_tiles<float2>(ctx->g, *tu).tsm : nl_tiles<double2>(ctx->g, *tu).tsm;
    if (zsm > NL_TILE_MAX_SMEM || tsm > NL_TILE_MAX_SMEM) {
        pf_set_error("pf_ctx_set_tuning: transform tiles need %zu / %zu bytes of shared memory (cap %zu)", zsm, tsm,
                     NL_TILE_MAX_SMEM);
        return PF_ERR_ARG;
    }
    return PF_OK;
}

// The fused-transform arguments of one pipe in its current pointer state.
static NLArgs make_nl_args(pf_ctx *ctx) {
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
    a.T = ctx->T;
    a.mpart = ctx->mpart;
    const bool mixed = ctx->cfg.precision == PF_PREC_MIXED;
    // FP32 transforms use the first 6*N*M*Z float2 of T; the curl fields follow
    a.curlf = mixed ? reinterpret_cast<float2 *>(ctx->T) + (size_t)6 * ctx->g.N * ctx->g.M * ctx->g.Z : nullptr;
    a.twz = mixed ? (const void *)ctx->twZf : (const void *)ctx->twZ;
    a.twt = mixed ? (const void *)ctx->twTf : (const void *)ctx->twT;
    int fzc = 0;
    size_t fsm = 0;
    if (mixed) {
        const NLTiles<float2> t = nl_tiles<float2>(ctx->g, ctx->tune);
        a.MC = t.MC;
        a.ZC = fused_plan(ctx->g, ctx->tune, true, &fzc, &fsm) ? fzc : t.ZC;
    } else {
        const NLTiles<double2> t = nl_tiles<double2>(ctx->g, ctx->tune);
        a.MC = t.MC;
        a.ZC = t.ZC;
    }
    return a;
}

// cur: the largest limit this call site asked for; the limit itself is kept
// per device by pf_raise_smem, which every call consults (a process may
// drive several devices)
template <typename K> static int raise_smem(K kernel, size_t bytes, size_t &cur) {
    PF_TRY(pf_raise_smem((const void *)kernel, bytes));
    cur = std::max(cur, bytes);
    return PF_OK;
}

template <typename C>
static int launch_nl(pf_ctx *ctx, const NLArgs &a) {
    const Geo &g = ctx->g;
    int fzc = 0;
    size_t fsm = 0;
    if (fused_plan(g, ctx->tune, sizeof(C) == 8, &fzc, &fsm)) {
        ProfScope ps_(ctx, PF_K_THFWD);
#define PF_CASE(ZL, TL)                                                   \
    if (g.Z == ZL && g.Th == TL) {                                        \
        static size_t set_ = 0;                                           \
        PF_TRY(raise_smem(k_nl_fused<ZL, TL>, fsm, set_));                \
        k_nl_fused<ZL, TL><<<g.N, FUSED_THREADS, fsm, ctx->stream>>>(a);  \
    }
        PF_NL_FUSED_PAIRS(PF_CASE)
#undef PF_CASE
        PF_LAUNCHED(ctx);
        return PF_OK;
    }
    const NLTiles<C> t = nl_tiles<C>(g, ctx->tune);
    const dim3 gz((g.M + t.MC - 1) / t.MC, g.N, 6), gt((g.Z + t.ZC - 1) / t.ZC, g.N), gf((g.M + t.MC - 1) / t.MC, g.N, 3);
    switch (g.Z) {
#define PF_CASE(L)                                                    \
    case L: {                                                         \
        static size_t set_ = 0;                                       \
        PF_TRY(raise_smem(k_nl_zinv<L, C>, t.zsm, set_));             \
        ProfScope ps_(ctx, PF_K_ZINV);                                \
        k_nl_zinv<L, C><<<gz, NL_THREADS, t.zsm, ctx->stream>>>(a);   \
    } break;
        PF_NL_LENGTHS(PF_CASE)
#undef PF_CASE
    default:
        pf_set_error("fused transform: unsupported Z=%d", g.Z);
        return PF_ERR_ARG;
    }
    PF_LAUNCHED(ctx);
    switch (g.Th) {
#define PF_CASE(L)                                                    \
    case L: {                                                         \
        static size_t set_ = 0;                                       \
        PF_TRY(raise_smem(k_nl_theta<L, C>, t.tsm, set_));            \
        ProfScope ps_(ctx, PF_K_THFWD);                               \
        k_nl_theta<L, C><<<gt, NL_THREADS, t.tsm, ctx->stream>>>(a);  \
    } break;
        PF_NL_LENGTHS(PF_CASE)
#undef PF_CASE
    default:
        pf_set_error("fused transform: unsupported Th=%d", g.Th);
        return PF_ERR_ARG;
    }
    PF_LAUNCHED(ctx);
    switch (g.Z) {
#define PF_CASE(L)                                                    \
    case L: {                                                         \
        static size_t set_ = 0;                                       \
        PF_TRY(raise_smem(k_nl_zfwd<L, C>, t.zsm, set_));             \
        ProfScope ps_(ctx, PF_K_ZFWD);                                \
        k_nl_zfwd<L, C><<<gf, NL_THREADS, t.zsm, ctx->stream>>>(a);   \
    } break;
        PF_NL_LENGTHS(PF_CASE)
#undef PF_CASE
    default:
        return PF_ERR_ARG;
    }
    PF_LAUNCHED(ctx);
    return PF_OK;
}

__global__ void k_nl_mean64_part(NLArgs a);
__global__ void k_nl_mean64_fin(NLArgs a);
static int mean_attrs();
static size_t mean_smem(int N);

// vel_transform + vel_nonlinear in three launches (five in mixed precision:
// first the FP64 mean-mode sums, which also leave curl(u) in FP32 for the z
// pass, last their reduction into the k=m=0 coefficients); CFL maxima per
// radial point are left in ctx->cflmax.
int pf_launch_nl_fused(pf_ctx *ctx) {
    const NLArgs a = make_nl_args(ctx);
    if (ctx->cfg.precision == PF_PREC_MIXED) {
        {
            ProfScope ps_(ctx, PF_K_ZINV);
            PF_TRY(mean_attrs());
            k_nl_mean64_part<<<(ctx->g.H + 31) / 32, MEAN_THREADS, mean_smem(ctx->g.N), ctx->stream>>>(a);
        }
        PF_LAUNCHED(ctx);
        PF_TRY(launch_nl<float2>(ctx, a));
        {
            ProfScope ps_(ctx, PF_K_ZFWD);
            k_nl_mean64_fin<<<(ctx->g.N + 3) / 4, 128, 0, ctx->stream>>>(a);
        }
        PF_LAUNCHED(ctx);
        return PF_OK;
    }
    return launch_nl<double2>(ctx, a);
}


// ------------------------------------------------- FP64 mean mode (mixed)
// With FP32 transforms the k=m=0 coefficient of u x curl(u) is replaced by
// its exact FP64 value.  On the 3/2-dealiased grid no product of retained
// modes aliases onto (0,0), so the grid mean equals the spectral sum
//   mean(f g) = Re f00 Re g00 + 2 sum_{k>=1} Re(f_k0 conj g_k0)
//             + 2 sum_{m>=1, all k} Re(f_km conj g_km)
// (the c2r transform ignores Im f00).  Two launches.  The first: one block
// per 32-mode chunk, u_t and u_z of those modes at every radial point staged
// in shared memory (each value read from HBM once), one warp per radial
// point at a time (lanes = modes), the curl formed from the staged rows and
// the chunk's sums written as partials.  The second: one warp per radial
// point adds the chunks' partials in a fixed order.
__device__ __forceinline__ void nl_mean64_part_body(const NLArgs &a, int chunk) {
    extern __shared__ double2 msm[];  // [2][N][32]: u_t, u_z of this chunk's modes
    const Geo &g = a.g;
    const int N = g.N, lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const int nh = chunk * 32 + lane;
    const bool live = nh < g.H;
    const size_t Hp = g.Hp;
    double2 *st = msm, *sz = msm + N * 32;
    for (int n = warp; n < N; n += nw) {
        const size_t at = (size_t)n * Hp + nh;
        st[n * 32 + lane] = live ? a.u[1][at] : make_double2(0.0, 0.0);
        sz[n * 32 + lane] = live ? a.u[2][at] : make_double2(0.0, 0.0);
    }
    __syncthreads();
    int k = 0, m = 0;
    if (live) mode_km(nh, g.K, k, m);
    const double k1a1 = g.alpha * k;
    const double *__restrict__ drb = a.dm.dr;
    for (int n = warp; n < N; n += nw) {
        double s0 = 0.0, s1 = 0.0, s2 = 0.0;
        if (live) {
            const double2 ur = a.u[0][(size_t)n * Hp + nh], ut = st[n * 32 + lane], uz = sz[n * 32 + lane];
            const double rm1 = a.dm.rp[2 * N + n];
            const double m1r1 = rm1 * g.Mp * m;
            const int lo = max(0, n - KL), hi = min(N - 1, n + KL);
            double2 dz = make_double2(0.0, 0.0), dt = dz;
            for (int j = lo; j <= hi; ++j) {  // d/dr of u_z and u_t (var_coll_meshmult)
                const double w = drb[(KL + n - j) * N + j];
                const double2 z = sz[j * 32 + lane], t = st[j * 32 + lane];
                dz.x = fma(w, z.x, dz.x);
                dz.y = fma(w, z.y, dz.y);
                dt.x = fma(w, t.x, dt.x);
                dt.y = fma(w, t.y, dt.y);
            }
            // curl (variables.f90:408-436)
            const double2 cr = make_double2(-uz.y * m1r1 + ut.y * k1a1, uz.x * m1r1 - ut.x * k1a1);
            const double2 ct = make_double2(-ur.y * k1a1 - dz.x, ur.x * k1a1 - dz.y);
            const double2 cz = make_double2(ut.x * rm1 + dt.x + ur.y * m1r1, ut.y * rm1 + dt.y - ur.x * m1r1);
            if (a.curlf) {  // the z pass's FP32 inputs of the curl components
                const size_t at = (size_t)n * Hp + nh, fs = (size_t)N * Hp;
                a.curlf[at] = make_float2((float)cr.x, (float)cr.y);
                a.curlf[fs + at] = make_float2((float)ct.x, (float)ct.y);
                a.curlf[2 * fs + at] = make_float2((float)cz.x, (float)cz.y);
            }
            const double w = (nh == 0) ? 1.0 : 2.0;
            auto dot = [&](double2 f, double2 h) { return nh == 0 ? f.x * h.x : f.x * h.x + f.y * h.y; };
            s0 = w * (dot(ut, cz) - dot(uz, ct));
            s1 = w * (dot(uz, cr) - dot(ur, cz));
            s2 = w * (dot(ur, ct) - dot(ut, cr));
        }
        for (int o = 16; o > 0; o >>= 1) {
            s0 += __shfl_xor_sync(0xffffffffu, s0, o);
            s1 += __shfl_xor_sync(0xffffffffu, s1, o);
            s2 += __shfl_xor_sync(0xffffffffu, s2, o);
        }
        if (lane == 0) {
            double *dst = a.mpart + ((size_t)chunk * N + n) * 3;
            dst[0] = s0;
            dst[1] = s1;
            dst[2] = s2;
        }
    }
}

__device__ __forceinline__ void nl_mean64_fin_body(const NLArgs &a, int n) {
    const Geo &g = a.g;
    const int lane = threadIdx.x & 31;
    const int nchunk = (g.H + 31) / 32;
    double t[3] = {0.0, 0.0, 0.0};
    for (int c = lane; c < nchunk; c += 32) {
        const double *src = a.mpart + ((size_t)c * g.N + n) * 3;
        t[0] += src[0];
        t[1] += src[1];
        t[2] += src[2];
    }
#pragma unroll
    for (int q = 0; q < 3; ++q)
        for (int o = 16; o > 0; o >>= 1) t[q] += __shfl_xor_sync(0xffffffffu, t[q], o);
    if (lane != 0) return;
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

static size_t mean_smem(int N) { return (size_t)2 * N * 32 * sizeof(double2); }
__global__ void __launch_bounds__(MEAN_THREADS) k_nl_mean64_part(NLArgs a) { nl_mean64_part_body(a, blockIdx.x); }
// one warp per radial point
__global__ void __launch_bounds__(128) k_nl_mean64_fin(NLArgs a) {
    const int n = blockIdx.x * 4 + (threadIdx.x >> 5);
    if (n < a.g.N) nl_mean64_fin_body(a, n);
}

// ------------------------------------------------------------------ batched
// One launch per (stage, transform length) covers the blocks of every pipe
// of a batch with that length: blk[b] = (pipe, block index within that pipe's
// own grid), and each block runs the lone-pipe body.  The launches of one
// stage for different lengths are independent and run concurrently (forked
// onto auxiliary streams, joined before the next stage).
template <int ZL, typename C>
__global__ void __launch_bounds__(NL_THREADS, (NLOcc<C, ZL>::zinv)) k_nl_zinv_b(const NLArgs *__restrict__ args, const int2 *__restrict__ blk) {
    const int2 pb = blk[blockIdx.x];
    const NLArgs a = args[pb.x];  // by value: stores through its pointers cannot alias it
    const int gx = (a.g.M + a.MC - 1) / a.MC;
    nl_zinv_body<ZL, C>(a, pb.y % gx, (pb.y / gx) % a.g.N, pb.y / (gx * a.g.N));
}

template <int TL, typename C>
__global__ void __launch_bounds__(NL_THREADS, (NLOcc<C, TL>::theta)) k_nl_theta_b(const NLArgs *__restrict__ args, const int2 *__restrict__ blk) {
    const int2 pb = blk[blockIdx.x];
    const NLArgs a = args[pb.x];
    const int gx = (a.g.Z + a.ZC - 1) / a.ZC;
    nl_theta_body<TL, C>(a, pb.y % gx, pb.y / gx);
}

template <int ZL, typename C>
__global__ void __launch_bounds__(NL_THREADS, (NLOcc<C, ZL>::zfwd)) k_nl_zfwd_b(const NLArgs *__restrict__ args, const int2 *__restrict__ blk) {
    const int2 pb = blk[blockIdx.x];
    const NLArgs a = args[pb.x];
    const int gx = (a.g.M + a.MC - 1) / a.MC;
    nl_zfwd_body<ZL, C>(a, pb.y % gx, (pb.y / gx) % a.g.N, pb.y / (gx * a.g.N));
}

template <int ZL, int TL>
__global__ void __launch_bounds__(FUSED_THREADS, 1) k_nl_fused_b(const NLArgs *__restrict__ args,
                                                                const int2 *__restrict__ blk) {
    const int2 pb = blk[blockIdx.x];
    const NLArgs a = args[pb.x];
    nl_fused_body<ZL, TL>(a, pb.y);
}

__global__ void __launch_bounds__(MEAN_THREADS) k_nl_mean64_part_batch(const NLArgs *__restrict__ args,
                                                                      const int2 *__restrict__ blk) {
    const int2 pb = blk[blockIdx.x];
    const NLArgs a = args[pb.x];
    nl_mean64_part_body(a, pb.y);
}
__global__ void __launch_bounds__(128) k_nl_mean64_fin_batch(const NLArgs *__restrict__ args,
                                                            const int2 *__restrict__ blk) {
    const int2 pb = blk[blockIdx.x];
    const NLArgs a = args[pb.x];
    const int n = pb.y * 4 + (threadIdx.x >> 5);
    if (n < a.g.N) nl_mean64_fin_body(a, n);
}

// ------------------------------------------------- work-list stage kernels
// One persistent launch per transform stage for every pipe of a
// mixed-precision batch, whatever its transform length.  The (pipe, tile)
// items of the stage sit in one list, longest lengths first; each resident
// block takes the next item from a device counter (the fetch of the item
// after it is in flight while the block works) and runs the lone-pipe body
// of that item's length, so the results are bitwise those of the per-length
// launches.  The last block to leave resets the counter for the stage's next
// launch.  FP32 lengths 36 to 192 (every length of the batched mix); the
// shorter ones hold whole rows in registers and keep their own launches.
#define PF_NL_WL_LENGTHS(X) X(36) X(48) X(72) X(96) X(144) X(192)

static bool wl_length_ok(int L) {
    switch (L) {
#define PF_CASE(L) case L:
        PF_NL_WL_LENGTHS(PF_CASE)
#undef PF_CASE
        return true;
    default:
        return false;
    }
}

// One item of stage ST (0 z inverse, 1 theta pass, 2 z forward) for one
// length: l = the block index within the pipe's own grid of that stage.  Not
// inlined, so each length's body gets the register allocation of its own
// per-length kernel instead of sharing one across every length.
template <int ST, int L>
__device__ __noinline__ void nl_wl_run(const NLArgs *__restrict__ args, int pipe, int l) {
    const NLArgs a = args[pipe];  // by value: stores through its pointers cannot alias it
    if constexpr (ST == 1) {
        const int gx = (a.g.Z + a.ZC - 1) / a.ZC;
        nl_theta_body<L, float2>(a, l % gx, l / gx);
    } else {
        const int gx = (a.g.M + a.MC - 1) / a.MC;
        const int bx = l % gx, by = (l / gx) % a.g.N, bz = l / (gx * a.g.N);
        if constexpr (ST == 0) nl_zinv_body<L, float2>(a, bx, by, bz);
        else nl_zfwd_body<L, float2>(a, bx, by, bz);
    }
}

template <int ST> __device__ __forceinline__ void nl_wl_item(const NLArgs *__restrict__ args, int pipe, int l) {
    const int len = ST == 1 ? args[pipe].g.Th : args[pipe].g.Z;
    switch (len) {
#define PF_CASE(L)                            \
    case L:                                   \
        nl_wl_run<ST, L>(args, pipe, l);      \
        break;
        PF_NL_WL_LENGTHS(PF_CASE)
#undef PF_CASE
    }
}

// ctr[0]: next item; ctr[1]: blocks that have left (both zero between launches)
template <int ST>
__global__ void __launch_bounds__(NL_THREADS, ST == 1 ? 6 : 5)
    k_nl_stage_wl(const NLArgs *__restrict__ args, const int2 *__restrict__ items, int nitems, unsigned *ctr) {
    __shared__ int next[2];
    if (threadIdx.x == 0) next[0] = (int)atomicAdd(&ctr[0], 1u);
    __syncthreads();
    int slot = 0, cur = next[0];
    while (cur < nitems) {
        if (threadIdx.x == 0) next[slot ^ 1] = (int)atomicAdd(&ctr[0], 1u);
        const int2 pb = items[cur];
        nl_wl_item<ST>(args, pb.x, pb.y);
        __syncthreads();  // the item's shared memory is free, next[slot ^ 1] is visible
        slot ^= 1;
        cur = next[slot];
    }
    if (threadIdx.x == 0) {
        __threadfence();  // this block's last fetch is done before it counts itself out
        if (atomicAdd(&ctr[1], 1u) == gridDim.x - 1) {
            ctr[0] = 0u;
            ctr[1] = 0u;
        }
    }
}

// shared-memory limit of the mean-mode partial-sum kernels (up to N = 128)
static int mean_attrs() {
    static bool set = false;
    if (!set) {
        const int bytes = (int)mean_smem(128);
        PF_CUDA(cudaFuncSetAttribute(k_nl_mean64_part, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
        PF_CUDA(cudaFuncSetAttribute(k_nl_mean64_part_batch, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
        set = true;
    }
    return PF_OK;
}

namespace {
struct NLGroup {
    int L;
    bool mixed;  // float2 (mixed precision) or double2 transforms
    int2 *blk;
    int nblk;
    size_t smem;
    int Th;      // one-block-per-radial-point groups: (Z, Th) = (L, Th)
};
constexpr int NLB_STAGES = 3;   // zinv, theta, zfwd
constexpr int NLB_MAXG = 24;    // (transform length, precision) pairs
}  // namespace

struct pf_nl_batch {
    int n;
    NLArgs *d_args[2];  // [pointer state]: 0 = as built, 1 = vel/prev swapped
    std::vector<NLGroup> groups[NLB_STAGES];
    int2 *mean_blk, *fin_blk;  // FP64 mean mode of the mixed-precision pipes: chunks, radial points
    int nmean, nfin;
    size_t mean_sm;
    cudaStream_t aux[NLB_MAXG];
    cudaEvent_t fork[NLB_STAGES], join[NLB_STAGES][NLB_MAXG];
    // pipes whose transforms run one block per radial point, one group per
    // (Z, Th): launched on streams of their own beside the three-pass stages
    std::vector<NLGroup> fgroups;
    cudaStream_t faux[NLB_MAXG];
    cudaEvent_t ffork, fjoin[NLB_MAXG];
    // work-list form (pf_batch_set_worklist): one persistent launch per
    // stage over the items of every group, in the groups' order
    bool wl;
    int2 *wl_items[NLB_STAGES];
    int wl_n[NLB_STAGES], wl_grid[NLB_STAGES];
    size_t wl_smem[NLB_STAGES];
    unsigned *wl_ctr;  // two counters per stage
};

bool pf_nl_batch_supported(pf_ctx *const *pipes, int n) {
    if (n <= 0) return false;
    for (int i = 0; i < n; ++i)
        if (!pf_nl_fused_supported(pipes[i])) return false;
    return true;
}

void pf_nl_batch_free(pf_nl_batch *b) {
    if (!b) return;
    for (int s = 0; s < 2; ++s) cudaFree(b->d_args[s]);
    for (int st = 0; st < NLB_STAGES; ++st) {
        for (NLGroup &gr : b->groups[st]) cudaFree(gr.blk);
        if (b->fork[st]) cudaEventDestroy(b->fork[st]);
        for (int k = 0; k < NLB_MAXG; ++k)
            if (b->join[st][k]) cudaEventDestroy(b->join[st][k]);
    }
    cudaFree(b->mean_blk);
    cudaFree(b->fin_blk);
    for (int st = 0; st < NLB_STAGES; ++st) cudaFree(b->wl_items[st]);
    cudaFree(b->wl_ctr);
    for (NLGroup &gr : b->fgroups) cudaFree(gr.blk);
    if (b->ffork) cudaEventDestroy(b->ffork);
    for (int k = 0; k < NLB_MAXG; ++k) {
        if (b->aux[k]) cudaStreamDestroy(b->aux[k]);
        if (b->faux[k]) cudaStreamDestroy(b->faux[k]);
        if (b->fjoin[k]) cudaEventDestroy(b->fjoin[k]);
    }
    delete b;
}

template <typename T> static int upload(T **d, const std::vector<T> &h) {
    PF_CUDA(cudaMalloc((void **)d, std::max<size_t>(1, h.size()) * sizeof(T)));
    if (!h.empty()) PF_CUDA(cudaMemcpy(*d, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice));
    return PF_OK;
}

static bool is_mixed(const pf_ctx *c) { return c->cfg.precision == PF_PREC_MIXED; }

template <typename C> static NLTiles<C> tiles_of(const pf_ctx *c) { return nl_tiles<C>(c->g, c->tune); }

static bool fused_of(const pf_ctx *c, int *ZC = nullptr, size_t *smem = nullptr) {
    int zc = 0;
    size_t sm = 0;
    const bool f = fused_plan(c->g, c->tune, is_mixed(c), &zc, &sm);
    if (ZC) *ZC = zc;
    if (smem) *smem = sm;
    return f;
}

// blocks of stage st for the pipes of one (length, precision) group
template <typename C>
static void nlb_group_map(int st, int L, bool mixed, pf_ctx *const *pipes, int n, std::vector<int2> &map,
                          size_t &smem) {
    for (int i = 0; i < n; ++i) {
        const Geo &g = pipes[i]->g;
        if ((st == 1 ? g.Th : g.Z) != L || is_mixed(pipes[i]) != mixed || fused_of(pipes[i])) continue;
        const NLTiles<C> t = tiles_of<C>(pipes[i]);
        int nb = 0;
        if (st == 0) nb = ((g.M + t.MC - 1) / t.MC) * g.N * 6;
        if (st == 1) nb = ((g.Z + t.ZC - 1) / t.ZC) * g.N;
        if (st == 2) nb = ((g.M + t.MC - 1) / t.MC) * g.N * 3;
        for (int l = 0; l < nb; ++l) map.push_back(make_int2(i, l));
        smem = std::max(smem, st == 1 ? t.tsm : t.zsm);
    }
}

// one group per (stage, transform length, precision), longest lengths first
static int nlb_groups(pf_nl_batch *b, pf_ctx *const *pipes, int n) {
    for (int st = 0; st < NLB_STAGES; ++st) {
        std::vector<std::pair<int, int>> keys;  // (L, mixed)
        for (int i = 0; i < n; ++i) {
            if (fused_of(pipes[i])) continue;
            const std::pair<int, int> k(st == 1 ? pipes[i]->g.Th : pipes[i]->g.Z, is_mixed(pipes[i]) ? 1 : 0);
            if (std::find(keys.begin(), keys.end(), k) == keys.end()) keys.push_back(k);
        }
        std::sort(keys.begin(), keys.end(), std::greater<std::pair<int, int>>());
        if ((int)keys.size() > NLB_MAXG) {
            pf_set_error("batched transforms: too many (length, precision) groups");
            return PF_ERR_ARG;
        }
        for (const auto &k : keys) {
            std::vector<int2> map;
            size_t smem = 0;
            if (k.second) nlb_group_map<float2>(st, k.first, true, pipes, n, map, smem);
            else nlb_group_map<double2>(st, k.first, false, pipes, n, map, smem);
            b->groups[st].push_back(NLGroup{k.first, k.second != 0, nullptr, (int)map.size(), smem, 0});
            PF_TRY(upload(&b->groups[st].back().blk, map));
        }
    }
    {  // one block per radial point: groups by (Z, Th), largest planes first
        std::vector<std::pair<int, int>> keys;
        for (int i = 0; i < n; ++i)
            if (fused_of(pipes[i])) {
                const std::pair<int, int> k(pipes[i]->g.Z, pipes[i]->g.Th);
                if (std::find(keys.begin(), keys.end(), k) == keys.end()) keys.push_back(k);
            }
        std::sort(keys.begin(), keys.end(), std::greater<std::pair<int, int>>());
        if ((int)keys.size() > NLB_MAXG) {
            pf_set_error("batched transforms: too many (Z, Th) groups");
            return PF_ERR_ARG;
        }
        for (const auto &k : keys) {
            std::vector<int2> map;
            size_t smem = 0;
            for (int i = 0; i < n; ++i) {
                size_t sm = 0;
                if (pipes[i]->g.Z != k.first || pipes[i]->g.Th != k.second || !fused_of(pipes[i], nullptr, &sm)) continue;
                for (int r = 0; r < pipes[i]->g.N; ++r) map.push_back(make_int2(i, r));
                smem = std::max(smem, sm);
            }
            b->fgroups.push_back(NLGroup{k.first, true, nullptr, (int)map.size(), smem, k.second});
            PF_TRY(upload(&b->fgroups.back().blk, map));
        }
    }
    std::vector<int2> mean, fin;
    b->mean_sm = 0;
    for (int i = 0; i < n; ++i)
        if (is_mixed(pipes[i])) {
            const Geo &g = pipes[i]->g;
            for (int l = 0; l < (g.H + 31) / 32; ++l) mean.push_back(make_int2(i, l));
            for (int l = 0; l < (g.N + 3) / 4; ++l) fin.push_back(make_int2(i, l));
            b->mean_sm = std::max(b->mean_sm, mean_smem(g.N));
        }
    b->nmean = (int)mean.size();
    b->nfin = (int)fin.size();
    PF_TRY(upload(&b->mean_blk, mean));
    return upload(&b->fin_blk, fin);
}

template <int ST> static int wl_plan(pf_nl_batch *b, int dev_sms) {
    static size_t set_ = 0;
    PF_TRY(raise_smem(k_nl_stage_wl<ST>, b->wl_smem[ST], set_));
    int per_sm = 0;
    PF_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_nl_stage_wl<ST>, NL_THREADS, b->wl_smem[ST]));
    if (per_sm < 1) {
        pf_set_error("batched transforms: work-list stage %d does not fit an SM", ST);
        return PF_ERR_ARG;
    }
    b->wl_grid[ST] = std::min(b->wl_n[ST], per_sm * dev_sms);
    return PF_OK;
}

// The work-list form of the three stages, when every three-pass group is in
// FP32 with a length the work-list kernels are built for; otherwise the
// batch keeps the per-length launches.
static int nlb_worklists(pf_nl_batch *b, pf_ctx *const *pipes, int n) {
    for (int st = 0; st < NLB_STAGES; ++st)
        for (const NLGroup &gr : b->groups[st])
            if (!gr.mixed || !wl_length_ok(gr.L)) return PF_OK;
    PF_CUDA(cudaMalloc((void **)&b->wl_ctr, 2 * NLB_STAGES * sizeof(unsigned)));
    PF_CUDA(cudaMemset(b->wl_ctr, 0, 2 * NLB_STAGES * sizeof(unsigned)));
    int dev = 0, sms = 0;
    PF_CUDA(cudaGetDevice(&dev));
    PF_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    for (int st = 0; st < NLB_STAGES; ++st) {
        std::vector<int2> items;
        size_t smem = 0;
        for (const NLGroup &gr : b->groups[st]) nlb_group_map<float2>(st, gr.L, true, pipes, n, items, smem);
        b->wl_n[st] = (int)items.size();
        b->wl_smem[st] = smem;
        PF_TRY(upload(&b->wl_items[st], items));
    }
    PF_TRY(wl_plan<0>(b, sms));
    PF_TRY(wl_plan<1>(b, sms));
    PF_TRY(wl_plan<2>(b, sms));
    b->wl = true;
    return PF_OK;
}

// Arguments of every pipe in both pointer states, and the per-group maps
// (and the work lists, when asked for and every group qualifies).
int pf_nl_batch_build(pf_ctx *const *pipes, int n, bool worklist, pf_nl_batch **out) {
    *out = nullptr;
    if (!pf_nl_batch_supported(pipes, n)) {
        pf_set_error("batched transforms: a transform length is not built");
        return PF_ERR_ARG;
    }
    pf_nl_batch *b = new pf_nl_batch();
    b->n = n;
    int s = PF_OK;
    std::vector<NLArgs> h(n);
    for (int st = 0; st < 2 && s == PF_OK; ++st) {
        for (int i = 0; i < n; ++i) {
            if (st) for (int c = 0; c < 3; ++c) std::swap(pipes[i]->vel[c].d, pipes[i]->prev[c].d);
            h[i] = make_nl_args(pipes[i]);
            if (st) for (int c = 0; c < 3; ++c) std::swap(pipes[i]->vel[c].d, pipes[i]->prev[c].d);
        }
        s = upload(&b->d_args[st], h);
    }
    if (s == PF_OK) s = nlb_groups(b, pipes, n);
    if (s == PF_OK && worklist) s = nlb_worklists(b, pipes, n);
    int ng = 0;
    for (int st = 0; st < NLB_STAGES; ++st) ng = std::max(ng, (int)b->groups[st].size());
    for (int st = 0; st < NLB_STAGES && s == PF_OK; ++st) {
        if (cudaEventCreateWithFlags(&b->fork[st], cudaEventDisableTiming) != cudaSuccess) s = PF_ERR_CUDA;
        for (size_t k = 0; k < b->groups[st].size() && s == PF_OK; ++k)
            if (cudaEventCreateWithFlags(&b->join[st][k], cudaEventDisableTiming) != cudaSuccess) s = PF_ERR_CUDA;
    }
    for (int k = 1; k < ng && s == PF_OK; ++k)
        if (cudaStreamCreateWithFlags(&b->aux[k], cudaStreamNonBlocking) != cudaSuccess) s = PF_ERR_CUDA;
    if (s == PF_OK && !b->fgroups.empty() && cudaEventCreateWithFlags(&b->ffork, cudaEventDisableTiming) != cudaSuccess)
        s = PF_ERR_CUDA;
    for (size_t k = 0; k < b->fgroups.size() && s == PF_OK; ++k)
        if (cudaStreamCreateWithFlags(&b->faux[k], cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventCreateWithFlags(&b->fjoin[k], cudaEventDisableTiming) != cudaSuccess)
            s = PF_ERR_CUDA;
    if (s != PF_OK) {
        if (s == PF_ERR_CUDA) pf_set_error("batched transforms: allocation failed");
        pf_nl_batch_free(b);
        return s;
    }
    *out = b;
    return PF_OK;
}

template <typename C> static int nlb_group_launch(int st, const NLGroup &gr, const NLArgs *args, cudaStream_t s) {
    switch (gr.L) {
#define PF_CASE(L)                                                                                 \
    case L: {                                                                                      \
        static size_t set_[NLB_STAGES] = {0, 0, 0};                                                \
        if (st == 0) {                                                                             \
            PF_TRY(raise_smem(k_nl_zinv_b<L, C>, gr.smem, set_[0]));                               \
            k_nl_zinv_b<L, C><<<gr.nblk, NL_THREADS, gr.smem, s>>>(args, gr.blk);                  \
        } else if (st == 1) {                                                                      \
            PF_TRY(raise_smem(k_nl_theta_b<L, C>, gr.smem, set_[1]));                              \
            k_nl_theta_b<L, C><<<gr.nblk, NL_THREADS, gr.smem, s>>>(args, gr.blk);                 \
        } else {                                                                                   \
            PF_TRY(raise_smem(k_nl_zfwd_b<L, C>, gr.smem, set_[2]));                               \
            k_nl_zfwd_b<L, C><<<gr.nblk, NL_THREADS, gr.smem, s>>>(args, gr.blk);                  \
        }                                                                                          \
    } break;
        PF_NL_LENGTHS(PF_CASE)
#undef PF_CASE
    default:
        pf_set_error("batched transforms: length %d not built", gr.L);
        return PF_ERR_ARG;
    }
    PF_CHECK_LAUNCH();
    return PF_OK;
}

static int nlb_fused_launch(const NLGroup &gr, const NLArgs *args, cudaStream_t s) {
#define PF_CASE(ZL, TL)                                                              \
    if (gr.L == ZL && gr.Th == TL) {                                                 \
        static size_t set_ = 0;                                                      \
        PF_TRY(raise_smem(k_nl_fused_b<ZL, TL>, gr.smem, set_));                     \
        k_nl_fused_b<ZL, TL><<<gr.nblk, FUSED_THREADS, gr.smem, s>>>(args, gr.blk);  \
        PF_CHECK_LAUNCH();                                                           \
        return PF_OK;                                                                \
    }
    PF_NL_FUSED_PAIRS(PF_CASE)
#undef PF_CASE
    pf_set_error("batched transforms: (Z, Th) = (%d, %d) not built as one block per radial point", gr.L, gr.Th);
    return PF_ERR_ARG;
}

// one stage: the first group on st, the others forked onto auxiliary streams
static int nlb_stage(pf_nl_batch *b, int stage, const NLArgs *args, cudaStream_t st, unsigned long long *nk) {
    if (b->wl) {
        if (b->wl_n[stage] == 0) return PF_OK;
        const int g = b->wl_grid[stage], n = b->wl_n[stage];
        const size_t sm = b->wl_smem[stage];
        unsigned *ctr = b->wl_ctr + 2 * stage;
        if (stage == 0) k_nl_stage_wl<0><<<g, NL_THREADS, sm, st>>>(args, b->wl_items[0], n, ctr);
        else if (stage == 1) k_nl_stage_wl<1><<<g, NL_THREADS, sm, st>>>(args, b->wl_items[1], n, ctr);
        else k_nl_stage_wl<2><<<g, NL_THREADS, sm, st>>>(args, b->wl_items[2], n, ctr);
        PF_CHECK_LAUNCH();
        ++*nk;
        return PF_OK;
    }
    const std::vector<NLGroup> &gs = b->groups[stage];
    if (gs.size() > 1) {
        PF_CUDA(cudaEventRecord(b->fork[stage], st));
        for (size_t k = 1; k < gs.size(); ++k) PF_CUDA(cudaStreamWaitEvent(b->aux[k], b->fork[stage], 0));
    }
    for (size_t k = 0; k < gs.size(); ++k) {
        cudaStream_t s = k ? b->aux[k] : st;
        if (gs[k].mixed) PF_TRY(nlb_group_launch<float2>(stage, gs[k], args, s));
        else PF_TRY(nlb_group_launch<double2>(stage, gs[k], args, s));
        ++*nk;
    }
    for (size_t k = 1; k < gs.size(); ++k) {
        PF_CUDA(cudaEventRecord(b->join[stage][k], b->aux[k]));
        PF_CUDA(cudaStreamWaitEvent(st, b->join[stage][k], 0));
    }
    return PF_OK;
}

// vel_transform + vel_nonlinear of every pipe: one launch per stage and
// (transform length, precision) group, plus the FP64 mean-mode launch when
// any pipe is in mixed precision; launches are counted into *nk.  state 0:
// the pointers the pipes held when the batch was built; 1: vel/prev swapped.
int pf_nl_batch_launch(pf_nl_batch *b, int state, cudaStream_t st, pf_stage_prof *prof, unsigned long long *nk) {
    const NLArgs *args = b->d_args[state];
    const int cats[NLB_STAGES] = {PF_K_ZINV, PF_K_THFWD, PF_K_ZFWD};
    // mixed precision: the FP64 mean-mode sums first; they leave curl(u) in
    // FP32 for the z pass
    if (b->nmean > 0) {
        StageScope ss_(prof, PF_K_ZINV, st);
        PF_TRY(mean_attrs());
        k_nl_mean64_part_batch<<<b->nmean, MEAN_THREADS, b->mean_sm, st>>>(args, b->mean_blk);
        PF_CHECK_LAUNCH();
        *nk += 1;
        // the pipes done one block per radial point, beside the three passes
        // of the others (they need the mean-mode pass's FP32 curl)
        if (!b->fgroups.empty()) {
            PF_CUDA(cudaEventRecord(b->ffork, st));
            for (size_t k = 0; k < b->fgroups.size(); ++k) {
                PF_CUDA(cudaStreamWaitEvent(b->faux[k], b->ffork, 0));
                PF_TRY(nlb_fused_launch(b->fgroups[k], args, b->faux[k]));
                PF_CUDA(cudaEventRecord(b->fjoin[k], b->faux[k]));
                ++*nk;
            }
        }
    }
    for (int stage = 0; stage < NLB_STAGES; ++stage) {
        StageScope ss_(prof, cats[stage], st);
        PF_TRY(nlb_stage(b, stage, args, st, nk));
    }
    if (b->nmean > 0) {
        StageScope ss_(prof, PF_K_ZFWD, st);
        for (size_t k = 0; k < b->fgroups.size(); ++k) PF_CUDA(cudaStreamWaitEvent(st, b->fjoin[k], 0));
        k_nl_mean64_fin_batch<<<b->nfin, 128, 0, st>>>(args, b->fin_blk);
        PF_CHECK_LAUNCH();
        *nk += 1;
    }
    return PF_OK;
}
