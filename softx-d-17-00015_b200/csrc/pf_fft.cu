// 3/2-dealiased Fourier transforms between spectral (coll) and physical space
// (transform.fftw3.f90:35-147) as batched mixed-radix Stockham FFTs staged
// through shared memory:
//   coll -> phys : z pass  (c2c length 3K, sign +1) over the M columns of each
//                  radial point, Hermitian fill of m=0 (transform.fftw3.f90:72-74);
//                  theta pass (c2r length 3M; two real rows packed per complex FFT)
//   phys -> coll : theta pass (r2c, scaled by 1/(9KM)), z pass (c2c, sign -1),
//                  truncation to |k|<K, m<M.
// FFTW's sign conventions are kept: +1 is the unnormalised backward transform;
// the c2r transform ignores the imaginary part of the theta DC bin.
#include <cmath>
#include "pf_internal.cuh"

static constexpr int FFT_THREADS = 256;

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
// multiply by sign*i
__device__ __forceinline__ double2 cmuli(double2 a, int sign) {
    return sign > 0 ? make_double2(-a.y, a.x) : make_double2(a.y, -a.x);
}

// B batches of length L (batch stride L) in `buf`; `tmp` is the ping-pong
// buffer; tw[t] = exp(+2 pi i t/L).  Returns the buffer holding the result.
// Stockham autosort: pass with radix r maps butterfly j (k = j mod Ns) to
// outputs (j/Ns)*Ns*r + k + q*Ns with twiddles W^(sign q k L/(Ns r)).
__device__ double2 *smem_fft(double2 *buf, double2 *tmp, int B, const FFTPlan &pl, const double2 *tw, int sign) {
    const int L = pl.L;
    double2 *src = buf, *dst = tmp;
    int Ns = 1;
    for (int s = 0; s < pl.nf; ++s) {
        const int r = pl.f[s];
        const int nb = L / r;
        const int stride = L / (Ns * r);
        for (int idx = threadIdx.x; idx < nb * B; idx += blockDim.x) {
            const int b = idx / nb, j = idx - b * nb;
            const int k = j % Ns;
            const double2 *sp = src + b * L;
            double2 *dp = dst + b * L;
            const int base = (j / Ns) * Ns * r + k;
            double2 v[16];
            for (int q = 0; q < r; ++q) {
                double2 x = sp[j + q * nb];
                if (q > 0 && k > 0) {
                    double2 w = tw[q * k * stride];
                    if (sign < 0) w.y = -w.y;
                    x = cmul(x, w);
                }
                v[q] = x;
            }
            if (r == 2) {
                dp[base] = cadd(v[0], v[1]);
                dp[base + Ns] = csub(v[0], v[1]);
            } else if (r == 4) {
                const double2 a = cadd(v[0], v[2]), b2 = csub(v[0], v[2]);
                const double2 c = cadd(v[1], v[3]), d = cmuli(csub(v[1], v[3]), sign);
                dp[base] = cadd(a, c);
                dp[base + Ns] = cadd(b2, d);
                dp[base + 2 * Ns] = csub(a, c);
                dp[base + 3 * Ns] = csub(b2, d);
            } else if (r == 3) {
                const double s3 = 0.86602540378443864676;  // sin(2 pi/3)
                const double2 t = cadd(v[1], v[2]);
                const double2 u = make_double2(v[0].x - 0.5 * t.x, v[0].y - 0.5 * t.y);
                const double2 w = cmuli(make_double2(s3 * (v[1].x - v[2].x), s3 * (v[1].y - v[2].y)), sign);
                dp[base] = cadd(v[0], t);
                dp[base + Ns] = cadd(u, w);
                dp[base + 2 * Ns] = csub(u, w);
            } else {  // generic small prime radix: direct DFT with table twiddles
                const int st = L / r;
                for (int q = 0; q < r; ++q) {
                    double2 acc = v[0];
                    for (int p = 1; p < r; ++p) {
                        double2 w = tw[((p * q) % r) * st];
                        if (sign < 0) w.y = -w.y;
                        acc = cadd(acc, cmul(v[p], w));
                    }
                    dp[base + q * Ns] = acc;
                }
            }
        }
        __syncthreads();
        double2 *t = src;
        src = dst;
        dst = t;
        Ns *= r;
    }
    return src;
}

struct SrcPtrs {
    const double2 *p[6];
};
struct PhysPtrs {
    double *p[6];
};
struct CPhysPtrs {
    const double *p[6];
};
struct DstPtrs {
    double2 *p[6];
};

// z pass, spectral -> (m, z) columns: grid (m-chunk, n, comp)
__global__ void k_zinv(SrcPtrs src, double2 *__restrict__ T, Geo g, FFTPlan pz, const double2 *__restrict__ twz,
                       int MC) {
    extern __shared__ double2 sm[];
    const int Z = g.Z, K = g.K;
    double2 *buf = sm, *tmp = sm + MC * Z, *tw = sm + 2 * MC * Z;
    const int comp = blockIdx.z, n = blockIdx.y, m0 = blockIdx.x * MC;
    const int mc = min(MC, g.M - m0);
    const double2 *f = src.p[comp] + (size_t)n * g.Hp;
    for (int i = threadIdx.x; i < Z; i += blockDim.x) tw[i] = twz[i];
    for (int idx = threadIdx.x; idx < mc * Z; idx += blockDim.x) {
        const int c = idx / Z, j = idx - c * Z;
        const int m = m0 + c;
        double2 v = make_double2(0.0, 0.0);
        if (m == 0) {
            if (j < K) v = f[j];
            else if (j >= 2 * K + 1) {
                v = f[Z - j];
                v.y = -v.y;
            }
        } else {
            const int base = m * (2 * K - 1);
            if (j < K) v = f[base + j];
            else if (j >= 2 * K + 1) v = f[base + (j - Z)];
        }
        buf[idx] = v;
    }
    __syncthreads();
    const double2 *res = smem_fft(buf, tmp, mc, pz, tw, +1);
    double2 *out = T + ((size_t)(comp * g.N + n) * g.M + m0) * Z;
    for (int idx = threadIdx.x; idx < mc * Z; idx += blockDim.x) out[idx] = res[idx];
}

// theta pass, (m, z) columns -> physical: grid (z-chunk, n); ncomp comps,
// ZC rows per block, two rows per complex FFT
__global__ void k_thinv(const double2 *__restrict__ T, PhysPtrs dst, int ncomp, Geo g, FFTPlan pt,
                        const double2 *__restrict__ twt, int ZC) {
    extern __shared__ double2 sm[];
    const int Th = g.Th, M = g.M, Z = g.Z;
    const int np = ZC / 2, B = ncomp * np;
    double2 *buf = sm, *tmp = sm + B * Th, *tw = sm + 2 * B * Th;
    const int n = blockIdx.y, z0 = blockIdx.x * ZC;
    for (int i = threadIdx.x; i < Th; i += blockDim.x) tw[i] = twt[i];
    for (int i = threadIdx.x; i < B * Th; i += blockDim.x) buf[i] = make_double2(0.0, 0.0);
    __syncthreads();
    for (int idx = threadIdx.x; idx < ncomp * M * np; idx += blockDim.x) {
        const int zp = idx % np, rest = idx / np;
        const int m = rest % M, comp = rest / M;
        const int za = z0 + 2 * zp, zb = za + 1;
        const double2 *col = T + ((size_t)(comp * g.N + n) * M + m) * Z;
        double2 a = (za < Z) ? col[za] : make_double2(0.0, 0.0);
        double2 b = (zb < Z) ? col[zb] : make_double2(0.0, 0.0);
        double2 *X = buf + (comp * np + zp) * Th;
        if (m == 0) {
            X[0] = make_double2(a.x, b.x);  // c2r: DC imaginary parts ignored
        } else {
            X[m] = make_double2(a.x - b.y, a.y + b.x);            // a + i b
            X[Th - m] = make_double2(a.x + b.y, -a.y + b.x);      // conj(a) + i conj(b)
        }
    }
    __syncthreads();
    const double2 *res = smem_fft(buf, tmp, B, pt, tw, +1);
    for (int idx = threadIdx.x; idx < ncomp * Th * ZC; idx += blockDim.x) {
        const int zz = idx % ZC, rest = idx / ZC;
        const int t = rest % Th, comp = rest / Th;
        const int z = z0 + zz;
        if (z >= Z) continue;
        const double2 v = res[(comp * np + zz / 2) * Th + t];
        dst.p[comp][((size_t)n * Th + t) * Z + z] = (zz & 1) ? v.y : v.x;
    }
}

// theta pass, physical -> (m, z) columns (scaled): grid (z-chunk, n).
// cross != 0: inputs are (r,t,z,curlr,curlt,curlz) and the three outputs are
// the components of u x curl(u) (velocity.f90:325-330).
__global__ void k_thfwd(CPhysPtrs src, int ncomp, int cross, double2 *__restrict__ T, Geo g, FFTPlan pt,
                        const double2 *__restrict__ twt, int ZC, double scale) {
    extern __shared__ double2 sm[];
    const int Th = g.Th, M = g.M, Z = g.Z;
    const int np = ZC / 2, B = ncomp * np;
    double2 *buf = sm, *tmp = sm + B * Th, *tw = sm + 2 * B * Th;
    const int n = blockIdx.y, z0 = blockIdx.x * ZC;
    for (int i = threadIdx.x; i < Th; i += blockDim.x) tw[i] = twt[i];
    double *bre = reinterpret_cast<double *>(buf);
    for (int idx = threadIdx.x; idx < ncomp * Th * ZC; idx += blockDim.x) {
        const int zz = idx % ZC, rest = idx / ZC;
        const int t = rest % Th, comp = rest / Th;
        const int z = z0 + zz;
        double v = 0.0;
        if (z < Z) {
            const size_t at = ((size_t)n * Th + t) * Z + z;
            if (cross) {
                const double ur = src.p[0][at], ut = src.p[1][at], uz = src.p[2][at];
                const double cr = src.p[3][at], ct = src.p[4][at], cz = src.p[5][at];
                if (comp == 0) v = ut * cz - uz * ct;
                else if (comp == 1) v = uz * cr - ur * cz;
                else v = ur * ct - ut * cr;
            } else {
                v = src.p[comp][at];
            }
            v = scale * v;
        }
        bre[2 * ((comp * np + zz / 2) * Th + t) + (zz & 1)] = v;
    }
    __syncthreads();
    const double2 *res = smem_fft(buf, tmp, B, pt, tw, -1);
    for (int idx = threadIdx.x; idx < ncomp * M * np; idx += blockDim.x) {
        const int zp = idx % np, rest = idx / np;
        const int m = rest % M, comp = rest / M;
        const double2 *X = res + (comp * np + zp) * Th;
        const double2 A = X[m], Bv = X[(Th - m) % Th];
        // separate the two packed real transforms
        const double2 a = make_double2(0.5 * (A.x + Bv.x), 0.5 * (A.y - Bv.y));
        const double2 b = make_double2(0.5 * (A.y + Bv.y), -0.5 * (A.x - Bv.x));
        double2 *col = T + ((size_t)(comp * g.N + n) * M + m) * Z;
        const int za = z0 + 2 * zp, zb = za + 1;
        if (za < Z) col[za] = a;
        if (zb < Z) col[zb] = b;
    }
}

// z pass, (m, z) columns -> spectral with truncation: grid (m-chunk, n, comp)
__global__ void k_zfwd(const double2 *__restrict__ T, DstPtrs dst, Geo g, FFTPlan pz,
                       const double2 *__restrict__ twz, int MC) {
    extern __shared__ double2 sm[];
    const int Z = g.Z, K = g.K;
    double2 *buf = sm, *tmp = sm + MC * Z, *tw = sm + 2 * MC * Z;
    const int comp = blockIdx.z, n = blockIdx.y, m0 = blockIdx.x * MC;
    const int mc = min(MC, g.M - m0);
    for (int i = threadIdx.x; i < Z; i += blockDim.x) tw[i] = twz[i];
    const double2 *in = T + ((size_t)(comp * g.N + n) * g.M + m0) * Z;
    for (int idx = threadIdx.x; idx < mc * Z; idx += blockDim.x) buf[idx] = in[idx];
    __syncthreads();
    const double2 *res = smem_fft(buf, tmp, mc, pz, tw, -1);
    double2 *f = dst.p[comp] + (size_t)n * g.Hp;
    for (int idx = threadIdx.x; idx < mc * (2 * K - 1); idx += blockDim.x) {
        const int c = idx / (2 * K - 1), kk = idx - c * (2 * K - 1) - (K - 1);
        const int m = m0 + c;
        if (m == 0) {
            if (kk >= 0) f[kk] = res[c * Z + kk];
        } else {
            f[m * (2 * K - 1) + kk] = res[c * Z + (kk >= 0 ? kk : Z + kk)];
        }
    }
}

static size_t zpass_smem(const pf_ctx *ctx, int MC) { return (size_t)(2 * MC + 1) * ctx->g.Z * sizeof(double2); }
static size_t thpass_smem(const pf_ctx *ctx, int ncomp, int ZC) {
    return ((size_t)2 * ncomp * (ZC / 2) + 1) * ctx->g.Th * sizeof(double2);
}

static const size_t kSmemBudget = 200 * 1024;

static int pick_mc(const pf_ctx *ctx) {
    int MC = ctx->g.M;
    while (MC > 1 && zpass_smem(ctx, MC) > 96 * 1024) --MC;
    return MC;
}
static int pick_zc(const pf_ctx *ctx, int ncomp) {
    int ZC = 16;
    while (ZC > 2 && thpass_smem(ctx, ncomp, ZC) > kSmemBudget) ZC -= 2;
    return ZC;
}

static int set_smem(const void *fn, size_t bytes) { return pf_raise_smem(fn, bytes); }

int pf_launch_coll2phys(pf_ctx *ctx, int ncomp, const double2 *const *src, double *const *dst) {
    const Geo &g = ctx->g;
    SrcPtrs sp{};
    PhysPtrs pp{};
    for (int c = 0; c < ncomp; ++c) {
        sp.p[c] = src[c];
        pp.p[c] = dst[c];
    }
    const int MC = pick_mc(ctx);
    size_t sz = zpass_smem(ctx, MC);
    PF_TRY(set_smem((const void *)k_zinv, sz));
    dim3 gz((g.M + MC - 1) / MC, g.N, ncomp);
    {
        ProfScope ps_(ctx, PF_K_ZINV);
        k_zinv<<<gz, FFT_THREADS, sz, ctx->stream>>>(sp, (double2 *)ctx->T, g, ctx->planZ, ctx->twZ, MC);
    }
    PF_LAUNCHED(ctx);
    const int ZC = pick_zc(ctx, ncomp);
    sz = thpass_smem(ctx, ncomp, ZC);
    PF_TRY(set_smem((const void *)k_thinv, sz));
    dim3 gt((g.Z + ZC - 1) / ZC, g.N);
    {
        ProfScope ps_(ctx, PF_K_THINV);
        k_thinv<<<gt, FFT_THREADS, sz, ctx->stream>>>((const double2 *)ctx->T, pp, ncomp, g, ctx->planT, ctx->twT, ZC);
    }
    PF_LAUNCHED(ctx);
    return PF_OK;
}

int pf_launch_phys2coll(pf_ctx *ctx, int ncomp, const double *const *src, double2 *const *dst, bool cross) {
    const Geo &g = ctx->g;
    CPhysPtrs sp{};
    DstPtrs dp{};
    const int nin = cross ? 6 : ncomp;
    for (int c = 0; c < nin; ++c) sp.p[c] = src[c];
    for (int c = 0; c < ncomp; ++c) dp.p[c] = dst[c];
    const int ZC = pick_zc(ctx, ncomp);
    size_t sz = thpass_smem(ctx, ncomp, ZC);
    PF_TRY(set_smem((const void *)k_thfwd, sz));
    dim3 gt((g.Z + ZC - 1) / ZC, g.N);
    const double scale = 1.0 / (double)(g.Z * g.Th);  // transform.fftw3.f90:114
    {
        ProfScope ps_(ctx, PF_K_THFWD);
        k_thfwd<<<gt, FFT_THREADS, sz, ctx->stream>>>(sp, ncomp, cross ? 1 : 0, (double2 *)ctx->T, g, ctx->planT,
                                                       ctx->twT, ZC, scale);
    }
    PF_LAUNCHED(ctx);
    const int MC = pick_mc(ctx);
    sz = zpass_smem(ctx, MC);
    PF_TRY(set_smem((const void *)k_zfwd, sz));
    dim3 gz((g.M + MC - 1) / MC, g.N, ncomp);
    {
        ProfScope ps_(ctx, PF_K_ZFWD);
        k_zfwd<<<gz, FFT_THREADS, sz, ctx->stream>>>((const double2 *)ctx->T, dp, g, ctx->planZ, ctx->twZ, MC);
    }
    PF_LAUNCHED(ctx);
    return PF_OK;
}

// ------------------------------------------------------------ CFL maxima
// per radial point: max|u_r|, max|u_t|, max|u_z + 1 - r^2| (velocity.f90:459-467)
__global__ void k_maxphys(const double *__restrict__ pr, const double *__restrict__ pt,
                          const double *__restrict__ pz, double *out, DevMesh dm, Geo g) {
    const int n = blockIdx.x;
    const size_t plane = (size_t)g.Th * g.Z;
    const double base = 1.0 - dm.rp[4 * g.N + n] * dm.rp[4 * g.N + n];
    double a = 0.0, b = 0.0, c = 0.0;
    for (size_t i = threadIdx.x; i < plane; i += blockDim.x) {
        const size_t at = (size_t)n * plane + i;
        a = fmax(a, fabs(pr[at]));
        b = fmax(b, fabs(pt[at]));
        c = fmax(c, fabs(pz[at] + base));
    }
    __shared__ double s[3][32];
    for (int o = 16; o > 0; o >>= 1) {
        a = fmax(a, __shfl_xor_sync(0xffffffffu, a, o));
        b = fmax(b, __shfl_xor_sync(0xffffffffu, b, o));
        c = fmax(c, __shfl_xor_sync(0xffffffffu, c, o));
    }
    const int w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    if ((threadIdx.x & 31) == 0) {
        s[0][w] = a;
        s[1][w] = b;
        s[2][w] = c;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int i = 1; i < nw; ++i) {
            a = fmax(a, s[0][i]);
            b = fmax(b, s[1][i]);
            c = fmax(c, s[2][i]);
        }
        out[3 * n + 0] = a;
        out[3 * n + 1] = b;
        out[3 * n + 2] = c;
    }
}

int pf_launch_maxtstep(pf_ctx *ctx, double *dt3) {
    const Geo &g = ctx->g;
    std::vector<double> mx(3 * g.N);
    if (ctx->cfl_fused) {  // maxima left by the fused theta pass
        std::vector<unsigned long long> bits(3 * g.N);
        PF_CUDA(cudaMemcpyAsync(bits.data(), ctx->cflmax, bits.size() * sizeof(unsigned long long),
                                cudaMemcpyDeviceToHost, ctx->stream));
        PF_CUDA(cudaStreamSynchronize(ctx->stream));
        for (int i = 0; i < 3 * g.N; ++i) mx[i] = bits_to_double(bits[i]);
    } else {
    {
        ProfScope ps_(ctx, PF_K_EW);
        k_maxphys<<<g.N, 256, 0, ctx->stream>>>(ctx->phys[0].d, ctx->phys[1].d, ctx->phys[2].d, ctx->red, ctx->dm, g);
    }
    PF_LAUNCHED(ctx);
    PF_CUDA(cudaMemcpyAsync(mx.data(), ctx->red, mx.size() * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    PF_CUDA(cudaStreamSynchronize(ctx->stream));
    }
    const double PI = 3.1415926535897931;
    const std::vector<double> &r = ctx->hm.r;
    const int N = g.N;
    double dt[3] = {1e99, 1e99, 1e99};
    for (int n = 0; n < N; ++n) {
        double d;
        if (n == 0) d = r[1] - r[0];
        else if (n == N - 1) d = r[N - 1] - r[N - 2];
        else d = std::min(r[n] - r[n - 1], r[n + 1] - r[n]);
        if (mx[3 * n] != 0.0) dt[0] = std::min(dt[0], d / mx[3 * n]);
        d = 2.0 * PI / (double)(g.Th * g.Mp);
        if (mx[3 * n + 1] != 0.0) dt[1] = std::min(dt[1], d / mx[3 * n + 1]);
        d = 2.0 * PI / (g.alpha * g.Z);
        if (mx[3 * n + 2] != 0.0) dt[2] = std::min(dt[2], d / mx[3 * n + 2]);
    }
    for (int i = 0; i < 3; ++i) dt3[i] = dt[i];
    return PF_OK;
}

// ------------------------------------------------------------------ C ABI
extern "C" int pf_tra_coll2phys(const pf_coll *c, pf_phys *p) {
    PF_ARG(c && p && c->ctx == p->ctx, "pf_tra_coll2phys: bad argument");
    const double2 *src[1] = {c->d};
    double *dst[1] = {p->d};
    return pf_launch_coll2phys(c->ctx, 1, src, dst);
}

extern "C" int pf_tra_phys2coll(const pf_phys *p, pf_coll *c) {
    PF_ARG(c && p && c->ctx == p->ctx, "pf_tra_phys2coll: bad argument");
    const double *src[1] = {p->d};
    double2 *dst[1] = {c->d};
    return pf_launch_phys2coll(c->ctx, 1, src, dst, false);
}
