// Spectral -> physical transform of one coll field that allocates no device
// memory: the variant of var_coll2spec + tra_spec2phys for callers that
// cannot call cudaMalloc (for example a host code whose device memory is
// owned by another allocator or pool, a loop that must not allocate while a
// stream is being captured elsewhere, or a Fortran driver that only hands
// over device pointers it allocated itself).
//
// Its scratch is the file-scope array below, PF_NOALLOC_SCRATCH_BYTES
// (24 MiB) in size; every GPU that loads this library holds it until the
// process exits.  The first 64 KiB hold the twiddle tables of every built
// transform length, written once per device at set-up; the rest holds the
// (m, z) intermediate of the z pass.  All calls share the intermediate and it
// keeps the previous call's contents (nothing in it has to start at zero:
// every call writes every entry it later reads).  Calls that overlap on the
// GPU -- on different streams, or from different host threads without
// ordering -- race on it.
//
// Host code must not hand the array's name to a kernel: in host code the name
// denotes a host-side stand-in.  The first call made on a device, with that
// device current, does the set-up: it looks up the device address with
// cudaGetSymbolAddress and writes the twiddle tables with a synchronous copy.
// Make that first call before any stream capture.  Every later call only
// queues its two kernels on the caller's stream.  The address and the tables
// are kept per device ordinal for the life of the process; a cudaDeviceReset
// in the caller discards the tables, and this entry point is not usable on
// that device after one.
#include <cmath>
#include <mutex>
#include "pf_internal.cuh"
#include "pf_fftcore.cuh"

static __device__ __align__(256) unsigned char g_noalloc_scratch[PF_NOALLOC_SCRATCH_BYTES];

static constexpr size_t kTwiddleBytes = 64 * 1024;  // tables of all built lengths (21 KiB used)
static std::mutex g_noalloc_mu;
static void *g_noalloc_addr[256];

#define PF_NA_LENGTHS(X) X(12) X(15) X(18) X(24) X(36) X(48) X(72) X(96) X(144) X(192) X(288) X(384)
static const int kLengths[] = {
#define PF_CASE(L) L,
    PF_NA_LENGTHS(PF_CASE)
#undef PF_CASE
};
static constexpr int kNumLengths = (int)(sizeof(kLengths) / sizeof(kLengths[0]));

// offset (in double2 entries) of length L's table exp(+2 pi i t/L), t < L,
// in the twiddle region; -1 if L is not built
static int twiddle_offset(int L) {
    int off = 0;
    for (int i = 0; i < kNumLengths; ++i) {
        if (kLengths[i] == L) return off;
        off += kLengths[i];
    }
    return -1;
}

// Set-up, once per device: the scratch address, and the twiddle tables of
// every built length (rounded once from long double) written into its first
// kTwiddleBytes with a synchronous copy from host memory.
static int scratch_address(int dev, unsigned char **out) {
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (dev < 0 || dev >= 256) {
        pf_set_error("pf_tra_coll2phys_noalloc: device index %d out of range", dev);
        return PF_ERR_ARG;
    }
    if (!g_noalloc_addr[dev]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            pf_set_error("pf_tra_coll2phys_noalloc: cudaGetSymbolAddress failed: %s", cudaGetErrorString(e));
            return PF_ERR_CUDA;
        }
        std::vector<double2> tw;
        for (int i = 0; i < kNumLengths; ++i) {
            const int L = kLengths[i];
            for (int t = 0; t < L; ++t) {
                const long double a = 2.0L * 3.14159265358979323846264338327950288L * (long double)t / (long double)L;
                tw.push_back(make_double2((double)cosl(a), (double)sinl(a)));
            }
        }
        static_assert(kTwiddleBytes >= 1329 * sizeof(double2), "twiddle region too small");
        e = cudaMemcpy(p, tw.data(), tw.size() * sizeof(double2), cudaMemcpyHostToDevice);
        if (e != cudaSuccess) {
            pf_set_error("pf_tra_coll2phys_noalloc: twiddle set-up copy failed: %s", cudaGetErrorString(e));
            return PF_ERR_CUDA;
        }
        g_noalloc_addr[dev] = p;
    }
    *out = static_cast<unsigned char *>(g_noalloc_addr[dev]);
    return PF_OK;
}

// z pass: reference coll layout in (re[nh*N+n], im[...]), (m, z) columns out
template <int ZL>
__global__ void __launch_bounds__(256) k_na_zinv(const double *__restrict__ re, const double *__restrict__ im,
                                                 double2 *__restrict__ T, const double2 *__restrict__ twz, int N,
                                                 int K, int M, int MC) {
    extern __shared__ __align__(16) unsigned char smraw[];
    double2 *buf = reinterpret_cast<double2 *>(smraw);
    double2 *tmp = buf + MC * ZL, *tw = tmp + MC * ZL;
    const int n = blockIdx.y, m0 = blockIdx.x * MC;
    const int mc = min(MC, M - m0);
    for (int i = threadIdx.x; i < ZL; i += blockDim.x) tw[i] = twz[i];
    for (int idx = threadIdx.x; idx < mc * ZL; idx += blockDim.x) {
        const int c = idx / ZL, j = idx - c * ZL;
        const int m = m0 + c;
        double2 v = make_double2(0.0, 0.0);
        int nh = -1;
        bool conj = false;
        if (m == 0) {
            if (j < K) nh = j;
            else if (j >= 2 * K + 1) {
                nh = ZL - j;
                conj = true;
            }
        } else if (j < K) {
            nh = m * (2 * K - 1) + j;
        } else if (j >= 2 * K + 1) {
            nh = m * (2 * K - 1) + (j - ZL);
        }
        if (nh >= 0) {
            v = make_double2(re[(size_t)nh * N + n], im[(size_t)nh * N + n]);
            if (conj) v.y = -v.y;
        }
        buf[idx] = v;
    }
    __syncthreads();
    const double2 *res = smem_fft_t<ZL, +1>(buf, tmp, mc, tw);
    double2 *out = T + ((size_t)n * M + m0) * ZL;
    for (int idx = threadIdx.x; idx < mc * ZL; idx += blockDim.x) out[idx] = res[idx];
}

// theta pass (c2r, two real rows per complex FFT) into the phys layout
template <int TL>
__global__ void __launch_bounds__(256) k_na_thinv(const double2 *__restrict__ T, double *__restrict__ phys,
                                                  const double2 *__restrict__ twt, int M, int Z, int ZC) {
    extern __shared__ __align__(16) unsigned char smraw[];
    const int np = ZC / 2;
    double2 *buf = reinterpret_cast<double2 *>(smraw);
    double2 *tmp = buf + np * TL, *tw = tmp + np * TL;
    const int n = blockIdx.y, z0 = blockIdx.x * ZC;
    for (int i = threadIdx.x; i < TL; i += blockDim.x) tw[i] = twt[i];
    for (int i = threadIdx.x; i < np * TL; i += blockDim.x) buf[i] = make_double2(0.0, 0.0);
    __syncthreads();
    for (int idx = threadIdx.x; idx < M * np; idx += blockDim.x) {
        const int zp = idx % np, m = idx / np;
        const int za = z0 + 2 * zp, zb = za + 1;
        const double2 *col = T + ((size_t)n * M + m) * Z;
        const double2 a = (za < Z) ? col[za] : make_double2(0.0, 0.0);
        const double2 b = (zb < Z) ? col[zb] : make_double2(0.0, 0.0);
        double2 *X = buf + zp * TL;
        if (m == 0) {
            X[0] = make_double2(a.x, b.x);
        } else {
            X[m] = make_double2(a.x - b.y, a.y + b.x);
            X[TL - m] = make_double2(a.x + b.y, -a.y + b.x);
        }
    }
    __syncthreads();
    const double2 *res = smem_fft_t<TL, +1>(buf, tmp, np, tw);
    for (int idx = threadIdx.x; idx < TL * ZC; idx += blockDim.x) {
        const int zz = idx % ZC, t = idx / ZC;
        const int z = z0 + zz;
        if (z >= Z) continue;
        const double2 v = res[(zz / 2) * TL + t];
        phys[((size_t)n * TL + t) * Z + z] = (zz & 1) ? v.y : v.x;
    }
}

static bool na_length_ok(int L) {
    switch (L) {
#define PF_CASE(L) case L:
        PF_NA_LENGTHS(PF_CASE)
#undef PF_CASE
        return true;
    default:
        return false;
    }
}

extern "C" int pf_tra_coll2phys_noalloc(int N, int K, int M, const double *re, const double *im, double *phys,
                                        void *cuda_stream) {
    PF_ARG(re && im && phys, "pf_tra_coll2phys_noalloc: null pointer");
    PF_ARG(N >= 1 && K >= 1 && M >= 1, "pf_tra_coll2phys_noalloc: N, K, M must be >= 1");
    const int Z = 3 * K, Th = 3 * M;
    if (!na_length_ok(Z) || !na_length_ok(Th)) {
        pf_set_error("pf_tra_coll2phys_noalloc: transform lengths 3K=%d, 3M=%d are not among the built ones "
                     "(12 15 18 24 36 48 72 96 144 192 288 384)", Z, Th);
        return PF_ERR_ARG;
    }
    const size_t need = kTwiddleBytes + (size_t)N * M * Z * sizeof(double2);
    if (need > PF_NOALLOC_SCRATCH_BYTES) {
        pf_set_error("pf_tra_coll2phys_noalloc: N*M*3K*16 + 64 KiB = %zu bytes exceeds the %u-byte static scratch",
                     need, (unsigned)PF_NOALLOC_SCRATCH_BYTES);
        return PF_ERR_ARG;
    }
    int dev = 0;
    PF_CUDA(cudaGetDevice(&dev));
    unsigned char *scratch = nullptr;
    PF_TRY(scratch_address(dev, &scratch));
    cudaStream_t st = (cudaStream_t)cuda_stream;
    const double2 *tables = reinterpret_cast<const double2 *>(scratch);
    const double2 *twz = tables + twiddle_offset(Z);
    const double2 *twt = tables + twiddle_offset(Th);
    double2 *T = reinterpret_cast<double2 *>(scratch + kTwiddleBytes);
    int MC = M;
    while (MC > 1 && (size_t)(2 * MC + 1) * Z * sizeof(double2) > 60 * 1024) --MC;
    const size_t zsm = (size_t)(2 * MC + 1) * Z * sizeof(double2);
    const dim3 gz((M + MC - 1) / MC, N);
    switch (Z) {
#define PF_CASE(L)                                                                                        \
    case L:                                                                                               \
        PF_TRY(pf_raise_smem((const void *)k_na_zinv<L>, zsm));                                          \
        k_na_zinv<L><<<gz, 256, zsm, st>>>(re, im, T, twz, N, K, M, MC);                                   \
        break;
        PF_NA_LENGTHS(PF_CASE)
#undef PF_CASE
    }
    PF_CHECK_LAUNCH();
    const int ZC = 16;
    const size_t tsm = ((size_t)2 * (ZC / 2) + 1) * Th * sizeof(double2);
    const dim3 gt((Z + ZC - 1) / ZC, N);
    switch (Th) {
#define PF_CASE(L)                                                                                         \
    case L:                                                                                                \
        PF_TRY(pf_raise_smem((const void *)k_na_thinv<L>, tsm));                                          \
        k_na_thinv<L><<<gt, 256, tsm, st>>>(T, phys, twt, M, Z, ZC);                                        \
        break;
        PF_NA_LENGTHS(PF_CASE)
#undef PF_CASE
    }
    PF_CHECK_LAUNCH();
    return PF_OK;
}
