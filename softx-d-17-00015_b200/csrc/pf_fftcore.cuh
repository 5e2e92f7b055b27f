// Shared-memory mixed-radix Stockham FFT with the transform length known at
// compile time: the radix sequence (4s, then 2, 3, 5, 7) and all index
// arithmetic are constants, and each butterfly lives in registers.
//
// B batches of length L sit contiguously (batch stride L) in `src`; `dst` is
// the ping-pong buffer; tw[t] = exp(+2 pi i t / L).  SIGN=+1 is FFTW's
// unnormalised backward transform, SIGN=-1 the forward one.  The Stockham
// pass with radix R maps butterfly j (k = j mod Ns) to outputs
// (j/Ns)*Ns*R + k + q*Ns after twiddling input q by W^(SIGN q k L/(Ns R)).
#pragma once
#include <cuda_runtime.h>

template <typename C> struct CTraits;
template <> struct CTraits<double2> {
    using R = double;
    static __device__ __forceinline__ double2 make(double x, double y) { return make_double2(x, y); }
};
template <> struct CTraits<float2> {
    using R = float;
    static __device__ __forceinline__ float2 make(float x, float y) { return make_float2(x, y); }
};

template <typename C> __device__ __forceinline__ C c_add(C a, C b) { return CTraits<C>::make(a.x + b.x, a.y + b.y); }
template <typename C> __device__ __forceinline__ C c_sub(C a, C b) { return CTraits<C>::make(a.x - b.x, a.y - b.y); }
template <typename C> __device__ __forceinline__ C c_mul(C a, C b) {
    return CTraits<C>::make(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// a * (SIGN * i)
template <int SIGN, typename C> __device__ __forceinline__ C c_muli(C a) {
    return SIGN > 0 ? CTraits<C>::make(-a.y, a.x) : CTraits<C>::make(a.y, -a.x);
}
template <int SIGN, typename C> __device__ __forceinline__ C c_tw(C w) {
    return SIGN > 0 ? w : CTraits<C>::make(w.x, -w.y);
}

__host__ __device__ constexpr int fft_first_radix(int L) {
    return L % 4 == 0 ? 4 : L % 2 == 0 ? 2 : L % 3 == 0 ? 3 : L % 5 == 0 ? 5 : L % 7 == 0 ? 7 : L;
}
__host__ __device__ constexpr bool fft_supported(int L) {
    while (L > 1) {
        const int r = fft_first_radix(L);
        if (r > 7) return false;
        L /= r;
    }
    return true;
}

template <int R, int SIGN, typename C>
__device__ __forceinline__ void fft_dft(C (&v)[R], const C *tw, int L) {
    if constexpr (R == 2) {
        const C a = v[0];
        v[0] = c_add(a, v[1]);
        v[1] = c_sub(a, v[1]);
    } else if constexpr (R == 4) {
        const C a = c_add(v[0], v[2]), b = c_sub(v[0], v[2]);
        const C c = c_add(v[1], v[3]), d = c_muli<SIGN>(c_sub(v[1], v[3]));
        v[0] = c_add(a, c);
        v[1] = c_add(b, d);
        v[2] = c_sub(a, c);
        v[3] = c_sub(b, d);
    } else if constexpr (R == 3) {
        using T = typename CTraits<C>::R;
        const T s3 = (T)0.86602540378443864676;  // sin(2 pi / 3)
        const C t = c_add(v[1], v[2]);
        const C u = CTraits<C>::make(v[0].x - (T)0.5 * t.x, v[0].y - (T)0.5 * t.y);
        const C w = c_muli<SIGN>(CTraits<C>::make(s3 * (v[1].x - v[2].x), s3 * (v[1].y - v[2].y)));
        v[0] = c_add(v[0], t);
        v[1] = c_add(u, w);
        v[2] = c_sub(u, w);
    } else {  // small prime: direct DFT with table twiddles
        C o[R];
        const int st = L / R;
#pragma unroll
        for (int q = 0; q < R; ++q) {
            C acc = v[0];
#pragma unroll
            for (int p = 1; p < R; ++p) acc = c_add(acc, c_mul(v[p], c_tw<SIGN>(tw[((p * q) % R) * st])));
            o[q] = acc;
        }
#pragma unroll
        for (int q = 0; q < R; ++q) v[q] = o[q];
    }
}

template <int L, int R, int NS, int SIGN, typename C>
__device__ __forceinline__ void fft_pass(const C *__restrict__ src, C *__restrict__ dst, int B, const C *tw) {
    constexpr int NB = L / R;
    constexpr int STRIDE = L / (NS * R);
    for (int idx = threadIdx.x; idx < NB * B; idx += blockDim.x) {
        const int b = idx / NB, j = idx - b * NB;
        const int k = j % NS;
        const C *sp = src + b * L;
        C *dp = dst + b * L;
        C v[R];
#pragma unroll
        for (int q = 0; q < R; ++q) {
            C x = sp[j + q * NB];
            if (NS > 1 && q > 0) x = c_mul(x, c_tw<SIGN>(tw[q * k * STRIDE]));
            v[q] = x;
        }
        fft_dft<R, SIGN>(v, tw, L);
        const int base = (j / NS) * NS * R + k;
#pragma unroll
        for (int q = 0; q < R; ++q) dp[base + q * NS] = v[q];
    }
}

// Runs all passes; returns the buffer that holds the result.  Every thread
// of the block must call it (it synchronises between passes).
template <int L, int REM, int NS, int SIGN, typename C>
__device__ __forceinline__ C *fft_run(C *src, C *dst, int B, const C *tw) {
    if constexpr (REM == 1) {
        return src;
    } else {
        constexpr int R = fft_first_radix(REM);
        fft_pass<L, R, NS, SIGN>(src, dst, B, tw);
        __syncthreads();
        return fft_run<L, REM / R, NS * R, SIGN>(dst, src, B, tw);
    }
}

template <int L, int SIGN, typename C>
__device__ __forceinline__ C *smem_fft_t(C *buf, C *tmp, int B, const C *tw) {
    return fft_run<L, L, 1, SIGN>(buf, tmp, B, tw);
}

// ---------------------------------------------------------------------------
// Register codelets and the four-step transform.
//
// rfft_run<R>: an R-point FFT (R <= 32) of v[R] held in registers; every index
// is a compile-time constant so nothing spills to local memory.  Internal
// twiddles W_R^e are read from a table of exp(+2 pi i t/LT) at tw[e*tws]
// (LT = R*tws); all threads read the same entry, so the reads broadcast.
template <int R, int REM, int NS, int SIGN, typename C>
__device__ __forceinline__ void rfft_stage(const C (&src)[R], C (&dst)[R], const C *tw, int tws) {
    constexpr int RR = fft_first_radix(REM);
    constexpr int NB = R / RR;
    constexpr int STRIDE = R / (NS * RR);
#pragma unroll
    for (int j = 0; j < NB; ++j) {
        const int k = j % NS;
        C v[RR];
#pragma unroll
        for (int q = 0; q < RR; ++q) {
            C x = src[j + q * NB];
            if (NS > 1 && q > 0 && k > 0) x = c_mul(x, c_tw<SIGN>(tw[(q * k * STRIDE) * tws]));
            v[q] = x;
        }
        fft_dft<RR, SIGN>(v, tw, R * tws);
        const int base = (j / NS) * NS * RR + k;
#pragma unroll
        for (int q = 0; q < RR; ++q) dst[base + q * NS] = v[q];
    }
}

template <int R, int REM, int NS, int SIGN, typename C>
__device__ __forceinline__ void rfft_run(C (&a)[R], const C *tw, int tws) {
    if constexpr (REM > 1) {
        constexpr int RR = fft_first_radix(REM);
        C b[R];
        rfft_stage<R, REM, NS, SIGN>(a, b, tw, tws);
#pragma unroll
        for (int i = 0; i < R; ++i) a[i] = b[i];
        rfft_run<R, REM / RR, NS * RR, SIGN>(a, tw, tws);
    }
}

// L = L1 * L2 with both factors <= 32 and L1 as close to sqrt(L) as allowed
__host__ __device__ constexpr int fft4_l1(int L) {
    if (L <= 32) return L;
    int best = 0;
    for (int d = 1; d <= 32; ++d)
        if (L % d == 0 && L / d <= 32 && (best == 0 || (d * d <= L && d > best) || (best * best > L && d < best)))
            best = d;
    return best;
}
// padded row pitch of the transposed intermediate (odd, so 16-byte accesses
// of consecutive threads fall in distinct bank groups)
__host__ __device__ constexpr int fft4_yp(int L1) { return (L1 % 2 == 0) ? L1 + 1 : L1 + 2; }
// elements one row occupies in shared memory
__host__ __device__ constexpr int fft4_pitch(int L) {
    return fft4_l1(L) == L ? L : ((L / fft4_l1(L)) * fft4_yp(fft4_l1(L)) > L ? (L / fft4_l1(L)) * fft4_yp(fft4_l1(L)) : L);
}

// In-place FFT of B rows (row r at rows + r*RS, natural order in and out).
// tw: exp(+2 pi i t/L), t < L; tw2[k1*L2 + n2] = W_L^(n2*k1) (the four-step
// twiddles, laid out so consecutive threads read consecutive entries).
// All threads of the block must call it; it synchronises internally.
template <int L, int SIGN, typename C>
__device__ __forceinline__ void fft4_rows(C *rows, int B, int RS, const C *tw, const C *tw2) {
    constexpr int L1 = fft4_l1(L);
    constexpr int L2 = L / L1;
    if constexpr (L2 == 1) {
        for (int b = threadIdx.x; b < B; b += blockDim.x) {
            C v[L];
#pragma unroll
            for (int i = 0; i < L; ++i) v[i] = rows[b * RS + i];
            rfft_run<L, L, 1, SIGN>(v, tw, 1);
#pragma unroll
            for (int i = 0; i < L; ++i) rows[b * RS + i] = v[i];
        }
        __syncthreads();
    } else {
        constexpr int YP = fft4_yp(L1);
        // each pass of these loops covers whole rows, because a row is read
        // in one layout and rewritten in the other (blockDim.x >= 32 >= L1, L2)
        const int rp1 = blockDim.x / L2;
        // step 1: L1-point transforms over n1 of x[L2*n1 + n2], twiddle, transpose
        for (int b0 = 0; b0 < B; b0 += rp1) {
            const int b = b0 + (int)threadIdx.x / L2, n2 = (int)threadIdx.x % L2;
            const bool act = (int)threadIdx.x < rp1 * L2 && b < B;
            C v[L1];
            if (act) {
#pragma unroll
                for (int i = 0; i < L1; ++i) v[i] = rows[b * RS + L2 * i + n2];
            }
            __syncthreads();
            if (act) {
                rfft_run<L1, L1, 1, SIGN>(v, tw, L2);
#pragma unroll
                for (int k1 = 0; k1 < L1; ++k1) {
                    C w = v[k1];
                    if (k1 > 0 && n2 > 0) w = c_mul(w, c_tw<SIGN>(tw2[k1 * L2 + n2]));
                    rows[b * RS + n2 * YP + k1] = w;
                }
            }
        }
        __syncthreads();
        // step 2: L2-point transforms over n2, output X[k1 + L1*k2]
        const int rp2 = blockDim.x / L1;
        for (int b0 = 0; b0 < B; b0 += rp2) {
            const int b = b0 + (int)threadIdx.x / L1, k1 = (int)threadIdx.x % L1;
            const bool act = (int)threadIdx.x < rp2 * L1 && b < B;
            C v[L2];
            if (act) {
#pragma unroll
                for (int i = 0; i < L2; ++i) v[i] = rows[b * RS + i * YP + k1];
            }
            __syncthreads();
            if (act) {
                rfft_run<L2, L2, 1, SIGN>(v, tw, L1);
#pragma unroll
                for (int k2 = 0; k2 < L2; ++k2) rows[b * RS + k1 + L1 * k2] = v[k2];
            }
        }
        __syncthreads();
    }
}

// Fill the tables a four-step transform of length L needs (in shared memory).
template <int L, typename C>
__device__ __forceinline__ void fft4_tables(C *tw, C *tw2, const C *__restrict__ gtw) {
    constexpr int L1 = fft4_l1(L);
    constexpr int L2 = L / L1;
    for (int i = threadIdx.x; i < L; i += blockDim.x) tw[i] = gtw[i];
    for (int i = threadIdx.x; i < L; i += blockDim.x) {
        const int k1 = i / L2, n2 = i - k1 * L2;
        tw2[i] = gtw[(k1 * n2) % L];
    }
}

// ---------------------------------------------------------------------------
// Stockham passes of radix 8 or 6 where the length allows (else as above),
// each butterfly an in-register codelet (rfft_run): a length-384 row takes
// three passes (8, 8, 6) instead of five (4, 4, 4, 2, 3), so three barriers
// and shared-memory round trips instead of five.
__host__ __device__ constexpr int fft_big_radix(int L) {
    return L % 8 == 0 ? 8 : L % 6 == 0 ? 6 : fft_first_radix(L);
}

template <int L, int R, int NS, int SIGN, typename C>
__device__ __forceinline__ void fft_pass_big(const C *__restrict__ src, C *__restrict__ dst, int B, const C *tw) {
    constexpr int NB = L / R;
    constexpr int STRIDE = L / (NS * R);
    for (int idx = threadIdx.x; idx < NB * B; idx += blockDim.x) {
        const int b = idx / NB, j = idx - b * NB;
        const int k = j % NS;
        const C *sp = src + b * L;
        C *dp = dst + b * L;
        C v[R];
#pragma unroll
        for (int q = 0; q < R; ++q) {
            C x = sp[j + q * NB];
            if (NS > 1 && q > 0) x = c_mul(x, c_tw<SIGN>(tw[q * k * STRIDE]));
            v[q] = x;
        }
        if constexpr (R == 8 || R == 6) rfft_run<R, R, 1, SIGN>(v, tw, L / R);
        else fft_dft<R, SIGN>(v, tw, L);
        const int base = (j / NS) * NS * R + k;
#pragma unroll
        for (int q = 0; q < R; ++q) dp[base + q * NS] = v[q];
    }
}

template <int L, int REM, int NS, int SIGN, typename C>
__device__ __forceinline__ C *fft_run_big(C *src, C *dst, int B, const C *tw) {
    if constexpr (REM == 1) {
        return src;
    } else {
        constexpr int R = fft_big_radix(REM);
        fft_pass_big<L, R, NS, SIGN>(src, dst, B, tw);
        __syncthreads();
        return fft_run_big<L, REM / R, NS * R, SIGN>(dst, src, B, tw);
    }
}

// ---------------------------------------------------------------------------
// Per-length choice between the four-step transform (one shared-memory
// transpose, codelets in registers) and the multi-pass Stockham transform
// (a ping-pong buffer of B*L, radix-8/6 register codelets, low register use).  FP64 lengths above 192
// need ~165 registers per thread in the four-step form, which caps occupancy
// at one 256-thread block per SM; they use Stockham.
template <int L, typename C> struct FFTRows {
    static constexpr bool four = (sizeof(C) == 8) || (L <= 192);
    static constexpr int pitch = four ? fft4_pitch(L) : L;
    // shared-memory elements for B rows plus the two tables
    static __host__ __device__ constexpr int smem_elems(int B) { return (four ? B * pitch : 2 * B * L) + 2 * L; }
    // rows at `rows` (B rows, pitch `pitch`); `scratch` = rows + B*pitch
    template <int SIGN>
    static __device__ __forceinline__ void run(C *rows, int B, const C *tw, const C *tw2) {
        if constexpr (four) {
            fft4_rows<L, SIGN>(rows, B, pitch, tw, tw2);
        } else {
            C *res = fft_run_big<L, L, 1, SIGN>(rows, rows + B * L, B, tw);
            if (res != rows) {
                for (int i = threadIdx.x; i < B * L; i += blockDim.x) rows[i] = res[i];
                __syncthreads();
            }
        }
    }
};
