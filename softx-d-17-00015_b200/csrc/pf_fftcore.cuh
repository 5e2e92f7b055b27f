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
