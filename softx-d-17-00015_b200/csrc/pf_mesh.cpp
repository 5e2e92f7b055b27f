// Radial mesh and finite-difference weights, computed once per context on the
// host in FP64 and uploaded (precompute only; meshs.f90:66-225, cheby.f:2-108).
#include <cmath>
#include <cstring>
#include <vector>
#include "pf_internal.cuh"

static const double kPI = 3.1415926535897931;  // d_PI, parameters.f90:51

// d/dx of a shifted-Chebyshev series a[0..M-1] on [0,1] (cheby.f:69-108)
static void cheb_deriv(const std::vector<double> &a, std::vector<double> &ax) {
    const int M = (int)a.size();
    ax.assign(M, 0.0);
    if (M == 1) return;
    if (M == 2) { ax[0] = 2.0 * a[1]; return; }
    if (M == 3) { ax[0] = 2.0 * a[1]; ax[1] = 8.0 * a[2]; return; }
    if (M == 4) {
        ax[0] = 2.0 * a[1] + 6.0 * a[3];
        ax[1] = 8.0 * a[2];
        ax[2] = 12.0 * a[3];
        return;
    }
    ax[M - 2] = -4.0 * (1.0 - M) * a[M - 1];
    ax[M - 3] = -4.0 * (2.0 - M) * a[M - 2];
    for (int J = M - 3; J >= 2; --J) ax[J - 1] = 4.0 * J * a[J] + ax[J + 1];
    ax[0] = 2.0 * a[1] + ax[2] / 2.0;
}

// Clenshaw evaluation at x of a shifted-Chebyshev series (cheby.f:38-67)
static double cheb_eval(const std::vector<double> &a, double x) {
    const int M = (int)a.size();
    std::vector<double> b(M + 3, 0.0);
    const double xa = 2.0 * x - 1.0, xb = 2.0 * xa;
    for (int J = M - 1; J >= 0; --J) b[J + 1] = xb * b[J + 2] - b[J + 3] + a[J];
    return b[1] - xa * b[2];
}

// nd-th derivative of T_m(2x-1) at x (cheby.f:2-36)
static double cheby(int m, int nd, double x) {
    if (m == 0) return nd == 0 ? 1.0 : 0.0;
    std::vector<double> a(m + 1, 0.0), ax;
    a[m] = 1.0;
    for (int i = 0; i < nd; ++i) {
        cheb_deriv(a, ax);
        a = ax;
    }
    return cheb_eval(a, x);
}

// In-place inverse of an n x n row-major matrix (Gauss-Jordan, partial pivoting).
static bool invert(int n, std::vector<double> &A) {
    std::vector<double> I(n * n, 0.0);
    for (int i = 0; i < n; ++i) I[i * n + i] = 1.0;
    for (int c = 0; c < n; ++c) {
        int p = c;
        for (int r = c + 1; r < n; ++r)
            if (std::fabs(A[r * n + c]) > std::fabs(A[p * n + c])) p = r;
        if (A[p * n + c] == 0.0) return false;
        if (p != c)
            for (int k = 0; k < n; ++k) {
                std::swap(A[p * n + k], A[c * n + k]);
                std::swap(I[p * n + k], I[c * n + k]);
            }
        const double inv = 1.0 / A[c * n + c];
        for (int k = 0; k < n; ++k) {
            A[c * n + k] *= inv;
            I[c * n + k] *= inv;
        }
        for (int r = 0; r < n; ++r) {
            if (r == c) continue;
            const double f = A[r * n + c];
            if (f == 0.0) continue;
            for (int k = 0; k < n; ++k) {
                A[r * n + k] -= f * A[c * n + k];
                I[r * n + k] -= f * I[c * n + k];
            }
        }
    }
    A = I;
    return true;
}

// Weights w(1..n) with sum_j w_j f(x_j) = f^(i)(x0) (meshs.f90:200-225)
static bool mes_weights(int i, int n, const double *x, double x0, double *w) {
    double xl = x0, xr = x0;
    for (int j = 0; j < n; ++j) {
        xl = std::min(xl, x[j]);
        xr = std::max(xr, x[j]);
    }
    std::vector<double> A(n * n), d(n);
    const double x0_ = (x0 - xl) / (xr - xl);
    for (int j = 0; j < n; ++j) {
        for (int p = 0; p < n; ++p) A[p * n + j] = cheby(j, 0, (x[p] - xl) / (xr - xl));
        d[j] = cheby(j, i, x0_);
    }
    if (!invert(n, A)) return false;
    double s = 1.0;
    for (int q = 0; q < i; ++q) s *= (xr - xl);
    for (int j = 0; j < n; ++j) {
        double acc = 0.0;
        for (int k = 0; k < n; ++k) acc += d[k] * A[k * n + j];
        w[j] = acc / s;
    }
    return true;
}

int pf_build_mesh(int N, const double *custom_r, HostMesh &hm) {
    hm.r.assign(N, 0.0);
    if (custom_r) {  // mesh.in (meshs.f90:76-88)
        for (int n = 0; n < N; ++n) hm.r[n] = custom_r[n];
        if (hm.r[0] < 0.0) { pf_set_error("mes_precompute: mesh.in err 2"); return PF_ERR_ARG; }
        if (std::fabs(hm.r[N - 1] - 1.0) > 1e-8) {
            pf_set_error("mes_precompute: mesh.in err 3");
            return PF_ERR_ARG;
        }
    } else {  // default mesh (meshs.f90:90-99)
        const int N_ = N + (int)std::sqrt((double)N);
        for (int n = N_ - N + 1; n <= N_; ++n)
            hm.r[n - N_ + N - 1] = 0.5 * (1.0 + std::cos(kPI * (N_ - n) / (double)N_));
        for (int it = 0; it < 10; ++it) {
            const double dr = 1.5 * hm.r[0] - 0.5 * hm.r[1];
            for (int n = 0; n < N; ++n) hm.r[n] = hm.r[n] * (1.0 + dr) - dr;
        }
    }
    const std::vector<double> &r = hm.r;
    hm.rp.assign(7 * N, 0.0);
    for (int n = 0; n < N; ++n) {
        const double x = r[n];
        hm.rp[0 * N + n] = 1.0 / (x * x * x);
        hm.rp[1 * N + n] = 1.0 / (x * x);
        hm.rp[2 * N + n] = 1.0 / x;
        hm.rp[3 * N + n] = 1.0;
        hm.rp[4 * N + n] = x;
        hm.rp[5 * N + n] = x * x;
        hm.rp[6 * N + n] = x * x * x;
    }
    std::vector<double> r_(N + 1);
    r_[0] = 0.0;
    for (int n = 0; n < N; ++n) r_[n + 1] = r[n];
    double w[NBAND];
    // dr(i) bands (meshs.f90:149-159)
    hm.dr.assign(KL * NBAND * N, 0.0);
    for (int n = 1; n <= N; ++n) {
        const int l = std::max(1, n - KL), rr = std::min(n + KL, N), nn = rr - l + 1;
        for (int i = 1; i <= KL; ++i) {
            if (!mes_weights(i, nn, &r_[l], r_[n], w)) goto singular;
            for (int j = l; j <= rr; ++j)
                hm.dr[((i - 1) * NBAND + (KL + n - j)) * N + (j - 1)] = w[j - l];
        }
    }
    // dr0 / dr1 extrapolation weights (meshs.f90:161-164)
    hm.dr0.assign((KL + 1) * (KL + 1), 0.0);
    hm.dr1.assign((KL + 1) * (KL + 1), 0.0);
    for (int i = 0; i <= KL; ++i) {
        if (!mes_weights(i, KL + 1, &r_[1], r_[0], &hm.dr0[i * (KL + 1)])) goto singular;
        if (!mes_weights(i, KL + 1, &r_[N - KL], r_[N], &hm.dr1[i * (KL + 1)])) goto singular;
    }
    // radLap = drr + (1/r) dr (meshs.f90:166-174)
    hm.radLap.assign(NBAND * N, 0.0);
    for (int j = 1; j <= N; ++j) {
        const int l = std::max(1, j - KL), rr = std::min(j + KL, N);
        for (int n = l; n <= rr; ++n) {
            const int row = KL + n - j;
            hm.radLap[row * N + (j - 1)] = hm.dr[(1 * NBAND + row) * N + (j - 1)]
                                         + hm.dr[(0 * NBAND + row) * N + (j - 1)] / r_[n];
        }
    }
    // intrdr quadrature of  f r dr  (meshs.f90:176-192)
    hm.intrdr.assign(N, 0.0);
    {
        double A[NBAND][NBAND];
        for (int n = 1; n <= N; ++n) {
            const int l = std::max(1, n - KL), rr = std::min(n + KL, N), nn = rr - l + 1;
            for (int i = 1; i <= nn; ++i) {
                if (!mes_weights(i - 1, nn, &r_[l], r_[n], w)) goto singular;
                for (int q = 0; q < nn; ++q) A[i - 1][q] = w[q];
            }
            double c = 1.0, e = 1.0;
            for (int i = 1; i <= nn; ++i) {
                c = c * (r_[std::min(n + 1, N)] - r_[n]) / (double)i;
                e = e * (r_[std::max(0, n - 1)] - r_[n]) / (double)i;
                for (int q = 0; q < nn; ++q)
                    hm.intrdr[l - 1 + q] = hm.intrdr[l - 1 + q] + 0.5 * (c - e) * A[i - 1][q] * r_[n];
            }
        }
    }
    return PF_OK;
singular:
    pf_set_error("matrix inversion error 1");
    return PF_ERR_SINGULAR;
}

// Factor L into radices (4 first, then 2, 3, 5, 7, 11, 13).
int pf_make_plan(int L, FFTPlan &p) {
    p.L = L;
    p.nf = 0;
    int rem = L;
    const int rads[] = {4, 2, 3, 5, 7, 11, 13};
    for (int ri = 0; ri < 7 && rem > 1; ++ri) {
        const int r = rads[ri];
        while (rem % r == 0) {
            if (p.nf >= 16) return PF_ERR_ARG;
            p.f[p.nf++] = r;
            rem /= r;
        }
    }
    if (rem != 1) {
        pf_set_error("FFT length %d has a prime factor > 13", L);
        return PF_ERR_ARG;
    }
    return PF_OK;
}
