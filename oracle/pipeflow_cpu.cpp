// CPU restatement of the openpipeflow timestep in C++ with OpenMP.
//
// TEST INFRASTRUCTURE, not the product: it times the reference's algorithm
// on the host cores (the reference's FFTW+MPI build cannot be compiled here)
// and cross-checks the numpy oracle.  The set-up work of vel_matrices (the
// clustered mesh, the banded LU factors, the influence matrices) comes from
// the numpy oracle (oracle/pipeflow_oracle.py) through pfc_set_*; this file
// restates the work of every timestep:
//   main.f90:20-44 / newton.f90:740-762   the loop body            pfc_timestep
//   velocity.f90:61-74                     vel_imposesym (mean mode)
//   velocity.f90:304-361                   vel_transform, vel_nonlinear, vel_addHPF
//   transform.fftw3.f90:65-147             tra_spec2phys, tra_phys2spec (own FFT)
//   variables.f90:378-481                  meshmult, curl, grad, div
//   velocity.f90:152-298, 367-432          adjustFlux, adjPPE, evalBC, vel_step,
//                                          vel_predictor, vel_corrector
//   timestep.f90:102-253                   lumesh_invert (dgbtrs + dtbsv
//                                          semantics), meshmult, zerobc,
//                                          nlincorr, measurecorr, check_cgce
// Fields are (N, H) row-major arrays [n*H + nh], Re and Im apart, as the
// numpy oracle holds them.  OpenMP splits the per-mode work over modes and
// the transforms over radial points.
#include <algorithm>
#include <cmath>
#include <complex>
#include <cstring>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {
constexpr int KL = 4;             // i_KL (parameters.f90:43)
constexpr int KV = 2 * KL;        // superdiagonals of U after pivoting
constexpr int LDAB = 3 * KL + 1;  // rows of a LAPACK band
constexpr double PI = 3.14159265358979323846;
using cd = std::complex<double>;

// ------------------------------------------------------------------ FFT
// Mixed-radix Stockham transform (radices 4, 2, 3, 5, then any odd prime),
// exp(sign * 2 pi i j k / L), unscaled (FFTW's convention).  Each pass reads
// the previous buffer and writes the other; the twiddles of every pass are
// tabulated at set-up.
struct FFT {
    int L = 0;
    std::vector<int> rad;
    std::vector<cd> wp;                 // exp(+2 pi i t / L)
    std::vector<std::vector<cd>> twp;   // per pass: twiddle of (j mod Ns, q), sign +1
    void init(int n) {
        L = n;
        wp.resize(n);
        for (int t = 0; t < n; ++t) {
            const long double a = 2.0L * 3.14159265358979323846264338327950288L * t / n;
            wp[t] = cd((double)cosl(a), (double)sinl(a));
        }
        rad.clear();
        int r = n;
        for (int p : {4, 2, 3, 5, 7})
            while (r % p == 0) {
                rad.push_back(p);
                r /= p;
            }
        for (int p = 11; r > 1; p += 2)
            while (r % p == 0) {
                rad.push_back(p);
                r /= p;
            }
        twp.clear();
        int Ns = 1;
        for (int p : rad) {
            const int stride = L / (Ns * p);
            std::vector<cd> t((size_t)Ns * p);
            for (int k = 0; k < Ns; ++k)
                for (int q = 0; q < p; ++q) t[(size_t)k * p + q] = wp[((size_t)q * k * stride) % L];
            twp.push_back(std::move(t));
            Ns *= p;
        }
    }
    template <int SIGN> static cd tw(cd w) { return SIGN > 0 ? w : std::conj(w); }
    template <int SIGN> static cd muli(cd a) { return SIGN > 0 ? cd(-a.imag(), a.real()) : cd(a.imag(), -a.real()); }
    template <int SIGN> void pass(const cd *src, cd *dst, int p, int Ns, const std::vector<cd> &t) const {
        const int NB = L / p;
        cd v[64];
        for (int jb = 0; jb < NB; jb += Ns)
            for (int k = 0; k < Ns; ++k) {
            const int j = jb + k;
            for (int q = 0; q < p; ++q) {
                cd x = src[j + q * NB];
                if (q > 0 && Ns > 1) x *= tw<SIGN>(t[(size_t)k * p + q]);
                v[q] = x;
            }
            if (p == 2) {
                const cd a = v[0];
                v[0] = a + v[1];
                v[1] = a - v[1];
            } else if (p == 4) {
                const cd a = v[0] + v[2], b = v[0] - v[2], c = v[1] + v[3], d = muli<SIGN>(v[1] - v[3]);
                v[0] = a + c;
                v[1] = b + d;
                v[2] = a - c;
                v[3] = b - d;
            } else if (p == 3) {
                const double s3 = 0.86602540378443864676;
                const cd tt = v[1] + v[2];
                const cd u = v[0] - 0.5 * tt;
                const cd w = muli<SIGN>(s3 * (v[1] - v[2]));
                v[0] = v[0] + tt;
                v[1] = u + w;
                v[2] = u - w;
            } else {  // direct DFT of a small prime
                cd o[64];
                const int st = L / p;
                for (int q = 0; q < p; ++q) {
                    cd acc = v[0];
                    for (int r = 1; r < p; ++r) acc += v[r] * tw<SIGN>(wp[(size_t)((r * q) % p) * st]);
                    o[q] = acc;
                }
                for (int q = 0; q < p; ++q) v[q] = o[q];
            }
            const int base = jb * p + k;
            for (int q = 0; q < p; ++q) dst[base + q * Ns] = v[q];
            }
    }
    // out = transform(in); work holds L values
    void run(const cd *in, cd *out, int sign, cd *work) const {
        const int np = (int)rad.size();
        if (np == 0) {
            out[0] = in[0];
            return;
        }
        // end in `out`: choose the first buffer by the parity of the pass count
        cd *a = (np % 2 == 1) ? out : work, *b = (np % 2 == 1) ? work : out;
        const cd *src = in;
        int Ns = 1;
        for (int i = 0; i < np; ++i) {
            cd *dst = (i % 2 == 0) ? a : b;
            if (sign > 0) pass<+1>(src, dst, rad[i], Ns, twp[i]);
            else pass<-1>(src, dst, rad[i], Ns, twp[i]);
            src = dst;
            Ns *= rad[i];
        }
    }
};

struct Coll {
    std::vector<double> re, im;
    void init(size_t n) {
        re.assign(n, 0.0);
        im.assign(n, 0.0);
    }
};

struct LU {
    std::vector<double> ab;  // [nh][LDAB][N]
    std::vector<int> ipiv;   // [nh][N], 1-based
};

struct Lt {
    std::vector<double> off;   // [2KL+1][N]
    std::vector<double> diag;  // [N][H]
};
}  // namespace

struct pfc_pipe {
    int N, K, M, Mp, H, Z, Th;
    double alpha, Re, implicit, dterr_tol, courant;
    int const_flux, pcn;
    std::vector<double> drb;  // d/dr band [2KL+1][N]: drb[(KL+n-j)*N + j]
    std::vector<double> rm1, velU, velUp, intrdr;
    std::vector<double> dr1;  // [KL+1][KL+1] row-major: dr1[j*(KL+1) + i]
    std::vector<int> kk, mm;
    LU LNp, LDp, LDm, LDz;
    Lt Ltp, Ltm, Ltz;
    std::vector<double> Ainv;  // [nh][4][4]
    std::vector<double> U;     // [6][N][H]
    std::vector<double> Ui;
    double flux_d1 = 1.0;
    Coll ur, ut, uz, Nr, Nt, Nz, ur_, ut_, uz_, Nr_, Nt_, Nz_;
    std::vector<double> phys[6];  // [n][Th][Z]
    FFT fz, ft;
    double Pr0 = 0.0, dt = 0.01, t = 0.0, dterr = 0.0, corr_dt = 0.0, lasterr = 1e99;
    int it = 0, step = 0, failed = 0;
};

namespace {
size_t NH(const pfc_pipe *p) { return (size_t)p->N * p->H; }

// d = A b + c with a band shared by all modes and an optional per-mode
// diagonal (timestep.f90:130-154, variables.f90:378-402), column order
void band_matvec(const pfc_pipe *p, const double *off, const double *diag, const Coll &b, const Coll *c, Coll &d) {
    const int N = p->N, H = p->H;
    Coll out;
    if (c) out = *c;
    else out.init(NH(p));
    constexpr int CH = 64;  // modes per task, innermost so rows are read contiguously
#pragma omp parallel for schedule(static)
    for (int h0 = 0; h0 < H; h0 += CH) {
        const int h1 = std::min(H, h0 + CH);
        for (int j = 0; j < N; ++j)
            for (int n = std::max(0, j - KL); n <= std::min(j + KL, N - 1); ++n) {
                const double w = off[(KL + n - j) * N + j];
                const bool own = (n == j && diag);
                double *ore = &out.re[(size_t)n * H], *oim = &out.im[(size_t)n * H];
                const double *bre = &b.re[(size_t)j * H], *bim = &b.im[(size_t)j * H];
                for (int nh = h0; nh < h1; ++nh) {
                    const double a = own ? diag[(size_t)j * H + nh] : w;
                    ore[nh] = ore[nh] + a * bre[nh];
                    oim[nh] = oim[nh] + a * bim[nh];
                }
            }
    }
    d = std::move(out);
}

void curl(const pfc_pipe *p, const Coll &r, const Coll &t, const Coll &z, Coll &orr, Coll &ot, Coll &oz) {
    const int N = p->N, H = p->H;
    Coll dz, dt;
    band_matvec(p, p->drb.data(), nullptr, z, nullptr, dz);
    band_matvec(p, p->drb.data(), nullptr, t, nullptr, dt);
    orr.init(NH(p));
    ot.init(NH(p));
    oz.init(NH(p));
#pragma omp parallel for schedule(static)
    for (int n = 0; n < N; ++n)
        for (int nh = 0; nh < H; ++nh) {
            const size_t i = (size_t)n * H + nh;
            const double m1r1 = p->rm1[n] * p->Mp * p->mm[nh], k1a1 = p->alpha * p->kk[nh], rm1 = p->rm1[n];
            orr.re[i] = -z.im[i] * m1r1 + t.im[i] * k1a1;
            orr.im[i] = z.re[i] * m1r1 - t.re[i] * k1a1;
            ot.re[i] = -r.im[i] * k1a1 - dz.re[i];
            ot.im[i] = r.re[i] * k1a1 - dz.im[i];
            oz.re[i] = t.re[i] * rm1 + dt.re[i] + r.im[i] * m1r1;
            oz.im[i] = t.im[i] * rm1 + dt.im[i] - r.re[i] * m1r1;
        }
}

// coll -> phys (transform.fftw3.f90:65-102): z c2c sign +1, then theta c2r
void spec2phys(pfc_pipe *p, const Coll &c, std::vector<double> &out) {
    const int N = p->N, K = p->K, M = p->M, Z = p->Z, Th = p->Th, H = p->H;
    out.assign((size_t)N * Th * Z, 0.0);
#pragma omp parallel for schedule(dynamic)
    for (int n = 0; n < N; ++n) {
        std::vector<cd> Y((size_t)M * Z), col(Z), row(Th), res(Th), work(std::max(Z, Th));
        const double *re = &c.re[(size_t)n * H], *im = &c.im[(size_t)n * H];
        for (int m = 0; m < M; ++m) {
            std::fill(col.begin(), col.end(), cd(0.0, 0.0));
            if (m == 0) {
                for (int k = 0; k < K; ++k) col[k] = cd(re[k], im[k]);
                for (int k = 1; k < K; ++k) col[Z - k] = cd(re[k], -im[k]);
            } else {
                const int base = m * (2 * K - 1);
                for (int k = 0; k < K; ++k) col[k] = cd(re[base + k], im[base + k]);
                for (int k = 1; k < K; ++k) col[Z - k] = cd(re[base - k], im[base - k]);
            }
            p->fz.run(col.data(), &Y[(size_t)m * Z], +1, work.data());
        }
        // c2r: the Hermitian extension of the M retained modes (DC imag
        // ignored); two z rows share one complex transform, a + i b
        for (int z = 0; z < Z; z += 2) {
            const bool two = z + 1 < Z;
            std::fill(row.begin(), row.end(), cd(0.0, 0.0));
            const cd ib(0.0, 1.0);
            row[0] = cd(Y[z].real(), two ? Y[z + 1].real() : 0.0);
            for (int m = 1; m < M; ++m) {
                const cd a = Y[(size_t)m * Z + z], b = two ? Y[(size_t)m * Z + z + 1] : cd(0.0, 0.0);
                row[m] = a + ib * b;
                row[Th - m] = std::conj(a) + ib * std::conj(b);
            }
            p->ft.run(row.data(), res.data(), +1, work.data());
            for (int t = 0; t < Th; ++t) {
                out[((size_t)n * Th + t) * Z + z] = res[t].real();
                if (two) out[((size_t)n * Th + t) * Z + z + 1] = res[t].imag();
            }
        }
    }
}

// phys -> coll (transform.fftw3.f90:108-147): scale, theta r2c, z c2c sign -1
void phys2spec(pfc_pipe *p, const std::vector<double> &ph, Coll &c) {
    const int N = p->N, K = p->K, M = p->M, Z = p->Z, Th = p->Th, H = p->H;
    const double scale = 1.0 / (double)(Z * Th);
    c.init(NH(p));
#pragma omp parallel for schedule(dynamic)
    for (int n = 0; n < N; ++n) {
        std::vector<cd> Y((size_t)M * Z), row(Th), res(Th), col(Z), X(Z), work(std::max(Z, Th));
        // r2c of two z rows at once: F = FFT(a + i b), A_m = (F_m + conj F_-m)/2,
        // B_m = (F_m - conj F_-m)/(2i)
        for (int z = 0; z < Z; z += 2) {
            const bool two = z + 1 < Z;
            for (int t = 0; t < Th; ++t)
                row[t] = cd(scale * ph[((size_t)n * Th + t) * Z + z], two ? scale * ph[((size_t)n * Th + t) * Z + z + 1] : 0.0);
            p->ft.run(row.data(), res.data(), -1, work.data());
            for (int m = 0; m < M; ++m) {
                const cd f = res[m], g = std::conj(res[(Th - m) % Th]);
                Y[(size_t)m * Z + z] = 0.5 * (f + g);
                if (two) Y[(size_t)m * Z + z + 1] = cd(0.0, -0.5) * (f - g);
            }
        }
        double *re = &c.re[(size_t)n * H], *im = &c.im[(size_t)n * H];
        for (int m = 0; m < M; ++m) {
            for (int z = 0; z < Z; ++z) col[z] = Y[(size_t)m * Z + z];
            p->fz.run(col.data(), X.data(), -1, work.data());
            if (m == 0) {
                for (int k = 0; k < K; ++k) {
                    re[k] = X[k].real();
                    im[k] = X[k].imag();
                }
            } else {
                const int base = m * (2 * K - 1);
                for (int k = 0; k < K; ++k) {
                    re[base + k] = X[k].real();
                    im[base + k] = X[k].imag();
                }
                for (int k = 1; k < K; ++k) {
                    re[base - k] = X[Z - k].real();
                    im[base - k] = X[Z - k].imag();
                }
            }
        }
    }
}

// dgbtrs ('N') then dtbsv ('U', 'N', non-unit) on one right-hand side x
void gbsolve(const double *ab, const int *ipiv, int N, double *x) {
    for (int j = 0; j < N - 1; ++j) {
        const int lm = std::min(KL, N - 1 - j);
        const int l = ipiv[j] - 1;
        if (l != j) std::swap(x[l], x[j]);
        const double temp = -x[j];
        for (int i = 1; i <= lm; ++i) x[j + i] = x[j + i] + ab[(KV + i) * N + j] * temp;
    }
    for (int j = N - 1; j >= 0; --j) {
        if (x[j] != 0.0) {
            x[j] = x[j] / ab[KV * N + j];
            const double temp = x[j];
            for (int i = j - 1; i >= std::max(0, j - KV); --i) x[i] = x[i] - temp * ab[(KV + i - j) * N + j];
        }
    }
}

// tim_lumesh_invert (timestep.f90:102-123), in place
void lumesh_invert(const pfc_pipe *p, int BC, const LU &A, Coll &b) {
    const int N = p->N, H = p->H;
#pragma omp parallel for schedule(static)
    for (int nh = 0; nh < H; ++nh) {
        std::vector<double> xr(N), xi(N);
        if (BC == 1 && p->kk[nh] == 0 && p->mm[nh] == 0) {
            for (int n = 0; n < N; ++n) b.re[(size_t)n * H + nh] = b.im[(size_t)n * H + nh] = 0.0;
            continue;
        }
        for (int n = 0; n < N; ++n) {
            xr[n] = b.re[(size_t)n * H + nh];
            xi[n] = b.im[(size_t)n * H + nh];
        }
        const double *ab = &A.ab[(size_t)nh * LDAB * N];
        const int *ip = &A.ipiv[(size_t)nh * N];
        gbsolve(ab, ip, N, xr.data());
        gbsolve(ab, ip, N, xi.data());
        for (int n = 0; n < N; ++n) {
            b.re[(size_t)n * H + nh] = xr[n];
            b.im[(size_t)n * H + nh] = xi[n];
        }
    }
}

void zerobc(const pfc_pipe *p, Coll &a) {
    const int H = p->H, N = p->N;
    for (int nh = 0; nh < H; ++nh) {
        a.re[nh] = a.im[nh] = 0.0;
        a.re[(size_t)(N - 1) * H + nh] = a.im[(size_t)(N - 1) * H + nh] = 0.0;
    }
}

void rt2pm(const Coll &r, const Coll &t, Coll &up, Coll &um) {
    const size_t n = r.re.size();
    Coll a, b;
    a.init(n);
    b.init(n);
    for (size_t i = 0; i < n; ++i) {
        a.re[i] = r.re[i] - t.im[i];
        a.im[i] = r.im[i] + t.re[i];
        b.re[i] = r.re[i] + t.im[i];
        b.im[i] = r.im[i] - t.re[i];
    }
    up = std::move(a);
    um = std::move(b);
}

void pm2rt(const Coll &up, const Coll &um, Coll &r, Coll &t) {
    const size_t n = up.re.size();
    Coll a, b;
    a.init(n);
    b.init(n);
    for (size_t i = 0; i < n; ++i) {
        a.re[i] = 0.5 * (up.re[i] + um.re[i]);
        a.im[i] = 0.5 * (up.im[i] + um.im[i]);
        b.re[i] = 0.5 * (up.im[i] - um.im[i]);
        b.im[i] = -0.5 * (up.re[i] - um.re[i]);
    }
    r = std::move(a);
    t = std::move(b);
}

void imposesym0(pfc_pipe *p) {
    for (int n = 0; n < p->N; ++n) {
        const size_t i = (size_t)n * p->H;
        p->ur.re[i] = 0.0;
        p->ur.im[i] = 0.0;
        p->ut.im[i] = 0.0;
        p->uz.im[i] = 0.0;
    }
}

// vel_transform + vel_nonlinear + vel_addHPF (velocity.f90:304-361)
void transform_nonlinear(pfc_pipe *p) {
    const int N = p->N, H = p->H;
    Coll cr, ct, cz;
    curl(p, p->ur, p->ut, p->uz, cr, ct, cz);
    const Coll *src[6] = {&p->ur, &p->ut, &p->uz, &cr, &ct, &cz};
    for (int i = 0; i < 6; ++i) spec2phys(p, *src[i], p->phys[i]);
    const size_t np = p->phys[0].size();
    std::vector<double> q(np);
    Coll *dst[3] = {&p->Nr, &p->Nt, &p->Nz};
    const int A[3][4] = {{1, 5, 2, 4}, {2, 3, 0, 5}, {0, 4, 1, 3}};  // u x curl u (velocity.f90:325-329)
    for (int c = 0; c < 3; ++c) {
        const double *a = p->phys[A[c][0]].data(), *b = p->phys[A[c][1]].data();
        const double *e = p->phys[A[c][2]].data(), *f = p->phys[A[c][3]].data();
#pragma omp parallel for schedule(static)
        for (long long i = 0; i < (long long)np; ++i) q[i] = a[i] * b[i] - e[i] * f[i];
        phys2spec(p, q, *dst[c]);
    }
    // vel_addHPF
#pragma omp parallel for schedule(static)
    for (int n = 0; n < N; ++n)
        for (int nh = 0; nh < H; ++nh) {
            const size_t i = (size_t)n * H + nh;
            const double a = p->alpha * p->kk[nh] * p->velU[n], b = -p->velUp[n];
            p->Nr.re[i] = p->Nr.re[i] + a * p->ur.im[i];
            p->Nr.im[i] = p->Nr.im[i] - a * p->ur.re[i];
            p->Nt.re[i] = p->Nt.re[i] + a * p->ut.im[i];
            p->Nt.im[i] = p->Nt.im[i] - a * p->ut.re[i];
            p->Nz.re[i] = p->Nz.re[i] + a * p->uz.im[i] + b * p->ur.re[i];
            p->Nz.im[i] = p->Nz.im[i] - a * p->uz.re[i] + b * p->ur.im[i];
        }
    if (p->const_flux) {
        double s = 0.0;
        for (int j = 0; j <= KL; ++j) s += p->uz.re[(size_t)(N - KL - 1 + j) * H] * p->dr1[j * (KL + 1) + 1];
        p->Pr0 = s / (-2.0);
        for (int n = 0; n < N; ++n) p->Nz.re[(size_t)n * H] = p->Nz.re[(size_t)n * H] + 4.0 * p->Pr0 / p->Re;
    }
}

// vel_evalBC (velocity.f90:262-298) for one mode
void evalBC(const pfc_pipe *p, const Coll &up, const Coll &um, const Coll &uz, int nh, double BRe[4],
            double BIm[4]) {
    const int N = p->N, H = p->H, n = N - 1;
    const size_t at = (size_t)n * H + nh;
    const double m_ = (double)(p->mm[nh] * p->Mp), a_ = p->alpha * p->kk[nh];
    const double urRe = 0.5 * (up.re[at] + um.re[at]), urIm = 0.5 * (up.im[at] + um.im[at]);
    const double utRe = 0.5 * (up.im[at] - um.im[at]), utIm = -0.5 * (up.re[at] - um.re[at]);
    double sr = 0.0, si = 0.0;
    for (int j = 0; j <= KL; ++j) {
        const size_t aj = (size_t)(N - KL - 1 + j) * H + nh;
        sr += p->dr1[j * (KL + 1) + 1] * (up.re[aj] + um.re[aj]);
        si += p->dr1[j * (KL + 1) + 1] * (up.im[aj] + um.im[aj]);
    }
    const double drRe = 0.5 * sr, drIm = 0.5 * si;
    const double d = p->rm1[n];
    BRe[0] = up.re[at];
    BIm[0] = up.im[at];
    BRe[1] = um.re[at];
    BIm[1] = um.im[at];
    BRe[2] = -uz.im[at];
    BIm[2] = uz.re[at];
    BRe[3] = urRe * d + drRe - d * m_ * utIm - a_ * uz.im[at];
    BIm[3] = urIm * d + drIm + d * m_ * utRe + a_ * uz.re[at];
}

// vel_step (velocity.f90:367-394)
void vel_step(pfc_pipe *p) {
    const int N = p->N, H = p->H;
    Coll c1, c2, a, b;
    rt2pm(p->Nr, p->Nt, c1, c2);
    rt2pm(p->ur_, p->ut_, a, b);
    band_matvec(p, p->Ltp.off.data(), p->Ltp.diag.data(), a, &c1, p->ur);
    band_matvec(p, p->Ltm.off.data(), p->Ltm.diag.data(), b, &c2, p->ut);
    band_matvec(p, p->Ltz.off.data(), p->Ltz.diag.data(), p->uz_, &p->Nz, p->uz);
    {  // vel_adjPPE(1): project with the pressure Poisson solve
        Coll r, t;
        pm2rt(p->ur, p->ut, r, t);
        Coll dr;
        band_matvec(p, p->drb.data(), nullptr, r, nullptr, dr);
        Coll dv;
        dv.init(NH(p));
#pragma omp parallel for schedule(static)
        for (int n = 0; n < N; ++n)
            for (int nh = 0; nh < H; ++nh) {
                const size_t i = (size_t)n * H + nh;
                const double rm1 = p->rm1[n], m1r1 = rm1 * p->Mp * p->mm[nh], k1a1 = p->alpha * p->kk[nh];
                dv.re[i] = r.re[i] * rm1 + dr.re[i] - t.im[i] * m1r1 - p->uz.im[i] * k1a1;
                dv.im[i] = r.im[i] * rm1 + dr.im[i] + t.re[i] * m1r1 + p->uz.re[i] * k1a1;
            }
        zerobc(p, dv);
        lumesh_invert(p, 1, p->LNp, dv);
        Coll gr;
        band_matvec(p, p->drb.data(), nullptr, dv, nullptr, gr);
        Coll gt, gz;
        gt.init(NH(p));
        gz.init(NH(p));
        for (int n = 0; n < N; ++n)
            for (int nh = 0; nh < H; ++nh) {
                const size_t i = (size_t)n * H + nh;
                const double m1r1 = p->rm1[n] * p->Mp * p->mm[nh], k1a1 = p->alpha * p->kk[nh];
                gt.re[i] = -dv.im[i] * m1r1;
                gt.im[i] = dv.re[i] * m1r1;
                gz.re[i] = -dv.im[i] * k1a1;
                gz.im[i] = dv.re[i] * k1a1;
            }
        Coll gp, gm;
        rt2pm(gr, gt, gp, gm);
        for (size_t i = 0; i < NH(p); ++i) {
            p->ur.re[i] = p->ur.re[i] - gp.re[i];
            p->ur.im[i] = p->ur.im[i] - gp.im[i];
            p->ut.re[i] = p->ut.re[i] - gm.re[i];
            p->ut.im[i] = p->ut.im[i] - gm.im[i];
            p->uz.re[i] = p->uz.re[i] - gz.re[i];
            p->uz.im[i] = p->uz.im[i] - gz.im[i];
        }
    }
    zerobc(p, p->ur);
    zerobc(p, p->ut);
    zerobc(p, p->uz);
    lumesh_invert(p, 0, p->LDp, p->ur);
    lumesh_invert(p, 0, p->LDm, p->ut);
    lumesh_invert(p, 0, p->LDz, p->uz);
    // vel_adjPPE(2): influence-matrix correction
#pragma omp parallel for schedule(static)
    for (int nh = 1; nh < H; ++nh) {
        double BRe[4], BIm[4], aR[4], aI[4];
        evalBC(p, p->ur, p->ut, p->uz, nh, BRe, BIm);
        const double *A = &p->Ainv[(size_t)nh * 16];
        for (int i = 0; i < 4; ++i) {
            double sr = 0.0, si = 0.0;
            for (int j = 0; j < 4; ++j) {
                sr += A[i * 4 + j] * BRe[j];
                si += A[i * 4 + j] * BIm[j];
            }
            aR[i] = -sr;
            aI[i] = -si;
        }
        for (int n = 0; n < N; ++n) {
            const size_t i = (size_t)n * H + nh;
            auto Uv = [&](int q) { return p->U[((size_t)q * N + n) * H + nh]; };
            p->ur.re[i] = p->ur.re[i] + aR[0] * Uv(0);
            p->ur.im[i] = p->ur.im[i] + aI[0] * Uv(0);
            p->ut.re[i] = p->ut.re[i] + aR[1] * Uv(1);
            p->ut.im[i] = p->ut.im[i] + aI[1] * Uv(1);
            p->uz.re[i] = p->uz.re[i] - aI[2] * Uv(2);
            p->uz.im[i] = p->uz.im[i] + aR[2] * Uv(2);
            p->ur.re[i] = p->ur.re[i] + aR[3] * Uv(3);
            p->ur.im[i] = p->ur.im[i] + aI[3] * Uv(3);
            p->ut.re[i] = p->ut.re[i] + aR[3] * Uv(4);
            p->ut.im[i] = p->ut.im[i] + aI[3] * Uv(4);
            p->uz.re[i] = p->uz.re[i] - aI[3] * Uv(5);
            p->uz.im[i] = p->uz.im[i] + aR[3] * Uv(5);
        }
    }
    Coll r, t;
    pm2rt(p->ur, p->ut, r, t);
    p->ur = std::move(r);
    p->ut = std::move(t);
    if (p->const_flux) {  // vel_adjustFlux(1)
        double s = 0.0;
        for (int n = 0; n < N; ++n) s += p->uz.re[(size_t)n * H] * p->intrdr[n];
        const double d3 = -(2.0 * s) / p->flux_d1;
        for (int n = 0; n < N; ++n) p->uz.re[(size_t)n * H] = p->uz.re[(size_t)n * H] + d3 * p->Ui[n];
        p->Pr0 = p->Pr0 + d3 * p->Re / 4.0;
    }
    imposesym0(p);
}

void corrector(pfc_pipe *p) {
    Coll r = p->ur, t = p->ut, z = p->uz;
    const double d1 = p->implicit, d2 = 1.0 - p->implicit;
    Coll *Nn[3] = {&p->Nr, &p->Nt, &p->Nz}, *Np[3] = {&p->Nr_, &p->Nt_, &p->Nz_};
    for (int c = 0; c < 3; ++c)
        for (size_t i = 0; i < NH(p); ++i) {
            Nn[c]->re[i] = d1 * Nn[c]->re[i] + d2 * Np[c]->re[i];
            Nn[c]->im[i] = d1 * Nn[c]->im[i] + d2 * Np[c]->im[i];
        }
    vel_step(p);
    double e = 0.0;
    const Coll *o[3] = {&r, &t, &z}, *nw[3] = {&p->ur, &p->ut, &p->uz};
    for (int c = 0; c < 3; ++c)
        for (size_t i = 0; i < NH(p); ++i) {
            const double a = o[c]->re[i] - nw[c]->re[i], b = o[c]->im[i] - nw[c]->im[i];
            e = std::max(e, a * a + b * b);
        }
    p->dterr = std::max(p->dterr, std::sqrt(e));
}

// tim_check_cgce (timestep.f90:214-253)
void check_cgce(pfc_pipe *p) {
    if (p->it == 1) {
        p->corr_dt = p->dterr > 0.0 ? p->dt * std::sqrt(p->dterr_tol / p->dterr) : INFINITY;
        p->lasterr = 1e99;
    }
    if (p->dt < 1e-9 && p->step > 30) {
        p->failed = 1;
        p->it = 0;
    } else if (p->it == p->pcn) {
        p->it = 0;
    } else if (p->it > 10) {
        p->failed = 2;
        p->it = 0;
    } else if (p->dterr > p->lasterr) {
        if (p->dterr > 2.0 * p->dterr_tol) p->failed = 3;
        if (p->dterr < 2.0 * p->dterr_tol) p->corr_dt = p->dt / (10.0 * p->courant);
        p->it = 0;
    } else if (p->dterr > p->dterr_tol) {
        p->lasterr = p->dterr;
        p->it = p->it + 1;
    } else {
        p->it = 0;
    }
    p->dterr = 0.0;
}

void copy_in(const double *src, std::vector<double> &dst, size_t n) { dst.assign(src, src + n); }
}  // namespace

extern "C" {

int pfc_threads() {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

void pfc_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

// drb: d/dr band [2KL+1][N]; rm1, velU, velUp, intrdr: [N]; dr1: [KL+1][KL+1]
// row-major (dr1[j][i] = weight of point N-1-KL+j for the i-th derivative at r=1)
pfc_pipe *pfc_create(int N, int K, int M, int Mp, double alpha, double Re, double implicit, int const_flux,
                     double dterr_tol, double courant, const double *drb, const double *rm1, const double *velU,
                     const double *velUp, const double *intrdr, const double *dr1) {
    pfc_pipe *p = new pfc_pipe();
    p->N = N;
    p->K = K;
    p->M = M;
    p->Mp = Mp;
    p->H = (2 * K - 1) * M - (K - 1);
    p->Z = 3 * K;
    p->Th = 3 * M;
    p->alpha = alpha;
    p->Re = Re;
    p->implicit = implicit;
    p->const_flux = const_flux;
    p->dterr_tol = dterr_tol;
    p->courant = courant;
    p->pcn = -1;
    copy_in(drb, p->drb, (size_t)(2 * KL + 1) * N);
    copy_in(rm1, p->rm1, N);
    copy_in(velU, p->velU, N);
    copy_in(velUp, p->velUp, N);
    copy_in(intrdr, p->intrdr, N);
    copy_in(dr1, p->dr1, (KL + 1) * (KL + 1));
    for (int m = 0; m < M; ++m)
        for (int k = -(K - 1); k < K; ++k) {
            if (m == 0 && k < 0) continue;
            p->kk.push_back(k);
            p->mm.push_back(m);
        }
    p->fz.init(p->Z);
    p->ft.init(p->Th);
    Coll *all[12] = {&p->ur, &p->ut, &p->uz, &p->Nr, &p->Nt, &p->Nz, &p->ur_, &p->ut_, &p->uz_, &p->Nr_, &p->Nt_, &p->Nz_};
    for (Coll *c : all) c->init(NH(p));
    return p;
}

void pfc_destroy(pfc_pipe *p) { delete p; }

// which: 0 LNp, 1 LDp, 2 LDm, 3 LDz; ab [H][LDAB][N], ipiv [H][N] (1-based)
void pfc_set_lu(pfc_pipe *p, int which, const double *ab, const int *ipiv) {
    LU *L[4] = {&p->LNp, &p->LDp, &p->LDm, &p->LDz};
    copy_in(ab, L[which]->ab, (size_t)p->H * LDAB * p->N);
    L[which]->ipiv.assign(ipiv, ipiv + (size_t)p->H * p->N);
}

// which: 0 Ltp, 1 Ltm, 2 Ltz; off [2KL+1][N], diag [N][H]
void pfc_set_lt(pfc_pipe *p, int which, const double *off, const double *diag) {
    Lt *L[3] = {&p->Ltp, &p->Ltm, &p->Ltz};
    copy_in(off, L[which]->off, (size_t)(2 * KL + 1) * p->N);
    copy_in(diag, L[which]->diag, NH(p));
}

// Ainv [H][4][4] (mode 0 unused), U [6][N][H], Ui [N]
void pfc_set_influence(pfc_pipe *p, const double *Ainv, const double *U, const double *Ui, double flux_d1) {
    copy_in(Ainv, p->Ainv, (size_t)p->H * 16);
    copy_in(U, p->U, (size_t)6 * NH(p));
    copy_in(Ui, p->Ui, p->N);
    p->flux_d1 = flux_d1;
}

void pfc_set_state(pfc_pipe *p, const double *urr, const double *uri, const double *utr, const double *uti,
                   const double *uzr, const double *uzi, double dt, double Pr0) {
    copy_in(urr, p->ur.re, NH(p));
    copy_in(uri, p->ur.im, NH(p));
    copy_in(utr, p->ut.re, NH(p));
    copy_in(uti, p->ut.im, NH(p));
    copy_in(uzr, p->uz.re, NH(p));
    copy_in(uzi, p->uz.im, NH(p));
    p->dt = dt;
    p->Pr0 = Pr0;
}

void pfc_get_state(const pfc_pipe *p, double *urr, double *uri, double *utr, double *uti, double *uzr,
                   double *uzi) {
    const size_t n = NH(p) * sizeof(double);
    std::memcpy(urr, p->ur.re.data(), n);
    std::memcpy(uri, p->ur.im.data(), n);
    std::memcpy(utr, p->ut.re.data(), n);
    std::memcpy(uti, p->ut.im.data(), n);
    std::memcpy(uzr, p->uz.re.data(), n);
    std::memcpy(uzi, p->uz.im.data(), n);
}

// One pass of the main.f90 loop body (orbit = 0: corrector to convergence)
// or of steporbit's (orbit = 1: one corrector); fixed dt.  Returns the
// corrector passes, or a negative number when tim_check_cgce failed.
int pfc_timestep(pfc_pipe *p, int orbit) {
    imposesym0(p);
    transform_nonlinear(p);
    p->ur_ = p->ur;
    p->ut_ = p->ut;
    p->uz_ = p->uz;
    p->Nr_ = p->Nr;
    p->Nt_ = p->Nt;
    p->Nz_ = p->Nz;
    vel_step(p);
    int nc = 0;
    p->it = 1;
    for (;;) {
        transform_nonlinear(p);
        corrector(p);
        ++nc;
        if (orbit) {
            imposesym0(p);
            check_cgce(p);
            break;
        }
        check_cgce(p);
        if (p->it == 0) break;
    }
    p->t += p->dt;
    p->step += 1;
    return p->failed ? -p->failed : nc;
}
}
