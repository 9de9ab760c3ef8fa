// Project-written CPU implementation of the FFTW 3 API subset declared in
// fftw3.h (test infrastructure: lets the reference's own sources build here).
//
// Transforms follow FFTW's documented, unnormalised definitions:
//   c2c   Y_k = sum_j X_j exp(sign 2 pi i j k / n)
//   r2c   the first n/2+1 outputs of the forward c2c of a real input
//   c2r   the real inverse of a Hermitian half spectrum (imaginary parts of
//         the DC and, for even n, Nyquist bins are ignored)
//   REDFT00 (n points)  Y_k = x_0 + (-1)^k x_{n-1} + 2 sum_{j=1}^{n-2} x_j cos(pi j k/(n-1))
// The engine is an iterative mixed-radix Stockham FFT (radix 4, 2, odd radices
// by symmetric pairs, per-pass twiddle tables); even-length real transforms are packed into a
// half-length complex FFT; REDFT00 is the real part of the r2c transform of
// the even extension of length 2(n-1).
#include "fftw3.h"

#include <cmath>
#include <complex>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <vector>

namespace {
using cd = std::complex<double>;

// Odd-radix butterfly by symmetric pairs: y_q = x_0 + sum_t [ (x_t + x_{R-t}) cos(2 pi t q/R)
//   + sign * i (x_t - x_{R-t}) sin(2 pi t q/R) ].
template <int R>
inline void bfly_odd(cd *v, const double *cs, const double *sn, int sign) {
    constexpr int h = R / 2;
    double sr[h + 1], si[h + 1], dr[h + 1], di[h + 1];
    for (int t = 1; t <= h; ++t) {
        sr[t] = v[t].real() + v[R - t].real();
        si[t] = v[t].imag() + v[R - t].imag();
        dr[t] = v[t].real() - v[R - t].real();
        di[t] = v[t].imag() - v[R - t].imag();
    }
    double y0r = v[0].real(), y0i = v[0].imag();
    for (int t = 1; t <= h; ++t) { y0r += sr[t]; y0i += si[t]; }
    cd out[R];
    out[0] = cd(y0r, y0i);
    for (int q = 1; q <= h; ++q) {
        double rr = v[0].real(), ri = v[0].imag(), ir = 0.0, ii = 0.0;
        for (int t = 1; t <= h; ++t) {
            const int idx = (t * q) % R;
            rr += cs[idx] * sr[t];
            ri += cs[idx] * si[t];
            ir += sn[idx] * dr[t];
            ii += sn[idx] * di[t];
        }
        // sign * i * (ir + i ii) = sign * (-ii + i ir)
        const double ar = -sign * ii, ai = sign * ir;
        out[q] = cd(rr + ar, ri + ai);
        out[R - q] = cd(rr - ar, ri - ai);
    }
    for (int q = 0; q < R; ++q) v[q] = out[q];
}

struct Cfft {
    struct Pass {
        int R, ns, m;
        std::vector<cd> tw;  // [k < ns][q = 1..R-1]: exp(sign 2 pi i q k / (ns R))
    };
    int n = 0;
    int sign = -1;
    std::vector<Pass> pass;
    std::vector<cd> root;       // exp(sign 2 pi i k / n), generic radices
    double cs[16][16], sn[16][16];  // per odd radix: cos/sin(2 pi m / R)

    static cd polar_exact(long double num, long double den, int sign) {
        const long double a = 2.0L * 3.141592653589793238462643383279502884L * num / den;
        return cd(static_cast<double>(std::cos(a)), static_cast<double>(sign * std::sin(a)));
    }

    Cfft(int n_, int sign_) : n(n_), sign(sign_) {
        std::vector<int> radix;
        int m = n;
        while (m % 4 == 0) { radix.push_back(4); m /= 4; }
        while (m % 2 == 0) { radix.push_back(2); m /= 2; }
        for (int p = 3; m > 1; p += 2)
            while (m % p == 0) { radix.push_back(p); m /= p; }
        root.resize(n);
        for (int k = 0; k < n; ++k) root[k] = polar_exact(k, n, sign);
        for (int R = 3; R < 16; R += 2)
            for (int q = 0; q < R; ++q) {
                const cd w = polar_exact(q, R, 1);
                cs[R][q] = w.real();
                sn[R][q] = w.imag();
            }
        int ns = 1;
        for (int R : radix) {
            Pass p;
            p.R = R;
            p.ns = ns;
            p.m = n / R;
            p.tw.resize(static_cast<size_t>(ns) * (R - 1));
            for (int k = 0; k < ns; ++k)
                for (int q = 1; q < R; ++q)
                    p.tw[static_cast<size_t>(k) * (R - 1) + q - 1] =
                        polar_exact(static_cast<long double>(q) * k, static_cast<long double>(ns) * R, sign);
            pass.push_back(std::move(p));
            ns *= R;
        }
    }

    template <int R>
    void run_pass(const Pass &p, const cd *src, cd *dst) const {
        const int m = p.m, ns = p.ns;
        cd v[R > 0 ? R : 1];
        for (int j0 = 0; j0 < m; j0 += ns) {
            for (int k = 0; k < ns; ++k) {
                const int j = j0 + k;
                const cd *tw = p.tw.data() + static_cast<size_t>(k) * (R - 1);
                v[0] = src[j];
                for (int q = 1; q < R; ++q) v[q] = src[j + q * m] * tw[q - 1];
                if (R == 2) {
                    const cd a = v[0], b = v[1];
                    v[0] = a + b;
                    v[1] = a - b;
                } else if (R == 4) {
                    const cd a = v[0] + v[2], b = v[0] - v[2];
                    const cd c = v[1] + v[3], d = v[1] - v[3];
                    const cd di = sign < 0 ? cd(d.imag(), -d.real()) : cd(-d.imag(), d.real());
                    v[0] = a + c;
                    v[1] = b + di;
                    v[2] = a - c;
                    v[3] = b - di;
                } else {
                    bfly_odd<R>(v, cs[R], sn[R], sign);
                }
                cd *o = dst + j0 * R + k;
                for (int q = 0; q < R; ++q) o[q * ns] = v[q];
            }
        }
    }

    void run_generic(const Pass &p, const cd *src, cd *dst) const {
        const int R = p.R, m = p.m, ns = p.ns;
        std::vector<cd> v(R), out(R);
        for (int j0 = 0; j0 < m; j0 += ns)
            for (int k = 0; k < ns; ++k) {
                const int j = j0 + k;
                const cd *tw = p.tw.data() + static_cast<size_t>(k) * (R - 1);
                v[0] = src[j];
                for (int q = 1; q < R; ++q) v[q] = src[j + q * m] * tw[q - 1];
                for (int q = 0; q < R; ++q) {
                    cd s = v[0];
                    for (int t = 1; t < R; ++t)
                        s += v[t] * root[(static_cast<long>(t) * q % R) * (n / R)];
                    out[q] = s;
                }
                cd *o = dst + j0 * R + k;
                for (int q = 0; q < R; ++q) o[q * ns] = out[q];
            }
    }

    // Result in `data`; `work` has n elements of scratch.
    void run(cd *data, cd *work) const {
        if (n <= 1) return;
        cd *src = data, *dst = work;
        for (const Pass &p : pass) {
            switch (p.R) {
            case 2: run_pass<2>(p, src, dst); break;
            case 3: run_pass<3>(p, src, dst); break;
            case 4: run_pass<4>(p, src, dst); break;
            case 5: run_pass<5>(p, src, dst); break;
            case 7: run_pass<7>(p, src, dst); break;
            case 11: run_pass<11>(p, src, dst); break;
            case 13: run_pass<13>(p, src, dst); break;
            default: run_generic(p, src, dst); break;
            }
            std::swap(src, dst);
        }
        if (src != data) std::memcpy(data, src, sizeof(cd) * n);
    }
};

enum class Kind { C2C, R2C, C2R, REDFT00 };

struct Scratch {
    std::vector<cd> a, b, c;
};
thread_local Scratch tls;

int g_nthreads = 1;
void (*g_loop)(void *(*)(char *), char *, size_t, int, void *) = nullptr;
void *g_loop_data = nullptr;
}  // namespace

struct cdns_fftw_plan_s {
    Kind kind;
    int n;            // logical length (REDFT00: number of points)
    int howmany;
    int istride, idist, ostride, odist;
    void *in, *out;
    int nthreads;
    std::unique_ptr<Cfft> full;  // length n complex (c2c, odd real lengths)
    std::unique_ptr<Cfft> half;  // length n/2 (even real transforms)
    std::vector<cd> tw;          // exp(-2 pi i k / n) for packed real transforms
    int m_real = 0;              // real length for r2c/c2r (REDFT00: 2(n-1))
};

namespace {
void setup_real(cdns_fftw_plan_s *p, int len, int sign) {
    p->m_real = len;
    if (len % 2 == 0 && len >= 2) {
        p->half.reset(new Cfft(len / 2, sign));
        p->tw.resize(len / 2 + 1);
        for (int k = 0; k <= len / 2; ++k) {
            const long double a = 2.0L * 3.141592653589793238462643383279502884L *
                                  static_cast<long double>(k) / static_cast<long double>(len);
            p->tw[k] = cd(static_cast<double>(std::cos(a)), static_cast<double>(-std::sin(a)));
        }
    } else {
        p->full.reset(new Cfft(len, sign));
    }
}

// Forward real transform of x[0..len) -> X[0..len/2].
void r2c_line(const cdns_fftw_plan_s *p, const double *x, cd *X) {
    const int len = p->m_real;
    auto &a = tls.a, &b = tls.b;
    if (p->half) {
        const int h = len / 2;
        a.resize(h); b.resize(h);
        for (int m = 0; m < h; ++m) a[m] = cd(x[2 * m], x[2 * m + 1]);
        p->half->run(a.data(), b.data());
        for (int k = 0; k <= h; ++k) {
            const cd zk = a[k % h];
            const cd zc = std::conj(a[(h - k) % h]);
            const cd e = 0.5 * (zk + zc);
            const cd o = cd(0.0, -0.5) * (zk - zc);
            X[k] = e + p->tw[k] * o;
        }
    } else {
        a.resize(len); b.resize(len);
        for (int j = 0; j < len; ++j) a[j] = cd(x[j], 0.0);
        p->full->run(a.data(), b.data());
        for (int k = 0; k <= len / 2; ++k) X[k] = a[k];
    }
}

// Backward real transform of the Hermitian half spectrum X[0..len/2] -> x.
void c2r_line(const cdns_fftw_plan_s *p, const cd *X, double *x) {
    const int len = p->m_real;
    auto &a = tls.a, &b = tls.b;
    if (p->half) {
        const int h = len / 2;
        a.resize(h); b.resize(h);
        for (int k = 0; k < h; ++k) {
            cd xk = X[k];
            cd xn = X[h - k];
            if (k == 0) { xk = cd(xk.real(), 0.0); xn = cd(xn.real(), 0.0); }
            const cd xc = std::conj(xn);
            // tw is exp(-2 pi i k/len); the backward twiddle is its conjugate.
            a[k] = (xk + xc) + cd(0.0, 1.0) * std::conj(p->tw[k]) * (xk - xc);
        }
        p->half->run(a.data(), b.data());
        for (int m = 0; m < h; ++m) {
            x[2 * m] = a[m].real();
            x[2 * m + 1] = a[m].imag();
        }
    } else {
        a.resize(len); b.resize(len);
        for (int k = 0; k <= len / 2; ++k) a[k] = X[k];
        a[0] = cd(a[0].real(), 0.0);
        for (int k = len / 2 + 1; k < len; ++k) a[k] = std::conj(X[len - k]);
        p->full->run(a.data(), b.data());
        for (int j = 0; j < len; ++j) x[j] = a[j].real();
    }
}

void run_range(const cdns_fftw_plan_s *p, void *in, void *out, int t0, int t1) {
    const int n = p->n;
    auto &c = tls.c;
    for (int t = t0; t < t1; ++t) {
        switch (p->kind) {
        case Kind::C2C: {
            const cd *src = static_cast<const cd *>(in) + static_cast<long>(t) * p->idist;
            cd *dst = static_cast<cd *>(out) + static_cast<long>(t) * p->odist;
            c.resize(2 * n);
            for (int j = 0; j < n; ++j) c[j] = src[static_cast<long>(j) * p->istride];
            p->full->run(c.data(), c.data() + n);
            for (int j = 0; j < n; ++j) dst[static_cast<long>(j) * p->ostride] = c[j];
            break;
        }
        case Kind::R2C: {
            const double *src = static_cast<const double *>(in) + static_cast<long>(t) * p->idist;
            cd *dst = static_cast<cd *>(out) + static_cast<long>(t) * p->odist;
            c.resize(n + n / 2 + 1);
            double *xr = reinterpret_cast<double *>(c.data());
            for (int j = 0; j < n; ++j) xr[j] = src[static_cast<long>(j) * p->istride];
            cd *X = c.data() + (n + 1) / 2;
            r2c_line(p, xr, X);
            for (int k = 0; k <= n / 2; ++k) dst[static_cast<long>(k) * p->ostride] = X[k];
            break;
        }
        case Kind::C2R: {
            const cd *src = static_cast<const cd *>(in) + static_cast<long>(t) * p->idist;
            double *dst = static_cast<double *>(out) + static_cast<long>(t) * p->odist;
            c.resize(n / 2 + 1 + (n + 1) / 2 + 1);
            cd *X = c.data();
            for (int k = 0; k <= n / 2; ++k) X[k] = src[static_cast<long>(k) * p->istride];
            double *xr = reinterpret_cast<double *>(c.data() + n / 2 + 1);
            c2r_line(p, X, xr);
            for (int j = 0; j < n; ++j) dst[static_cast<long>(j) * p->ostride] = xr[j];
            break;
        }
        case Kind::REDFT00: {
            const double *src = static_cast<const double *>(in) + static_cast<long>(t) * p->idist;
            double *dst = static_cast<double *>(out) + static_cast<long>(t) * p->odist;
            const int len = p->m_real;  // 2(n-1)
            c.resize(len / 2 + (len / 2 + 1) + 1);
            double *e = reinterpret_cast<double *>(c.data());
            for (int j = 0; j < n; ++j) e[j] = src[static_cast<long>(j) * p->istride];
            for (int j = 1; j < n - 1; ++j) e[len - j] = e[j];
            cd *X = c.data() + len / 2;
            r2c_line(p, e, X);
            for (int k = 0; k < n; ++k) dst[static_cast<long>(k) * p->ostride] = X[k].real();
            break;
        }
        }
    }
}

struct Job {
    const cdns_fftw_plan_s *p;
    void *in, *out;
    int t0, t1;
};

void *job_work(char *data) {
    Job *j = reinterpret_cast<Job *>(data);
    run_range(j->p, j->in, j->out, j->t0, j->t1);
    return nullptr;
}

void execute(const cdns_fftw_plan_s *p, void *in, void *out) {
    const int jobs = std::min(p->nthreads, p->howmany);
    if (jobs > 1 && g_loop) {
        std::vector<Job> list(jobs);
        for (int i = 0; i < jobs; ++i)
            list[i] = Job{p, in, out, static_cast<int>(static_cast<long>(p->howmany) * i / jobs),
                          static_cast<int>(static_cast<long>(p->howmany) * (i + 1) / jobs)};
        g_loop(job_work, reinterpret_cast<char *>(list.data()), sizeof(Job), jobs, g_loop_data);
        return;
    }
    run_range(p, in, out, 0, p->howmany);
}

cdns_fftw_plan_s *make(Kind k, int rank, const int *n, int howmany, void *in, int istride,
                       int idist, void *out, int ostride, int odist) {
    if (rank != 1 || !n || n[0] < 1 || howmany < 0) {
        std::fprintf(stderr, "fftw shim: only rank-1 transforms are provided\n");
        std::abort();
    }
    auto *p = new cdns_fftw_plan_s();
    p->kind = k;
    p->n = n[0];
    p->howmany = howmany;
    p->istride = istride;
    p->idist = idist;
    p->ostride = ostride;
    p->odist = odist;
    p->in = in;
    p->out = out;
    p->nthreads = g_nthreads;
    return p;
}
}  // namespace

extern "C" {

fftw_plan fftw_plan_many_dft(int rank, const int *n, int howmany, fftw_complex *in, const int *,
                             int istride, int idist, fftw_complex *out, const int *, int ostride,
                             int odist, int sign, unsigned) {
    auto *p = make(Kind::C2C, rank, n, howmany, in, istride, idist, out, ostride, odist);
    p->full.reset(new Cfft(n[0], sign));
    return p;
}

fftw_plan fftw_plan_many_dft_r2c(int rank, const int *n, int howmany, double *in, const int *,
                                 int istride, int idist, fftw_complex *out, const int *,
                                 int ostride, int odist, unsigned) {
    auto *p = make(Kind::R2C, rank, n, howmany, in, istride, idist, out, ostride, odist);
    setup_real(p, n[0], -1);
    return p;
}

fftw_plan fftw_plan_many_dft_c2r(int rank, const int *n, int howmany, fftw_complex *in,
                                 const int *, int istride, int idist, double *out, const int *,
                                 int ostride, int odist, unsigned) {
    auto *p = make(Kind::C2R, rank, n, howmany, in, istride, idist, out, ostride, odist);
    setup_real(p, n[0], +1);
    return p;
}

fftw_plan fftw_plan_many_r2r(int rank, const int *n, int howmany, double *in, const int *,
                             int istride, int idist, double *out, const int *, int ostride,
                             int odist, const fftw_r2r_kind *kind, unsigned) {
    if (!kind || kind[0] != FFTW_REDFT00 || n[0] < 2) {
        std::fprintf(stderr, "fftw shim: only REDFT00 with n >= 2 is provided\n");
        std::abort();
    }
    auto *p = make(Kind::REDFT00, rank, n, howmany, in, istride, idist, out, ostride, odist);
    setup_real(p, 2 * (n[0] - 1), -1);
    return p;
}

fftw_plan fftw_plan_dft_1d(int n, fftw_complex *in, fftw_complex *out, int sign, unsigned f) {
    return fftw_plan_many_dft(1, &n, 1, in, nullptr, 1, n, out, nullptr, 1, n, sign, f);
}
fftw_plan fftw_plan_dft_r2c_1d(int n, double *in, fftw_complex *out, unsigned f) {
    return fftw_plan_many_dft_r2c(1, &n, 1, in, nullptr, 1, n, out, nullptr, 1, n / 2 + 1, f);
}
fftw_plan fftw_plan_dft_c2r_1d(int n, fftw_complex *in, double *out, unsigned f) {
    return fftw_plan_many_dft_c2r(1, &n, 1, in, nullptr, 1, n / 2 + 1, out, nullptr, 1, n, f);
}
fftw_plan fftw_plan_r2r_1d(int n, double *in, double *out, fftw_r2r_kind kind, unsigned f) {
    return fftw_plan_many_r2r(1, &n, 1, in, nullptr, 1, n, out, nullptr, 1, n, &kind, f);
}

void fftw_execute(const fftw_plan p) { execute(p, p->in, p->out); }
void fftw_execute_dft(const fftw_plan p, fftw_complex *in, fftw_complex *out) { execute(p, in, out); }
void fftw_execute_dft_r2c(const fftw_plan p, double *in, fftw_complex *out) { execute(p, in, out); }
void fftw_execute_dft_c2r(const fftw_plan p, fftw_complex *in, double *out) { execute(p, in, out); }
void fftw_execute_r2r(const fftw_plan p, double *in, double *out) { execute(p, in, out); }
void fftw_destroy_plan(fftw_plan p) { delete p; }

int fftw_alignment_of(double *p) { return static_cast<int>(reinterpret_cast<std::uintptr_t>(p) % 16); }
int fftw_init_threads(void) { return 1; }
void fftw_plan_with_nthreads(int nthreads) { g_nthreads = nthreads > 0 ? nthreads : 1; }
void fftw_cleanup_threads(void) {}
void fftw_cleanup(void) {}
void fftw_threads_set_callback(void (*loop)(void *(*)(char *), char *, size_t, int, void *),
                               void *data) {
    g_loop = loop;
    g_loop_data = data;
}
int fftw_import_wisdom_from_filename(const char *) { return 0; }
int fftw_export_wisdom_to_filename(const char *filename) {
    // No planner state to save; write an empty marker so callers see success.
    FILE *f = std::fopen(filename, "w");
    if (!f) return 0;
    std::fputs("(cdns-fftw-shim-wisdom)\n", f);
    std::fclose(f);
    return 1;
}
void *fftw_malloc(size_t n) { return std::aligned_alloc(64, (n + 63) / 64 * 64); }
void fftw_free(void *p) { std::free(p); }

}  // extern "C"
