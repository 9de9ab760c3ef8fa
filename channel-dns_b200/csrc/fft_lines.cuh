// Batched complex FFT of interleaved lines in shared memory.
//
// L lines of length n are stored interleaved: element (pos, line) sits at
// buf[pos*L + line], so a warp's lanes touch consecutive 16-byte words in
// every pass (no bank conflicts).  The transform is an iterative mixed-radix
// Stockham autosort FFT (radix 4, 2, 3, 5, 7, and a direct DFT for other
// small primes) that ping-pongs between two buffers; it is unnormalised with
// the FFTW sign convention: SIGN=-1 forward, SIGN=+1 backward.
#pragma once

#include "cdns_common.cuh"

namespace cdns {

constexpr int kMaxRadix = 16;

// roots[k] = exp(-2 pi i k / n); SIGN=+1 uses the conjugate.
template <int SIGN> __device__ inline double2 root_of(const double2 *roots, int k) {
    const double2 r = roots[k];
    return SIGN < 0 ? r : mk(r.x, -r.y);
}

template <int SIGN>
__device__ inline void dft_small(double2 *v, int R, const double2 *roots, int n) {
    if (R == 2) {
        const double2 a = v[0], b = v[1];
        v[0] = cadd(a, b);
        v[1] = csub(a, b);
        return;
    }
    if (R == 4) {
        const double2 a = cadd(v[0], v[2]), b = csub(v[0], v[2]);
        const double2 c = cadd(v[1], v[3]), d = csub(v[1], v[3]);
        // SIGN*i*d
        const double2 di = SIGN < 0 ? mk(d.y, -d.x) : mk(-d.y, d.x);
        v[0] = cadd(a, c);
        v[1] = cadd(b, di);
        v[2] = csub(a, c);
        v[3] = csub(b, di);
        return;
    }
    if (R == 3) {
        // y0 = a+b+c ; y1,2 = a - (b+c)/2 +- SIGN*i*(sqrt3/2)(b-c)
        const double s3 = 0.86602540378443864676;
        const double2 t = cadd(v[1], v[2]);
        const double2 d = csub(v[1], v[2]);
        const double2 m = mk(v[0].x - 0.5 * t.x, v[0].y - 0.5 * t.y);
        const double2 r = SIGN < 0 ? mk(s3 * d.y, -s3 * d.x) : mk(-s3 * d.y, s3 * d.x);
        v[0] = cadd(v[0], t);
        v[1] = cadd(m, r);
        v[2] = csub(m, r);
        return;
    }
    // Odd R: pair terms t and R-t (real parts share cosines, imaginary parts
    // share sines), halving the multiplications of a direct DFT.
    double2 out[kMaxRadix];
    const int step = n / R;
    const int h = R / 2;
    double2 s[kMaxRadix / 2 + 1], dd[kMaxRadix / 2 + 1];
    for (int t = 1; t <= h; ++t) {
        s[t] = cadd(v[t], v[R - t]);
        dd[t] = csub(v[t], v[R - t]);
    }
    double2 y0 = v[0];
    for (int t = 1; t <= h; ++t) y0 = cadd(y0, s[t]);
    out[0] = y0;
    for (int q = 1; q <= h; ++q) {
        double2 re = v[0];
        double2 im = mk(0.0, 0.0);
        for (int t = 1; t <= h; ++t) {
            const double2 w = roots[((t * q) % R) * step];  // exp(-2 pi i tq/R)
            re.x += w.x * s[t].x;
            re.y += w.x * s[t].y;
            im.x += w.y * dd[t].x;
            im.y += w.y * dd[t].y;
        }
        // forward: y_q = re + i*im_part, where sum w.y*dd carries sin(-..)
        // term i*(w.y)*dd ; backward flips the sign of the sine.
        const double2 iim = SIGN < 0 ? mk(-im.y, im.x) : mk(im.y, -im.x);
        out[q] = cadd(re, iim);
        out[R - q] = csub(re, iim);
    }
    for (int q = 0; q < R; ++q) v[q] = out[q];
}

// Runs all passes; returns the buffer holding the result (a or b).  Every
// thread of the block must call it (it synchronises between passes).
template <int SIGN>
__device__ double2 *fft_lines(double2 *a, double2 *b, int L, const FftPlan &P,
                              const double2 *roots) {
    const int n = P.n;
    double2 *src = a, *dst = b;
    int ns = 1;
    for (int p = 0; p < P.nrad; ++p) {
        const int R = P.radix[p];
        const int m = n / R;
        const int tstep = n / (ns * R);
        const int work = m * L;
        for (int w = threadIdx.x; w < work; w += blockDim.x) {
            const int line = w % L;
            const int j = w / L;
            const int k = j % ns;
            double2 v[kMaxRadix];
            for (int q = 0; q < R; ++q) {
                double2 x = src[(j + q * m) * L + line];
                if (k) x = cmul(x, root_of<SIGN>(roots, q * k * tstep));
                v[q] = x;
            }
            dft_small<SIGN>(v, R, roots, n);
            const int base = (j / ns) * ns * R + k;
            for (int q = 0; q < R; ++q) dst[(base + q * ns) * L + line] = v[q];
        }
        __syncthreads();
        double2 *t = src;
        src = dst;
        dst = t;
        ns *= R;
    }
    return src;
}

}  // namespace cdns
