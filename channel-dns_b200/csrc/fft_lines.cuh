// Batched complex FFT of interleaved lines for sm_100a.
//
// L lines of length n are stored interleaved: element (pos, line) sits at
// buf[pos*L + line], so a warp's lanes touch consecutive 16-byte words in
// every pass.  The transform is an iterative mixed-radix Stockham autosort
// FFT, unnormalised, with the FFTW sign convention (SIGN=-1 forward, +1
// backward).  Every pass is instantiated for its radix at compile time
// (radix 2, 3, 4, 5, 7 with literal twiddle constants; other odd radices up
// to 13 from the root table), so the R values of a butterfly stay in
// registers.  Two drivers:
//   fft_lines  shared memory in, shared memory out (ping-pong buffers);
//   fft_run    the first pass reads through a source functor and the last
//              pass writes through a destination functor (global memory),
//              middle passes ping-pong in shared memory.
#pragma once

#include "cdns_common.cuh"

namespace cdns {

constexpr int kMaxRadix = 16;

// roots[k] = exp(-2 pi i k / n); SIGN=+1 uses the conjugate.
template <int SIGN, class C> __device__ __forceinline__ C root_of(const C *roots, int k) {
    const C r = roots[k];
    return SIGN < 0 ? r : mkc<C>(r.x, -r.y);
}

// A twiddle table exp(-2 pi i k / n): in FP32 each entry carries the residue
// of its rounding (lo), added by a second product, so that the transform is
// the exact DFT up to random arithmetic rounding (no systematic operator error).
template <class C> struct Twiddles {
    const C *hi, *lo;   // lo is used by the FP32 form only
    template <int SIGN> __device__ __forceinline__ C at(int k) const { return root_of<SIGN>(hi, k); }
    template <int SIGN> __device__ __forceinline__ C mul(C v, int k) const {
        const C w = root_of<SIGN>(hi, k);
        if constexpr (sizeof(C) == 8) {
            return cadd(cmul(v, w), cmul(v, root_of<SIGN>(lo, k)));
        } else {
            return cmul(v, w);
        }
    }
};

// cos / sin (2 pi i / R) for 0 <= i < R, folded to literals after unrolling.
template <int R> __device__ __forceinline__ double kcos(int i);
template <int R> __device__ __forceinline__ double ksin(int i);
template <> __device__ __forceinline__ double kcos<3>(int i) { return i == 0 ? 1.0 : -0.5; }
template <> __device__ __forceinline__ double ksin<3>(int i) {
    return i == 0 ? 0.0 : (i == 1 ? 0.8660254037844386 : -0.8660254037844386);
}
template <> __device__ __forceinline__ double kcos<5>(int i) {
    const int a = i <= 2 ? i : 5 - i;
    return a == 0 ? 1.0 : (a == 1 ? 0.30901699437494745 : -0.8090169943749475);
}
template <> __device__ __forceinline__ double ksin<5>(int i) {
    const int a = i <= 2 ? i : 5 - i;
    const double s = a == 0 ? 0.0 : (a == 1 ? 0.9510565162951535 : 0.5877852522924731);
    return i <= 2 ? s : -s;
}
template <> __device__ __forceinline__ double kcos<7>(int i) {
    const int a = i <= 3 ? i : 7 - i;
    return a == 0 ? 1.0 : (a == 1 ? 0.6234898018587335 : (a == 2 ? -0.2225209339563144 : -0.9009688679024191));
}
template <> __device__ __forceinline__ double ksin<7>(int i) {
    const int a = i <= 3 ? i : 7 - i;
    const double s = a == 0 ? 0.0 : (a == 1 ? 0.7818314824680298 : (a == 2 ? 0.9749279121818236 : 0.4338837391175581));
    return i <= 3 ? s : -s;
}

// Odd radix by symmetric pairs: with s_t = x_t + x_{R-t}, d_t = x_t - x_{R-t},
// y_q = x_0 + sum_t s_t cos(2 pi t q/R) + SIGN i sum_t d_t sin(2 pi t q/R),
// y_{R-q} the same with the sine term negated.
template <int R, int SIGN, bool TABLE, class C>
__device__ __forceinline__ void bfly_odd(C (&v)[R], const C *roots, int n) {
    using T = typename CReal<C>::T;
    constexpr int h = R / 2;
    C s[h + 1], d[h + 1];
#pragma unroll
    for (int t = 1; t <= h; ++t) {
        s[t] = cadd(v[t], v[R - t]);
        d[t] = csub(v[t], v[R - t]);
    }
    C out[R];
    C y0 = v[0];
#pragma unroll
    for (int t = 1; t <= h; ++t) y0 = cadd(y0, s[t]);
    out[0] = y0;
#pragma unroll
    for (int q = 1; q <= h; ++q) {
        C re = v[0], im = mkc<C>(0.0, 0.0);
#pragma unroll
        for (int t = 1; t <= h; ++t) {
            const int i = (t * q) % R;
            T c, sn;
            if constexpr (TABLE) {
                const C w = roots[i * (n / R)];  // exp(-2 pi i i/R)
                c = w.x;
                sn = -w.y;
            } else {
                c = (T)kcos<R>(i);
                sn = (T)ksin<R>(i);
            }
            re.x += c * s[t].x;
            re.y += c * s[t].y;
            im.x += sn * d[t].x;
            im.y += sn * d[t].y;
            if constexpr (!TABLE && sizeof(T) == 4) {
                // FP32: add the rounding residue of the constant, so that the
                // butterfly is the exact DFT up to random arithmetic rounding
                const T cl = (T)(kcos<R>(i) - (double)c), sl = (T)(ksin<R>(i) - (double)sn);
                re.x += cl * s[t].x;
                re.y += cl * s[t].y;
                im.x += sl * d[t].x;
                im.y += sl * d[t].y;
            }
        }
        const C iim = SIGN < 0 ? mkc<C>(im.y, -im.x) : mkc<C>(-im.y, im.x);
        out[q] = cadd(re, iim);
        out[R - q] = csub(re, iim);
    }
#pragma unroll
    for (int q = 0; q < R; ++q) v[q] = out[q];
}

template <int R, int SIGN, class C>
__device__ __forceinline__ void bfly(C (&v)[R], const C *roots, int n) {
    if constexpr (R == 1) {
        return;
    } else if constexpr (R == 2) {
        const C a = v[0], b = v[1];
        v[0] = cadd(a, b);
        v[1] = csub(a, b);
    } else if constexpr (R == 4) {
        const C a = cadd(v[0], v[2]), b = csub(v[0], v[2]);
        const C c = cadd(v[1], v[3]), d = csub(v[1], v[3]);
        const C di = SIGN < 0 ? mkc<C>(d.y, -d.x) : mkc<C>(-d.y, d.x);  // SIGN i d
        v[0] = cadd(a, c);
        v[1] = cadd(b, di);
        v[2] = csub(a, c);
        v[3] = csub(b, di);
    } else if constexpr (R == 3 || R == 5 || R == 7) {
        bfly_odd<R, SIGN, false>(v, roots, n);
    } else {
        bfly_odd<R, SIGN, true>(v, roots, n);
    }
}

// Source / destination functors over interleaved shared-memory lines.
struct SmemSrc {
    const double2 *buf;
    int L;
    __device__ __forceinline__ double2 operator()(int pos, int line) const { return buf[pos * L + line]; }
};
struct SmemDst {
    double2 *buf;
    int L;
    __device__ __forceinline__ void operator()(int pos, int line, double2 v) const { buf[pos * L + line] = v; }
};

// One Stockham pass of radix R over L lines: span ns (product of the radices
// already applied).  Each work item (j, line) reads R inputs at stride n/R,
// twiddles them by w^(q k), k = j mod ns, and writes R outputs at stride ns.
template <int R, int SIGN, class Src, class Dst>
__device__ __forceinline__ void pass_ct(int n, int L, int ns, const double2 *roots, const Src &src,
                                        const Dst &dst) {
    const int m = n / R;
    const int tstep = n / (ns * R);
    const int total = m * L;
    for (int w = threadIdx.x; w < total; w += blockDim.x) {
        const int j = w / L;
        const int line = w - j * L;
        const int k = j % ns;
        double2 v[R];
#pragma unroll
        for (int q = 0; q < R; ++q) v[q] = src(j + q * m, line);
        if (k) {
#pragma unroll
            for (int q = 1; q < R; ++q) v[q] = cmul(v[q], root_of<SIGN>(roots, q * k * tstep));
        }
        bfly<R, SIGN>(v, roots, n);
        const int base = (j / ns) * ns * R + k;
#pragma unroll
        for (int q = 0; q < R; ++q) dst(base + q * ns, line, v[q]);
    }
}

// Radices 9, 11 and 13 (meshes outside the usual 2^a 3^b 5^c 7^d sizes) run in
// a separate non-inlined function so that they do not raise the register
// budget of the kernels that use the common radices.
template <int SIGN, class Src, class Dst>
__device__ __noinline__ void pass_rare(int R, int n, int L, int ns, const double2 *roots,
                                       const Src &src, const Dst &dst) {
    switch (R) {
    case 9: pass_ct<9, SIGN>(n, L, ns, roots, src, dst); break;
    case 11: pass_ct<11, SIGN>(n, L, ns, roots, src, dst); break;
    case 13: pass_ct<13, SIGN>(n, L, ns, roots, src, dst); break;
    default: break;  // plans only hold radices 2, 3, 4, 5, 7, 9, 11, 13
    }
}

template <int SIGN, class Src, class Dst>
__device__ __forceinline__ void pass_dispatch(int R, int n, int L, int ns, const double2 *roots,
                                              const Src &src, const Dst &dst) {
    switch (R) {
    case 1: pass_ct<1, SIGN>(n, L, ns, roots, src, dst); break;
    case 2: pass_ct<2, SIGN>(n, L, ns, roots, src, dst); break;
    case 3: pass_ct<3, SIGN>(n, L, ns, roots, src, dst); break;
    case 4: pass_ct<4, SIGN>(n, L, ns, roots, src, dst); break;
    case 5: pass_ct<5, SIGN>(n, L, ns, roots, src, dst); break;
    case 7: pass_ct<7, SIGN>(n, L, ns, roots, src, dst); break;
    default: pass_rare<SIGN>(R, n, L, ns, roots, src, dst); break;
    }
}

// Shared memory in and out; returns the buffer holding the result (a or b).
// Every thread of the block must call it (it synchronises between passes).
template <int SIGN>
__device__ double2 *fft_lines(double2 *a, double2 *b, int L, const FftPlan &P, const double2 *roots) {
    const int n = P.n;
    double2 *src = a, *dst = b;
    int ns = 1;
    for (int p = 0; p < P.nrad; ++p) {
        const int R = P.radix[p];
        pass_dispatch<SIGN>(R, n, L, ns, roots, SmemSrc{src, L}, SmemDst{dst, L});
        __syncthreads();
        double2 *t = src;
        src = dst;
        dst = t;
        ns *= R;
    }
    return src;
}

// First pass reads through `gsrc(pos, line)`, last pass writes through
// `gdst(pos, line, value)`; middle passes ping-pong between a and b.
template <int SIGN, class GSrc, class GDst>
__device__ void fft_run(double2 *a, double2 *b, int L, const FftPlan &P, const double2 *roots,
                        const GSrc &gsrc, const GDst &gdst) {
    const int n = P.n;
    if (P.nrad <= 1) {
        pass_dispatch<SIGN>(P.nrad == 1 ? P.radix[0] : 1, n, L, 1, roots, gsrc, gdst);
        return;
    }
    int ns = 1;
    pass_dispatch<SIGN>(P.radix[0], n, L, ns, roots, gsrc, SmemDst{a, L});
    __syncthreads();
    ns *= P.radix[0];
    double2 *cur = a, *oth = b;
    for (int p = 1; p < P.nrad - 1; ++p) {
        pass_dispatch<SIGN>(P.radix[p], n, L, ns, roots, SmemSrc{cur, L}, SmemDst{oth, L});
        __syncthreads();
        double2 *t = cur;
        cur = oth;
        oth = t;
        ns *= P.radix[p];
    }
    pass_dispatch<SIGN>(P.radix[P.nrad - 1], n, L, ns, roots, SmemSrc{cur, L}, gdst);
}

}  // namespace cdns
