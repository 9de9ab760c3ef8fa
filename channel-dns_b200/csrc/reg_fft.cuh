// In-register DFTs for sm_100a: a length-N DFT (N <= 16) held by one thread,
// composed as N = A x B of the radix-2/3/4/5/7 butterflies of fft_lines.cuh
// (unnormalised, FFTW sign convention: SIGN = -1 forward, +1 backward).
// A length n = N1 x N2 transform then needs a single exchange through shared
// memory between its two steps:
//   step 1 (thread n2):  Y[k1] = W_n^(n2 k1) sum_n1 x[n2 + N2 n1] W_N1^(n1 k1)
//   step 2 (thread k1):  X[k1 + N1 k2] = sum_n2 Y_n2[k1] W_N2^(n2 k2)
#pragma once

#include "fft_lines.cuh"

namespace cdns {

// N = A x B with A, B in {1, 2, 3, 4, 5, 7}.
template <int N> struct RegSplit;
template <> struct RegSplit<2> { static constexpr int A = 2, B = 1; };
template <> struct RegSplit<3> { static constexpr int A = 3, B = 1; };
template <> struct RegSplit<4> { static constexpr int A = 4, B = 1; };
template <> struct RegSplit<6> { static constexpr int A = 2, B = 3; };
template <> struct RegSplit<7> { static constexpr int A = 7, B = 1; };
template <> struct RegSplit<8> { static constexpr int A = 2, B = 4; };
template <> struct RegSplit<9> { static constexpr int A = 3, B = 3; };
template <> struct RegSplit<10> { static constexpr int A = 2, B = 5; };
template <> struct RegSplit<12> { static constexpr int A = 3, B = 4; };
template <> struct RegSplit<14> { static constexpr int A = 2, B = 7; };
template <> struct RegSplit<16> { static constexpr int A = 4, B = 4; };

// exp(-2 pi i k / N), N <= 16, as literals (cos and -sin of 2 pi k / N,
// correctly rounded), so that twiddles that are the same in every lane need
// no table loads.
template <int N> __device__ __forceinline__ double2 kroot(int k);
template <> __device__ __forceinline__ double2 kroot<2>(int k) {
    constexpr double c[2] = {1.0, -1.0};
    constexpr double s[2] = {0.0, 0.0};
    return make_double2(c[k], s[k]);
}
template <> __device__ __forceinline__ double2 kroot<3>(int k) {
    constexpr double c[3] = {1.0, -0.5, -0.5};
    constexpr double s[3] = {0.0, -0.8660254037844386, 0.8660254037844386};
    return make_double2(c[k], s[k]);
}
template <> __device__ __forceinline__ double2 kroot<4>(int k) {
    constexpr double c[4] = {1.0, 0.0, -1.0, 0.0};
    constexpr double s[4] = {0.0, -1.0, 0.0, 1.0};
    return make_double2(c[k], s[k]);
}
template <> __device__ __forceinline__ double2 kroot<5>(int k) {
    constexpr double c[5] = {1.0, 0.30901699437494745, -0.8090169943749475, -0.8090169943749475, 0.30901699437494745};
    constexpr double s[5] = {0.0, -0.9510565162951535, -0.5877852522924731, 0.5877852522924731, 0.9510565162951535};
    return make_double2(c[k], s[k]);
}
template <> __device__ __forceinline__ double2 kroot<6>(int k) {
    constexpr double c[6] = {1.0, 0.5, -0.5, -1.0, -0.5, 0.5};
    constexpr double s[6] = {0.0, -0.8660254037844386, -0.8660254037844386, 0.0, 0.8660254037844386, 0.8660254037844386};
    return make_double2(c[k], s[k]);
}
template <> __device__ __forceinline__ double2 kroot<7>(int k) {
    constexpr double c[7] = {1.0, 0.6234898018587335, -0.2225209339563144, -0.9009688679024191, -0.9009688679024191, -0.2225209339563144, 0.6234898018587335};
    constexpr double s[7] = {0.0, -0.7818314824680298, -0.9749279121818236, -0.4338837391175581, 0.4338837391175581, 0.9749279121818236, 0.7818314824680298};
    return make_double2(c[k], s[k]);
}
template <> __device__ __forceinline__ double2 kroot<8>(int k) {
    constexpr double c[8] = {1.0, 0.7071067811865476, 0.0, -0.7071067811865476, -1.0, -0.7071067811865476, 0.0, 0.7071067811865476};
    constexpr double s[8] = {0.0, -0.7071067811865476, -1.0, -0.7071067811865476, 0.0, 0.7071067811865476, 1.0, 0.7071067811865476};
    return make_double2(c[k], s[k]);
}
template <> __device__ __forceinline__ double2 kroot<9>(int k) {
    constexpr double c[9] = {1.0, 0.766044443118978, 0.17364817766693036, -0.5, -0.9396926207859084, -0.9396926207859084, -0.5, 0.17364817766693036, 0.766044443118978};
    constexpr double s[9] = {0.0, -0.6427876096865394, -0.984807753012208, -0.8660254037844386, -0.3420201433256687, 0.3420201433256687, 0.8660254037844386, 0.984807753012208, 0.6427876096865394};
    return make_double2(c[k], s[k]);
}
template <> __device__ __forceinline__ double2 kroot<10>(int k) {
    constexpr double c[10] = {1.0, 0.8090169943749475, 0.30901699437494745, -0.30901699437494745, -0.8090169943749475, -1.0, -0.8090169943749475, -0.30901699437494745, 0.30901699437494745, 0.8090169943749475};
    constexpr double s[10] = {0.0, -0.5877852522924731, -0.9510565162951535, -0.9510565162951535, -0.5877852522924731, 0.0, 0.5877852522924731, 0.9510565162951535, 0.9510565162951535, 0.5877852522924731};
    return make_double2(c[k], s[k]);
}
template <> __device__ __forceinline__ double2 kroot<11>(int k) {
    constexpr double c[11] = {1.0, 0.8412535328311812, 0.41541501300188644, -0.14231483827328514, -0.6548607339452851, -0.9594929736144974, -0.9594929736144974, -0.6548607339452851, -0.14231483827328514, 0.41541501300188644, 0.8412535328311812};
    constexpr double s[11] = {0.0, -0.5406408174555976, -0.9096319953545183, -0.9898214418809327, -0.7557495743542583, -0.28173255684142967, 0.28173255684142967, 0.7557495743542583, 0.9898214418809327, 0.9096319953545183, 0.5406408174555976};
    return make_double2(c[k], s[k]);
}
template <> __device__ __forceinline__ double2 kroot<12>(int k) {
    constexpr double c[12] = {1.0, 0.8660254037844386, 0.5, 0.0, -0.5, -0.8660254037844386, -1.0, -0.8660254037844386, -0.5, 0.0, 0.5, 0.8660254037844386};
    constexpr double s[12] = {0.0, -0.5, -0.8660254037844386, -1.0, -0.8660254037844386, -0.5, 0.0, 0.5, 0.8660254037844386, 1.0, 0.8660254037844386, 0.5};
    return make_double2(c[k], s[k]);
}
template <> __device__ __forceinline__ double2 kroot<13>(int k) {
    constexpr double c[13] = {1.0, 0.8854560256532099, 0.5680647467311558, 0.12053668025532305, -0.3546048870425356, -0.7485107481711011, -0.970941817426052, -0.970941817426052, -0.7485107481711011, -0.3546048870425356, 0.12053668025532305, 0.5680647467311558, 0.8854560256532099};
    constexpr double s[13] = {0.0, -0.46472317204376856, -0.8229838658936564, -0.992708874098054, -0.9350162426854148, -0.6631226582407952, -0.23931566428755777, 0.23931566428755777, 0.6631226582407952, 0.9350162426854148, 0.992708874098054, 0.8229838658936564, 0.46472317204376856};
    return make_double2(c[k], s[k]);
}
template <> __device__ __forceinline__ double2 kroot<14>(int k) {
    constexpr double c[14] = {1.0, 0.9009688679024191, 0.6234898018587335, 0.2225209339563144, -0.2225209339563144, -0.6234898018587335, -0.9009688679024191, -1.0, -0.9009688679024191, -0.6234898018587335, -0.2225209339563144, 0.2225209339563144, 0.6234898018587335, 0.9009688679024191};
    constexpr double s[14] = {0.0, -0.4338837391175581, -0.7818314824680298, -0.9749279121818236, -0.9749279121818236, -0.7818314824680298, -0.4338837391175581, 0.0, 0.4338837391175581, 0.7818314824680298, 0.9749279121818236, 0.9749279121818236, 0.7818314824680298, 0.4338837391175581};
    return make_double2(c[k], s[k]);
}
template <> __device__ __forceinline__ double2 kroot<15>(int k) {
    constexpr double c[15] = {1.0, 0.9135454576426009, 0.6691306063588582, 0.30901699437494745, -0.10452846326765347, -0.5, -0.8090169943749475, -0.9781476007338057, -0.9781476007338057, -0.8090169943749475, -0.5, -0.10452846326765347, 0.30901699437494745, 0.6691306063588582, 0.9135454576426009};
    constexpr double s[15] = {0.0, -0.4067366430758002, -0.7431448254773942, -0.9510565162951535, -0.9945218953682733, -0.8660254037844386, -0.5877852522924731, -0.20791169081775934, 0.20791169081775934, 0.5877852522924731, 0.8660254037844386, 0.9945218953682733, 0.9510565162951535, 0.7431448254773942, 0.4067366430758002};
    return make_double2(c[k], s[k]);
}
template <> __device__ __forceinline__ double2 kroot<16>(int k) {
    constexpr double c[16] = {1.0, 0.9238795325112867, 0.7071067811865476, 0.3826834323650898, 0.0, -0.3826834323650898, -0.7071067811865476, -0.9238795325112867, -1.0, -0.9238795325112867, -0.7071067811865476, -0.3826834323650898, 0.0, 0.3826834323650898, 0.7071067811865476, 0.9238795325112867};
    constexpr double s[16] = {0.0, -0.3826834323650898, -0.7071067811865476, -0.9238795325112867, -1.0, -0.9238795325112867, -0.7071067811865476, -0.3826834323650898, 0.0, 0.3826834323650898, 0.7071067811865476, 0.9238795325112867, 1.0, 0.9238795325112867, 0.7071067811865476, 0.3826834323650898};
    return make_double2(c[k], s[k]);
}

// v * exp(SIGN 2 pi i k / N) with the literal root: the exact cases (+-1, +-i)
// fold to sign changes and swaps after unrolling; FP32 adds the product by the
// rounding residue of the constant (the exact DFT up to arithmetic rounding).
template <int N, int SIGN, class C> __device__ __forceinline__ C mul_kroot(C v, int k) {
    using T = typename CReal<C>::T;
    const double2 w = kroot<N>(k);
    const double wr = w.x, wi = SIGN < 0 ? w.y : -w.y;
    if (wi == 0.0 && wr == -1.0) return C{-v.x, -v.y};
    if (wr == 0.0 && wi == 1.0) return C{-v.y, v.x};
    if (wr == 0.0 && wi == -1.0) return C{v.y, -v.x};
    const T hr = (T)wr, hi = (T)wi;
    C out{v.x * hr - v.y * hi, v.x * hi + v.y * hr};
    if constexpr (sizeof(T) == 4) {
        const T lr = (T)(wr - (double)hr), li = (T)(wi - (double)hi);
        out = C{out.x + (v.x * lr - v.y * li), out.y + (v.x * li + v.y * lr)};
    }
    return out;
}

// X[c + A d] = sum_m v[m] W_N^(m (c + A d)), W_N = exp(SIGN 2 pi i / N), in place.
// The twiddles are literals (kroot); tw and rstride are not read.
template <int N, int SIGN, class C>
__device__ __forceinline__ void dft_reg(C (&v)[N], const Twiddles<C> &, int) {
    constexpr int A = RegSplit<N>::A, B = RegSplit<N>::B;
    if constexpr (B == 1) {
        bfly<A, SIGN>(v, static_cast<const C *>(nullptr), 0);
    } else {
        C y[N];
        // m = b + B a: radix-A DFTs over a, twiddled by W_N^(b c)
#pragma unroll
        for (int b = 0; b < B; ++b) {
            C t[A];
#pragma unroll
            for (int a = 0; a < A; ++a) t[a] = v[b + B * a];
            bfly<A, SIGN>(t, static_cast<const C *>(nullptr), 0);
#pragma unroll
            for (int c = 0; c < A; ++c)
                y[b * A + c] = (b * c == 0) ? t[c] : mul_kroot<N, SIGN>(t[c], (b * c) % N);
        }
        // radix-B DFTs over b
#pragma unroll
        for (int c = 0; c < A; ++c) {
            C t[B];
#pragma unroll
            for (int b = 0; b < B; ++b) t[b] = y[b * A + c];
            bfly<B, SIGN>(t, static_cast<const C *>(nullptr), 0);
#pragma unroll
            for (int d = 0; d < B; ++d) v[c + A * d] = t[d];
        }
    }
}

}  // namespace cdns
