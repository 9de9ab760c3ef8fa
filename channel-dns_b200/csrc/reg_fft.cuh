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

// X[c + A d] = sum_m v[m] W_N^(m (c + A d)), W_N = exp(SIGN 2 pi i / N), in place.
// tw.hi[m * rstride] = exp(-2 pi i m / N) for 0 <= m < N.
template <int N, int SIGN, class C>
__device__ __forceinline__ void dft_reg(C (&v)[N], const Twiddles<C> &tw, int rstride) {
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
                y[b * A + c] = (b * c == 0) ? t[c] : tw.template mul<SIGN>(t[c], ((b * c) % N) * rstride);
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
