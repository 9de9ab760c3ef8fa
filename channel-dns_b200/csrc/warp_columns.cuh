// Warp-per-column building blocks for sm_100a.
//
// A warp owns one spectral column (kz, kx) and keeps its NYS+1 Chebyshev
// coefficients in registers: lane L = 2h + p holds, for every field, the
// coefficients of parity p at y = 2(E h + e) + p, e = 0..E-1.  Recurrences in
// y that couple one parity (Chebyshev derivatives, tau elimination sweeps)
// become first-order affine recurrences along the 16 lanes of a parity: a
// sequential pass over a lane's E coefficients, a 4-level shuffle scan, and a
// carry-in.  Blocks of kColsPerBlock warps stage the planar [kz][y][kx]
// spectral layout through swizzled shared-memory tiles so that global
// accesses are coalesced rows of kColsPerBlock columns.
#pragma once

#include "cdns_common.cuh"

namespace cdns {

constexpr int kColsPerBlock = 8;
constexpr unsigned kFull = 0xffffffffu;

// ---- warp primitives -------------------------------------------------------
__device__ __forceinline__ double2 shfl2(double2 v, int src) {
    return mk(__shfl_sync(kFull, v.x, src), __shfl_sync(kFull, v.y, src));
}
__device__ __forceinline__ double2 shfl2_up(double2 v, int d) {
    return mk(__shfl_up_sync(kFull, v.x, d), __shfl_up_sync(kFull, v.y, d));
}
__device__ __forceinline__ double2 shfl2_down(double2 v, int d) {
    return mk(__shfl_down_sync(kFull, v.x, d), __shfl_down_sync(kFull, v.y, d));
}
__device__ __forceinline__ double2 shfl2_xor(double2 v, int m) {
    return mk(__shfl_xor_sync(kFull, v.x, m), __shfl_xor_sync(kFull, v.y, m));
}
// Sum over the 16 lanes of one parity; every lane of the parity gets the
// same value (IEEE addition commutes).
__device__ __forceinline__ double2 sum_parity(double2 v) {
#pragma unroll
    for (int m = 2; m < 32; m <<= 1) v = cadd(v, shfl2_xor(v, m));
    return v;
}
__device__ __forceinline__ double2 sum_warp(double2 v) {
#pragma unroll
    for (int m = 1; m < 32; m <<= 1) v = cadd(v, shfl2_xor(v, m));
    return v;
}
__device__ __forceinline__ double sum_warp(double v) {
#pragma unroll
    for (int m = 1; m < 32; m <<= 1) v += __shfl_xor_sync(kFull, v, m);
    return v;
}

__device__ __forceinline__ int lane_id() { return threadIdx.x & 31; }

// y of element e in this lane.
template <int E> __device__ __forceinline__ int ycoef(int e) {
    const int L = lane_id();
    return 2 * (E * (L >> 1) + e) + (L & 1);
}

// Value of coefficient y (uniform across the warp) broadcast to all lanes.
template <int E> __device__ __forceinline__ double2 elem(const double2 (&x)[E], int y) {
    const int m = y >> 1, h = m / E, e = m - h * E;
    double2 v = x[0];
#pragma unroll
    for (int k = 1; k < E; ++k)
        if (k == e) v = x[k];
    return shfl2(v, 2 * h + (y & 1));
}

// In-place solution of X_y = B_y + A_y X_{y+2} (suffix direction, per parity);
// elements beyond the chain carry A = 0, B = 0.
template <int E> __device__ __forceinline__ void affine_suffix(double (&A)[E], double2 (&B)[E]) {
    const int L = lane_id();
#pragma unroll
    for (int e = E - 2; e >= 0; --e) {
        B[e] = cadd(B[e], cscale(A[e], B[e + 1]));
        A[e] = A[e] * A[e + 1];
    }
    double a = A[0];
    double2 b = B[0];
#pragma unroll
    for (int d = 2; d < 32; d <<= 1) {
        const double a2 = __shfl_down_sync(kFull, a, d);
        const double2 b2 = shfl2_down(b, d);
        if (L + d < 32) {
            b = cadd(b, cscale(a, b2));
            a = a * a2;
        }
    }
    double2 carry = shfl2_down(b, 2);
    if (L + 2 >= 32) carry = mk(0.0, 0.0);
#pragma unroll
    for (int e = 0; e < E; ++e) B[e] = cadd(B[e], cscale(A[e], carry));
}
template <int E> __device__ __forceinline__ void affine_suffix(double (&A)[E], double (&B)[E]) {
    const int L = lane_id();
#pragma unroll
    for (int e = E - 2; e >= 0; --e) {
        B[e] = B[e] + A[e] * B[e + 1];
        A[e] = A[e] * A[e + 1];
    }
    double a = A[0], b = B[0];
#pragma unroll
    for (int d = 2; d < 32; d <<= 1) {
        const double a2 = __shfl_down_sync(kFull, a, d);
        const double b2 = __shfl_down_sync(kFull, b, d);
        if (L + d < 32) {
            b = b + a * b2;
            a = a * a2;
        }
    }
    double carry = __shfl_down_sync(kFull, b, 2);
    if (L + 2 >= 32) carry = 0.0;
#pragma unroll
    for (int e = 0; e < E; ++e) B[e] = B[e] + A[e] * carry;
}
// In-place solution of Z_y = B_y + A_y Z_{y-2} (prefix direction, per parity).
template <int E> __device__ __forceinline__ void affine_prefix(double (&A)[E], double2 (&B)[E]) {
    const int L = lane_id();
#pragma unroll
    for (int e = 1; e < E; ++e) {
        B[e] = cadd(B[e], cscale(A[e], B[e - 1]));
        A[e] = A[e] * A[e - 1];
    }
    double a = A[E - 1];
    double2 b = B[E - 1];
#pragma unroll
    for (int d = 2; d < 32; d <<= 1) {
        const double a2 = __shfl_up_sync(kFull, a, d);
        const double2 b2 = shfl2_up(b, d);
        if (L >= d) {
            b = cadd(b, cscale(a, b2));
            a = a * a2;
        }
    }
    double2 carry = shfl2_up(b, 2);
    if (L < 2) carry = mk(0.0, 0.0);
#pragma unroll
    for (int e = 0; e < E; ++e) B[e] = cadd(B[e], cscale(A[e], carry));
}
// In-place suffix sums S_y = sum_{j >= y, j = y mod 2} S_j.
template <int E> __device__ __forceinline__ void suffix_sum(double2 (&S)[E]) {
    const int L = lane_id();
#pragma unroll
    for (int e = E - 2; e >= 0; --e) S[e] = cadd(S[e + 1], S[e]);
    double2 b = S[0];
#pragma unroll
    for (int d = 2; d < 32; d <<= 1) {
        const double2 t = shfl2_down(b, d);
        if (L + d < 32) b = cadd(t, b);
    }
    double2 carry = shfl2_down(b, 2);
    if (L + 2 >= 32) carry = mk(0.0, 0.0);
#pragma unroll
    for (int e = 0; e < E; ++e) S[e] = cadd(carry, S[e]);
}

// Diagonal of the tau boundary rows (src/solver/eqsolve_pv.cpp:64-128).
__device__ __forceinline__ double tau_func(double a, double b, int y) {
    const int q = y & 1;
    if (a == 0.0 && b == 0.0) return (double)((1 - q) * y * y + q);
    return a + b * y * y;
}

// In-place prefix sums S_y = sum_{j <= y, j = y mod 2} S_j.
template <int E> __device__ __forceinline__ void prefix_sum(double2 (&S)[E]) {
    const int L = lane_id();
#pragma unroll
    for (int e = 1; e < E; ++e) S[e] = cadd(S[e - 1], S[e]);
    double2 b = S[E - 1];
#pragma unroll
    for (int d = 2; d < 32; d <<= 1) {
        const double2 t = shfl2_up(b, d);
        if (L >= d) b = cadd(t, b);
    }
    double2 carry = shfl2_up(b, 2);
    if (L < 2) carry = mk(0.0, 0.0);
#pragma unroll
    for (int e = 0; e < E; ++e) S[e] = cadd(carry, S[e]);
}

// Chebyshev derivative (src/solver/vector_ops.cpp:17-25):
// d_k = sum_{j > k, j = k+1 mod 2} 2 j f_j, d_0 halved.  f is zero beyond ny.
template <int E> __device__ __forceinline__ void deriv_warp(int ny, const double2 (&f)[E], double2 (&d)[E]) {
    const int L = lane_id(), p = L & 1;
    double2 S[E];
#pragma unroll
    for (int e = 0; e < E; ++e) {
        const int y = ycoef<E>(e);
        S[e] = (y <= ny) ? cscale((double)(2 * y), f[e]) : mk(0.0, 0.0);
    }
    suffix_sum<E>(S);
    // d(y) = S(y + 1): the neighbour of opposite parity
    double2 a[E];
#pragma unroll
    for (int e = 0; e < E; ++e) a[e] = shfl2_xor(S[e], 1);
    double2 c = shfl2_down(S[0], 1);
    if (L == 31) c = mk(0.0, 0.0);
#pragma unroll
    for (int e = 0; e < E; ++e) {
        const int y = ycoef<E>(e);
        const double2 nx = (p == 0) ? a[e] : (e + 1 < E ? a[(e + 1) % E] : c);
        d[e] = (y < ny) ? nx : mk(0.0, 0.0);
        if (y == 0) d[e] = cscale(0.5, d[e]);
    }
}

// Shared-memory tile [ncy][kColsPerBlock] of complex values with the column
// slot swizzled by y, so that both a row of kColsPerBlock columns (staging)
// and the E-strided y coefficients of one column (a warp) are free of bank
// conflicts.
template <int E> __device__ __forceinline__ int tile_slot(int y, int l) {
    const int g = (2 * (y / (2 * E)) + (y & 1)) & (kColsPerBlock - 1);
    return y * kColsPerBlock + (l ^ g);
}

// Elements per lane for NYS + 1 coefficients (1, 2, 4 or 8; 0 if too many).
inline int lane_elems(const Dims &d) {
    const int e = (d.ncy + 31) / 32;
    return e <= 1 ? 1 : e <= 2 ? 2 : e <= 4 ? 4 : e <= 8 ? 8 : 0;
}

}  // namespace cdns
