// Fine-grid (3/2 product grid) transforms of the channel-dns nonlinear term,
// written for sm_100a.  Stage layout in HBM (complex<double>):
//
//   spectral   S[c][kz][y][kx]          (c = component, Ns per component)
//   Ypys       F[f][j][kz][kx]          after the Chebyshev synthesis (j = GL point)
//   Zphys      G[f][j][z][kx]           after the inverse z FFT
//   Xspec      H[f][j][z][kx]           products after the forward x FFT
//   Zspec      F[f][j][kz][kx]          after the forward z FFT
//
// The Chebyshev (y) synthesis and analysis live in chebyshev.cu; this file
// holds the Fourier directions (src/fft/transforms.cpp:615-741): the analysis
// keeps x1/NX2 before the z FFT and x1/NZ2 after it.
#include <algorithm>
#include <cstdlib>
#include <type_traits>

#include "cdns_kernels.cuh"
#include "fft_lines.cuh"
#include "reg_fft.cuh"

namespace cdns {

// ---------------------------------------------------------------------------
// K2: inverse z FFT.  Block = one (field, y point) plane x TL kx lines.  The
// first Stockham pass reads the kz in [-NZS, NZS] coefficients straight from
// HBM into the NZ2 slots (negative Nyquist slot wins at a full z spectrum,
// src/fft/transforms.cpp:715-732); the last pass writes z-physical rows.
// ---------------------------------------------------------------------------
// The coarse-grid transform (coarse = true, src/fft/transforms.cpp:560-572)
// instead sums the two Nyquist coefficients into the shared slot.
template <class C> struct ZExpandSrc {
    const C *Fp;   // one (field, y point) plane [kz][kx]
    int nkx, kx0, NZS, n;
    bool coarse;
    __device__ __forceinline__ C operator()(int z, int line) const {
        const int kx = kx0 + line;
        if (kx >= nkx) return mkc<C>(0, 0);
        int kz;
        if (z <= NZS) {
            if (z == n - NZS) {
                if (coarse) return cadd(Fp[(2 * NZS) * nkx + kx], Fp[kx]);
                kz = -NZS;
            } else {
                kz = z;
            }
        } else if (z >= n - NZS) {
            kz = z - n;
        } else {
            return mkc<C>(0, 0);
        }
        return Fp[(kz + NZS) * nkx + kx];
    }
};
template <class C> struct RowDst {
    C *p;   // [pos][kx]
    int nkx, kx0;
    __device__ __forceinline__ void operator()(int pos, int line, C v) const {
        const int kx = kx0 + line;
        if (kx < nkx) p[(long long)pos * nkx + kx] = v;
    }
};
template <class C> struct RowSrc {
    const C *p;
    int nkx, kx0;
    __device__ __forceinline__ C operator()(int pos, int line) const {
        const int kx = kx0 + line;
        return kx < nkx ? p[(long long)pos * nkx + kx] : mkc<C>(0, 0);
    }
};
// Forward z: keep kz in [-NZS, NZS] scaled by 1/NZ2 (src/fft/transforms.cpp:658-665);
// at a full z spectrum slot NZS feeds both kz = +NZS and kz = -NZS, halved on
// the coarse grid (coarse = true, src/fft/transforms.cpp:506-511).
template <class C> struct ZTruncDst {
    C *Fp;
    int nkx, kx0, NZS, n;
    typename CReal<C>::T invn;
    bool coarse;
    __device__ __forceinline__ void operator()(int z, int line, C v) const {
        const int kx = kx0 + line;
        if (kx >= nkx) return;
        C s = cscale(invn, v);
        if (coarse && z <= NZS && z >= n - NZS) s = cscale((typename CReal<C>::T)0.5, s);
        if (z <= NZS) Fp[(z + NZS) * nkx + kx] = s;
        if (z >= n - NZS) Fp[(z - n + NZS) * nkx + kx] = s;
    }
};

__global__ void __launch_bounds__(256, 2)
k_z_backward(Dims d, FftPlan P, const double2 *__restrict__ roots, const double2 *__restrict__ F,
             double2 *__restrict__ G, int TL, bool coarse) {
    extern __shared__ double2 sm[];
    const int n = d.NZ2;
    double2 *s_root = sm;
    double2 *a = sm + n;
    double2 *b = a + n * TL;
    const int f = blockIdx.z, j = blockIdx.y, kx0 = blockIdx.x * TL;
    for (int i = threadIdx.x; i < n; i += blockDim.x) s_root[i] = roots[i];
    __syncthreads();
    const ZExpandSrc<double2> src{F + ((long long)f * d.ny2 + j) * d.fcol, d.nkx, kx0, d.NZS, n, coarse};
    const RowDst<double2> dst{G + ((long long)f * d.ny2 + j) * (long long)n * d.nkx, d.nkx, kx0};
    fft_run<+1>(a, b, TL, P, s_root, src, dst);
}

__global__ void __launch_bounds__(256, 2)
k_z_forward(Dims d, FftPlan P, const double2 *__restrict__ roots, const double2 *__restrict__ H,
            double2 *__restrict__ F, int TL, bool coarse) {
    extern __shared__ double2 sm[];
    const int n = d.NZ2;
    double2 *s_root = sm;
    double2 *a = sm + n;
    double2 *b = a + n * TL;
    const int f = blockIdx.z, j = blockIdx.y, kx0 = blockIdx.x * TL;
    for (int i = threadIdx.x; i < n; i += blockDim.x) s_root[i] = roots[i];
    __syncthreads();
    const RowSrc<double2> src{H + ((long long)f * d.ny2 + j) * (long long)n * d.nkx, d.nkx, kx0};
    const ZTruncDst<double2> dst{F + ((long long)f * d.ny2 + j) * d.fcol, d.nkx, kx0, d.NZS, n, 1.0 / (double)n,
                                 coarse};
    fft_run<-1>(a, b, TL, P, s_root, src, dst);
}

// Register form of the z transforms for NZ2 = N1 x N2: threads t = n2 TL + l
// (step 1) and t = k1 TL + l (step 2) over TL kx lines, one shared-memory
// exchange S[k1][n2][l]; loads and stores run along kx.
// Shared twiddle table of the register forms: n double2 slots, holding the
// FP64 roots, or the FP32 roots and their rounding residues.
template <class C> __device__ __forceinline__ Twiddles<C> load_twiddles(double2 *sm_d, const double2 *roots, int n) {
    C *hi = reinterpret_cast<C *>(sm_d);
    C *lo = sizeof(C) == 8 ? hi + n : hi;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const double2 r = roots[i];
        hi[i] = cto<C>(r);
        if (sizeof(C) == 8) lo[i] = mkc<C>(r.x - (double)hi[i].x, r.y - (double)hi[i].y);
    }
    return Twiddles<C>{hi, lo};
}
// Inter-step twiddles of an N1 x N2 register transform (N2 <= 16) as N1 rows of
// 16: entry (k1, s) = exp(-2 pi i s k1 / n), in 16 N1 double2 slots (FP32: the
// roots and their rounding residues).  The view returned is offset to the
// calling lane's column s = sub, so that row k1 is at index 16 k1.
template <int N1, class C>
__device__ __forceinline__ Twiddles<C> load_lane_twiddles(double2 *sm_d, const double2 *roots, int n, int sub) {
    C *hi = reinterpret_cast<C *>(sm_d);
    C *lo = sizeof(C) == 8 ? hi + 16 * N1 : hi;
    for (int i = threadIdx.x; i < 16 * N1; i += blockDim.x) {
        const double2 r = roots[((i & 15) * (i >> 4)) % n];
        hi[i] = cto<C>(r);
        if (sizeof(C) == 8) lo[i] = mkc<C>(r.x - (double)hi[i].x, r.y - (double)hi[i].y);
    }
    return Twiddles<C>{hi + sub, lo + sub};
}

// Row stride of fft2_lines' exchange between k1 groups: N2 TL padded to = TL
// (mod 8), so that a quarter-warp whose threads span two k1 groups touches 8
// distinct 16-byte bank groups (unpadded, N2 TL = 0 mod 8 for the even N2 used).
__host__ __device__ constexpr int fft2_kstride(int n2, int tl) { return n2 * tl + (((tl - n2 * tl) % 8) + 8) % 8; }

template <int N1, int N2, int SIGN, class C, class Src, class Dst>
__device__ __forceinline__ void fft2_lines(int TL, const Twiddles<C> &tw, C *S, const Src &src, const Dst &dst) {
    const int KS = fft2_kstride(N2, TL);
    constexpr int NM = N1 > N2 ? N1 : N2;
    const int t = threadIdx.x;
    C v[NM];
    const bool a1 = t < N2 * TL;
    const int n2 = t / TL, l1 = t - (t / TL) * TL;
    if (a1) {
#pragma unroll
        for (int n1 = 0; n1 < N1; ++n1) v[n1] = src(n2 + N2 * n1, l1);
    }
    __syncthreads();   // s_root complete
    if (a1) {
        C(&w)[N1] = reinterpret_cast<C(&)[N1]>(v);
        dft_reg<N1, SIGN>(w, tw, N2);
#pragma unroll
        for (int k1 = 0; k1 < N1; ++k1)
            S[k1 * KS + n2 * TL + l1] = (k1 == 0 || n2 == 0) ? w[k1] : tw.template mul<SIGN>(w[k1], n2 * k1);
    }
    __syncthreads();
    if (t < N1 * TL) {
        const int k1 = t / TL, l = t - (t / TL) * TL;
#pragma unroll
        for (int m = 0; m < N2; ++m) v[m] = S[k1 * KS + m * TL + l];
        C(&w)[N2] = reinterpret_cast<C(&)[N2]>(v);
        dft_reg<N2, SIGN>(w, tw, N1);
#pragma unroll
        for (int k2 = 0; k2 < N2; ++k2) dst(k1 + N1 * k2, l, w[k2]);
    }
}

template <int N1, int N2, class C>
__global__ void __launch_bounds__(16 * 17)
k_z_backward_r(Dims d, const double2 *__restrict__ roots, const C *__restrict__ F, C *__restrict__ G, int TL,
               bool coarse) {
    extern __shared__ double2 sm_d[];
    constexpr int n = N1 * N2;
    C *S = reinterpret_cast<C *>(sm_d + n);
    const int f = blockIdx.z, j = blockIdx.y, kx0 = blockIdx.x * TL;
    const Twiddles<C> tw = load_twiddles<C>(sm_d, roots, n);
    const ZExpandSrc<C> src{F + ((long long)f * d.ny2 + j) * d.fcol, d.nkx, kx0, d.NZS, n, coarse};
    const RowDst<C> dst{G + ((long long)f * d.ny2 + j) * (long long)n * d.nkx, d.nkx, kx0};
    fft2_lines<N1, N2, +1>(TL, tw, S, src, dst);
}

template <int N1, int N2, class C>
__global__ void __launch_bounds__(16 * 17)
k_z_forward_r(Dims d, const double2 *__restrict__ roots, const C *__restrict__ H, C *__restrict__ F, int TL,
              bool coarse) {
    extern __shared__ double2 sm_d[];
    constexpr int n = N1 * N2;
    C *S = reinterpret_cast<C *>(sm_d + n);
    const int f = blockIdx.z, j = blockIdx.y, kx0 = blockIdx.x * TL;
    const Twiddles<C> tw = load_twiddles<C>(sm_d, roots, n);
    const RowSrc<C> src{H + ((long long)f * d.ny2 + j) * (long long)n * d.nkx, d.nkx, kx0};
    // FP32: no 1/NZ2 here (not exact in FP32); the FP64 y analysis applies 1/(NX2 NZ2)
    const ZTruncDst<C> dst{F + ((long long)f * d.ny2 + j) * d.fcol, d.nkx, kx0, d.NZS, n,
                           (typename CReal<C>::T)(sizeof(C) == 8 ? 1.0 : 1.0 / (double)n), coarse};
    fft2_lines<N1, N2, -1>(TL, tw, S, src, dst);
}

// The pencil rank's fused exchange: the same transforms, the spectral side
// read from and written to every rank's column buffer (PeerCols) at the
// slab's global y point pc.j0 + j.  Fine-grid conventions (FP64).
struct ZExpandPeers {
    PeerCols pc;
    int f, jg, nkx, kx0, nkz, NZS, n;
    __device__ __forceinline__ double2 operator()(int z, int line) const {
        const int kx = kx0 + line;
        if (kx >= nkx) return mk(0.0, 0.0);
        int kz;
        if (z <= NZS) kz = (z == n - NZS) ? -NZS : z;
        else if (z >= n - NZS) kz = z - n;
        else return mk(0.0, 0.0);
        return pc.col[kx][((long long)(f * pc.ny2 + jg) * nkz + (kz + NZS)) * pc.width[kx]];
    }
};
struct ZTruncPeers {
    PeerCols pc;
    int f, jg, nkx, kx0, nkz, NZS, n;
    double invn;
    __device__ __forceinline__ void operator()(int z, int line, double2 v) const {
        const int kx = kx0 + line;
        if (kx >= nkx) return;
        const double2 s = cscale(invn, v);
        double2 *p = pc.col[kx];
        const long long row = (long long)(f * pc.ny2 + jg) * nkz;
        const int w = pc.width[kx];
        if (z <= NZS) p[(row + z + NZS) * w] = s;
        if (z >= n - NZS) p[(row + z - n + NZS) * w] = s;
    }
};

template <int N1, int N2>
__global__ void __launch_bounds__(16 * 17)
k_z_backward_peers(Dims d, const double2 *__restrict__ roots, PeerCols pc, double2 *__restrict__ G, int TL) {
    extern __shared__ double2 sm_d[];
    constexpr int n = N1 * N2;
    double2 *S = sm_d + n;
    const int f = blockIdx.z, j = blockIdx.y, kx0 = blockIdx.x * TL;
    const Twiddles<double2> tw = load_twiddles<double2>(sm_d, roots, n);
    const ZExpandPeers src{pc, f, pc.j0 + j, d.nkx, kx0, d.nkz, d.NZS, n};
    const RowDst<double2> dst{G + ((long long)f * d.ny2 + j) * (long long)n * d.nkx, d.nkx, kx0};
    fft2_lines<N1, N2, +1>(TL, tw, S, src, dst);
}

template <int N1, int N2>
__global__ void __launch_bounds__(16 * 17)
k_z_forward_peers(Dims d, const double2 *__restrict__ roots, const double2 *__restrict__ H, PeerCols pc, int TL) {
    extern __shared__ double2 sm_d[];
    constexpr int n = N1 * N2;
    double2 *S = sm_d + n;
    const int f = blockIdx.z, j = blockIdx.y, kx0 = blockIdx.x * TL;
    const Twiddles<double2> tw = load_twiddles<double2>(sm_d, roots, n);
    const RowSrc<double2> src{H + ((long long)f * d.ny2 + j) * (long long)n * d.nkx, d.nkx, kx0};
    const ZTruncPeers dst{pc, f, pc.j0 + j, d.nkx, kx0, d.nkz, d.NZS, n, 1.0 / (double)n};
    fft2_lines<N1, N2, -1>(TL, tw, S, src, dst);
}

// ---------------------------------------------------------------------------
// Chebyshev synthesis and analysis as a DCT-I of N + 1 points, N = NY2 =
// N1 x N2, through one length-N complex FFT per column (FP64).  For x_0..x_N,
//   Y_j = (x_0 + (-1)^j x_N)/2 + sum_{n=1}^{N-1} x_n cos(pi n j / N):
// with y_n = (x_n + x_{N-n})/2 - sin(pi n / N)(x_n - x_{N-n}) (n < N) and
// Z = DFT_N(y), the even outputs are Y_2k = (Z_k + Z_{N-k})/2 and the odd ones
// follow by a prefix sum, Y_{2k+1} = Y_1 + sum_{q=1..k} i (Z_q - Z_{N-q})/2,
// with Y_1 = (x_0 - x_N)/2 + sum_{n=1}^{N-1} x_n cos(pi n / N).
//   synthesis (ANA = false): x_0 = 2 c_0, x_k = c_k (k <= NYS), 0 beyond;
//             f_j = Y_j for j = 0..N (the doubled c_0 and the z expansion's
//             0.5 of the reference cancel, as in k_ysynth).
//   analysis  (ANA = true):  x_j = F_j;  S_0 = Y_0 / N, S_k = 2 Y_k / N
//             (the scalings 1/(2 NY2) and 1/NY2 with the DCT-I's doubled
//             interior sum), k <= NYS.
// Block = one (field, kz) plane x TL kx lines (TL a compile-time width), 16 TL
// threads: thread t owns line l = t mod TL and row group r = t / TL (rows
// r, r + 16, ...), so that in every phase consecutive threads touch
// consecutive lines -- coalesced global rows along kx and conflict-free
// shared rows [n][l].  Phases (barriers between):
//   load x_n (n = 0..N) and each thread's partial of Y_1's sum over its rows;
//   Z = DFT_N(y) (fft2_lines; the exchange aliases x, read before its barrier);
//   even outputs from Z pairs, stored from registers, and each thread's chunk
//   of the odd outputs' prefix sum (16 consecutive-k chunks per line);
//   the carry of the earlier chunks (a fixed-order sum of their totals) and
//   the odd outputs, stored from registers.  Stores run along kx (11-16 lines of
//   one row per thread group), as the loads do.
// Shared memory: twiddles [N], x / exchange [(N+1)][TL] (or the padded
// exchange), Z [N][TL], partials [16][TL] (Y_1's, then the chunk totals), Y_1 [TL].
// ---------------------------------------------------------------------------
struct YdctSrc {
    const double2 *X;
    const double *cosy;
    int TL, N;
    __device__ __forceinline__ double2 operator()(int n, int l) const {
        const double2 a = X[n * TL + l], b = X[(N - n) * TL + l];
        const double s = cosy[(n + (3 * N) / 2) % (2 * N)];   // sin(pi n / N)
        return csub(cscale(0.5, cadd(a, b)), cscale(s, csub(a, b)));
    }
};
struct YdctDst {
    double2 *Z;
    int TL;
    __device__ __forceinline__ void operator()(int k, int l, double2 v) const { Z[k * TL + l] = v; }
};

constexpr int kYdctRows = 16;   // row groups of the DCT kernel (16 TL threads)
// x / exchange region of the DCT kernel: the N + 1 rows, or the padded exchange
__host__ __device__ constexpr int ydct_xslots(int n1, int n2, int tl) {
    return (n1 * n2 + 1) * tl > n1 * fft2_kstride(n2, tl) ? (n1 * n2 + 1) * tl : n1 * fft2_kstride(n2, tl);
}
__host__ __device__ constexpr size_t ydct_slots(int n1, int n2, int tl) {
    return (size_t)n1 * n2 + (size_t)ydct_xslots(n1, n2, tl) + (size_t)n1 * n2 * tl + (size_t)kYdctRows * tl + tl;
}

// Operands of the DCT kernels; CT is the stage buffer's complex type (double2,
// or float2 for the mixed form's FP32 stages).  Synthesis: spectral
// spec0 / spec1 (fields f < nsplit / the rest), coefficient k weighted by
// in0 (k = 0) or in1, -> F, row j weighted by outE (j = 0, N) or outI; with
// `mean` (FP32 stages) the (kz, kx) = (0, 0) column goes to mean[f][j] in FP64
// and zeros to F.  Analysis: F, row j weighted by inE (j = 0, N) or inI, ->
// spectral S, coefficient k scaled by s0 (k = 0) or sk.  The forward
// transforms take unit weights and s0 = 1/N, sk = 2/N (times 1 / (NX2 NZ2) for
// FP32 stages, whose z and x analyses leave it out); the discrete adjoint's
// transposed stages take other weights (launch_ydct_adjoint_*).
template <class CT> struct YdctArgs {
    const double2 *spec0 = nullptr, *spec1 = nullptr;
    int nsplit = 0;
    const CT *Fin = nullptr;
    CT *Fout = nullptr;
    double2 *S = nullptr;
    double *mean = nullptr;
    double in0 = 1.0, in1 = 1.0, outE = 1.0, outI = 1.0;   // synthesis weights
    double inE = 1.0, inI = 1.0, s0 = 0.0, sk = 0.0;       // analysis weights and scales
};

template <int N1, int N2, bool ANA, int TL, class CT>
__global__ void __launch_bounds__(16 * TL)
k_ydct_r(Dims d, const double2 *__restrict__ roots, const double *__restrict__ cosy, YdctArgs<CT> A) {
    constexpr int N = N1 * N2;
    constexpr int R = kYdctRows;
    constexpr int M = N / 2 - 1;                // odd outputs beyond Y_1: k = 1..M
    constexpr int CH = (N / 2 + R) / R;         // k = 0..N/2 in R chunks of CH
    extern __shared__ double2 sm_d[];
    double2 *X = sm_d + N;
    double2 *Z = X + ydct_xslots(N1, N2, TL);
    double2 *P = Z + N * TL;
    double2 *Y1 = P + R * TL;
    const int f = blockIdx.z, kzi = blockIdx.y, kx0 = blockIdx.x * TL;
    const int t = threadIdx.x;
    const int l = t % TL, r = t / TL;
    const int nkx = d.nkx, ncy = d.ncy, kx = kx0 + l;
    const bool lok = kx < nkx;
    const Twiddles<double2> tw = load_twiddles<double2>(sm_d, roots, N);
    // ---- x_n, n = 0..N, and partials of Y_1 = sum_{n=1}^{N-1} x_n cos(pi n / N)
    // rows n = r + R i: all loads of a thread are issued before the first use
    constexpr int NI = N / R + 1;
    double2 y1 = mk(0.0, 0.0);
    double2 xv[NI];
    if (!ANA) {
        const double2 *S = (f < A.nsplit ? A.spec0 + (long long)f * d.Ns : A.spec1 + (long long)(f - A.nsplit) * d.Ns) +
                           (long long)kzi * ncy * nkx + kx;
#pragma unroll
        for (int i = 0; i < NI; ++i) {
            const int n = r + R * i;
            xv[i] = (n <= N && n < ncy && lok) ? S[(long long)n * nkx] : mk(0.0, 0.0);
        }
#pragma unroll
        for (int i = 0; i < NI; ++i) {
            const int n = r + R * i;
            if (n > N) break;
            double2 v = cscale(n == 0 ? A.in0 : A.in1, xv[i]);
            if (n == 0) v = cadd(v, v);
            X[n * TL + l] = v;
            if (n >= 1 && n < N) y1 = cadd(y1, cscale(cosy[n], v));
        }
    } else {
        const CT *F = A.Fin + (long long)f * d.ny2 * d.fcol + (long long)kzi * nkx + kx;
#pragma unroll
        for (int i = 0; i < NI; ++i) {
            const int n = r + R * i;
            xv[i] = (n <= N && lok) ? cto<double2>(F[(long long)n * d.fcol]) : mk(0.0, 0.0);
        }
#pragma unroll
        for (int i = 0; i < NI; ++i) {
            const int n = r + R * i;
            if (n > N) break;
            const double2 v = cscale(n == 0 || n == N ? A.inE : A.inI, xv[i]);
            X[n * TL + l] = v;
            if (n >= 1 && n < N) y1 = cadd(y1, cscale(cosy[n], v));
        }
    }
    P[r * TL + l] = y1;
    __syncthreads();
    if (r == 0) {
        double2 acc = cscale(0.5, csub(X[l], X[N * TL + l]));
#pragma unroll
        for (int q = 0; q < R; ++q) acc = cadd(acc, P[q * TL + l]);
        Y1[l] = acc;
    }
    // ---- Z = DFT_N(y) (the exchange buffer aliases X: read before its barrier)
    fft2_lines<N1, N2, -1>(TL, tw, X, YdctSrc{X, cosy, TL, N}, YdctDst{Z, TL});
    __syncthreads();
    // ---- outputs, stored from registers as they are formed ----------------
    // (row j of the line: synthesis F_j, j = 0..N; analysis S_j, j <= NYS)
    CT *Fo = nullptr;
    double2 *So = nullptr;
    if (!ANA) Fo = A.Fout + (long long)f * d.ny2 * d.fcol + (long long)kzi * nkx + kx;
    else So = A.S + (long long)f * d.Ns + (long long)kzi * ncy * nkx + kx;
    // mean profile (kz, kx) = (0, 0) of FP32 stages: kept in FP64, out of the
    // FP32 buffer (its imaginary part is round-off of a real profile)
    const bool to_mean = !ANA && A.mean && kzi == d.NZS && kx == 0;
    auto out = [&](int j, double2 v) {
        if (!lok) return;
        if (!ANA) {
            if (to_mean) {
                A.mean[f * d.ny2 + j] = v.x;
                Fo[(long long)j * d.fcol] = mkc<CT>(0.0, 0.0);
            } else {
                Fo[(long long)j * d.fcol] = cto<CT>(cscale(j == 0 || j == N ? A.outE : A.outI, v));
            }
        } else if (j < ncy) {
            So[(long long)j * nkx] = cscale(j == 0 ? A.s0 : A.sk, v);
        }
    };
    // ---- even outputs X_2k = (Z_k + Z_{N-k}) / 2; chunk sums of i (Z_q - Z_{N-q}) / 2
    double2 part[CH];
    double2 run = mk(0.0, 0.0);
#pragma unroll
    for (int c = 0; c < CH; ++c) {
        const int k = r * CH + c;
        if (k <= N / 2) {
            const double2 zk = Z[k * TL + l], zm = Z[((N - k) % N) * TL + l];
            out(2 * k, cscale(0.5, cadd(zk, zm)));
            if (k >= 1 && k <= M) {
                const double2 dz = csub(zk, zm);
                run = cadd(run, mk(-0.5 * dz.y, 0.5 * dz.x));
            }
        }
        part[c] = run;
    }
    P[r * TL + l] = run;
    __syncthreads();
    // ---- odd outputs X_{2k+1} = Y_1 + sum_{q=1..k} i (Z_q - Z_{N-q}) / 2 -------
    double2 carry = mk(0.0, 0.0);
    for (int q = 0; q < r; ++q) carry = cadd(carry, P[q * TL + l]);
    const double2 y = Y1[l];
    if (r == 0) out(1, y);
#pragma unroll
    for (int c = 0; c < CH; ++c) {
        const int k = r * CH + c;
        if (k >= 1 && k <= M) out(2 * k + 1, cadd(y, cadd(carry, part[c])));
    }
}

// ---------------------------------------------------------------------------
// K3: inverse x FFT of the six fields, u x omega, forward x FFT of the three
// products.  Block = RW rows (z, j); real rows are packed in pairs into one
// complex line (a + i b); c2r drops the imaginary parts of the DC and Nyquist
// bins as FFTW does.  Products: N = u x omega (src/solver/vector_ops.cpp:263-269),
// packed as (N0 + i N1) and (N2 of row r + i N2 of row r+1).  Loads and stores
// run along kx so that a warp touches contiguous HBM.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256, 2)
k_x_cross(Dims d, FftPlan P, const double2 *__restrict__ roots, const double2 *__restrict__ G,
          double2 *__restrict__ H, int RW) {
    extern __shared__ double2 sm[];
    const int n = d.NX2;
    double2 *s_root = sm;
    const int L = 3 * RW;
    double2 *a = sm + n;
    double2 *b = a + n * L;
    const int j = blockIdx.y, z0 = blockIdx.x * RW;
    for (int i = threadIdx.x; i < n; i += blockDim.x) s_root[i] = roots[i];
    const long long fstride = (long long)d.ny2 * d.NZ2 * d.nkx;
    const double2 *Gj = G + (long long)j * d.NZ2 * d.nkx;
    const int nyq = (n % 2 == 0) ? n / 2 : -1;
    const int nkx = d.nkx;
    // zero band between the retained modes and their mirrors
    const int zlo = d.NXS + 1, zhi = n - d.NXS;  // slots [zlo, zhi) are zero
    for (int i = threadIdx.x; i < (zhi - zlo) * L; i += blockDim.x) {
        const int k = zlo + i / L, line = i - (i / L) * L;
        a[k * L + line] = mk(0, 0);
    }
    // retained modes and their Hermitian mirrors, one (row, pair, kx) per thread
    for (int i = threadIdx.x; i < L * nkx; i += blockDim.x) {
        const int line = i / nkx, m = i - (i / nkx) * nkx;
        const int r = line / 3, p = line - (line / 3) * 3;
        const int z = z0 + r;
        double2 A = mk(0, 0), B = mk(0, 0);
        if (z < d.NZ2) {
            const double2 *row = Gj + (long long)z * nkx + m;
            A = row[(2 * p) * fstride];
            B = row[(2 * p + 1) * fstride];
        }
        if (m == 0 || m == nyq) {
            A.y = 0.0;
            B.y = 0.0;
        }
        a[m * L + line] = mk(A.x - B.y, A.y + B.x);
        if (m != 0 && m != nyq) a[(n - m) * L + line] = mk(A.x + B.y, B.x - A.y);
    }
    __syncthreads();
    double2 *res = fft_lines<+1>(a, b, L, P, s_root);
    double2 *oth = (res == a) ? b : a;
    // products, packed into 3 lines per pair of rows; one thread per
    // (point, row pair) so every shared-memory element has a single writer.
    const int npair = (RW + 1) / 2;
    const int L2 = 3 * npair;
    for (int i = threadIdx.x; i < n * npair; i += blockDim.x) {
        const int x = i / npair, pr = i - (i / npair) * npair;
        double n2[2] = {0.0, 0.0};
        for (int odd = 0; odd < 2; ++odd) {
            const int r = 2 * pr + odd;
            if (r >= RW) {
                oth[x * L2 + 3 * pr + odd] = mk(0, 0);
                continue;
            }
            const double2 p0 = res[x * L + 3 * r];
            const double2 p1 = res[x * L + 3 * r + 1];
            const double2 p2 = res[x * L + 3 * r + 2];
            const double uu = p0.x, vv = p0.y, ww = p1.x, ox = p1.y, oy = p2.x, oz = p2.y;
            const double n0 = vv * oz - ww * oy;
            const double n1 = ww * ox - uu * oz;
            n2[odd] = uu * oy - vv * ox;
            oth[x * L2 + 3 * pr + odd] = mk(n0, n1);
        }
        oth[x * L2 + 3 * pr + 2] = mk(n2[0], n2[1]);
    }
    __syncthreads();
    double2 *res2 = fft_lines<-1>(oth, res, L2, P, s_root);
    const double invn = 1.0 / (double)n;
    for (int i = threadIdx.x; i < RW * 3 * nkx; i += blockDim.x) {
        const int rf = i / nkx, k = i - (i / nkx) * nkx;
        const int r = rf / 3, f = rf - (rf / 3) * 3;
        const int z = z0 + r;
        if (z >= d.NZ2) continue;
        const int km = (n - k) % n;
        const int pr = r >> 1, odd = r & 1;
        const int line = (f < 2) ? 3 * pr + odd : 3 * pr + 2;
        const double2 P0 = res2[k * L2 + line];
        const double2 Pm = res2[km * L2 + line];
        // unpack: A = (P + conj Pm)/2, B = (P - conj Pm)/(2i)
        const bool takeA = (f == 0) || (f == 2 && !odd);
        const double2 out = takeA ? mk(0.5 * (P0.x + Pm.x), 0.5 * (P0.y - Pm.y))
                                  : mk(0.5 * (P0.y + Pm.y), -0.5 * (P0.x - Pm.x));
        H[(long long)f * fstride + ((long long)j * d.NZ2 + z) * nkx + k] = cscale(invn, out);
    }
}

// ---------------------------------------------------------------------------
// K3, register form for NX2 = N1 x N2 (N1, N2 <= 16): the same transform with
// every length-NX2 FFT done as two in-register DFT steps and one shared-memory
// exchange.  16 lanes per line (a half-warp), RW rows per block, RW even.
//   phase 1  lanes (line, n2): gather the Hermitian spectrum slots
//            m = n2 + N2 n1 from HBM, N1-point DFT, twiddle -> S
//   phase 2  lanes (line, k1): N2-point DFT -> physical rows P[line][x]
//   phase 3  lanes (out line, n2): products at x = n2 + N2 n1 from P,
//            N1-point DFT, twiddle -> S
//   phase 4  lanes (out line, k1): N2-point DFT, Hermitian unpack with the
//            partner lane (k1' = N1 - k1) by shuffle, modes k <= NXS -> HBM
// S and P share one buffer; every phase reads into registers before a
// barrier and writes after it.
// ---------------------------------------------------------------------------
// SPLIT (N1, N2 even): the forward phases 3 and 4 give each of the 1.5 RW
// forward lines two slots (one warp, lanes h = 0, 1 of a pair sub, sub + 16):
// each N-point DFT step is split by decimation in time into its even (h = 0)
// and odd (h = 1) samples, N/2-point DFTs on each lane, the odd half twiddled
// by W_N^k, and the butterfly X_k = E_k + W^k O_k, X_{k+N/2} = E_k - W^k O_k
// exchanged by __shfl_xor(16): lane h then holds outputs k + h N/2.  So all
// 3 RW slots work in every phase (without SPLIT, half of them idle in 3, 4).
// FP64 is held to 3 blocks per SM (at most 112 registers; left free, the
// compiler moves all twiddle loads of a phase ahead and takes 138); FP32 has
// no minimum (with one it takes 64 registers instead of 56).
constexpr int kRWr = 4;   // rows per block of the register-form x stage (at most)
// exchange buffer of k_x_cross_r in complex elements for rw rows: the step-1
// output of 3 rw lines ([line][k1][n2], rows padded to n2 + 1; larger than their
// physical rows)
__host__ __device__ constexpr int xcross_buf_elems(int n1, int n2, int rw) { return 3 * rw * n1 * (n2 + 1); }
template <int N1, int N2, class C, bool MEAN, bool SPLIT = false>
__global__ void __launch_bounds__(16 * 3 * 4, sizeof(C) == 16 ? 3 : 0)
k_x_cross_r(Dims d, const double2 *__restrict__ roots, const C *__restrict__ G, C *__restrict__ H, int RW,
            const double *__restrict__ mean) {
    using T = typename CReal<C>::T;
    constexpr int n = N1 * N2;
    constexpr int SP = N2 + 1;   // padded row of the step-1 output
    extern __shared__ double2 sm_d[];
    C *buf = reinterpret_cast<C *>(sm_d + n + 16 * N1);
    T *n2s = reinterpret_cast<T *>(buf + xcross_buf_elems(N1, N2, RW));   // [RW][n], SPLIT only
    const int L = 3 * RW, L2 = 3 * (RW / 2);
    const int slot = threadIdx.x >> 4, sub = threadIdx.x & 15;
    const int j = blockIdx.y, z0 = blockIdx.x * RW;
    const int nkx = d.nkx, nxs = d.NXS;
    const long long fstride = (long long)d.ny2 * d.NZ2 * nkx;
    const C *Gj = G + (long long)j * d.NZ2 * nkx;
    const Twiddles<C> tw = load_twiddles<C>(sm_d, roots, n);
    // FP64: the inter-step twiddles W_n^(sub k1) as rows k1 of 16 lanes, so
    // that the 16 lanes of a line read 16 consecutive entries (no bank
    // conflicts).  FP32 reads them from the root table at index sub k1.
    Twiddles<C> tws = tw;
    if constexpr (sizeof(C) == 16) tws = load_lane_twiddles<N1, C>(sm_d + n, roots, n, sub);
    // FP32 skips the product by the unit twiddle of lane 0 (without that
    // branch the loads of all its twiddles move ahead: 80 registers, not 56)
    constexpr bool FP32 = sizeof(C) == 8;
    auto inter = [&](auto sign, C v, int k1) -> C {
        constexpr int SIGN = decltype(sign)::value;
        if constexpr (sizeof(C) == 16) return tws.template mul<SIGN>(v, 16 * k1);
        else return tw.template mul<SIGN>(v, sub * k1);
    };
    const int nyq = (n % 2 == 0) ? n / 2 : -1;
    C v[N1 > N2 ? N1 : N2];

    // ---- phase 1: spectrum gather, N1-point DFTs over n1 (backward) --------
    const bool act1 = slot < L && sub < N2;
    if (act1) {
        const int r = slot / 3, pl = slot - (slot / 3) * 3;
        const int z = z0 + r;
        const C *rowA = Gj + (long long)z * nkx + (2 * pl) * fstride;
        const C *rowB = rowA + fstride;
#pragma unroll
        for (int n1 = 0; n1 < N1; ++n1) {
            const int m = sub + N2 * n1;
            C x = mkc<C>(0.0, 0.0);
            if (z < d.NZ2) {
                if (m <= nxs) {
                    C A = rowA[m], B = rowB[m];
                    if (m == 0 || m == nyq) {
                        A.y = 0.0;
                        B.y = 0.0;
                    }
                    x = mkc<C>(A.x - B.y, A.y + B.x);
                } else if (m >= n - nxs && m != nyq) {
                    const C A = rowA[n - m], B = rowB[n - m];
                    x = mkc<C>(A.x + B.y, B.x - A.y);
                }
            }
            v[n1] = x;
        }
    }
    __syncthreads();   // twiddles complete
    if (act1) {
        C(&w)[N1] = reinterpret_cast<C(&)[N1]>(v);
        dft_reg<N1, +1>(w, tw, N2);
#pragma unroll
        for (int k1 = 0; k1 < N1; ++k1) {
            const C t = (k1 == 0 || (FP32 && sub == 0)) ? w[k1] : inter(std::integral_constant<int, +1>{}, w[k1], k1);
            buf[(slot * N1 + k1) * SP + sub] = t;
        }
    }
    __syncthreads();
    // ---- phase 2: N2-point DFTs over n2 -> physical rows ------------------
    const bool act2 = slot < L && sub < N1;
    if (act2) {
#pragma unroll
        for (int n2 = 0; n2 < N2; ++n2) v[n2] = buf[(slot * N1 + sub) * SP + n2];
    }
    __syncthreads();
    if (act2) {
        C(&w)[N2] = reinterpret_cast<C(&)[N2]>(v);
        dft_reg<N2, +1>(w, tw, N1);
#pragma unroll
        for (int k2 = 0; k2 < N2; ++k2) buf[slot * n + sub + N1 * k2] = w[k2];
    }
    __syncthreads();
    // ---- phase 3: products u x omega, N1-point DFTs (forward) -------------
    T mu = 0, mv = 0, mw = 0, mox = 0, moy = 0, moz = 0;
    if constexpr (MEAN) {
        const int ny2 = d.ny2;
        mu = (T)mean[j];
        mv = (T)mean[ny2 + j];
        mw = (T)mean[2 * ny2 + j];
        mox = (T)mean[3 * ny2 + j];
        moy = (T)mean[4 * ny2 + j];
        moz = (T)mean[5 * ny2 + j];
    }
    if constexpr (SPLIT) {
        static_assert(N1 % 2 == 0 && N2 % 2 == 0, "lane-pair split needs even factors");
        constexpr int H1 = N1 / 2, H2 = N2 / 2;
        const int ol = slot >> 1, h = slot & 1;   // forward line, half (lanes sub and sub + 16)
        const int pr = ol / 3, kind = ol - (ol / 3) * 3;
        // ---- phase 3: products at x = sub + N2 (2m + h), N1/2-point DFTs --------
        const bool act3 = ol < L2 && sub < N2;
        if (act3) {
#pragma unroll
            for (int m = 0; m < H1; ++m) {
                const int x = sub + N2 * (2 * m + h);
                auto prod = [&](int r, T &n0, T &n1v, T &n2v) {
                    const C p0 = buf[(3 * r) * n + x];
                    const C p1 = buf[(3 * r + 1) * n + x];
                    const C p2 = buf[(3 * r + 2) * n + x];
                    const T uu = p0.x, vv = p0.y, ww = p1.x, ox = p1.y, oy = p2.x, oz = p2.y;
                    n0 = vv * oz - ww * oy;
                    n1v = ww * ox - uu * oz;
                    n2v = uu * oy - vv * ox;
                    if constexpr (MEAN) {
                        n0 += (mv * oz - mw * oy) + (vv * moz - ww * moy);
                        n1v += (mw * ox - mu * oz) + (ww * mox - uu * moz);
                        n2v += (mu * oy - mv * ox) + (uu * moy - vv * mox);
                    }
                };
                // lines (N0 + i N1) of rows 2 pr, 2 pr + 1 leave N2 in n2s for the
                // line N2(2 pr) + i N2(2 pr + 1), which reads it after the barrier
                if (kind < 2) {
                    T a0, a1, a2;
                    prod(2 * pr + kind, a0, a1, a2);
                    v[m] = mkc<C>(a0, a1);
                    n2s[(2 * pr + kind) * n + x] = a2;
                }
            }
        }
        __syncthreads();
        if (act3) {
            if (kind == 2) {
#pragma unroll
                for (int m = 0; m < H1; ++m) {
                    const int x = sub + N2 * (2 * m + h);
                    v[m] = mkc<C>(n2s[(2 * pr) * n + x], n2s[(2 * pr + 1) * n + x]);
                }
            }
            C(&w)[H1] = reinterpret_cast<C(&)[H1]>(v);
            dft_reg<H1, -1>(w, tw, 2 * N2);
            if (h) {
#pragma unroll
                for (int k = 1; k < H1; ++k) w[k] = mul_kroot<N1, -1>(w[k], k);   // W_N1^k
            }
        }
#pragma unroll
        for (int k = 0; k < H1; ++k) {
            C q;
            q.x = __shfl_xor_sync(0xffffffffu, v[k].x, 16);
            q.y = __shfl_xor_sync(0xffffffffu, v[k].y, 16);
            if (!act3) continue;
            const C xk = h ? csub(q, v[k]) : cadd(v[k], q);
            const int k1 = k + h * H1;
            buf[(ol * N1 + k1) * SP + sub] = (k1 == 0 || (FP32 && sub == 0)) ? xk : inter(std::integral_constant<int, -1>{}, xk, k1);
        }
        __syncthreads();
        // ---- phase 4: N2/2-point DFTs over n2 = 2m + h, unpack, modes k <= NXS ---
        const bool act4 = ol < L2 && sub < N1;
        if (act4) {
#pragma unroll
            for (int m = 0; m < H2; ++m) v[m] = buf[(ol * N1 + sub) * SP + 2 * m + h];
            C(&w)[H2] = reinterpret_cast<C(&)[H2]>(v);
            dft_reg<H2, -1>(w, tw, 2 * N1);
            if (h) {
#pragma unroll
                for (int k = 1; k < H2; ++k) w[k] = mul_kroot<N2, -1>(w[k], k);   // W_N2^k
            }
        }
#pragma unroll
        for (int k = 0; k < H2; ++k) {
            C q;
            q.x = __shfl_xor_sync(0xffffffffu, v[k].x, 16);
            q.y = __shfl_xor_sync(0xffffffffu, v[k].y, 16);
            v[k] = h ? csub(q, v[k]) : cadd(v[k], q);   // P[sub + N1 (h H2 + k)]
        }
        // partner of q = k1 + N1 k2 (k2 = h H2 + c) is n - q: for k1 > 0 lane
        // (1 - h, N1 - k1), c' = H2 - 1 - c; for k1 = 0 lane (1 - h, 0), c' = H2 - c
        // (c = 0: the lane itself).  Lanes k1 = 0 serve only the k1 = 0 lane of the
        // other half, so each lane sends the register its readers want: one
        // shuffle per output.
        const int pA = 16 * (1 - h) + (sub < N1 ? (N1 - sub) % N1 : sub);
        const T invn = (T)(sizeof(C) == 8 ? 1.0 : 1.0 / (double)n);
#pragma unroll
        for (int c = 0; c < H2; ++c) {
            const C send = sub == 0 ? v[(H2 - c) % H2] : v[H2 - 1 - c];
            C pa;
            pa.x = __shfl_sync(0xffffffffu, send.x, pA);
            pa.y = __shfl_sync(0xffffffffu, send.y, pA);
            const int k = sub + N1 * (h * H2 + c);
            if (!act4 || k > nxs) continue;
            const C pm = (sub == 0 && c == 0) ? v[0] : pa;
            const C p0 = v[c];
            const C outA = cscale(invn, mkc<C>(T(0.5) * (p0.x + pm.x), T(0.5) * (p0.y - pm.y)));
            const C outB = cscale(invn, mkc<C>(T(0.5) * (p0.y + pm.y), T(-0.5) * (p0.x - pm.x)));
            if (kind < 2) {
                const int z = z0 + 2 * pr + kind;
                if (z < d.NZ2) {
                    C *hp = H + ((long long)j * d.NZ2 + z) * nkx + k;
                    hp[0] = outA;            // N0
                    hp[fstride] = outB;      // N1
                }
            } else {
                const int z = z0 + 2 * pr;
                C *hp = H + 2 * fstride + ((long long)j * d.NZ2 + z) * nkx + k;
                if (z < d.NZ2) hp[0] = outA;                 // N2 of row r
                if (z + 1 < d.NZ2) hp[nkx] = outB;           // N2 of row r+1
            }
        }
    } else {
        // out lines per row pair (r, r+1): (N0 + i N1)(r), (N0 + i N1)(r+1), N2(r) + i N2(r+1)
        const bool act3 = slot < L2 && sub < N2;
        if (act3) {
            const int pr = slot / 3, kind = slot - (slot / 3) * 3;
    #pragma unroll
            for (int n1 = 0; n1 < N1; ++n1) {
                const int x = sub + N2 * n1;
                auto prod = [&](int r, T &n0, T &n1v, T &n2v) {
                    const C p0 = buf[(3 * r) * n + x];
                    const C p1 = buf[(3 * r + 1) * n + x];
                    const C p2 = buf[(3 * r + 2) * n + x];
                    const T uu = p0.x, vv = p0.y, ww = p1.x, ox = p1.y, oy = p2.x, oz = p2.y;
                    n0 = vv * oz - ww * oy;
                    n1v = ww * ox - uu * oz;
                    n2v = uu * oy - vv * ox;
                    if constexpr (MEAN) {
                        // fluctuations about the FP64 mean profiles: + M x om' + u' x M_om
                        // (M x M_om is added to the mean mode in FP64 after the analysis)
                        n0 += (mv * oz - mw * oy) + (vv * moz - ww * moy);
                        n1v += (mw * ox - mu * oz) + (ww * mox - uu * moz);
                        n2v += (mu * oy - mv * ox) + (uu * moy - vv * mox);
                    }
                };
                T a0, a1, a2, b0, b1, b2;
                if (kind < 2) {
                    prod(2 * pr + kind, a0, a1, a2);
                    v[n1] = mkc<C>(a0, a1);
                } else {
                    prod(2 * pr, a0, a1, a2);
                    prod(2 * pr + 1, b0, b1, b2);
                    v[n1] = mkc<C>(a2, b2);
                }
            }
        }
        __syncthreads();
        if (act3) {
            C(&w)[N1] = reinterpret_cast<C(&)[N1]>(v);
            dft_reg<N1, -1>(w, tw, N2);
    #pragma unroll
            for (int k1 = 0; k1 < N1; ++k1) {
                const C t = (k1 == 0 || (FP32 && sub == 0)) ? w[k1] : inter(std::integral_constant<int, -1>{}, w[k1], k1);
                buf[(slot * N1 + k1) * SP + sub] = t;
            }
        }
        __syncthreads();
        // ---- phase 4: N2-point DFTs, unpack, modes k <= NXS -------------------
        const bool act4 = slot < L2 && sub < N1;
        if (act4) {
    #pragma unroll
            for (int n2 = 0; n2 < N2; ++n2) v[n2] = buf[(slot * N1 + sub) * SP + n2];
            C(&w)[N2] = reinterpret_cast<C(&)[N2]>(v);
            dft_reg<N2, -1>(w, tw, N1);
        }
        // partner of frequency k1 + N1 k2 is n - k = k1' + N1 k2' with
        // k1' = (N1 - k1) mod N1, k2' = N2 - 1 - k2 (k1 > 0) or (N2 - k2) mod N2 (k1 = 0)
        const int lane = threadIdx.x & 31;
        const int partner = (lane & 16) + (sub < N1 ? (N1 - sub) % N1 : sub);
        const int pr = slot / 3, kind = slot - (slot / 3) * 3;
        // FP32: no 1/NX2 here (not exact in FP32); the FP64 y analysis applies 1/(NX2 NZ2)
        const T invn = (T)(sizeof(C) == 8 ? 1.0 : 1.0 / (double)n);
    #pragma unroll
        for (int k2 = 0; k2 < N2; ++k2) {
            C pm;
            pm.x = __shfl_sync(0xffffffffu, v[N2 - 1 - k2].x, partner);
            pm.y = __shfl_sync(0xffffffffu, v[N2 - 1 - k2].y, partner);
            const int k = sub + N1 * k2;
            if (!act4 || k > nxs) continue;
            if (sub == 0) pm = v[(N2 - k2) % N2];
            const C p0 = v[k2];
            const C outA = cscale(invn, mkc<C>(T(0.5) * (p0.x + pm.x), T(0.5) * (p0.y - pm.y)));
            const C outB = cscale(invn, mkc<C>(T(0.5) * (p0.y + pm.y), T(-0.5) * (p0.x - pm.x)));
            if (kind < 2) {
                const int z = z0 + 2 * pr + kind;
                if (z < d.NZ2) {
                    C *h = H + ((long long)j * d.NZ2 + z) * nkx + k;
                    h[0] = outA;            // N0
                    h[fstride] = outB;      // N1
                }
            } else {
                const int z = z0 + 2 * pr;
                C *h = H + 2 * fstride + ((long long)j * d.NZ2 + z) * nkx + k;
                if (z < d.NZ2) h[0] = outA;                 // N2 of row r
                if (z + 1 < d.NZ2) h[nkx] = outB;           // N2 of row r+1
            }
        }
    }
}

// ---------------------------------------------------------------------------
// K3, half-warp form for NX2 = N1 x N2 (N1, N2 <= 16).  A half-warp (16
// lanes) owns a pair of rows (A, B) of the flattened row index R = j NZ2 + z
// from the spectral gather to the spectral store, so it synchronises with
// __syncwarp only (the twiddle table is the block's one barrier).  Per row:
//   three inverse lines (u + i v), (w + i om_x), (om_y + i om_z): lanes n2
//     gather Z[n2 + N2 n1] and do the N1-point DFT, twiddle, exchange through
//     the half-warp's scratch, lanes k1 do the N2-point DFT -> the line at
//     x = k1 + N1 k2 in lane k1's registers; the first two lines are kept
//     lane-private in shared memory (no exchange: lane k1 reads back what it
//     wrote) for
//   the products N = u x omega at the same x points, in registers; then
//   the forward line (N0 + i N1) of the row: lane a = k1 holds x = a + N1 b,
//     so the N2-point DFT over b runs on its registers, twiddle, exchange,
//     lanes q1 do the N1-point DFT -> P[q1 + N2 q2]; Hermitian unpack with
//     the partner lane (N2 - q1) by shuffle, modes q <= NXS -> HBM.
// N2 of row A waits lane-private in shared memory; with row B's it forms the
// third forward line N2(A) + i N2(B).  Rows past the end (an odd row count)
// are neither read nor written.
// ---------------------------------------------------------------------------
constexpr int kXHWarps = 2;   // warps per block of the half-warp form
__host__ __device__ constexpr int xh_scratch(int n1, int n2) {
    return n1 * (n2 + 1) > n2 * (n1 + 1) ? n1 * (n2 + 1) : n2 * (n1 + 1);
}
// bytes of one half-warp's shared memory: scratch, two stashed lines, N2 of row A
__host__ __device__ constexpr int xh_bytes(int n1, int n2, int elem) {
    return elem * (xh_scratch(n1, n2) + 2 * n1 * n2) + (elem / 2) * n1 * n2;
}

template <int N1, int N2, class C, bool MEAN>
__global__ void __launch_bounds__(32 * kXHWarps)
k_x_cross_h(Dims d, const double2 *__restrict__ roots, const C *__restrict__ G, C *__restrict__ H,
            const double *__restrict__ mean) {
    using T = typename CReal<C>::T;
    constexpr int n = N1 * N2;
    constexpr int NV = N1 > N2 ? N1 : N2;
    constexpr int SP1 = N2 + 1, SP2 = N1 + 1;   // padded scratch rows (inverse, forward)
    extern __shared__ double2 sm_d[];
    const Twiddles<C> tw = load_twiddles<C>(sm_d, roots, n);
    const int hw = threadIdx.x >> 4, sub = threadIdx.x & 15;
    char *mine = reinterpret_cast<char *>(sm_d + n) + hw * xh_bytes(N1, N2, (int)sizeof(C));
    C *S = reinterpret_cast<C *>(mine);                        // exchange scratch
    C *P = S + xh_scratch(N1, N2);                             // stashed lines [2][N2][N1]
    T *Q = reinterpret_cast<T *>(P + 2 * n);                   // N2 of row A [N2][N1]
    const long long rows = (long long)d.ny2 * d.NZ2;
    const long long rA = 2 * ((long long)blockIdx.x * (2 * kXHWarps) + hw);
    const int nkx = d.nkx, nxs = d.NXS;
    const long long fstride = rows * nkx;
    const int nyq = (n % 2 == 0) ? n / 2 : -1;
    const int lane = threadIdx.x & 31;
    const int partner = (lane & 16) + (sub < N2 ? (N2 - sub) % N2 : sub);
    // FP32: no 1/NX2 here (not exact in FP32); the FP64 y analysis applies 1/(NX2 NZ2)
    const T invn = (T)(sizeof(C) == 8 ? 1.0 : 1.0 / (double)n);
    __syncthreads();   // twiddles complete; no block-wide barrier below
    C v[NV];

    // forward FFT of the line in v (lane a < N1: v[b] = p[a + N1 b]), unpack
    // of the two real spectra, stores of modes q <= NXS: outA to dstA, outB to dstB
    auto forward_store = [&](C *dstA, C *dstB, bool okA, bool okB) {
        if (sub < N1) {
            C(&w)[N2] = reinterpret_cast<C(&)[N2]>(v);
            dft_reg<N2, -1>(w, tw, N1);
#pragma unroll
            for (int q1 = 0; q1 < N2; ++q1)
                S[q1 * SP2 + sub] = (q1 == 0 || sub == 0) ? w[q1] : tw.template mul<-1>(w[q1], sub * q1);
        }
        __syncwarp();
        if (sub < N2) {
#pragma unroll
            for (int a = 0; a < N1; ++a) v[a] = S[sub * SP2 + a];
            C(&w)[N1] = reinterpret_cast<C(&)[N1]>(v);
            dft_reg<N1, -1>(w, tw, N2);
        }
#pragma unroll
        for (int q2 = 0; q2 < N1; ++q2) {
            C pm;
            pm.x = __shfl_sync(0xffffffffu, v[N1 - 1 - q2].x, partner);
            pm.y = __shfl_sync(0xffffffffu, v[N1 - 1 - q2].y, partner);
            const int q = sub + N2 * q2;
            if (sub >= N2 || q > nxs) continue;
            if (sub == 0) pm = v[(N1 - q2) % N1];
            const C p0 = v[q2];
            if (okA) dstA[q] = cscale(invn, mkc<C>(T(0.5) * (p0.x + pm.x), T(0.5) * (p0.y - pm.y)));
            if (okB) dstB[q] = cscale(invn, mkc<C>(T(0.5) * (p0.y + pm.y), T(-0.5) * (p0.x - pm.x)));
        }
        __syncwarp();   // scratch free for the next exchange
    };

#pragma unroll 1
    for (int rr = 0; rr < 2; ++rr) {
        const long long row = rA + rr;
        const bool live = row < rows;
        // ---- three inverse lines ------------------------------------------
#pragma unroll 1
        for (int line = 0; line < 3; ++line) {
            if (sub < N2) {
                const C *rowA = G + (2 * line) * fstride + row * nkx;
                const C *rowB = rowA + fstride;
#pragma unroll
                for (int n1 = 0; n1 < N1; ++n1) {
                    const int m = sub + N2 * n1;
                    C x = mkc<C>(0.0, 0.0);
                    if (live) {
                        if (m <= nxs) {
                            C A = rowA[m], B = rowB[m];
                            if (m == 0 || m == nyq) {
                                A.y = 0.0;
                                B.y = 0.0;
                            }
                            x = mkc<C>(A.x - B.y, A.y + B.x);
                        } else if (m >= n - nxs && m != nyq) {
                            const C A = rowA[n - m], B = rowB[n - m];
                            x = mkc<C>(A.x + B.y, B.x - A.y);
                        }
                    }
                    v[n1] = x;
                }
                C(&w)[N1] = reinterpret_cast<C(&)[N1]>(v);
                dft_reg<N1, +1>(w, tw, N2);
#pragma unroll
                for (int k1 = 0; k1 < N1; ++k1)
                    S[k1 * SP1 + sub] = (k1 == 0 || sub == 0) ? w[k1] : tw.template mul<+1>(w[k1], sub * k1);
            }
            __syncwarp();
            if (sub < N1) {
#pragma unroll
                for (int n2 = 0; n2 < N2; ++n2) v[n2] = S[sub * SP1 + n2];
                C(&w)[N2] = reinterpret_cast<C(&)[N2]>(v);
                dft_reg<N2, +1>(w, tw, N1);
                if (line < 2) {
#pragma unroll
                    for (int k2 = 0; k2 < N2; ++k2) P[(line * N2 + k2) * N1 + sub] = w[k2];
                }
            }
            __syncwarp();
        }
        // ---- products u x omega at x = sub + N1 k2 -------------------------
        if (sub < N1) {
            T mu = 0, mv = 0, mw = 0, mox = 0, moy = 0, moz = 0;
            if constexpr (MEAN) {
                const int ny2 = d.ny2;
                const int j = live ? (int)(row / d.NZ2) : 0;
                mu = (T)mean[j];
                mv = (T)mean[ny2 + j];
                mw = (T)mean[2 * ny2 + j];
                mox = (T)mean[3 * ny2 + j];
                moy = (T)mean[4 * ny2 + j];
                moz = (T)mean[5 * ny2 + j];
            }
#pragma unroll
            for (int k2 = 0; k2 < N2; ++k2) {
                const C p0 = P[k2 * N1 + sub];
                const C p1 = P[(N2 + k2) * N1 + sub];
                const T uu = p0.x, vv = p0.y, ww = p1.x, ox = p1.y, oy = v[k2].x, oz = v[k2].y;
                T n0 = vv * oz - ww * oy;
                T n1v = ww * ox - uu * oz;
                T n2v = uu * oy - vv * ox;
                if constexpr (MEAN) {
                    // fluctuations about the FP64 mean profiles: + M x om' + u' x M_om
                    // (M x M_om is added to the mean mode in FP64 after the analysis)
                    n0 += (mv * oz - mw * oy) + (vv * moz - ww * moy);
                    n1v += (mw * ox - mu * oz) + (ww * mox - uu * moz);
                    n2v += (mu * oy - mv * ox) + (uu * moy - vv * mox);
                }
                v[k2] = mkc<C>(n0, n1v);
                if (rr == 0) {
                    Q[k2 * N1 + sub] = n2v;
                } else {
                    P[k2 * N1 + sub] = mkc<C>(Q[k2 * N1 + sub], n2v);   // third line N2(A) + i N2(B)
                }
            }
        }
        // ---- forward line (N0 + i N1) of this row -------------------------
        forward_store(H + row * nkx, H + fstride + row * nkx, live, live);
    }
    // ---- third forward line N2(A) + i N2(B) -------------------------------
    if (sub < N1) {
#pragma unroll
        for (int b = 0; b < N2; ++b) v[b] = P[b * N1 + sub];
    }
    forward_store(H + 2 * fstride + rA * nkx, H + 2 * fstride + (rA + 1) * nkx, rA < rows, rA + 1 < rows);
}

// ---------------------------------------------------------------------------
// Transpose of K3 in the register form (NX2 = N1 x N2, FP64): k_x_adjoint's
// algebra with the layout of k_x_cross_r.  16 lanes per line, RW rows per
// block; five inverse lines per row, (u, v), (w, om_x), (om_y, om_z),
// (lP_0, lP_1), (lP_2, 0), and three forward lines per row, (lu, lv),
// (lw, lom_x), (lom_y, lom_z).  Phase 1 reads lH (fields 0..2 of L) and
// phase 4 writes lG (fields 0..5 of L) for the block's own rows only.
// ---------------------------------------------------------------------------
template <int N1, int N2>
__global__ void __launch_bounds__(16 * 5 * 2)
k_x_adjoint_r(Dims d, const double2 *__restrict__ roots, const double2 *__restrict__ G, double2 *__restrict__ Lb,
              int RW) {
    using C = double2;
    constexpr int n = N1 * N2;
    constexpr int SP = N2 + 1;
    extern __shared__ double2 sm_d[];
    C *buf = sm_d + n;
    const int L = 5 * RW, L3 = 3 * RW;
    const int slot = threadIdx.x >> 4, sub = threadIdx.x & 15;
    const int j = blockIdx.y, z0 = blockIdx.x * RW;
    const int nkx = d.nkx, nxs = d.NXS;
    const long long fstride = (long long)d.ny2 * d.NZ2 * nkx;
    const C *Gj = G + (long long)j * d.NZ2 * nkx;
    C *Lj = Lb + (long long)j * d.NZ2 * nkx;
    const Twiddles<C> tw = load_twiddles<C>(sm_d, roots, n);
    const int nyq = (n % 2 == 0) ? n / 2 : -1;
    C v[N1 > N2 ? N1 : N2];

    // ---- phase 1: spectrum gather, N1-point DFTs (backward) ---------------
    const bool act1 = slot < L && sub < N2;
    if (act1) {
        const int r = slot / 5, q = slot - (slot / 5) * 5;
        const int z = z0 + r;
        const bool lam = q >= 3, hasB = q != 4;
        const C *rowA = q < 3 ? Gj + (long long)z * nkx + (2 * q) * fstride
                              : Lj + (long long)z * nkx + (q == 3 ? 0 : 2) * fstride;
        const C *rowB = rowA + fstride;
#pragma unroll
        for (int n1 = 0; n1 < N1; ++n1) {
            const int m = sub + N2 * n1;
            C x = mk(0.0, 0.0);
            if (z < d.NZ2) {
                const int mm = m <= nxs ? m : n - m;
                if (m <= nxs || (m >= n - nxs && m != nyq)) {
                    C A = rowA[mm], B = hasB ? rowB[mm] : mk(0.0, 0.0);
                    if (lam && mm > 0) {
                        A = cscale(0.5, A);
                        B = cscale(0.5, B);
                    }
                    if (mm == 0 || mm == nyq) {
                        A.y = 0.0;
                        B.y = 0.0;
                    }
                    x = m <= nxs ? mk(A.x - B.y, A.y + B.x) : mk(A.x + B.y, B.x - A.y);
                }
            }
            v[n1] = x;
        }
    }
    __syncthreads();   // twiddles complete
    if (act1) {
        C(&w)[N1] = reinterpret_cast<C(&)[N1]>(v);
        dft_reg<N1, +1>(w, tw, N2);
#pragma unroll
        for (int k1 = 0; k1 < N1; ++k1)
            buf[(slot * N1 + k1) * SP + sub] = (k1 == 0 || sub == 0) ? w[k1] : tw.template mul<+1>(w[k1], sub * k1);
    }
    __syncthreads();
    // ---- phase 2: N2-point DFTs -> physical rows --------------------------
    const bool act2 = slot < L && sub < N1;
    if (act2) {
#pragma unroll
        for (int n2 = 0; n2 < N2; ++n2) v[n2] = buf[(slot * N1 + sub) * SP + n2];
    }
    __syncthreads();
    if (act2) {
        C(&w)[N2] = reinterpret_cast<C(&)[N2]>(v);
        dft_reg<N2, +1>(w, tw, N1);
#pragma unroll
        for (int k2 = 0; k2 < N2; ++k2) buf[slot * n + sub + N1 * k2] = w[k2];
    }
    __syncthreads();
    // ---- phase 3: lu = om x lP, lom = lP x u; N1-point DFTs (forward) -----
    const bool act3 = slot < L3 && sub < N2;
    if (act3) {
        const int r = slot / 3, q = slot - (slot / 3) * 3;
        const C *P = buf + (5 * r) * n;
#pragma unroll
        for (int n1 = 0; n1 < N1; ++n1) {
            const int x = sub + N2 * n1;
            const C p0 = P[x], p1 = P[n + x], p2 = P[2 * n + x], p3 = P[3 * n + x], p4 = P[4 * n + x];
            const double uu = p0.x, vv = p0.y, ww = p1.x, ox = p1.y, oy = p2.x, oz = p2.y;
            const double l0 = p3.x, l1 = p3.y, l2 = p4.x;
            C t;
            if (q == 0) t = mk(oy * l2 - oz * l1, oz * l0 - ox * l2);
            else if (q == 1) t = mk(ox * l1 - oy * l0, l1 * ww - l2 * vv);
            else t = mk(l2 * uu - l0 * ww, l0 * vv - l1 * uu);
            v[n1] = t;
        }
    }
    __syncthreads();
    if (act3) {
        C(&w)[N1] = reinterpret_cast<C(&)[N1]>(v);
        dft_reg<N1, -1>(w, tw, N2);
#pragma unroll
        for (int k1 = 0; k1 < N1; ++k1)
            buf[(slot * N1 + k1) * SP + sub] = (k1 == 0 || sub == 0) ? w[k1] : tw.template mul<-1>(w[k1], sub * k1);
    }
    __syncthreads();
    // ---- phase 4: N2-point DFTs, unpack, modes k <= NXS (x 2 for k >= 1) --
    const bool act4 = slot < L3 && sub < N1;
    if (act4) {
#pragma unroll
        for (int n2 = 0; n2 < N2; ++n2) v[n2] = buf[(slot * N1 + sub) * SP + n2];
        C(&w)[N2] = reinterpret_cast<C(&)[N2]>(v);
        dft_reg<N2, -1>(w, tw, N1);
    }
    const int lane = threadIdx.x & 31;
    const int partner = (lane & 16) + (sub < N1 ? (N1 - sub) % N1 : sub);
    const int r = slot / 3, q = slot - (slot / 3) * 3;
    const int z = z0 + r;
#pragma unroll
    for (int k2 = 0; k2 < N2; ++k2) {
        C pm;
        pm.x = __shfl_sync(0xffffffffu, v[N2 - 1 - k2].x, partner);
        pm.y = __shfl_sync(0xffffffffu, v[N2 - 1 - k2].y, partner);
        const int k = sub + N1 * k2;
        if (!act4 || k > nxs || z >= d.NZ2) continue;
        if (sub == 0) pm = v[(N2 - k2) % N2];
        const C p0 = v[k2];
        C outA = mk(0.5 * (p0.x + pm.x), 0.5 * (p0.y - pm.y));
        C outB = mk(0.5 * (p0.y + pm.y), -0.5 * (p0.x - pm.x));
        if (k == 0) {
            outA.y = 0.0;
            outB.y = 0.0;
        } else {
            outA = cscale(2.0, outA);
            outB = cscale(2.0, outB);
        }
        C *h = Lj + (2 * q) * fstride + (long long)z * nkx + k;
        h[0] = outA;
        h[fstride] = outB;
    }
}

// ---------------------------------------------------------------------------
// Output reduction, x stage (coarse grid): c2r of the five z-physical fields
// u, v, w, p, div (nf = 5; nf = 4: no divergence, div taken as 0) of RW rows
// (z, j) per block, then per point the moment
// terms of Statistics::reduce (src/sim/statistics.cpp:58-86) and div^2 of
// Diagnostics::evaluate (src/sim/diagnostics.cpp:62-72), summed over the
// block's points into partial[j][blockIdx.x][kMomentSlots]:
//   0-3 u v w p, 4-6 uu vv ww, 7-9 uv vw wu, 10-12 pu pv pw, 13 pp,
//   14-16 u^3 v^3 w^3, 17-19 u^4 v^4 w^4, 20 div^2, 21 finite flag (1/0),
// with p = p_raw - (uu + vv + ww)/2.  If phys is set the block also writes
// u, v, w, p_raw to phys[4][NZ][NY+1][NX] (the snapshot of to_physical).
// Lines per row: (u, v), (w, p), (div, 0); a full-spectrum Nyquist bin is
// doubled (the coarse c2r convention).
// ---------------------------------------------------------------------------
constexpr int kMomentSlots = 22;

struct MomentAcc {
    double s[21];
    bool ok;
    __device__ __forceinline__ void init() {
#pragma unroll
        for (int k = 0; k < 21; ++k) s[k] = 0.0;
        ok = true;
    }
    __device__ __forceinline__ void add(double u, double v, double w, double praw, double dv) {
        const double uu = u * u, vv = v * v, ww = w * w;
        const double p = praw - 0.5 * (uu + vv + ww);
        ok = ok && isfinite(u) && isfinite(v) && isfinite(w) && isfinite(praw) && isfinite(p) && isfinite(dv);
        s[0] += u; s[1] += v; s[2] += w; s[3] += p;
        s[4] += uu; s[5] += vv; s[6] += ww;
        s[7] += u * v; s[8] += v * w; s[9] += w * u;
        s[10] += p * u; s[11] += p * v; s[12] += p * w; s[13] += p * p;
        s[14] += uu * u; s[15] += vv * v; s[16] += ww * w;
        s[17] += uu * uu; s[18] += vv * vv; s[19] += ww * ww;
        s[20] += dv * dv;
    }
    // block sum (fixed order) into out[0..21]; red holds 32 x kMomentSlots doubles
    __device__ void store(double *red, double *out) {
        const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
        double f = ok ? 1.0 : 0.0;
#pragma unroll
        for (int k = 0; k < 21; ++k)
            for (int m = 16; m > 0; m >>= 1) s[k] += __shfl_xor_sync(0xffffffffu, s[k], m);
        for (int m = 16; m > 0; m >>= 1) f = fmin(f, __shfl_xor_sync(0xffffffffu, f, m));
        if (lane == 0) {
#pragma unroll
            for (int k = 0; k < 21; ++k) red[wid * kMomentSlots + k] = s[k];
            red[wid * kMomentSlots + 21] = f;
        }
        __syncthreads();
        if (threadIdx.x < kMomentSlots) {
            const int k = threadIdx.x;
            double t = red[k];
            for (int q = 1; q < nw; ++q) t = (k == 21) ? fmin(t, red[q * kMomentSlots + k]) : t + red[q * kMomentSlots + k];
            out[k] = t;
        }
    }
};

template <int N1, int N2>
__global__ void __launch_bounds__(16 * 3 * 4)
k_x_moments_r(Dims d, const double2 *__restrict__ roots, const double2 *__restrict__ G, int RW,
              double *__restrict__ partial, double *__restrict__ phys, int nf) {
    using C = double2;
    constexpr int n = N1 * N2;
    constexpr int SP = N2 + 1;
    extern __shared__ double2 sm_d[];
    C *buf = sm_d + n;
    __shared__ double red[32 * kMomentSlots];
    const int L = 3 * RW;
    const int slot = threadIdx.x >> 4, sub = threadIdx.x & 15;
    const int j = blockIdx.y, z0 = blockIdx.x * RW;
    const int nkx = d.nkx, nxs = d.NXS;
    const long long fstride = (long long)d.ny2 * d.NZ2 * nkx;
    const C *Gj = G + (long long)j * d.NZ2 * nkx;
    const Twiddles<C> tw = load_twiddles<C>(sm_d, roots, n);
    const int nyq = (n % 2 == 0) ? n / 2 : -1;
    C v[N1 > N2 ? N1 : N2];
    const bool act1 = slot < L && sub < N2;
    if (act1) {
        const int r = slot / 3, q = slot - (slot / 3) * 3;
        const int z = z0 + r;
        const C *rowA = Gj + (long long)z * nkx + (2 * q) * fstride;
        const C *rowB = rowA + fstride;
#pragma unroll
        for (int n1 = 0; n1 < N1; ++n1) {
            const int m = sub + N2 * n1;
            C x = mk(0.0, 0.0);
            if (z < d.NZ2) {
                const int mm = m <= nxs ? m : n - m;
                if (m <= nxs || (m >= n - nxs && m != nyq)) {
                    C A = (2 * q < nf) ? rowA[mm] : mk(0.0, 0.0), B = q < 2 ? rowB[mm] : mk(0.0, 0.0);
                    if (mm == 0 || mm == nyq) {
                        A.y = 0.0;
                        B.y = 0.0;
                    }
                    if (mm == nyq) {
                        A.x *= 2.0;
                        B.x *= 2.0;
                    }
                    x = m <= nxs ? mk(A.x - B.y, A.y + B.x) : mk(A.x + B.y, B.x - A.y);
                }
            }
            v[n1] = x;
        }
    }
    __syncthreads();
    if (act1) {
        C(&w)[N1] = reinterpret_cast<C(&)[N1]>(v);
        dft_reg<N1, +1>(w, tw, N2);
#pragma unroll
        for (int k1 = 0; k1 < N1; ++k1)
            buf[(slot * N1 + k1) * SP + sub] = (k1 == 0 || sub == 0) ? w[k1] : tw.template mul<+1>(w[k1], sub * k1);
    }
    __syncthreads();
    const bool act2 = slot < L && sub < N1;
    if (act2) {
#pragma unroll
        for (int n2 = 0; n2 < N2; ++n2) v[n2] = buf[(slot * N1 + sub) * SP + n2];
    }
    __syncthreads();
    if (act2) {
        C(&w)[N2] = reinterpret_cast<C(&)[N2]>(v);
        dft_reg<N2, +1>(w, tw, N1);
#pragma unroll
        for (int k2 = 0; k2 < N2; ++k2) buf[slot * n + sub + N1 * k2] = w[k2];
    }
    __syncthreads();
    MomentAcc acc;
    acc.init();
    const int ny1 = d.ny2;
    for (int i = threadIdx.x; i < RW * n; i += blockDim.x) {
        const int r = i / n, x = i - (i / n) * n;
        const int z = z0 + r;
        if (z >= d.NZ2) continue;
        const C a = buf[(3 * r) * n + x], b = buf[(3 * r + 1) * n + x], c = buf[(3 * r + 2) * n + x];
        acc.add(a.x, a.y, b.x, b.y, c.x);
        if (phys) {
            const long long o = ((long long)z * ny1 + j) * n + x, fs = (long long)d.NZ2 * ny1 * n;
            phys[o] = a.x;
            phys[fs + o] = a.y;
            phys[2 * fs + o] = b.x;
            phys[3 * fs + o] = b.y;
        }
    }
    acc.store(red, partial + ((long long)j * gridDim.x + blockIdx.x) * kMomentSlots);
}

// Stockham form of k_x_moments_r for any NX.
__global__ void __launch_bounds__(256)
k_x_moments(Dims d, FftPlan P, const double2 *__restrict__ roots, const double2 *__restrict__ G, int RW,
            double *__restrict__ partial, double *__restrict__ phys, int nf) {
    extern __shared__ double2 sm[];
    __shared__ double red[32 * kMomentSlots];
    const int n = d.NX2;
    double2 *s_root = sm;
    const int L = 3 * RW;
    double2 *a = sm + n;
    double2 *b = a + n * L;
    const int j = blockIdx.y, z0 = blockIdx.x * RW;
    for (int i = threadIdx.x; i < n; i += blockDim.x) s_root[i] = roots[i];
    const long long fstride = (long long)d.ny2 * d.NZ2 * d.nkx;
    const double2 *Gj = G + (long long)j * d.NZ2 * d.nkx;
    const int nyq = (n % 2 == 0) ? n / 2 : -1;
    for (int i = threadIdx.x; i < n * L; i += blockDim.x) {
        const int k = i / L, line = i - (i / L) * L;
        const int r = line / 3, q = line - (line / 3) * 3;
        const int z = z0 + r;
        double2 A = mk(0, 0), B = mk(0, 0);
        int m;
        bool mirror;
        if (k <= d.NXS) { m = k; mirror = false; }
        else if (k >= n - d.NXS && k != nyq) { m = n - k; mirror = true; }
        else { m = -1; mirror = false; }
        if (m >= 0 && z < d.NZ2) {
            const double2 *row = Gj + (long long)z * d.nkx + m + (2 * q) * fstride;
            if (2 * q < nf) A = row[0];
            if (q < 2) B = row[fstride];
            if (m == 0 || m == nyq) { A.y = 0.0; B.y = 0.0; }
            if (m == nyq) { A.x *= 2.0; B.x *= 2.0; }
        }
        a[i] = mirror ? mk(A.x + B.y, B.x - A.y) : mk(A.x - B.y, A.y + B.x);
    }
    __syncthreads();
    const double2 *res = fft_lines<+1>(a, b, L, P, s_root);
    MomentAcc acc;
    acc.init();
    const int ny1 = d.ny2;
    for (int i = threadIdx.x; i < RW * n; i += blockDim.x) {
        const int r = i / n, x = i - (i / n) * n;
        const int z = z0 + r;
        if (z >= d.NZ2) continue;
        const double2 p0 = res[x * L + 3 * r], p1 = res[x * L + 3 * r + 1], p2 = res[x * L + 3 * r + 2];
        acc.add(p0.x, p0.y, p1.x, p1.y, p2.x);
        if (phys) {
            const long long o = ((long long)z * ny1 + j) * n + x, fs = (long long)d.NZ2 * ny1 * n;
            phys[o] = p0.x;
            phys[fs + o] = p0.y;
            phys[2 * fs + o] = p1.x;
            phys[3 * fs + o] = p1.y;
        }
    }
    acc.store(red, partial + ((long long)j * gridDim.x + blockIdx.x) * kMomentSlots);
}

// ---------------------------------------------------------------------------
// Single-field x transforms for the standalone fine transform (tests and
// to-physical output): c2r / r2c of one real field [z][j][x].
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(128)
k_x_c2r(Dims d, FftPlan P, const double2 *__restrict__ roots, const double2 *__restrict__ G,
        double *__restrict__ phys, int RW, double nyq_scale) {
    extern __shared__ double2 sm[];
    const int n = d.NX2;
    double2 *s_root = sm;
    const int L = (RW + 1) / 2;  // two real rows per complex line
    double2 *a = sm + n;
    double2 *b = a + n * L;
    const int j = blockIdx.y, z0 = blockIdx.x * RW;
    for (int i = threadIdx.x; i < n; i += blockDim.x) s_root[i] = roots[i];
    const int nyq = (n % 2 == 0) ? n / 2 : -1;
    for (int i = threadIdx.x; i < n * L; i += blockDim.x) {
        const int k = i / L, line = i - (i / L) * L;
        double2 A = mk(0, 0), B = mk(0, 0);
        int m;
        bool mirror;
        if (k <= d.NXS) { m = k; mirror = false; }
        else if (k >= n - d.NXS && k != nyq) { m = n - k; mirror = true; }
        else { m = -1; mirror = false; }
        if (m >= 0) {
            const int za = z0 + 2 * line, zb = za + 1;
            if (za < d.NZ2 && za < z0 + RW) A = G[((long long)j * d.NZ2 + za) * d.nkx + m];
            if (zb < d.NZ2 && zb < z0 + RW) B = G[((long long)j * d.NZ2 + zb) * d.nkx + m];
            if (m == 0 || m == nyq) { A.y = 0.0; B.y = 0.0; }
            if (m == nyq) { A.x *= nyq_scale; B.x *= nyq_scale; }
        }
        a[i] = mirror ? mk(A.x + B.y, B.x - A.y) : mk(A.x - B.y, A.y + B.x);
    }
    __syncthreads();
    const double2 *res = fft_lines<+1>(a, b, L, P, s_root);
    for (int i = threadIdx.x; i < n * RW; i += blockDim.x) {
        const int x = i / RW, r = i - (i / RW) * RW;
        const int z = z0 + r;
        if (z >= d.NZ2) continue;
        const double2 v = res[x * L + (r >> 1)];
        phys[((long long)z * d.ny2 + j) * n + x] = (r & 1) ? v.y : v.x;
    }
}

__global__ void __launch_bounds__(128)
k_x_r2c(Dims d, FftPlan P, const double2 *__restrict__ roots, const double *__restrict__ phys,
        double2 *__restrict__ H, int RW, double nyq_scale) {
    extern __shared__ double2 sm[];
    const int n = d.NX2;
    double2 *s_root = sm;
    const int L = (RW + 1) / 2;
    double2 *a = sm + n;
    double2 *b = a + n * L;
    const int j = blockIdx.y, z0 = blockIdx.x * RW;
    for (int i = threadIdx.x; i < n; i += blockDim.x) s_root[i] = roots[i];
    for (int i = threadIdx.x; i < n * L; i += blockDim.x) {
        const int x = i / L, line = i - (i / L) * L;
        const int za = z0 + 2 * line, zb = za + 1;
        double va = 0, vb = 0;
        if (za < d.NZ2 && za < z0 + RW) va = phys[((long long)za * d.ny2 + j) * n + x];
        if (zb < d.NZ2 && zb < z0 + RW) vb = phys[((long long)zb * d.ny2 + j) * n + x];
        a[i] = mk(va, vb);
    }
    __syncthreads();
    const double2 *res = fft_lines<-1>(a, b, L, P, s_root);
    const double invn = 1.0 / (double)n;
    for (int i = threadIdx.x; i < d.nkx * RW; i += blockDim.x) {
        const int k = i / RW, r = i - (i / RW) * RW;
        const int z = z0 + r;
        if (z >= d.NZ2) continue;
        const int km = (n - k) % n;
        const double2 P0 = res[k * L + (r >> 1)];
        const double2 Pm = res[km * L + (r >> 1)];
        const double2 out = (r & 1) ? mk(0.5 * (P0.y + Pm.y), -0.5 * (P0.x - Pm.x))
                                    : mk(0.5 * (P0.x + Pm.x), 0.5 * (P0.y - Pm.y));
        H[((long long)j * d.NZ2 + z) * d.nkx + k] = cscale(2 * k == n ? invn * nyq_scale : invn, out);
    }
}

// ---------------------------------------------------------------------------
// Transpose of K3 (discrete adjoint) about the fields G of the forward step:
// with P = u x omega = c2r(G) products and H = r2c(P) / NX2 (modes k <= NXS),
//   lP    = c2r(Y),  Y_0 = lH_0, Y_k = lH_k / 2       (the 1/NX2 is applied
//                                                      by the caller's tables)
//   lu    = omega x lP,  lomega = lP x u
//   lG_0  = sum_x l(x) (real),  lG_k = 2 sum_x l(x) e^{-2 pi i k x / NX2}.
// L holds lH in fields 0..2 on entry and lG in fields 0..5 on return; a block
// reads and writes only its own rows, so the update is in place.  Block = RW
// rows (z, j); inverse lines per row: (u, v), (w, om_x), (om_y, om_z),
// (lP_0, lP_1), (lP_2, 0); forward lines: (lu, lv), (lw, lom_x), (lom_y, lom_z).
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256, 2)
k_x_adjoint(Dims d, FftPlan P, const double2 *__restrict__ roots, const double2 *__restrict__ G,
            double2 *__restrict__ Lb, int RW) {
    extern __shared__ double2 sm[];
    const int n = d.NX2;
    double2 *s_root = sm;
    const int L5 = 5 * RW, L3 = 3 * RW;
    double2 *a = sm + n;
    double2 *b = a + n * L5;
    const int j = blockIdx.y, z0 = blockIdx.x * RW;
    for (int i = threadIdx.x; i < n; i += blockDim.x) s_root[i] = roots[i];
    const long long fstride = (long long)d.ny2 * d.NZ2 * d.nkx;
    const double2 *Gj = G + (long long)j * d.NZ2 * d.nkx;
    double2 *Lj = Lb + (long long)j * d.NZ2 * d.nkx;
    const int nyq = (n % 2 == 0) ? n / 2 : -1;
    const int nkx = d.nkx;
    const int zlo = d.NXS + 1, zhi = n - d.NXS;   // slots [zlo, zhi) are zero
    for (int i = threadIdx.x; i < (zhi - zlo) * L5; i += blockDim.x) {
        const int k = zlo + i / L5, line = i - (i / L5) * L5;
        a[k * L5 + line] = mk(0, 0);
    }
    for (int i = threadIdx.x; i < L5 * nkx; i += blockDim.x) {
        const int line = i / nkx, m = i - (i / nkx) * nkx;
        const int r = line / 5, q = line - (line / 5) * 5;
        const int z = z0 + r;
        double2 A = mk(0, 0), B = mk(0, 0);
        if (z < d.NZ2) {
            const long long o = (long long)z * nkx + m;
            if (q < 3) {
                A = Gj[(2 * q) * fstride + o];
                B = Gj[(2 * q + 1) * fstride + o];
            } else {
                const double h = m == 0 ? 1.0 : 0.5;
                A = cscale(h, Lj[(q == 3 ? 0 : 2) * fstride + o]);
                if (q == 3) B = cscale(h, Lj[fstride + o]);
            }
        }
        if (m == 0 || m == nyq) {
            A.y = 0.0;
            B.y = 0.0;
        }
        a[m * L5 + line] = mk(A.x - B.y, A.y + B.x);
        if (m != 0 && m != nyq) a[(n - m) * L5 + line] = mk(A.x + B.y, B.x - A.y);
    }
    __syncthreads();
    double2 *res = fft_lines<+1>(a, b, L5, P, s_root);
    double2 *oth = (res == a) ? b : a;
    for (int i = threadIdx.x; i < n * RW; i += blockDim.x) {
        const int x = i / RW, r = i - (i / RW) * RW;
        const double2 p0 = res[x * L5 + 5 * r], p1 = res[x * L5 + 5 * r + 1], p2 = res[x * L5 + 5 * r + 2];
        const double2 p3 = res[x * L5 + 5 * r + 3], p4 = res[x * L5 + 5 * r + 4];
        const double uu = p0.x, vv = p0.y, ww = p1.x, ox = p1.y, oy = p2.x, oz = p2.y;
        const double l0 = p3.x, l1 = p3.y, l2 = p4.x;
        oth[x * L3 + 3 * r] = mk(oy * l2 - oz * l1, oz * l0 - ox * l2);        // omega x lP
        oth[x * L3 + 3 * r + 1] = mk(ox * l1 - oy * l0, l1 * ww - l2 * vv);    // ..., (lP x u)_x
        oth[x * L3 + 3 * r + 2] = mk(l2 * uu - l0 * ww, l0 * vv - l1 * uu);    // (lP x u)_y, _z
    }
    __syncthreads();
    double2 *res2 = fft_lines<-1>(oth, res, L3, P, s_root);
    for (int i = threadIdx.x; i < RW * 6 * nkx; i += blockDim.x) {
        const int rf = i / nkx, k = i - (i / nkx) * nkx;
        const int r = rf / 6, f = rf - (rf / 6) * 6;
        const int z = z0 + r;
        if (z >= d.NZ2) continue;
        const int km = (n - k) % n;
        const int line = 3 * r + (f >> 1);
        const double2 P0 = res2[k * L3 + line];
        const double2 Pm = res2[km * L3 + line];
        // unpack A = (P + conj Pm)/2, B = (P - conj Pm)/(2i); the c2r transpose doubles k >= 1
        double2 out = (f & 1) ? mk(0.5 * (P0.y + Pm.y), -0.5 * (P0.x - Pm.x))
                              : mk(0.5 * (P0.x + Pm.x), 0.5 * (P0.y - Pm.y));
        out = (k == 0) ? mk(out.x, 0.0) : cscale(2.0, out);
        Lj[f * fstride + (long long)z * nkx + k] = out;
    }
}

// ---------------------------------------------------------------------------
// Host launchers
// ---------------------------------------------------------------------------
namespace {
constexpr int kRW = 4;
constexpr int kRWs = 8;
}  // namespace

// Lines per z-FFT block: the width in [8, 17] that tiles NXS+1 with the least
// padding (13 for 65 modes).
constexpr int kMaxZLines = 17;   // z-transform (and y FFT form) kx lines per block: 8..17
int z_lines(const Dims &d) {
    if (d.ztl >= 8 && d.ztl <= kMaxZLines) return d.ztl;
    int best = 16, waste = 1 << 30;
    for (int tl = 17; tl >= 8; --tl) {
        const int w = ((d.nkx + tl - 1) / tl) * tl - d.nkx;
        if (w < waste) { waste = w; best = tl; }
    }
    return best;
}

template <typename Fn> bool with_xsplit(int nx2, Fn &&fn);
// kx lines per block of the DCT kernels: of {8, 11, 13, 16}, the width that
// keeps the most threads per SM on real lines -- blocks per SM by shared
// memory (228 KB, 1 KB reserved per block) x 16 TL threads x nkx / (nkx
// padded to TL) -- the wider one on a tie; CDNS_YDCT_LINES fixes it.
int ydct_lines(const Dims &d) {
    const char *e = std::getenv("CDNS_YDCT_LINES");
    const int forced = e ? std::atoi(e) : 0;
    if (forced == 8 || forced == 11 || forced == 13 || forced == 16) return forced;
    int n1 = 1, n2 = d.NY2;
    with_xsplit(d.NY2, [&](auto a, auto b) {
        n1 = decltype(a)::value;
        n2 = decltype(b)::value;
    });
    int best = 16;
    double best_useful = -1.0;
    for (int tl : {16, 13, 11, 8}) {
        const size_t bytes = sizeof(double2) * ydct_slots(n1, n2, tl) + 1024;
        const int blocks = (int)std::min<size_t>((228u * 1024u) / bytes, 2048 / (16 * tl));
        const int padded = ((d.nkx + tl - 1) / tl) * tl;
        const double useful = (double)blocks * 16 * tl * d.nkx / padded;
        if (useful > best_useful) {
            best_useful = useful;
            best = tl;
        }
    }
    return best;
}
template <typename Fn> void with_ydct_lines(int tl, Fn &&fn) {
    switch (tl) {
    case 8: fn(std::integral_constant<int, 8>{}); break;
    case 11: fn(std::integral_constant<int, 11>{}); break;
    case 13: fn(std::integral_constant<int, 13>{}); break;
    default: fn(std::integral_constant<int, 16>{}); break;
    }
}
size_t smem_ydct(int n1, int n2, int tl) { return sizeof(double2) * ydct_slots(n1, n2, tl); }
// Dims with the widest line tile, for raising the kernels' shared-memory limits
Dims widest_lines(Dims d) {
    d.ztl = kMaxZLines;
    return d;
}

size_t smem_zfft(const Dims &d) { return sizeof(double2) * (size_t)d.NZ2 * (1 + 2 * z_lines(d)); }
size_t smem_xcross(const Dims &d) { return sizeof(double2) * (size_t)d.NX2 * (1 + 2 * 3 * kRW); }
constexpr int kRWa = 2;
size_t smem_xadjoint(const Dims &d) { return sizeof(double2) * (size_t)d.NX2 * (1 + 2 * 5 * kRWa); }
size_t smem_xsingle(const Dims &d) {
    return sizeof(double2) * (size_t)d.NX2 * (1 + 2 * ((kRWs + 1) / 2));
}

// NX2 / NZ2 = N1 x N2 with a register form; others use the Stockham form
// (FP64 only).
template <typename Fn> bool with_xsplit(int nx2, Fn &&fn) {
    switch (nx2) {
    case 32: fn(std::integral_constant<int, 4>{}, std::integral_constant<int, 8>{}); return true;
    case 48: fn(std::integral_constant<int, 6>{}, std::integral_constant<int, 8>{}); return true;
    case 64: fn(std::integral_constant<int, 8>{}, std::integral_constant<int, 8>{}); return true;
    case 72: fn(std::integral_constant<int, 8>{}, std::integral_constant<int, 9>{}); return true;
    case 96: fn(std::integral_constant<int, 8>{}, std::integral_constant<int, 12>{}); return true;
    case 144: fn(std::integral_constant<int, 12>{}, std::integral_constant<int, 12>{}); return true;
    case 192: fn(std::integral_constant<int, 12>{}, std::integral_constant<int, 16>{}); return true;
    case 128: fn(std::integral_constant<int, 8>{}, std::integral_constant<int, 16>{}); return true;
    case 196: fn(std::integral_constant<int, 14>{}, std::integral_constant<int, 14>{}); return true;
    default: return false;
    }
}

constexpr int kRWm = 4;    // rows per block of the output-reduction x stage
size_t smem_xmoments_r(int n1, int n2) {
    const size_t L = 3 * kRWm;
    const size_t s1 = L * n1 * (n2 + 1), s2 = L * n1 * n2;
    return sizeof(double2) * (n1 * n2 + (s1 > s2 ? s1 : s2));
}
size_t smem_xmoments(const Dims &d) { return sizeof(double2) * (size_t)d.NX2 * (1 + 2 * 3 * kRWm); }
size_t smem_zfft_r(const Dims &d, int n1, int n2, size_t elem) {
    // twiddles, then the exchange of fft2_lines: n1 rows of the padded k1 stride
    return sizeof(double2) * n1 * n2 + elem * ((size_t)n1 * fft2_kstride(n2, z_lines(d)));
}
constexpr int kRWar = 2;   // rows per block of the register-form x adjoint (16 * 5 * kRWar threads)
size_t smem_xadjoint_r(int n1, int n2) {
    const size_t L = 5 * kRWar;
    const size_t s1 = L * n1 * (n2 + 1), s2 = L * n1 * n2;
    return sizeof(double2) * (n1 * n2 + (s1 > s2 ? s1 : s2));
}
size_t smem_xcross_h(int n1, int n2, size_t elem) {
    return sizeof(double2) * n1 * n2 + (size_t)(2 * kXHWarps) * xh_bytes(n1, n2, (int)elem);
}
size_t smem_xcross_r(int n1, int n2, size_t elem, int rw = kRWr) {
    return sizeof(double2) * (n1 * n2 + 16 * n1) + elem * xcross_buf_elems(n1, n2, rw) + (elem / 2) * rw * n1 * n2;
}

template <class C> cudaError_t configure_register_forms(const Dims &d) {
    cudaError_t e = cudaSuccess;
    with_xsplit(d.NX2, [&](auto a, auto b) {
        constexpr int N1 = decltype(a)::value, N2 = decltype(b)::value;
        e = raise_smem(k_x_cross_r<N1, N2, C, sizeof(C) == 8>, smem_xcross_r(N1, N2, sizeof(C)));
        if constexpr (N1 % 2 == 0 && N2 % 2 == 0)
            if (e == cudaSuccess)
                e = raise_smem(k_x_cross_r<N1, N2, C, sizeof(C) == 8, true>, smem_xcross_r(N1, N2, sizeof(C)));
        if (e == cudaSuccess)
            e = raise_smem(k_x_cross_h<N1, N2, C, sizeof(C) == 8>, smem_xcross_h(N1, N2, sizeof(C)));
        if (e == cudaSuccess && sizeof(C) == 16) e = raise_smem(k_x_adjoint_r<N1, N2>, smem_xadjoint_r(N1, N2));
        if (e == cudaSuccess && sizeof(C) == 16) e = raise_smem(k_x_moments_r<N1, N2>, smem_xmoments_r(N1, N2));
    });
    if (e != cudaSuccess) return e;
    with_xsplit(d.NZ2, [&](auto a, auto b) {
        constexpr int N1 = decltype(a)::value, N2 = decltype(b)::value;
        const int sm = (int)smem_zfft_r(widest_lines(d), N1, N2, sizeof(C));
        e = raise_smem(k_z_backward_r<N1, N2, C>, sm);
        if (e == cudaSuccess)
            e = raise_smem(k_z_forward_r<N1, N2, C>, sm);
        if (e == cudaSuccess && sizeof(C) == 16) e = raise_smem(k_z_backward_peers<N1, N2>, sm);
        if (e == cudaSuccess && sizeof(C) == 16) e = raise_smem(k_z_forward_peers<N1, N2>, sm);
    });
    return e;
}

cudaError_t configure_ydct(const Dims &d) {
    cudaError_t e = cudaSuccess;
    with_xsplit(d.NY2, [&](auto a, auto b) {
        constexpr int N1 = decltype(a)::value, N2 = decltype(b)::value;
        with_ydct_lines(ydct_lines(d), [&](auto w) {
            constexpr int TL = decltype(w)::value;
            const int sm = (int)smem_ydct(N1, N2, TL);
            e = raise_smem(k_ydct_r<N1, N2, true, TL, double2>, sm);
            if (e == cudaSuccess) e = raise_smem(k_ydct_r<N1, N2, false, TL, double2>, sm);
            if (e == cudaSuccess) e = raise_smem(k_ydct_r<N1, N2, true, TL, float2>, sm);
            if (e == cudaSuccess) e = raise_smem(k_ydct_r<N1, N2, false, TL, float2>, sm);
        });
    });
    return e;
}

bool register_forms(const Dims &d) {
    return with_xsplit(d.NX2, [](auto, auto) {}) && with_xsplit(d.NZ2, [](auto, auto) {});
}

cudaError_t configure_transform_kernels(const Dims &d) {
    cudaError_t e = configure_register_forms<double2>(d);
    if (e != cudaSuccess) return e;
    e = configure_ydct(d);
    if (e != cudaSuccess) return e;
    e = configure_register_forms<float2>(d);
    if (e != cudaSuccess) return e;
    e = raise_smem(k_z_backward, (int)smem_zfft(widest_lines(d)));
    if (e != cudaSuccess) return e;
    e = raise_smem(k_z_forward, (int)smem_zfft(widest_lines(d)));
    if (e != cudaSuccess) return e;
    e = raise_smem(k_x_cross, (int)smem_xcross(d));
    if (e != cudaSuccess) return e;
    e = raise_smem(k_x_adjoint, (int)smem_xadjoint(d));
    if (e != cudaSuccess) return e;
    e = raise_smem(k_x_moments, (int)smem_xmoments(d));
    if (e != cudaSuccess) return e;
    e = raise_smem(k_x_c2r, (int)smem_xsingle(d));
    if (e != cudaSuccess) return e;
    e = raise_smem(k_x_r2c, (int)smem_xsingle(d));
    return e;
}

template <class C>
bool z_backward_r(const Dims &d, const double2 *roots, const C *F, C *G, int nf, cudaStream_t s,
                  bool coarse = false) {
    const int tl = z_lines(d);
    dim3 grid((d.nkx + tl - 1) / tl, d.ny2, nf);
    return with_xsplit(d.NZ2, [&](auto a, auto b) {
        constexpr int N1 = decltype(a)::value, N2 = decltype(b)::value;
        k_z_backward_r<N1, N2, C><<<grid, (N1 > N2 ? N1 : N2) * tl, smem_zfft_r(d, N1, N2, sizeof(C)), s>>>(
            d, roots, F, G, tl, coarse);
    });
}
template <class C, bool MEAN>
bool x_cross_r(const Dims &d, const double2 *roots, const C *G, C *H, const double *mean, cudaStream_t s) {
    if (d.xrw == 1) {   // half-warp form: 4 kXHWarps rows per block
        const long long rows = (long long)d.ny2 * d.NZ2;
        const int per = 4 * kXHWarps;
        return with_xsplit(d.NX2, [&](auto a, auto b) {
            constexpr int N1 = decltype(a)::value, N2 = decltype(b)::value;
            k_x_cross_h<N1, N2, C, MEAN><<<(unsigned)((rows + per - 1) / per), 32 * kXHWarps,
                                           smem_xcross_h(N1, N2, sizeof(C)), s>>>(d, roots, G, H, mean);
        });
    }
    const int rw = (d.xrw == 2 || d.xrw == 4) ? d.xrw : kRWr;   // even, at most kRWr
    return with_xsplit(d.NX2, [&](auto a, auto b) {
        constexpr int N1 = decltype(a)::value, N2 = decltype(b)::value;
        dim3 grid((d.NZ2 + rw - 1) / rw, d.ny2);
        if constexpr (N1 % 2 == 0 && N2 % 2 == 0) {
            if (d.xrw == 3 || d.xrw == 5) {   // 4 or 2 rows, forward phases split over lane pairs
                const int srw = d.xrw == 3 ? 4 : 2;
                dim3 sgrid((d.NZ2 + srw - 1) / srw, d.ny2);
                k_x_cross_r<N1, N2, C, MEAN, true><<<sgrid, 16 * 3 * srw, smem_xcross_r(N1, N2, sizeof(C), srw), s>>>(
                    d, roots, G, H, srw, mean);
                return;
            }
        }
        k_x_cross_r<N1, N2, C, MEAN><<<grid, 16 * 3 * rw, smem_xcross_r(N1, N2, sizeof(C)), s>>>(
            d, roots, G, H, rw, mean);
    });
}
template <class C>
bool z_forward_r(const Dims &d, const double2 *roots, const C *H, C *F, int nf, cudaStream_t s,
                 bool coarse = false) {
    const int tl = z_lines(d);
    dim3 grid((d.nkx + tl - 1) / tl, d.ny2, nf);
    return with_xsplit(d.NZ2, [&](auto a, auto b) {
        constexpr int N1 = decltype(a)::value, N2 = decltype(b)::value;
        k_z_forward_r<N1, N2, C><<<grid, (N1 > N2 ? N1 : N2) * tl, smem_zfft_r(d, N1, N2, sizeof(C)), s>>>(
            d, roots, H, F, tl, coarse);
    });
}

bool launch_z_backward_peers(const Dims &d, const double2 *roots, const PeerCols &pc, double2 *G,
                             cudaStream_t s) {
    const int tl = z_lines(d);
    dim3 grid((d.nkx + tl - 1) / tl, d.ny2, 6);
    return with_xsplit(d.NZ2, [&](auto a, auto b) {
        constexpr int N1 = decltype(a)::value, N2 = decltype(b)::value;
        k_z_backward_peers<N1, N2><<<grid, (N1 > N2 ? N1 : N2) * tl, smem_zfft_r(d, N1, N2, sizeof(double2)), s>>>(
            d, roots, pc, G, tl);
    });
}

bool launch_z_forward_peers(const Dims &d, const double2 *roots, const double2 *H, const PeerCols &pc,
                            cudaStream_t s) {
    const int tl = z_lines(d);
    dim3 grid((d.nkx + tl - 1) / tl, d.ny2, 3);
    return with_xsplit(d.NZ2, [&](auto a, auto b) {
        constexpr int N1 = decltype(a)::value, N2 = decltype(b)::value;
        k_z_forward_peers<N1, N2><<<grid, (N1 > N2 ? N1 : N2) * tl, smem_zfft_r(d, N1, N2, sizeof(double2)), s>>>(
            d, roots, H, pc, tl);
    });
}

void launch_z_backward(const Dims &d, const FftPlan &P, const double2 *roots, const double2 *F,
                       double2 *G, int nf, cudaStream_t s, bool coarse) {
    if (z_backward_r(d, roots, F, G, nf, s, coarse)) return;
    const int tl = z_lines(d);
    dim3 grid((d.nkx + tl - 1) / tl, d.ny2, nf);
    k_z_backward<<<grid, 256, smem_zfft(d), s>>>(d, P, roots, F, G, tl, coarse);
}

void launch_x_cross(const Dims &d, const FftPlan &P, const double2 *roots, const double2 *G,
                    double2 *H, cudaStream_t s) {
    if (x_cross_r<double2, false>(d, roots, G, H, nullptr, s)) return;
    dim3 grid((d.NZ2 + kRW - 1) / kRW, d.ny2);
    k_x_cross<<<grid, 256, smem_xcross(d), s>>>(d, P, roots, G, H, kRW);
}

void launch_z_forward(const Dims &d, const FftPlan &P, const double2 *roots, const double2 *H,
                      double2 *F, int nf, cudaStream_t s, bool coarse) {
    if (z_forward_r(d, roots, H, F, nf, s, coarse)) return;
    const int tl = z_lines(d);
    dim3 grid((d.nkx + tl - 1) / tl, d.ny2, nf);
    k_z_forward<<<grid, 256, smem_zfft(d), s>>>(d, P, roots, H, F, tl, coarse);
}

// FP32 stage buffers (mixed precision): register forms only.
void launch_z_backward(const Dims &d, const double2 *roots, const float2 *F, float2 *G, int nf, cudaStream_t s) {
    z_backward_r(d, roots, F, G, nf, s);
}
void launch_x_cross(const Dims &d, const double2 *roots, const float2 *G, float2 *H, const double *mean,
                    cudaStream_t s) {
    x_cross_r<float2, true>(d, roots, G, H, mean, s);
}
void launch_z_forward(const Dims &d, const double2 *roots, const float2 *H, float2 *F, int nf, cudaStream_t s) {
    z_forward_r(d, roots, H, F, nf, s);
}

void launch_x_adjoint(const Dims &d, const FftPlan &P, const double2 *roots, const double2 *G, double2 *L,
                      cudaStream_t s) {
    const bool reg = with_xsplit(d.NX2, [&](auto a, auto b) {
        constexpr int N1 = decltype(a)::value, N2 = decltype(b)::value;
        dim3 grid((d.NZ2 + kRWar - 1) / kRWar, d.ny2);
        k_x_adjoint_r<N1, N2><<<grid, 16 * 5 * kRWar, smem_xadjoint_r(N1, N2), s>>>(d, roots, G, L, kRWar);
    });
    if (reg) return;
    dim3 grid((d.NZ2 + kRWa - 1) / kRWa, d.ny2);
    k_x_adjoint<<<grid, 256, smem_xadjoint(d), s>>>(d, P, roots, G, L, kRWa);
}

bool ydct_available(const Dims &d, const Tables &t) {
    return t.root_y && d.NY2 % 2 == 0 && with_xsplit(d.NY2, [](auto, auto) {});
}

template <class CT>
bool ydct(const Dims &d, const Tables &t, int nf, bool ana, const YdctArgs<CT> &A, cudaStream_t s) {
    if (!ydct_available(d, t)) return false;
    const int tl = ydct_lines(d);
    dim3 grid((d.nkx + tl - 1) / tl, d.nkz, nf);
    return with_xsplit(d.NY2, [&](auto a, auto b) {
        constexpr int N1 = decltype(a)::value, N2 = decltype(b)::value;
        with_ydct_lines(tl, [&](auto w) {
            constexpr int TL = decltype(w)::value;
            const size_t sm = smem_ydct(N1, N2, TL);
            if (ana)
                k_ydct_r<N1, N2, true, TL, CT><<<grid, 16 * TL, sm, s>>>(d, t.root_y, t.cosy, A);
            else
                k_ydct_r<N1, N2, false, TL, CT><<<grid, 16 * TL, sm, s>>>(d, t.root_y, t.cosy, A);
        });
    });
}
bool launch_ydct(const Dims &d, const Tables &t, const double2 *src0, const double2 *src1, int nsplit, int nf,
                 double2 *out, bool ana, cudaStream_t s) {
    YdctArgs<double2> A;
    if (ana) {
        A.Fin = src0;
        A.S = out;
        A.s0 = 1.0 / (double)d.NY2;
        A.sk = 2.0 / (double)d.NY2;
    } else {
        A.spec0 = src0;
        A.spec1 = src1;
        A.nsplit = nsplit;
        A.Fout = out;
    }
    return ydct(d, t, nf, ana, A, s);
}
bool launch_ydct_adjoint_analysis(const Dims &d, const Tables &t, const double2 *lS, int nf, double2 *F,
                                  cudaStream_t s) {
    // F_j = v_j xs sum_k s_k lS_k cos(pi j k / N): s_0 = 1/(2N), s_k = 1/N;
    // v_0 = v_N = 1, v_j = 2; xs = 1/(NX2 NZ2), the transposed x and z scalings
    const double N = (double)d.NY2, xs = 1.0 / ((double)d.NX2 * (double)d.NZ2);
    YdctArgs<double2> A;
    A.spec0 = lS;
    A.nsplit = nf;
    A.Fout = F;
    A.in0 = 1.0 / (2.0 * N);
    A.in1 = 1.0 / N;
    A.outE = xs;
    A.outI = 2.0 * xs;
    return ydct(d, t, nf, false, A, s);
}
bool launch_ydct_adjoint_synthesis(const Dims &d, const Tables &t, const double2 *F, int nf, double2 *S,
                                   double scale, cudaStream_t s) {
    // S_k = scale sum_{j=0..N} F_j cos(pi j k / N): the DCT-I with its end rows doubled
    YdctArgs<double2> A;
    A.Fin = F;
    A.S = S;
    A.inE = 2.0;
    A.s0 = scale;
    A.sk = scale;
    return ydct(d, t, nf, true, A, s);
}
bool launch_ydct_synthesis_fp32(const Dims &d, const Tables &t, const double2 *src0, const double2 *src1,
                                int nsplit, int nf, float2 *F, double *mean, cudaStream_t s) {
    YdctArgs<float2> A;
    A.spec0 = src0;
    A.spec1 = src1;
    A.nsplit = nsplit;
    A.Fout = F;
    A.mean = mean;
    return ydct(d, t, nf, false, A, s);
}
bool launch_ydct_analysis_fp32(const Dims &d, const Tables &t, const float2 *F, double2 *S, int nf,
                               cudaStream_t s) {
    YdctArgs<float2> A;
    A.Fin = F;
    A.S = S;
    const double sxz = 1.0 / ((double)d.NX2 * (double)d.NZ2);
    A.s0 = sxz / (double)d.NY2;
    A.sk = 2.0 * sxz / (double)d.NY2;
    return ydct(d, t, nf, true, A, s);
}

int moment_blocks(const Dims &d) { return (d.NZ2 + kRWm - 1) / kRWm; }

void launch_x_moments(const Dims &d, const FftPlan &P, const double2 *roots, const double2 *G, double *partial,
                      double *phys, int nf, cudaStream_t s) {
    dim3 grid(moment_blocks(d), d.ny2);
    const bool reg = with_xsplit(d.NX2, [&](auto a, auto b) {
        constexpr int N1 = decltype(a)::value, N2 = decltype(b)::value;
        k_x_moments_r<N1, N2><<<grid, 16 * 3 * kRWm, smem_xmoments_r(N1, N2), s>>>(d, roots, G, kRWm, partial, phys,
                                                                                 nf);
    });
    if (reg) return;
    k_x_moments<<<grid, 256, smem_xmoments(d), s>>>(d, P, roots, G, kRWm, partial, phys, nf);
}

// The coarse grid doubles (c2r) / halves (r2c) a full-spectrum x Nyquist bin
// (src/fft/transforms.cpp:486-487, 574-576); the fine grid does not.
void launch_x_c2r(const Dims &d, const FftPlan &P, const double2 *roots, const double2 *G,
                  double *phys, cudaStream_t s, bool coarse) {
    dim3 grid((d.NZ2 + kRWs - 1) / kRWs, d.ny2);
    k_x_c2r<<<grid, 128, smem_xsingle(d), s>>>(d, P, roots, G, phys, kRWs, coarse ? 2.0 : 1.0);
}

void launch_x_r2c(const Dims &d, const FftPlan &P, const double2 *roots, const double *phys,
                  double2 *H, cudaStream_t s, bool coarse) {
    dim3 grid((d.NZ2 + kRWs - 1) / kRWs, d.ny2);
    k_x_r2c<<<grid, 128, smem_xsingle(d), s>>>(d, P, roots, phys, H, kRWs, coarse ? 0.5 : 1.0);
}

}  // namespace cdns
