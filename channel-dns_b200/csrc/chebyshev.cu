// Chebyshev-direction kernels of the channel-dns nonlinear term for sm_100a:
// the spectral curl, the synthesis of Gauss-Lobatto values and the analysis
// back to Chebyshev coefficients (src/fft/transforms.cpp:615-741,
// src/solver/vector_ops.cpp:17-25, 112-151).
//
// Synthesis and analysis are FP64 matrix products against precomputed cosine
// matrices, folded by the parity of the Chebyshev index:
//   synthesis  E_j = sum_{k even} C_kj c_k,  O_j = sum_{k odd} C_kj c_k,
//              f_j = E_j + O_j,  f_{N-j} = E_j - O_j   (j <= N/2),
//              C_kj = w_k cos(pi j k / N), w_k = 1/2 at k = N, else 1
//              (the c_0 doubling of the DCT-I and the 0.5 z-expansion factor
//              of the reference cancel; both are powers of two);
//   analysis   S_k = s_k sum_{j <= N/2} A_jk (k even ? X_j + X_{N-j} : X_j - X_{N-j}),
//              A_jk = v_j cos(pi j k / N), v_0 = 1, else 2 (the middle point
//              j = N/2 enters once), s_0 = 1/(2N), s_k = 1/N.
// A block owns 32 consecutive spectral columns of one field; its warps run
// 8x8x4 FP64 MMA tiles (rows x real columns) of one parity each, with the
// column data and cosine rows streamed through shared memory by cp.async.
#include <algorithm>

#include "cdns_kernels.cuh"
#include "warp_columns.cuh"

namespace cdns {

namespace {
constexpr int kSynRows = 16;   // synthesis rows (j) per warp
constexpr int kAnaRows = 16;   // analysis rows (k of one parity) per warp
constexpr int kMaxGroups = 8;  // row groups per block (two warps each); more go to grid.z

int syn_groups(const Dims &d) { return (d.nyh + kSynRows - 1) / kSynRows; }
int ana_groups(const Dims &d) { return ((d.ncy + 1) / 2 + kAnaRows - 1) / kAnaRows; }

// ---------------------------------------------------------------------------
// Cosine matrices, built on the device from the cos(pi m / N) table:
//   csyn[k][j]        k < NYS+1, j < syn_groups * kSynRows (zero padded)
//   cana[j][p][m]     j <= N/2, k = 2m + p, m < ana_groups * kAnaRows
// ---------------------------------------------------------------------------
__global__ void k_cheb_tables(Dims d, const double *__restrict__ cosy, double *csyn, int jp,
                              double *cana, int kh) {
    const int N = d.NY2, twoN = 2 * N;
    const long long nsyn = (long long)d.ncy * jp;
    const long long nana = cana ? (long long)d.nyh * 2 * kh : 0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nsyn + nana;
         i += (long long)gridDim.x * blockDim.x) {
        if (i < nsyn) {
            const int k = (int)(i / jp), j = (int)(i - (i / jp) * jp);
            csyn[i] = (j < d.nyh) ? cosy[((long long)j * k) % twoN] * (k == N ? 0.5 : 1.0) : 0.0;
        } else {
            const long long q = i - nsyn;
            const int j = (int)(q / (2 * kh));
            const int r = (int)(q - (long long)j * 2 * kh);
            const int p = r / kh, m = r - (r / kh) * kh;
            const int k = 2 * m + p;
            cana[q] = (k < d.ncy) ? cosy[((long long)j * k) % twoN] * (j == 0 ? 1.0 : 2.0) : 0.0;
        }
    }
}

// Tables of the transposed Chebyshev stages (discrete adjoint), in the
// layouts of csyn and cana so that the synthesis kernel applies the
// transposed analysis and the analysis kernel the transposed synthesis:
//   csyn_t[k][j]    = s_k v_j cos(pi j k / N) * xs    (v_j, s_k of the analysis;
//                     xs = 1/(NX2 NZ2), the transposed x and z scalings)
//   cana_t[j][p][m] = cos(pi j k / N), k = 2m + p     (synthesis weights w_k = 1)
__global__ void k_cheb_tables_adjoint(Dims d, const double *__restrict__ cosy, double *csyn_t, int jp,
                                      double *cana_t, int kh, double xs) {
    const int N = d.NY2, twoN = 2 * N;
    const long long nsyn = (long long)d.ncy * jp;
    const long long nana = (long long)d.nyh * 2 * kh;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nsyn + nana;
         i += (long long)gridDim.x * blockDim.x) {
        if (i < nsyn) {
            const int k = (int)(i / jp), j = (int)(i - (i / jp) * jp);
            const double sk = k == 0 ? 1.0 / (2.0 * N) : 1.0 / (double)N;
            const double vj = j == 0 ? 1.0 : 2.0;
            csyn_t[i] = (j < d.nyh) ? cosy[((long long)j * k) % twoN] * (sk * vj * xs) : 0.0;
        } else {
            const long long q = i - nsyn;
            const int j = (int)(q / (2 * kh));
            const int r = (int)(q - (long long)j * 2 * kh);
            const int p = r / kh, m = r - (r / kh) * kh;
            const int k = 2 * m + p;
            cana_t[q] = (k < d.ncy) ? cosy[((long long)j * k) % twoN] : 0.0;
        }
    }
}

// ---------------------------------------------------------------------------
// Spectral curl, warp per column (src/solver/vector_ops.cpp:112-151):
//   om_x = dw/dy - i kz v,  om_y = i kz u - i kx w,  om_z = i kx v - du/dy,
// and the vorticity part of the pressure wall condition
// (src/solver/timestepper.cpp:26-43): bw = sum_k (i kx/Re om_z - i kz/Re om_x)
// with signs (+1, (-1)^(k+1)) for the (y = +1, y = -1) walls.
// ---------------------------------------------------------------------------
template <int E>
__global__ void __launch_bounds__(32 * kColsPerBlock)
k_curl(Dims d, Tables t, const double2 *__restrict__ u, double2 *__restrict__ om,
       double2 *__restrict__ bw, double re) {
    extern __shared__ double2 tile[];   // [3][ncy][kColsPerBlock]
    const int ncy = d.ncy, ny = d.NYS, nkx = d.nkx, ncol = d.ncol;
    const int S = ncy * kColsPerBlock;
    const int col0 = blockIdx.x * kColsPerBlock;
    const int tid = threadIdx.x, w = tid >> 5, L = tid & 31, p = L & 1;
    // the loads of kBatch rows of the tile are issued before the first store
    constexpr int kBatch = 4;
    for (int i0 = tid; i0 < S; i0 += kBatch * blockDim.x) {
        double2 v[kBatch][3];
#pragma unroll
        for (int b = 0; b < kBatch; ++b) {
            const int i = i0 + b * blockDim.x;
            const int y = i / kColsPerBlock, l = i - (i / kColsPerBlock) * kColsPerBlock;
            const int c2 = col0 + l;
            const bool ok = i < S && c2 < ncol;
            const int kzi = c2 / nkx, kx = c2 - (c2 / nkx) * nkx;
            const long long off = ((long long)kzi * ncy + y) * nkx + kx;
#pragma unroll
            for (int c = 0; c < 3; ++c) v[b][c] = ok ? u[c * d.Ns + off] : mk(0.0, 0.0);
        }
#pragma unroll
        for (int b = 0; b < kBatch; ++b) {
            const int i = i0 + b * blockDim.x;
            const int y = i / kColsPerBlock, l = i - (i / kColsPerBlock) * kColsPerBlock;
            if (i >= S || col0 + l >= ncol) continue;
            const int sl = tile_slot<E>(y, l);
#pragma unroll
            for (int c = 0; c < 3; ++c) tile[c * S + sl] = v[b][c];
        }
    }
    __syncthreads();
    const int col = col0 + w;
    if (col < ncol) {
        const int kzi = col / nkx, kx = col - kzi * nkx;
        const double ax = t.wavx[kx], az = t.wavz[kzi];
        double2 uu[E], vv[E], ww[E], du[E], dw[E];
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const int y = ycoef<E>(e);
            if (y <= ny) {
                const int sl = tile_slot<E>(y, w);
                uu[e] = tile[sl];
                vv[e] = tile[S + sl];
                ww[e] = tile[2 * S + sl];
            } else {
                uu[e] = vv[e] = ww[e] = mk(0.0, 0.0);
            }
        }
        deriv_warp<E>(ny, uu, du);
        deriv_warp<E>(ny, ww, dw);
        const double axr = ax / re, azr = az / re;
        double2 btop = mk(0, 0), bbot = mk(0, 0);
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const int y = ycoef<E>(e);
            if (y > ny) continue;
            const double2 ox = csub(dw[e], fderiv(az, vv[e]));
            const double2 oy = csub(fderiv(az, uu[e]), fderiv(ax, ww[e]));
            const double2 oz = csub(fderiv(ax, vv[e]), du[e]);
            const double2 wall = csub(fderiv(axr, oz), fderiv(azr, ox));
            btop = cadd(btop, wall);
            bbot = p ? cadd(bbot, wall) : csub(bbot, wall);
            const int sl = tile_slot<E>(y, w);
            tile[sl] = ox;
            tile[S + sl] = oy;
            tile[2 * S + sl] = oz;
        }
        btop = sum_warp(btop);
        bbot = sum_warp(bbot);
        if (L == 0 && bw) {
            bw[col] = btop;
            bw[ncol + col] = bbot;
        }
    }
    __syncthreads();
    for (int i = tid; i < S; i += blockDim.x) {
        const int y = i / kColsPerBlock, l = i - (i / kColsPerBlock) * kColsPerBlock;
        const int c2 = col0 + l;
        if (c2 >= ncol) continue;
        const int kzi = c2 / nkx, kx = c2 - (c2 / nkx) * nkx;
        const long long off = ((long long)kzi * ncy + y) * nkx + kx;
        const int sl = tile_slot<E>(y, l);
#pragma unroll
        for (int c = 0; c < 3; ++c) om[c * d.Ns + off] = tile[c * S + sl];
    }
}

// D (8x8) += A (8x4) B (4x8) on the FP64 tensor pipe.  Lane l = 4 g + t holds
// A[g][t], B[t][g] and D[g][2t], D[g][2t+1].
__device__ __forceinline__ void dmma(double &d0, double &d1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};\n"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}

// Staged rows are padded so that the four k (or j) rows of one fragment load
// fall on distinct bank quarters: complex rows of 32 columns take kXS = 34
// slots; double rows are padded to a stride = 4 (mod 16) / 2 (mod 8).
constexpr int kXS = 34;
__host__ __device__ inline int syn_cs(int jp) { return jp + ((4 - jp % 16) + 16) % 16; }
__host__ __device__ inline int ana_as(int kh) { return kh + ((2 - kh % 8) + 8) % 8; }

// ---------------------------------------------------------------------------
// Synthesis: F[f][j][col] for j = 0..NY2 from spectral fields
// (fields f < nsplit from src0, the rest from src1).  Grid (column tiles of
// 32, fields); block (32, 2 G): warp (g, p) accumulates, with 8x8x4 FP64 MMA,
// the parity-p sum of rows j = 16 g .. 16 g + 15 for the 32 columns (a 16 x 64
// real tile).  Coefficients and cosine rows stream through shared memory in
// chunks of KC rows of k (descending), split by parity, double-buffered with
// cp.async; odd-parity warps hand their sums to the even ones at the end.
// ---------------------------------------------------------------------------
constexpr int kSynKC = 16;
constexpr int kSynStages = 4;
constexpr int kSynTiles = 4;   // 16-row tiles per block (two warps each); more go to grid.z

template <class CO>
__global__ void __launch_bounds__(32 * 2 * kSynTiles, 2)
k_ysynth(Dims d, const double *__restrict__ csyn, int jp, const double2 *__restrict__ src0,
         const double2 *__restrict__ src1, int nsplit, CO *__restrict__ F, double *__restrict__ mean) {
    extern __shared__ double2 sm[];
    constexpr int KC = kSynKC, KH = KC / 2;
    constexpr int jw = kSynTiles * 16;   // cosine columns staged per block
    const int CS = syn_cs(jw);
    constexpr int NS = kSynStages;
    double2 *xs = sm;                                                // [NS][2 par][KH][kXS]
    double *cs = reinterpret_cast<double *>(sm + NS * 2 * KH * kXS); // [NS][2 par][KH][CS]
    const int lane = threadIdx.x, wy = threadIdx.y;
    const int tid = wy * 32 + lane, nthr = 32 * blockDim.y;
    const int jt = blockIdx.z * kSynTiles + (wy >> 1), par = wy & 1;
    const int jb = blockIdx.z * kSynTiles * 16;   // first row of this block
    const int g = lane >> 2, t = lane & 3;
    const int f = blockIdx.y, col0 = blockIdx.x * 32;
    const int ncol = d.ncol, ny = d.NYS, N = d.NY2;
    const double2 *X = f < nsplit ? src0 + (long long)f * d.Ns : src1 + (long long)(f - nsplit) * d.Ns;
    const int nchunk = (d.ncy + KC - 1) / KC;
    const int nxu = KC * 32, ncu = KC * (jw / 2);
    auto fetch = [&](int chunk, int buf) {
        const int khi = ny - chunk * KC;
        for (int u = tid; u < nxu + ncu; u += nthr) {
            if (u < nxu) {
                const int r = u >> 5, l = u & 31;
                const int k = khi - r, col = col0 + l;
                const bool ok = k >= 0 && col < ncol;
                const int kzi = ok ? col / d.nkx : 0, kx = ok ? col - kzi * d.nkx : 0;
                cp_async16(xs + ((buf * 2 + (k & 1)) * KH + (r >> 1)) * kXS + l,
                           X + ((long long)kzi * d.ncy + (ok ? k : 0)) * d.nkx + kx, ok ? 16 : 0);
            } else {
                const int c = u - nxu;
                const int r = c / (jw / 2), h = c - r * (jw / 2);
                const int k = khi - r;
                const bool ok = k >= 0 && jb + 2 * h < jp;
                cp_async16(cs + ((buf * 2 + (k & 1)) * KH + (r >> 1)) * CS + 2 * h,
                           csyn + (long long)(ok ? k : 0) * jp + (ok ? jb + 2 * h : 0), ok ? 16 : 0);
            }
        }
        cp_async_commit();
    };
    double acc[2][8][2];
#pragma unroll
    for (int mr = 0; mr < 2; ++mr)
#pragma unroll
        for (int q = 0; q < 8; ++q) acc[mr][q][0] = acc[mr][q][1] = 0.0;
    const int j0 = jt * 16;
    const bool jok = j0 < jp;   // warps past the last row tile only stage data
#pragma unroll
    for (int c = 0; c < NS - 1; ++c) {
        if (c < nchunk) fetch(c, c);
        else cp_async_commit();
    }
    for (int chunk = 0; chunk < nchunk; ++chunk) {
        const int buf = chunk % NS;
        cp_async_wait<NS - 2>();   // this chunk has landed
        __syncthreads();           // ... for every thread; the buffer refilled next was consumed last iteration
        if (chunk + NS - 1 < nchunk) fetch(chunk + NS - 1, (chunk + NS - 1) % NS);
        else cp_async_commit();
        const double *cb = cs + (buf * 2 + par) * KH * CS;
        const double2 *xb = xs + (buf * 2 + par) * KH * kXS;
#pragma unroll
        for (int st = 0; st < (jok ? KH / 4 : 0); ++st) {
            const int r = 4 * st + t;
            const double a0 = cb[r * CS + j0 - jb + g], a1 = cb[r * CS + j0 - jb + 8 + g];
            const double *xr = reinterpret_cast<const double *>(xb + r * kXS) + (g & 1);
#pragma unroll
            for (int q = 0; q < 8; ++q) {
                const double bq = xr[2 * (4 * q + (g >> 1))];
                dmma(acc[0][q][0], acc[0][q][1], a0, bq);
                dmma(acc[1][q][0], acc[1][q][1], a1, bq);
            }
        }
    }
    cp_async_wait<0>();
    __syncthreads();
    // combine: odd-parity warps hand their sums to the even-parity warps
    constexpr int kEXS = 36;
    double2 *ex = sm;   // [16 * kSynTiles][kEXS], rows relative to this block's first tile
    if (jok && par == 1) {
#pragma unroll
        for (int mr = 0; mr < 2; ++mr)
#pragma unroll
            for (int q = 0; q < 8; ++q) ex[(j0 - jb + 8 * mr + g) * kEXS + 4 * q + t] = mk(acc[mr][q][0], acc[mr][q][1]);
    }
    __syncthreads();
    if (jok && par == 0) {
        CO *Ff = F + (long long)f * d.ny2 * d.fcol + col0;
        const int zc = d.zc;   // the (kz, kx) = (0, 0) column
#pragma unroll
        for (int mr = 0; mr < 2; ++mr) {
            const int j = j0 + 8 * mr + g;
            if (j >= d.nyh) continue;
#pragma unroll
            for (int q = 0; q < 8; ++q) {
                const int c = 4 * q + t;
                if (col0 + c >= ncol) continue;
                const double2 o = ex[(j0 - jb + 8 * mr + g) * kEXS + c];
                const double2 e = mk(acc[mr][q][0], acc[mr][q][1]);
                if (mean && col0 + c == zc) {
                    // mean profile (kz, kx) = (0, 0): kept in FP64, out of the FP32 stages
                    // (its imaginary part is round-off of a real profile)
                    mean[f * d.ny2 + j] = e.x + o.x;
                    mean[f * d.ny2 + N - j] = e.x - o.x;
                    Ff[(long long)j * d.fcol + c] = mkc<CO>(0.0, 0.0);
                    if (N - j != j) Ff[(long long)(N - j) * d.fcol + c] = mkc<CO>(0.0, 0.0);
                    continue;
                }
                Ff[(long long)j * d.fcol + c] = cto<CO>(cadd(e, o));
                if (N - j != j) Ff[(long long)(N - j) * d.fcol + c] = cto<CO>(csub(e, o));
            }
        }
    }
}

// ---------------------------------------------------------------------------
// Analysis: S[f][k][col] (spectral, planar) from F[f][j][col].  Grid (column
// tiles of 32, fields); block (32, 2 G): warp (g, p) owns k = 2 m + p for
// m = 16 g .. 16 g + 15, accumulated with 8x8x4 FP64 MMA over chunks of JC
// points j; rows j and N - j are staged by cp.async and folded into
// X_j +- X_{N-j} as the B fragments are read.
// ---------------------------------------------------------------------------
constexpr int kAnaJC = 16;
constexpr int kAnaStages = 3;
// double2 slots taken by the staged rows of the analysis (j and N - j, all stages)
__host__ __device__ constexpr int ana_x_slots(int xs, int elem) {
    return (kAnaStages * 2 * kAnaJC * xs * elem + 15) / 16;
}

template <class CI>
__global__ void __launch_bounds__(32 * 2 * kMaxGroups)
k_yanalysis(Dims d, const double *__restrict__ cana, int kh, const CI *__restrict__ F,
            double2 *__restrict__ S, double s0, double sn) {
    // staged complex row of 32 columns: 34 slots for FP64, 36 for FP32 (16-byte units)
    constexpr bool F32 = sizeof(CI) == 8;
    constexpr int XS = F32 ? 36 : kXS;
    extern __shared__ double2 sm[];
    constexpr int JC = kAnaJC;
    const int AS = ana_as(kh);
    constexpr int NS = kAnaStages;
    CI *xab = reinterpret_cast<CI *>(sm);                                       // [NS][2 side][JC][XS]
    double *as = reinterpret_cast<double *>(sm + ana_x_slots(XS, sizeof(CI)));  // [NS][JC][2 par][AS]
    // folded rows e = X_j + X_{N-j}, o = X_j - X_{N-j} in FP64 [2][JC][kXS]: in place
    // over the stage buffer for FP64 input, a buffer of their own for FP32 input
    double2 *eo_f32 = reinterpret_cast<double2 *>(as + NS * JC * 2 * AS);
    const int lane = threadIdx.x, wy = threadIdx.y;
    const int tid = wy * 32 + lane, nthr = 32 * blockDim.y;
    const int kt = blockIdx.z * kMaxGroups + (wy >> 1), par = wy & 1;
    const int g = lane >> 2, t = lane & 3;
    const int f = blockIdx.y, col0 = blockIdx.x * 32;
    const int ncol = d.ncol, N = d.NY2;
    const CI *X = F + (long long)f * d.ny2 * d.fcol;
    const int nchunk = (d.nyh + JC - 1) / JC;
    // X units of 16 bytes (one double2 or two float2 columns), both sides; cosine double2 units
    constexpr int CPU_ = 16 / sizeof(CI), UPR = 32 / CPU_;
    const int nxu = 2 * JC * UPR, nau = JC * kh;
    auto fetch = [&](int chunk, int buf) {
        for (int u = tid; u < nxu + nau; u += nthr) {
            if (u < nxu) {
                const int side = u >= JC * UPR, v = u - side * JC * UPR;
                const int r = v / UPR, l = (v - r * UPR) * CPU_;
                const int j = chunk * JC + r, col = col0 + l;
                const int jj = side ? N - j : j;
                const bool ok = j < d.nyh && col < ncol && !(side && jj == j);
                const int bytes = ok ? (int)sizeof(CI) * min(CPU_, ncol - col) : 0;
                cp_async16(xab + ((buf * 2 + side) * JC + r) * XS + l,
                           X + (long long)(ok ? jj : 0) * d.fcol + (ok ? col : 0), bytes);
            } else {
                const int c = u - nxu;
                const int r = c / kh, rem = c - r * kh;
                const int p = rem / (kh / 2), h = rem - p * (kh / 2);
                const int j = chunk * JC + r;
                cp_async16(as + ((buf * JC + r) * 2 + p) * AS + 2 * h,
                           cana + (long long)(j < d.nyh ? j : 0) * 2 * kh + p * kh + 2 * h, j < d.nyh ? 16 : 0);
            }
        }
        cp_async_commit();
    };
    double acc[2][8][2];
#pragma unroll
    for (int mr = 0; mr < 2; ++mr)
#pragma unroll
        for (int q = 0; q < 8; ++q) acc[mr][q][0] = acc[mr][q][1] = 0.0;
    const int m0 = kt * 16;
    const bool kok = m0 < kh;   // warps past the last row tile only stage data
#pragma unroll
    for (int c = 0; c < NS - 1; ++c) {
        if (c < nchunk) fetch(c, c);
        else cp_async_commit();
    }
    for (int chunk = 0; chunk < nchunk; ++chunk) {
        const int buf = chunk % NS;
        cp_async_wait<NS - 2>();
        __syncthreads();
        if (chunk + NS - 1 < nchunk) fetch(chunk + NS - 1, (chunk + NS - 1) % NS);
        else cp_async_commit();
        // fold (and widen) this chunk once: eo[0] = e, eo[1] = o
        double2 *eo = F32 ? eo_f32 : reinterpret_cast<double2 *>(xab + buf * 2 * JC * XS);
        for (int i = tid; i < JC * 32; i += nthr) {
            const int r = i >> 5, l = i & 31;
            const double2 a = cto<double2>(xab[(buf * 2 * JC + r) * XS + l]);
            const double2 b = cto<double2>(xab[((buf * 2 + 1) * JC + r) * XS + l]);
            eo[r * kXS + l] = cadd(a, b);
            eo[(JC + r) * kXS + l] = csub(a, b);
        }
        __syncthreads();
#pragma unroll
        for (int st = 0; st < (kok ? JC / 4 : 0); ++st) {
            const int r = 4 * st + t;
            const double *ar = as + ((buf * JC + r) * 2 + par) * AS + m0 + g;
            const double a0 = ar[0], a1 = ar[8];
            const double *xr = reinterpret_cast<const double *>(eo + (par * JC + r) * kXS) + (g & 1);
#pragma unroll
            for (int q = 0; q < 8; ++q) {
                const double bq = xr[2 * (4 * q + (g >> 1))];
                dmma(acc[0][q][0], acc[0][q][1], a0, bq);
                dmma(acc[1][q][0], acc[1][q][1], a1, bq);
            }
        }
    }
    cp_async_wait<0>();
    double2 *Sf = S + (long long)f * d.Ns;
#pragma unroll
    for (int mr = 0; mr < 2; ++mr) {
        const int k = 2 * (m0 + 8 * mr + g) + par;
        if (!kok || k >= d.ncy) continue;
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            const int col = col0 + 4 * q + t;
            if (col >= ncol) continue;
            const int kzi = col / d.nkx, kx = col - kzi * d.nkx;
            Sf[((long long)kzi * d.ncy + k) * d.nkx + kx] = cscale(k == 0 ? s0 : sn, mk(acc[mr][q][0], acc[mr][q][1]));
        }
    }
}

// Mean x mean part of u x omega for the mixed path: P(j) = M_u(j) x M_om(j)
// of the FP64 mean profiles, analysed like k_yanalysis and added to the
// (kz, kx) = (0, 0) column of N.  Each block forms the products in shared
// memory; one warp per (component, coefficient) sums them.
__global__ void k_mean_products(Dims d, const double *__restrict__ cana, int kh, const double *__restrict__ mean,
                                double2 *__restrict__ S) {
    extern __shared__ double sp[];   // [3][NY2+1]
    const int N = d.NY2, ny2 = d.ny2;
    for (int j = threadIdx.x; j < ny2; j += blockDim.x) {
        const double mu = mean[j], mv = mean[ny2 + j], mw = mean[2 * ny2 + j];
        const double ox = mean[3 * ny2 + j], oy = mean[4 * ny2 + j], oz = mean[5 * ny2 + j];
        sp[j] = mv * oz - mw * oy;
        sp[ny2 + j] = mw * ox - mu * oz;
        sp[2 * ny2 + j] = mu * oy - mv * ox;
    }
    __syncthreads();
    // one warp per (component, coefficient): lanes stride over j, shuffle sum
    const int lane = threadIdx.x & 31;
    const int i = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (i >= 3 * d.ncy) return;
    const int c = i / d.ncy, k = i - (i / d.ncy) * d.ncy;
    const int p = k & 1, m = k >> 1;
    const double *P = sp + c * ny2;
    double acc = 0.0;
    for (int j = lane; j < d.nyh; j += 32) {
        const double x = (N - j == j) ? P[j] : (p ? P[j] - P[N - j] : P[j] + P[N - j]);
        acc += cana[(long long)j * 2 * kh + p * kh + m] * x;
    }
    acc = sum_warp(acc);
    if (lane == 0) {
        const double sc = k == 0 ? 1.0 / (2.0 * N) : 1.0 / (double)N;
        double2 *s = S + (long long)c * d.Ns + ((long long)d.NZS * d.ncy + k) * d.nkx;   // kx = 0
        s->x += sc * acc;
    }
}

size_t curl_smem(const Dims &d) { return sizeof(double2) * 3 * (size_t)d.ncy * kColsPerBlock; }
size_t syn_smem(const Dims &) {
    const size_t pipe = sizeof(double2) * kSynStages * 2 * (kSynKC / 2) * kXS +
                        sizeof(double) * kSynStages * 2 * (kSynKC / 2) * syn_cs(kSynTiles * 16);
    const size_t ex = sizeof(double2) * (size_t)kSynTiles * 16 * 36;
    return pipe > ex ? pipe : ex;
}
size_t ana_smem(const Dims &d, size_t elem) {
    const int kh = ana_groups(d) * kAnaRows;
    const int xs = elem == 16 ? kXS : 36;
    const size_t eo = elem == 16 ? 0 : sizeof(double2) * 2 * kAnaJC * kXS;
    return sizeof(double2) * ana_x_slots(xs, (int)elem) + sizeof(double) * kAnaStages * kAnaJC * 2 * ana_as(kh) + eo;
}
}  // namespace

void cheb_table_sizes(const Dims &d, size_t *nsyn, size_t *nana) {
    *nsyn = (size_t)d.ncy * syn_groups(d) * kSynRows;
    *nana = (size_t)d.nyh * 2 * ana_groups(d) * kAnaRows;
}

void launch_cheb_tables(const Dims &d, const double *cosy, double *csyn, double *cana, cudaStream_t s) {
    size_t ns, na;
    cheb_table_sizes(d, &ns, &na);
    if (!cana) na = 0;
    const long long n = (long long)(ns + na);
    const int blocks = (int)std::min<long long>((n + 255) / 256, 4096);
    k_cheb_tables<<<blocks, 256, 0, s>>>(d, cosy, csyn, syn_groups(d) * kSynRows, cana,
                                         ana_groups(d) * kAnaRows);
}

void launch_cheb_tables_adjoint(const Dims &d, const double *cosy, double *csyn_t, double *cana_t,
                                cudaStream_t s) {
    size_t ns, na;
    cheb_table_sizes(d, &ns, &na);
    const long long n = (long long)(ns + na);
    const int blocks = (int)std::min<long long>((n + 255) / 256, 4096);
    k_cheb_tables_adjoint<<<blocks, 256, 0, s>>>(d, cosy, csyn_t, syn_groups(d) * kSynRows, cana_t,
                                                 ana_groups(d) * kAnaRows,
                                                 1.0 / ((double)d.NX2 * (double)d.NZ2));
}

cudaError_t configure_cheb_kernels(const Dims &d) {
    cudaError_t e = raise_smem(k_ysynth<double2>, (int)syn_smem(d));
    if (e == cudaSuccess)
        e = raise_smem(k_ysynth<float2>, (int)syn_smem(d));
    if (e == cudaSuccess)
        e = raise_smem(k_yanalysis<double2>, (int)ana_smem(d, sizeof(double2)));
    if (e == cudaSuccess)
        e = raise_smem(k_yanalysis<float2>, (int)ana_smem(d, sizeof(float2)));
    if (e != cudaSuccess) return e;
    const int sm = (int)curl_smem(d);
    switch (lane_elems(d)) {
    case 1: return raise_smem(k_curl<1>, sm);
    case 2: return raise_smem(k_curl<2>, sm);
    case 4: return raise_smem(k_curl<4>, sm);
    case 8: return raise_smem(k_curl<8>, sm);
    default: return cudaErrorInvalidValue;
    }
}

void launch_curl(const Dims &d, const Tables &t, const double2 *u, double2 *om, double2 *bw, double re,
                 cudaStream_t s) {
    const int blocks = (d.ncol + kColsPerBlock - 1) / kColsPerBlock;
    const size_t sm = curl_smem(d);
    switch (lane_elems(d)) {
    case 1: k_curl<1><<<blocks, 32 * kColsPerBlock, sm, s>>>(d, t, u, om, bw, re); break;
    case 2: k_curl<2><<<blocks, 32 * kColsPerBlock, sm, s>>>(d, t, u, om, bw, re); break;
    case 4: k_curl<4><<<blocks, 32 * kColsPerBlock, sm, s>>>(d, t, u, om, bw, re); break;
    case 8: k_curl<8><<<blocks, 32 * kColsPerBlock, sm, s>>>(d, t, u, om, bw, re); break;
    default: break;
    }
}

template <class CO>
void ysynth(const Dims &d, const Tables &t, const double2 *src0, const double2 *src1, int nsplit, int nf, CO *F,
            double *mean, cudaStream_t s) {
    const int g = syn_groups(d);
    dim3 block(32, 2 * std::min(g, kSynTiles));
    dim3 grid((d.ncol + 31) / 32, nf, (g + kSynTiles - 1) / kSynTiles);
    k_ysynth<CO><<<grid, block, syn_smem(d), s>>>(d, t.csyn, g * kSynRows, src0, src1, nsplit, F, mean);
}
void launch_ysynth(const Dims &d, const Tables &t, const double2 *src0, const double2 *src1, int nsplit,
                   int nf, double2 *F, cudaStream_t s) {
    if ((t.yform & 1) && launch_ydct(d, t, src0, src1, nsplit, nf, F, false, s)) return;
    ysynth(d, t, src0, src1, nsplit, nf, F, static_cast<double *>(nullptr), s);
}
void launch_ysynth(const Dims &d, const Tables &t, const double2 *src0, const double2 *src1, int nsplit,
                   int nf, float2 *F, double *mean, cudaStream_t s) {
    if ((t.yform & 1) && launch_ydct_synthesis_fp32(d, t, src0, src1, nsplit, nf, F, mean, s)) return;
    ysynth(d, t, src0, src1, nsplit, nf, F, mean, s);
}

template <class CI>
void yanalysis(const Dims &d, const double *cana, const CI *F, double2 *S, int nf, double s0, double sn,
               cudaStream_t s) {
    const int g = ana_groups(d);
    dim3 block(32, 2 * std::min(g, kMaxGroups));
    dim3 grid((d.ncol + 31) / 32, nf, (g + kMaxGroups - 1) / kMaxGroups);
    k_yanalysis<CI><<<grid, block, ana_smem(d, sizeof(CI)), s>>>(d, cana, g * kAnaRows, F, S, s0, sn);
}
// Output scales of the analysis: s_0 = 1/(2N), s_k = 1/N; FP32 stage buffers
// arrive without the 1/(NX2 NZ2) of the x and z analyses.
template <class CI>
void yanalysis(const Dims &d, const Tables &t, const CI *F, double2 *S, int nf, cudaStream_t s) {
    const double sxz = sizeof(CI) == 8 ? 1.0 / ((double)d.NX2 * (double)d.NZ2) : 1.0;
    yanalysis(d, t.cana, F, S, nf, sxz / (2.0 * d.NY2), sxz / (double)d.NY2, s);
}
void launch_yanalysis(const Dims &d, const Tables &t, const double2 *F, double2 *S, int nf, cudaStream_t s) {
    if ((t.yform & 2) && launch_ydct(d, t, F, nullptr, 0, nf, S, true, s)) return;
    yanalysis(d, t, F, S, nf, s);
}
void launch_yanalysis(const Dims &d, const Tables &t, const float2 *F, double2 *S, int nf, cudaStream_t s) {
    if ((t.yform & 2) && launch_ydct_analysis_fp32(d, t, F, S, nf, s)) return;
    yanalysis(d, t, F, S, nf, s);
}

void launch_yanalysis_scaled(const Dims &d, const double *cana, const double2 *F, double2 *S, int nf,
                             double scale, cudaStream_t s) {
    yanalysis(d, cana, F, S, nf, scale, scale, s);
}

void launch_mean_products(const Dims &d, const Tables &t, const double *mean, double2 *S, cudaStream_t s) {
    const int warps = 3 * d.ncy, per_block = 8;
    k_mean_products<<<(warps + per_block - 1) / per_block, 32 * per_block, sizeof(double) * 3 * d.ny2, s>>>(
        d, t.cana, ana_groups(d) * kAnaRows, mean, S);
}

}  // namespace cdns
