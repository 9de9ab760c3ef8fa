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
// One thread owns one spectral column and MR output rows of one field; the 32
// lanes of a warp own 32 consecutive columns and read the same matrix entries
// (one broadcast load per pair of rows), so the kernels run at the FP64 FMA
// rate with coalesced column loads and stores.
#include <algorithm>

#include "cdns_kernels.cuh"
#include "warp_columns.cuh"

namespace cdns {

namespace {
constexpr int kSynRows = 14;   // synthesis rows (j) per thread
constexpr int kAnaRows = 16;   // analysis rows (k of one parity) per thread
constexpr int kMaxGroups = 8;  // row groups per block (two warps each)

// 16-byte asynchronous global -> shared copy; src_bytes = 0 writes zeros.
__device__ __forceinline__ void cp_async16(void *dst, const void *src, int src_bytes) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(sa), "l"(src), "r"(src_bytes)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N> __device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

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
    for (int i = tid; i < S; i += blockDim.x) {
        const int y = i / kColsPerBlock, l = i - (i / kColsPerBlock) * kColsPerBlock;
        const int c2 = col0 + l;
        if (c2 >= ncol) continue;
        const int kzi = c2 / nkx, kx = c2 - (c2 / nkx) * nkx;
        const long long off = ((long long)kzi * ncy + y) * nkx + kx;
        const int sl = tile_slot<E>(y, l);
#pragma unroll
        for (int c = 0; c < 3; ++c) tile[c * S + sl] = u[c * d.Ns + off];
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

// ---------------------------------------------------------------------------
// Synthesis: F[f][j][col] for j = 0..NY2 from spectral fields
// (fields f < nsplit from src0, the rest from src1).  Grid (column tiles of
// 32, fields); block (32, 2 G): warp (g, p) accumulates the parity-p sum of
// rows j = g MR .. g MR + MR - 1 for the 32 columns.  The coefficients flow
// through shared memory in chunks of KC rows of k (descending, as the
// reference's recurrences), the next chunk prefetched into registers while
// the current one is multiplied; the cosine rows of the chunk ride along.
// ---------------------------------------------------------------------------
constexpr int kSynKC = 16;

template <int MR>
__global__ void __launch_bounds__(32 * 2 * kMaxGroups)
k_ysynth(Dims d, const double *__restrict__ csyn, int jp, const double2 *__restrict__ src0,
         const double2 *__restrict__ src1, int nsplit, double2 *__restrict__ F) {
    extern __shared__ double2 sm[];
    constexpr int KC = kSynKC;
    double2 *xs = sm;                                            // [2][KC][32]
    double *cs = reinterpret_cast<double *>(sm + 2 * KC * 32);   // [2][KC][jp]
    const int lane = threadIdx.x, wy = threadIdx.y;
    const int tid = wy * 32 + lane, nthr = 32 * blockDim.y;
    const int g = wy >> 1, par = wy & 1;
    const int f = blockIdx.y, col0 = blockIdx.x * 32;
    const int ncol = d.ncol, ny = d.NYS, N = d.NY2;
    const double2 *X = f < nsplit ? src0 + (long long)f * d.Ns : src1 + (long long)(f - nsplit) * d.Ns;
    const int nchunk = (d.ncy + KC - 1) / KC;
    // staging of one chunk: X units (row r, lane l) and cosine double2 units
    const int nxu = KC * 32, ncu = KC * jp / 2;
    auto fetch = [&](int chunk, int buf) {
        const int khi = ny - chunk * KC;
        for (int u = tid; u < nxu + ncu; u += nthr) {
            if (u < nxu) {
                const int r = u >> 5, l = u & 31;
                const int k = khi - r, col = col0 + l;
                const bool ok = k >= 0 && col < ncol;
                const int kzi = ok ? col / d.nkx : 0, kx = ok ? col - kzi * d.nkx : 0;
                cp_async16(xs + buf * KC * 32 + u, X + ((long long)kzi * d.ncy + (ok ? k : 0)) * d.nkx + kx,
                           ok ? 16 : 0);
            } else {
                const int c = u - nxu;
                const int r = c / (jp / 2), h = c - r * (jp / 2);
                const int k = khi - r;
                cp_async16(reinterpret_cast<double2 *>(cs + buf * KC * jp) + c,
                           reinterpret_cast<const double2 *>(csyn + (long long)(k >= 0 ? k : 0) * jp) + h,
                           k >= 0 ? 16 : 0);
            }
        }
        cp_async_commit();
    };
    double2 acc[MR];
#pragma unroll
    for (int i = 0; i < MR; ++i) acc[i] = mk(0.0, 0.0);
    const int j0 = g * MR;
    fetch(0, 0);
    for (int chunk = 0; chunk < nchunk; ++chunk) {
        const int buf = chunk & 1;
        if (chunk + 1 < nchunk) {
            fetch(chunk + 1, buf ^ 1);
            cp_async_wait<1>();
        } else {
            cp_async_wait<0>();
        }
        __syncthreads();
        const int khi = ny - chunk * KC;
        // rows r of this chunk whose k = khi - r has parity par
        const int r0 = ((khi - par) & 1);
        for (int r = r0; r < KC; r += 2) {
            const double2 x = xs[(buf * KC + r) * 32 + lane];
            const double2 *c2 = reinterpret_cast<const double2 *>(cs + (buf * KC + r) * jp + j0);
#pragma unroll
            for (int i = 0; i < MR / 2; ++i) {
                const double2 c = c2[i];
                acc[2 * i].x += c.x * x.x;
                acc[2 * i].y += c.x * x.y;
                acc[2 * i + 1].x += c.y * x.x;
                acc[2 * i + 1].y += c.y * x.y;
            }
        }
        __syncthreads();
    }
    // combine: odd-parity warps hand their sums to the even-parity warps
    double2 *ex = sm;   // [G][MR][32]
    if (par == 1) {
#pragma unroll
        for (int i = 0; i < MR; ++i) ex[(g * MR + i) * 32 + lane] = acc[i];
    }
    __syncthreads();
    const int col = col0 + lane;
    if (par == 0 && col < ncol) {
        double2 *Ff = F + (long long)f * d.ny2 * ncol + col;
#pragma unroll
        for (int i = 0; i < MR; ++i) {
            const int j = j0 + i;
            if (j >= d.nyh) break;
            const double2 o = ex[(g * MR + i) * 32 + lane];
            Ff[(long long)j * ncol] = cadd(acc[i], o);
            if (N - j != j) Ff[(long long)(N - j) * ncol] = csub(acc[i], o);
        }
    }
}

// ---------------------------------------------------------------------------
// Analysis: S[f][k][col] (spectral, planar) from F[f][j][col].  Grid (column
// tiles of 32, fields); block (32, 2 G): warp (g, p) owns the MR coefficients
// k = 2 (g MR + i) + p.  Chunks of JC points j (ascending) are folded into
// e_j = X_j + X_{N-j}, o_j = X_j - X_{N-j} while staged in shared memory.
// ---------------------------------------------------------------------------
constexpr int kAnaJC = 16;

template <int MR>
__global__ void __launch_bounds__(32 * 2 * kMaxGroups)
k_yanalysis(Dims d, const double *__restrict__ cana, int kh, const double2 *__restrict__ F,
            double2 *__restrict__ S) {
    extern __shared__ double2 sm[];
    constexpr int JC = kAnaJC;
    double2 *xab = sm;                                           // [2][2 (j, N-j)][JC][32]
    double *as = reinterpret_cast<double *>(sm + 2 * 2 * JC * 32);   // [2][JC][2][kh]
    const int lane = threadIdx.x, wy = threadIdx.y;
    const int tid = wy * 32 + lane, nthr = 32 * blockDim.y;
    const int g = wy >> 1, par = wy & 1;
    const int f = blockIdx.y, col0 = blockIdx.x * 32;
    const int ncol = d.ncol, N = d.NY2;
    const double2 *X = F + (long long)f * d.ny2 * ncol;
    const int nchunk = (d.nyh + JC - 1) / JC;
    // staging of one chunk: rows j and N - j (zero for the middle point and
    // beyond N/2) and the cosine double2 units
    const int nxu = JC * 32, nau = JC * kh;
    auto fetch = [&](int chunk, int buf) {
        for (int u = tid; u < 2 * nxu + nau; u += nthr) {
            if (u < 2 * nxu) {
                const int side = u >= nxu, v = u - side * nxu;
                const int r = v >> 5, l = v & 31;
                const int j = chunk * JC + r, col = col0 + l;
                const int jj = side ? N - j : j;
                const bool ok = j < d.nyh && col < ncol && !(side && jj == j);
                cp_async16(xab + (buf * 2 + side) * JC * 32 + v, X + (long long)(ok ? jj : 0) * ncol + (ok ? col : 0),
                           ok ? 16 : 0);
            } else {
                const int c = u - 2 * nxu;
                const int r = c / kh, h = c - r * kh;
                const int j = chunk * JC + r;
                cp_async16(reinterpret_cast<double2 *>(as + buf * JC * 2 * kh) + c,
                           reinterpret_cast<const double2 *>(cana + (long long)(j < d.nyh ? j : 0) * 2 * kh) + h,
                           j < d.nyh ? 16 : 0);
            }
        }
        cp_async_commit();
    };
    double2 acc[MR];
#pragma unroll
    for (int i = 0; i < MR; ++i) acc[i] = mk(0.0, 0.0);
    const int m0 = g * MR;
    fetch(0, 0);
    for (int chunk = 0; chunk < nchunk; ++chunk) {
        const int buf = chunk & 1;
        if (chunk + 1 < nchunk) {
            fetch(chunk + 1, buf ^ 1);
            cp_async_wait<1>();
        } else {
            cp_async_wait<0>();
        }
        __syncthreads();
        const int rmax = min(JC, d.nyh - chunk * JC);
        for (int r = 0; r < rmax; ++r) {
            const double2 xa = xab[(buf * 2 * JC + r) * 32 + lane];
            const double2 xb = xab[((buf * 2 + 1) * JC + r) * 32 + lane];
            const double2 x = par ? csub(xa, xb) : cadd(xa, xb);
            const double2 *a2 = reinterpret_cast<const double2 *>(as + ((buf * JC + r) * 2 + par) * kh + m0);
#pragma unroll
            for (int i = 0; i < MR / 2; ++i) {
                const double2 a = a2[i];
                acc[2 * i].x += a.x * x.x;
                acc[2 * i].y += a.x * x.y;
                acc[2 * i + 1].x += a.y * x.x;
                acc[2 * i + 1].y += a.y * x.y;
            }
        }
        __syncthreads();
    }
    const int col = col0 + lane;
    if (col < ncol) {
        const int kzi = col / d.nkx, kx = col - kzi * d.nkx;
        double2 *Sf = S + (long long)f * d.Ns + (long long)kzi * d.ncy * d.nkx + kx;
        const double sn = 1.0 / (double)N, s0 = 1.0 / (2.0 * N);
#pragma unroll
        for (int i = 0; i < MR; ++i) {
            const int k = 2 * (m0 + i) + par;
            if (k < d.ncy) Sf[(long long)k * d.nkx] = cscale(k == 0 ? s0 : sn, acc[i]);
        }
    }
}

size_t curl_smem(const Dims &d) { return sizeof(double2) * 3 * (size_t)d.ncy * kColsPerBlock; }
size_t syn_smem(const Dims &d) {
    const size_t jp = (size_t)syn_groups(d) * kSynRows;
    const size_t pipe = sizeof(double2) * 2 * kSynKC * 32 + sizeof(double) * 2 * kSynKC * jp;
    const size_t ex = sizeof(double2) * jp * 32;
    return pipe > ex ? pipe : ex;
}
size_t ana_smem(const Dims &d) {
    const size_t kh = (size_t)ana_groups(d) * kAnaRows;
    return sizeof(double2) * 2 * 2 * kAnaJC * 32 + sizeof(double) * 2 * kAnaJC * 2 * kh;
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

cudaError_t configure_cheb_kernels(const Dims &d) {
    if (syn_groups(d) > kMaxGroups || ana_groups(d) > kMaxGroups) return cudaErrorInvalidValue;
    cudaError_t e = cudaFuncSetAttribute(k_ysynth<kSynRows>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)syn_smem(d));
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(k_yanalysis<kAnaRows>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)ana_smem(d));
    if (e != cudaSuccess) return e;
    const int sm = (int)curl_smem(d);
    switch (lane_elems(d)) {
    case 1: return cudaFuncSetAttribute(k_curl<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
    case 2: return cudaFuncSetAttribute(k_curl<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
    case 4: return cudaFuncSetAttribute(k_curl<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
    case 8: return cudaFuncSetAttribute(k_curl<8>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
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

void launch_ysynth(const Dims &d, const Tables &t, const double2 *src0, const double2 *src1, int nsplit,
                   int nf, double2 *F, cudaStream_t s) {
    const int g = syn_groups(d);
    dim3 block(32, 2 * g);
    dim3 grid((d.ncol + 31) / 32, nf);
    k_ysynth<kSynRows><<<grid, block, syn_smem(d), s>>>(d, t.csyn, g * kSynRows, src0, src1, nsplit, F);
}

void launch_yanalysis(const Dims &d, const Tables &t, const double2 *F, double2 *S, int nf, cudaStream_t s) {
    const int g = ana_groups(d);
    dim3 block(32, 2 * g);
    dim3 grid((d.ncol + 31) / 32, nf);
    k_yanalysis<kAnaRows><<<grid, block, ana_smem(d), s>>>(d, t.cana, g * kAnaRows, F, S);
}

}  // namespace cdns
