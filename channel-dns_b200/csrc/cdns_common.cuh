// Shared device-side definitions for the channel-dns B200 step.
//
// Spectral fields live in HBM component-planar: component c of a vector field
// is a contiguous complex<double> array [kz+NZS][y][kx] (the reference's
// per-component order, src/core/array4d.hpp:62-67, with the component index
// moved outermost).  The flattened column index col = kz_idx*nkx + kx numbers
// the independent (kz, kx) Fourier modes.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>

namespace cdns {

struct Dims {
    int NX2, NY2, NZ2;   // product (fine) grid: x points, y intervals, z points
    int NXS, NYS, NZS;   // retained modes
    int nkx, nkz, ncy;   // NXS+1, 2 NZS+1, NYS+1
    int ny2;             // NY2+1 Gauss-Lobatto points
    int ncol;            // nkz*nkx spectral columns
    int fcol;            // row stride (columns) of the y-physical stage buffer F:
                         // ncol, rounded up to even for FP32 stages (16-byte rows)
    int nyh;             // NY2/2+1 (half of the y points, symmetric pairs)
    long long Ns;        // nkz*ncy*nkx complex values per spectral component
    int ztl;             // kx lines per block of the z transforms (0: the padding rule)
    int xrw;             // register-form x stage: (z, y) rows per block (2 or 4; 0: 4), 3 or 5:
                         // 4 or 2 rows with the forward phases split over lane pairs (even N1,
                         // N2), or 1: the half-warp form (a half-warp per row pair)
    int kx0;             // global kx of local column kx = 0 (a pencil rank's kx block; else 0)
    int zc;              // local index of the (kz, kx) = (0, 0) column, -1 if not held here
};

// Read-only per-context tables in device memory.
struct Tables {
    const double *wavx;   // [nkx]  kx*2pi/XL
    const double *wavz;   // [nkz]  kz*2pi/ZL
    const double *WL, *WD, *WR;  // [ncy] Chebyshev integration weights
    const double *cosy;   // [2*NY2] cos(pi m / NY2)
    const double *csyn;   // Chebyshev synthesis matrix (chebyshev.cu)
    const double *cana;   // Chebyshev analysis matrix (chebyshev.cu)
    const double2 *root_x;  // [NX2] exp(-2 pi i k / NX2)
    const double2 *root_z;  // [NZ2] exp(-2 pi i k / NZ2)
    const double2 *root_y;  // [NY2] exp(-2 pi i k / NY2) (FFT form of the Chebyshev transforms)
    int yform;              // Chebyshev transforms in the FFT (DCT-I) form where NY2 splits:
                            // bit 0 the synthesis, bit 1 the analysis (else the FP64 MMA products)
};

struct FftPlan {
    int n;
    int nrad;
    int radix[12];
};

__host__ __device__ inline double2 mk(double re, double im) { return make_double2(re, im); }
__device__ inline double2 cadd(double2 a, double2 b) { return mk(a.x + b.x, a.y + b.y); }
__device__ inline double2 csub(double2 a, double2 b) { return mk(a.x - b.x, a.y - b.y); }
__device__ inline double2 cmul(double2 a, double2 b) {
    return mk(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ inline double2 cscale(double s, double2 a) { return mk(s * a.x, s * a.y); }
__device__ inline double2 cconj(double2 a) { return mk(a.x, -a.y); }
// (i*k)*(a+ib) in the reference's form (src/core/complex_ops.hpp:6-8)
__device__ inline double2 fderiv(double k, double2 v) { return mk(-k * v.y, k * v.x); }
// complex division in Smith's form (what libgcc's __divdc3 reduces to for
// finite operands)
__device__ inline double2 cdiv(double2 a, double2 b) {
    if (fabs(b.x) >= fabs(b.y)) {
        const double r = b.y / b.x;
        const double den = b.x + b.y * r;
        return mk((a.x + a.y * r) / den, (a.y - a.x * r) / den);
    }
    const double r = b.x / b.y;
    const double den = b.x * r + b.y;
    return mk((a.x * r + a.y) / den, (a.y * r - a.x) / den);
}
__device__ inline double2 cdivr(double2 a, double s) { return mk(a.x / s, a.y / s); }

// FP32 complex arithmetic (the mixed-precision transforms) and a complex-type
// trait so that butterflies and DFTs are written once for both widths.
__device__ inline float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ inline float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ inline float2 cmul(float2 a, float2 b) {
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ inline float2 cscale(float s, float2 a) { return make_float2(s * a.x, s * a.y); }

template <class C> struct CReal;
template <> struct CReal<double2> { using T = double; };
template <> struct CReal<float2> { using T = float; };
template <class C> __host__ __device__ inline C mkc(double re, double im);
template <> __host__ __device__ inline double2 mkc<double2>(double re, double im) { return make_double2(re, im); }
template <> __host__ __device__ inline float2 mkc<float2>(double re, double im) {
    return make_float2((float)re, (float)im);
}
// complex value converted between widths
template <class C, class S> __device__ inline C cto(S v) { return mkc<C>(v.x, v.y); }

// Raise a kernel's dynamic shared-memory limit to at least `bytes` (never
// lower it: contexts of different meshes share the kernel attribute).
template <class K> inline cudaError_t raise_smem(K *kernel, size_t bytes) {
    cudaFuncAttributes a{};
    cudaError_t e = cudaFuncGetAttributes(&a, kernel);
    if (e != cudaSuccess) return e;
    if ((size_t)a.maxDynamicSharedSizeBytes >= bytes) return cudaSuccess;
    return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

// Asynchronous global -> shared copies (cp.async, sm_80 and later): 16 bytes
// cached in L2 only, or 8 bytes; src_bytes below the size fills the rest
// with zeros (0: zeros only, the source is not read).
__device__ __forceinline__ void cp_async16(void *dst, const void *src, int src_bytes) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(sa), "l"(src), "r"(src_bytes)
                 : "memory");
}
__device__ __forceinline__ void cp_async8(void *dst, const void *src, int src_bytes) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(sa), "l"(src), "r"(src_bytes)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N> __device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// Error bits recorded on the device and read by the host after a step.
enum : unsigned { ERR_NONFINITE = 1u, ERR_PIVOT = 2u };

}  // namespace cdns
