// Fine-grid backward transform of one scalar field that allocates no device
// memory.  Its intermediate stage buffers (Chebyshev-synthesised and
// z-physical fields) and its tables live in one file-scope device array, so
// a caller that may not allocate -- one running under a memory pool or an
// embedding framework that owns every allocation, or inside a region where
// cudaMalloc would synchronise or is forbidden -- only passes its own input
// and output buffers.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <mutex>

#include "../../include/cdns.h"
#include "cdns_kernels.cuh"

namespace cdns {
namespace {

// Maximum scratch: 32 MiB, enough for product grids up to about 96^3.
constexpr size_t kScratchBytes = 32ull << 20;
__device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
std::atomic<unsigned char *> g_scratch_addr[kMaxDevices];
// The mesh whose tables the array of each device holds and for which the
// kernels' shared-memory limits were raised (guarded by g_setup_mutex).
struct TableMesh {
    bool valid = false;
    cdns_mesh_desc mesh{};
};
TableMesh g_table_mesh[kMaxDevices];

bool same_mesh(const cdns_mesh_desc &a, const cdns_mesh_desc &b) {
    return a.NX == b.NX && a.NY == b.NY && a.NZ == b.NZ && a.NXS == b.NXS && a.NYS == b.NYS && a.NZS == b.NZS &&
           a.NX2 == b.NX2 && a.NY2 == b.NY2 && a.NZ2 == b.NZ2 && a.XL == b.XL && a.ZL == b.ZL;
}

size_t align256(size_t b) { return (b + 255) / 256 * 256; }

bool factor(int n, FftPlan &p) {
    p.n = n;
    p.nrad = 0;
    int m = n;
    while (m % 4 == 0) { if (p.nrad >= 12) return false; p.radix[p.nrad++] = 4; m /= 4; }
    while (m % 2 == 0) { if (p.nrad >= 12) return false; p.radix[p.nrad++] = 2; m /= 2; }
    for (int q = 3; m > 1; q += 2)
        while (m % q == 0) {
            if (q > 13 || p.nrad >= 12) return false;
            p.radix[p.nrad++] = q;
            m /= q;
        }
    return true;
}

// Tables of the transform: wavenumbers, cos(pi m / NY2) and the x / z roots
// of unity exp(-2 pi i k / n), computed on the device.
__global__ void k_noalloc_tables(Dims d, double alx, double alz, double *wavx, double *wavz,
                                 double *cosy, double2 *root_x, double2 *root_z) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < d.nkx) wavx[i] = i * alx;
    if (i < d.nkz) wavz[i] = (i - d.NZS) * alz;
    if (i < 2 * d.NY2) {
        const int N = d.NY2;
        cosy[i] = (2 * i == N || 2 * i == 3 * N) ? 0.0 : cospi((double)i / (double)N);
    }
    if (i < d.NX2) {
        double s, c;
        sincospi(2.0 * (double)i / (double)d.NX2, &s, &c);
        root_x[i] = make_double2(c, -s);
    }
    if (i < d.NZ2) {
        double s, c;
        sincospi(2.0 * (double)i / (double)d.NZ2, &s, &c);
        root_z[i] = make_double2(c, -s);
    }
}

// Device address of the scratch array on the current device.  The first call
// on each device looks the address up (cudaGetSymbolAddress), which is not
// allowed inside stream capture.
int scratch_on_current_device(unsigned char **out) {
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return record_error(CDNS_ERR_CUDA, cudaGetErrorString(e));
    if (dev < 0 || dev >= kMaxDevices) return record_error(CDNS_ERR_ARG, "device index beyond 64");
    unsigned char *p = g_scratch_addr[dev].load(std::memory_order_acquire);
    if (!p) {
        std::lock_guard<std::mutex> lock(g_setup_mutex);
        p = g_scratch_addr[dev].load(std::memory_order_relaxed);
        if (!p) {
            e = cudaGetSymbolAddress((void **)&p, g_noalloc_scratch);
            if (e != cudaSuccess || !p)
                return record_error(CDNS_ERR_CUDA, "cudaGetSymbolAddress of the scratch array failed");
            g_scratch_addr[dev].store(p, std::memory_order_release);
        }
    }
    *out = p;
    return CDNS_OK;
}

}  // namespace
}  // namespace cdns

using namespace cdns;

extern "C" int cdns_transform_fine_backward_noalloc(const cdns_mesh_desc *m, const double *spectral,
                                                   double *physical, void *stream) {
    if (!m || !spectral || !physical) return record_error(CDNS_ERR_ARG, "null argument");
    if (m->NYS < 4 || m->NXS < 0 || m->NZS < 0 || m->NY2 < m->NYS || m->NX2 < 2 * m->NXS ||
        m->NZ2 < 2 * m->NZS || m->NX2 < 1 || m->NZ2 < 1 || !(m->XL > 0) || !(m->ZL > 0))
        return record_error(CDNS_ERR_ARG,
                            "invalid mesh: need NYS>=4, NY2>=NYS, NX2>=2 NXS, NZ2>=2 NZS");
    Dims d{};
    d.NX2 = m->NX2; d.NY2 = m->NY2; d.NZ2 = m->NZ2;
    d.NXS = m->NXS; d.NYS = m->NYS; d.NZS = m->NZS;
    d.nkx = m->NXS + 1; d.nkz = 2 * m->NZS + 1; d.ncy = m->NYS + 1; d.ny2 = m->NY2 + 1;
    d.ncol = d.nkx * d.nkz;
    d.fcol = d.ncol;
    d.zc = d.NZS * d.nkx;
    d.nyh = m->NY2 / 2 + 1;
    d.Ns = (long long)d.nkz * d.ncy * d.nkx;
    FftPlan px{}, pz{};
    if (!factor(d.NX2, px) || !factor(d.NZ2, pz))
        return record_error(CDNS_ERR_ARG, "NX2/NZ2 must factor into primes <= 13");
    // the limits cdns_create applies: configure_transform_kernels raises the
    // shared memory of every transform kernel for this mesh
    if ((size_t)16 * d.NZ2 * 35 > 220 * 1024 || (size_t)16 * d.NX2 * 25 > 220 * 1024)
        return record_error(CDNS_ERR_ARG, "mesh exceeds the shared-memory tiling limits");
    // scratch layout: tables, then the two stage buffers
    const size_t b_wavx = align256(sizeof(double) * d.nkx);
    const size_t b_wavz = align256(sizeof(double) * d.nkz);
    const size_t b_cos = align256(sizeof(double) * 2 * (size_t)d.NY2);
    const size_t b_rx = align256(sizeof(double2) * (size_t)d.NX2);
    const size_t b_rz = align256(sizeof(double2) * (size_t)d.NZ2);
    size_t nsyn, nana;
    cheb_table_sizes(d, &nsyn, &nana);
    const size_t b_syn = align256(sizeof(double) * nsyn);
    const size_t b_F = align256(sizeof(double2) * (size_t)d.ny2 * d.ncol);
    const size_t b_G = align256(sizeof(double2) * (size_t)d.ny2 * d.NZ2 * d.nkx);
    const size_t need = b_wavx + b_wavz + b_cos + b_rx + b_rz + b_syn + b_F + b_G;
    if (need > kScratchBytes) {
        char msg[200];
        std::snprintf(msg, sizeof msg,
                      "mesh needs %zu bytes of scratch; the allocation-free transform holds at most "
                      "%zu bytes (product grids up to about 96^3)", need, kScratchBytes);
        return record_error(CDNS_ERR_ARG, msg);
    }
    unsigned char *base = nullptr;
    int r = scratch_on_current_device(&base);
    if (r) return r;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return record_error(CDNS_ERR_CUDA, cudaGetErrorString(e));
    // tables and kernel limits once per device and mesh: a call with the mesh
    // of the previous call on this device only launches the transform
    bool fresh;
    {
        std::lock_guard<std::mutex> lock(g_setup_mutex);
        fresh = !g_table_mesh[dev].valid || !same_mesh(g_table_mesh[dev].mesh, *m);
        if (fresh) {
            g_table_mesh[dev].valid = false;
            e = configure_transform_kernels(d);
            if (e != cudaSuccess) return record_error(CDNS_ERR_CUDA, cudaGetErrorString(e));
            g_table_mesh[dev].mesh = *m;
            g_table_mesh[dev].valid = true;
        }
    }
    unsigned char *p = base;
    double *wavx = reinterpret_cast<double *>(p); p += b_wavx;
    double *wavz = reinterpret_cast<double *>(p); p += b_wavz;
    double *cosy = reinterpret_cast<double *>(p); p += b_cos;
    double2 *root_x = reinterpret_cast<double2 *>(p); p += b_rx;
    double2 *root_z = reinterpret_cast<double2 *>(p); p += b_rz;
    double *csyn = reinterpret_cast<double *>(p); p += b_syn;
    double2 *F = reinterpret_cast<double2 *>(p); p += b_F;
    double2 *G = reinterpret_cast<double2 *>(p);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const double pi = std::acos(-1.0);
    const int nt = std::max(std::max(d.nkx, d.nkz), std::max(2 * d.NY2, std::max(d.NX2, d.NZ2)));
    if (fresh) {
        k_noalloc_tables<<<(nt + 127) / 128, 128, 0, s>>>(d, 2.0 * pi / m->XL, 2.0 * pi / m->ZL, wavx,
                                                           wavz, cosy, root_x, root_z);
        launch_cheb_tables(d, cosy, csyn, nullptr, s);
        e = cudaGetLastError();
        if (e != cudaSuccess) {
            std::lock_guard<std::mutex> lock(g_setup_mutex);
            g_table_mesh[dev].valid = false;
            return record_error(CDNS_ERR_CUDA, cudaGetErrorString(e));
        }
    }
    Tables t{};
    t.csyn = csyn;
    t.wavx = wavx;
    t.wavz = wavz;
    t.cosy = cosy;
    t.root_x = root_x;
    t.root_z = root_z;
    // Every element of F and G is written before it is read, so nothing in
    // the scratch needs clearing between calls.
    launch_ysynth(d, t, reinterpret_cast<const double2 *>(spectral), nullptr, 1, 1, F, s);
    launch_z_backward(d, pz, root_z, F, G, 1, s);
    launch_x_c2r(d, px, root_x, G, physical, s);
    e = cudaGetLastError();
    if (e != cudaSuccess) return record_error(CDNS_ERR_CUDA, cudaGetErrorString(e));
    return CDNS_OK;
}
