// Layout conversion between the reference's interleaved-component arrays
// ([..][c], src/core/array4d.hpp:62-67) and the component-planar device
// layout ([c][..]).
#include "cdns_kernels.cuh"

namespace cdns {

__global__ void k_deinterleave(const double2 *__restrict__ src, double2 *__restrict__ dst,
                               long long n, int nc) {
    const long long total = n * nc;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        const long long e = i / nc;
        const int c = (int)(i - e * nc);
        dst[c * n + e] = src[i];
    }
}

__global__ void k_interleave(const double2 *__restrict__ src, double2 *__restrict__ dst,
                             long long n, int nc) {
    const long long total = n * nc;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        const long long e = i / nc;
        const int c = (int)(i - e * nc);
        dst[i] = src[c * n + e];
    }
}

static int grid_for(long long total) {
    long long b = (total + 255) / 256;
    if (b > 148 * 32) b = 148 * 32;
    return (int)(b < 1 ? 1 : b);
}

void launch_deinterleave(const double2 *src, double2 *dst, long long n, int nc, cudaStream_t s) {
    k_deinterleave<<<grid_for(n * nc), 256, 0, s>>>(src, dst, n, nc);
}

void launch_interleave(const double2 *src, double2 *dst, long long n, int nc, cudaStream_t s) {
    k_interleave<<<grid_for(n * nc), 256, 0, s>>>(src, dst, n, nc);
}

}  // namespace cdns
