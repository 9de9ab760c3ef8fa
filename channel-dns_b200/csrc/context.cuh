// Internal view of a cdns context, shared by the translation units that
// orchestrate the forward step (context.cu) and its discrete adjoint
// (adjoint_run.cu).  Not part of the C ABI.
#pragma once

#include <cuda_runtime.h>

#include <cstdlib>
#include <string>
#include <vector>

#include "../../include/cdns.h"
#include "cdns_kernels.cuh"

namespace cdns {

// Records msg as the calling thread's last error (cdns_last_error) and returns code.
int fail(int code, const std::string &msg);

constexpr int kStages = 7;
constexpr int kMaxProfSteps = 256;

struct AdjointWork;   // adjoint_run.cu
void adjoint_release(AdjointWork *w);
size_t adjoint_bytes(const AdjointWork *w);
struct OutputWork;    // output.cu
void output_release(OutputWork *w);
size_t output_bytes(const OutputWork *w);
struct PencilWork;    // pencil.cu
void pencil_release(PencilWork *w);
// Rank `rank` of a `ranks`-way pencil decomposition of mesh m: the kx block
// [kx0, kx0 + nkx) and the fine-grid y slab [j0, j0 + nj) (the reference's
// block rule, src/core/mesh.cpp:20-85).  Non-zero (with the error recorded)
// if the decomposition would leave a rank an empty block.
int pencil_blocks(const cdns_mesh_desc &m, int ranks, int rank, int &kx0, int &nkx, int &j0, int &nj);
// Radix plan of a length-n Stockham FFT (false if n has a prime factor > 13).
bool plan_fft(int n, FftPlan &p);

}  // namespace cdns

#define CK(call)                                                                                  \
    do {                                                                                          \
        cudaError_t e_ = (call);                                                                  \
        if (e_ != cudaSuccess)                                                                    \
            return ::cdns::fail(CDNS_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

struct cdns_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    cdns_mesh_desc mesh{};
    cdns::Dims d{};
    cdns::Tables t{};
    cdns::FftPlan px{}, pz{};
    cdns::PhysParams pp{};
    double DT = 0.0;
    std::vector<void *> allocs;
    size_t bytes = 0;
    // state (component planar)
    double2 *U[2] = {nullptr, nullptr};   // velocity / previous velocity
    double2 *Nb[2] = {nullptr, nullptr};  // nonlinear term, current / previous
    double2 *Bb[2] = {nullptr, nullptr};  // pressure wall data, current / previous
    int cur = 0;                          // U[cur] = u, Nb[cur] = next N, Bb[cur] = next B
    double2 *p = nullptr, *bw = nullptr, *bc_v = nullptr, *bc_p = nullptr;
    double2 *F = nullptr, *G = nullptr, *H = nullptr, *aux = nullptr, *aux2 = nullptr, *zero3 = nullptr;
    double2 *om = nullptr;                // vorticity of the velocity being transformed
    bool mixed = false;                   // FP32 fine-grid stages (CDNS_PRECISION_MIXED)
    double *mean = nullptr;               // mixed: FP64 (kz, kx) = (0, 0) profiles [6][NY2+1]
    double *phys = nullptr;
    double *dpdx = nullptr;
    unsigned *err = nullptr;
    cdns::SolverState st{};
    double g_setup = NAN;
    bool have_velocity = false;
    cudaGraphExec_t graph[2] = {nullptr, nullptr};
    bool prof = false;
    int prof_steps = 0;
    std::vector<cudaEvent_t> ev;
    cdns::AdjointWork *adj = nullptr;     // discrete-adjoint workspace, made on first use
    cdns::OutputWork *outw = nullptr;     // coarse-grid output workspace, made on first use
    cdns::PencilWork *pen = nullptr;      // pencil rank: y-slab stage buffers and exchange maps

    template <typename T> int alloc(T *&ptr, size_t count) {
        void *p = nullptr;
        const size_t b = sizeof(T) * (count ? count : 1);
        // CDNS_DEVICE_BYTES_CAP=<bytes>: refuse allocations past a cap (host-side
        // injection of an out-of-memory failure for tests)
        if (const char *cap = std::getenv("CDNS_DEVICE_BYTES_CAP")) {
            const unsigned long long limit = std::strtoull(cap, nullptr, 10);
            if (limit > 0 && bytes + b > limit)
                return cdns::fail(CDNS_ERR_NOMEM, "device allocation cap (CDNS_DEVICE_BYTES_CAP) reached");
        }
        cudaError_t e = cudaMalloc(&p, b);
        if (e != cudaSuccess)
            return cdns::fail(CDNS_ERR_NOMEM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
        // Zero on the context stream: a cudaMemset on the legacy default stream
        // is not ordered against this non-blocking stream and could land after
        // the kernels that fill the buffer.
        e = cudaMemsetAsync(p, 0, b, stream);
        if (e != cudaSuccess) return cdns::fail(CDNS_ERR_CUDA, cudaGetErrorString(e));
        allocs.push_back(p);
        bytes += b;
        ptr = static_cast<T *>(p);
        return CDNS_OK;
    }
};

namespace cdns {

// Multistep coefficients of iteration it (src/sim/simulation.cpp:36-45).
void step_coefficients(int it, double dt, double re, double &a0, double &a1, double &b0, double &b1,
                       double &g);
// Nonlinear stages u -> N (planar spectral) and bw; G_fp64 (FP64 contexts)
// receives the z-physical fields of u and omega, c->G if null.
void enqueue_nonlinear(cdns_ctx *c, const double2 *u, double2 *N, bool prof, int step_slot,
                       double2 *G_fp64 = nullptr);
// The column solve of a step from U[cur], Nb[cur], bw and the stored history
// (RHS assembly, pressure and velocity solves, zero-mode and flow corrections).
void enqueue_solve(cdns_ctx *c, double a0, double a1, double b0, double b1, double g_v);
// Solver state of c for wall-normal Helmholtz constant g_v (no-op if current).
int do_setup(cdns_ctx *c, double g_v);
// Entry points that transform or step the whole channel refuse a pencil rank.
int require_whole(const cdns_ctx *c);
// Sets up the pencil workspace of a rank context made by cdns_create's body.
int pencil_init(cdns_ctx *c, int ranks, int rank);
// One step of cdns_step: setup if g changed, then the step (graph replay for it >= 3).
int one_step(cdns_ctx *c, int it);
// Launch shapes of c (z line width, Chebyshev transform forms): cached or timed (tune.cu).
int tune_context(cdns_ctx *c, bool force);

struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev) {
        cudaGetDevice(&prev);
        if (prev != dev) cudaSetDevice(dev);
    }
    ~DeviceGuard() {
        if (prev >= 0) cudaSetDevice(prev);
    }
};

}  // namespace cdns
