// Output reduction of the channel-dns step on the device for sm_100a: the
// output branch of Simulation::run (src/sim/simulation.cpp:226-235) --
// FieldIO::to_physical (src/io/field_io.cpp:199-220), Statistics::reduce
// (src/sim/statistics.cpp:55-110) and Diagnostics::evaluate
// (src/sim/diagnostics.cpp:14-80) -- and the coarse-grid transform
// Transforms::channel_xyzfft (src/fft/transforms.cpp:452-582).
//
// The coarse grid (NX x (NY+1) x NZ) runs the fine-grid kernels with the
// coarse mesh as their Dims and its own tables: the Chebyshev synthesis and
// analysis on NY+1 points, the z transforms with the coarse Nyquist
// conventions (halve and mirror / sum at a full spectrum) and a fused x stage
// that synthesises u, v, w, p and the divergence of each (z, y) row and sums
// the per-plane moments in the same kernel, so the physical fields never go
// to HBM unless a snapshot is asked for.  Only (NY+1) x 22 plane sums come
// back to the host, where EKT, TKE and the divergence L2 norm are formed in
// the reference's order.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>

#include "context.cuh"
#include "warp_columns.cuh"

namespace cdns {

struct OutputWork {
    Dims dc{};          // coarse grid as a Dims: NX2 = NX, NY2 = NY, NZ2 = NZ
    Tables tc{};        // spectral tables of the context, coarse cosine tables and roots
    FftPlan px{}, pz{};
    std::vector<void *> allocs;
    size_t bytes = 0;
    double2 *pd = nullptr;       // [2][Ns] pressure copy, spectral divergence
    double2 *F = nullptr;        // [5][NY+1][ncol] y-physical
    double2 *G = nullptr;        // [5][NY+1][NZ][nkx] z-physical
    double *partial = nullptr;   // [NY+1][blocks][22]
    double *planes = nullptr;    // [NY+1][22]
    double *phys = nullptr;      // [4][NZ][NY+1][NX] snapshot (made on first request)
    unsigned *flag = nullptr;    // spectral finite check
    std::vector<double> ccw;     // Clenshaw-Curtis weights / 2
    double *stats = nullptr;     // running means [20][NY+1] + dpdx, dpdz means
    long long count = 0;         // samples accumulated
};

void output_release(OutputWork *w) {
    if (!w) return;
    for (void *p : w->allocs) cudaFree(p);
    delete w;
}

size_t output_bytes(const OutputWork *w) { return w ? w->bytes : 0; }

namespace {

template <typename T> int oalloc(cdns_ctx *c, OutputWork *w, T *&p, size_t n) {
    void *q = nullptr;
    const size_t b = sizeof(T) * (n ? n : 1);
    cudaError_t e = cudaMalloc(&q, b);
    if (e != cudaSuccess) return fail(CDNS_ERR_NOMEM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
    e = cudaMemsetAsync(q, 0, b, c->stream);
    if (e != cudaSuccess) return fail(CDNS_ERR_CUDA, cudaGetErrorString(e));
    w->allocs.push_back(q);
    w->bytes += b;
    p = static_cast<T *>(q);
    return CDNS_OK;
}

// Spectral divergence (src/solver/vector_ops.cpp:90-105), the pressure copied
// beside it, and a finite check of the spectral velocity and pressure
// (src/io/field_io.cpp:205-215).  Warp per column for the y derivative.
template <int E>
__global__ void __launch_bounds__(32 * kColsPerBlock)
k_divergence(Dims d, Tables t, const double2 *__restrict__ u, const double2 *__restrict__ p,
             double2 *__restrict__ pd, unsigned *__restrict__ flag) {
    extern __shared__ double2 tile[];   // [ncy][kColsPerBlock]: v, then dv/dy
    const int ncy = d.ncy, ny = d.NYS, nkx = d.nkx, ncol = d.ncol;
    const int S = ncy * kColsPerBlock;
    const int col0 = blockIdx.x * kColsPerBlock;
    const int tid = threadIdx.x, w = tid >> 5;
    bool ok = true;
    for (int i = tid; i < S; i += blockDim.x) {
        const int y = i / kColsPerBlock, l = i - (i / kColsPerBlock) * kColsPerBlock;
        const int c2 = col0 + l;
        if (c2 >= ncol) continue;
        const int kzi = c2 / nkx, kx = c2 - (c2 / nkx) * nkx;
        const long long off = ((long long)kzi * ncy + y) * nkx + kx;
        tile[tile_slot<E>(y, l)] = u[d.Ns + off];
    }
    __syncthreads();
    const int col = col0 + w;
    if (col < ncol) {
        double2 vv[E], dv[E];
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const int y = ycoef<E>(e);
            vv[e] = y <= ny ? tile[tile_slot<E>(y, w)] : mk(0.0, 0.0);
        }
        deriv_warp<E>(ny, vv, dv);
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const int y = ycoef<E>(e);
            if (y <= ny) tile[tile_slot<E>(y, w)] = dv[e];
        }
    }
    __syncthreads();
    for (int i = tid; i < S; i += blockDim.x) {
        const int y = i / kColsPerBlock, l = i - (i / kColsPerBlock) * kColsPerBlock;
        const int c2 = col0 + l;
        if (c2 >= ncol) continue;
        const int kzi = c2 / nkx, kx = c2 - (c2 / nkx) * nkx;
        const long long off = ((long long)kzi * ncy + y) * nkx + kx;
        const double2 a = u[off], b = u[d.Ns + off], c = u[2 * d.Ns + off], q = p[off];
        ok = ok && isfinite(a.x) && isfinite(a.y) && isfinite(b.x) && isfinite(b.y) && isfinite(c.x) &&
             isfinite(c.y) && isfinite(q.x) && isfinite(q.y);
        pd[off] = q;
        pd[d.Ns + off] = cadd(cadd(fderiv(t.wavx[kx], a), tile[tile_slot<E>(y, l)]), fderiv(t.wavz[kzi], c));
    }
    if (__any_sync(kFull, !ok) && (tid & 31) == 0) atomicOr(flag, 1u);
}

// Plane sums of the x-stage partials in a fixed order (one block per plane).
__global__ void k_plane_finalize(int nblocks, const double *__restrict__ partial, double *__restrict__ planes) {
    constexpr int K = 22;
    const int j = blockIdx.x, k = threadIdx.x;
    if (k >= K) return;
    const double *p = partial + (long long)j * nblocks * K;
    double t = p[k];
    for (int b = 1; b < nblocks; ++b) t = (k == 21) ? fmin(t, p[b * K + k]) : t + p[b * K + k];
    planes[j * K + k] = t;
}

// Statistics::accumulate (src/sim/statistics.cpp:117-139) on the device:
// running means (old * count + sample) / (count + 1) of the plane moments
// scaled by 1/(NX NZ), in the layout [20][NY+1]:
//   0-2 velocity mean, 3 pressure mean, 4-9 velocity second moments (uu vv
//   ww uv vw wu), 10 pressure second, 11-13 pressure-velocity, 14-16
//   velocity third, 17-19 velocity fourth; then the dpdx and dpdz means.
__global__ void k_stats_accumulate(int ny1, double scale, long long count, const double *__restrict__ planes,
                                   const double *__restrict__ dpdx, double *__restrict__ stats) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    const double cn = (double)count, cn1 = (double)(count + 1);
    auto upd = [&](int slot, double sample) {
        double &o = stats[(long long)slot * ny1 + j];
        o = (o * cn + sample) / cn1;
    };
    if (j < ny1) {
        const double *sm = planes + (long long)j * 22;
        upd(3, sm[3] * scale);
        upd(10, sm[13] * scale);
        for (int c = 0; c < 3; ++c) {
            upd(c, sm[c] * scale);
            upd(4 + c, sm[4 + c] * scale);
            upd(7 + c, sm[7 + c] * scale);
            upd(11 + c, sm[10 + c] * scale);
            upd(14 + c, sm[14 + c] * scale);
            upd(17 + c, sm[17 + c] * scale);
        }
    }
    if (j == 0) {
        double *dm = stats + 20LL * ny1;
        dm[0] = (dm[0] * cn + dpdx[0]) / cn1;
        dm[1] = (dm[1] * cn + dpdx[1]) / cn1;
    }
}

size_t div_smem(const Dims &d) { return sizeof(double2) * (size_t)d.ncy * kColsPerBlock; }

template <int E> cudaError_t configure_div_e(const Dims &d) { return raise_smem(k_divergence<E>, (int)div_smem(d)); }

void launch_divergence(const Dims &d, const Tables &t, const double2 *u, const double2 *p, double2 *pd,
                       unsigned *flag, cudaStream_t s) {
    const int blocks = (d.ncol + kColsPerBlock - 1) / kColsPerBlock;
    const size_t sm = div_smem(d);
    switch (lane_elems(d)) {
    case 1: k_divergence<1><<<blocks, 32 * kColsPerBlock, sm, s>>>(d, t, u, p, pd, flag); break;
    case 2: k_divergence<2><<<blocks, 32 * kColsPerBlock, sm, s>>>(d, t, u, p, pd, flag); break;
    case 4: k_divergence<4><<<blocks, 32 * kColsPerBlock, sm, s>>>(d, t, u, p, pd, flag); break;
    case 8: k_divergence<8><<<blocks, 32 * kColsPerBlock, sm, s>>>(d, t, u, p, pd, flag); break;
    default: break;
    }
}

// Clenshaw-Curtis weights on the NY+1 Gauss-Lobatto points divided by the
// height 2 (src/sim/diagnostics.cpp:18-36).
std::vector<double> clenshaw_curtis(int n) {
    std::vector<double> w(n + 1);
    const double pi = std::acos(-1.0);
    for (int j = 0; j <= n; ++j) {
        const double theta = pi * j / n;
        double weight;
        if (j == 0 || j == n) {
            weight = 1.0 / (n * n - (n % 2 == 0 ? 1.0 : 0.0));
        } else {
            double value = 1.0;
            for (int k = 1; k <= (n - 1) / 2; ++k) value -= 2.0 * std::cos(2 * k * theta) / (4.0 * k * k - 1.0);
            if (n % 2 == 0) value -= std::cos(n * theta) / (n * n - 1.0);
            weight = 2.0 * value / n;
        }
        w[j] = weight / 2.0;
    }
    return w;
}

int ensure_output(cdns_ctx *c, bool snapshot) {
    const Dims &d = c->d;   // (FP64 state in both precision modes; the coarse stages are FP64)
    if (!c->outw) {
        OutputWork *w = new OutputWork;
        c->outw = w;
        Dims &dc = w->dc;
        dc = d;
        dc.NX2 = c->mesh.NX;
        dc.NY2 = c->mesh.NY;
        dc.NZ2 = c->mesh.NZ;
        dc.ny2 = c->mesh.NY + 1;
        dc.nyh = c->mesh.NY / 2 + 1;
        dc.fcol = d.ncol;
        if (!(dc.NX2 >= 2 * d.NXS && dc.NZ2 >= 2 * d.NZS && dc.NY2 >= d.NYS))
            return fail(CDNS_ERR_ARG, "coarse grid smaller than the spectral modes");
        if (!plan_fft(dc.NX2, w->px) || !plan_fft(dc.NZ2, w->pz))
            return fail(CDNS_ERR_ARG, "coarse NX / NZ has a prime factor above 13");
        // coarse tables: cos(pi m / NY), m < 2 NY, exact zeros; roots of NX and NZ
        const long double pil = 3.141592653589793238462643383279502884L;
        std::vector<double> cosy(2 * (size_t)dc.NY2);
        for (int mm = 0; mm < 2 * dc.NY2; ++mm) {
            if (2 * mm == dc.NY2 || 2 * mm == 3 * dc.NY2) cosy[mm] = 0.0;
            else cosy[mm] = (double)cosl(pil * (long double)mm / (long double)dc.NY2);
        }
        auto roots = [&](int nn) {
            std::vector<double2> rr(nn);
            for (int k = 0; k < nn; ++k) {
                const long double a = 2.0L * pil * (long double)k / (long double)nn;
                rr[k] = make_double2((double)cosl(a), (double)(-sinl(a)));
            }
            return rr;
        };
        const auto rx = roots(dc.NX2), rz = roots(dc.NZ2), ry = roots(dc.NY2);
        size_t nsyn, nana;
        cheb_table_sizes(dc, &nsyn, &nana);
        double *cy = nullptr, *csyn = nullptr, *cana = nullptr;
        double2 *rxd = nullptr, *rzd = nullptr, *ryd = nullptr;
        const size_t Ns = (size_t)d.Ns, ny1 = dc.ny2;
        int r = 0;
        if ((r = oalloc(c, w, cy, cosy.size())) || (r = oalloc(c, w, csyn, nsyn)) || (r = oalloc(c, w, cana, nana)) ||
            (r = oalloc(c, w, rxd, rx.size())) || (r = oalloc(c, w, rzd, rz.size())) ||
            (r = oalloc(c, w, ryd, ry.size())) ||
            (r = oalloc(c, w, w->pd, 2 * Ns)) || (r = oalloc(c, w, w->F, 5 * ny1 * d.ncol)) ||
            (r = oalloc(c, w, w->G, 5 * ny1 * dc.NZ2 * d.nkx)) ||
            (r = oalloc(c, w, w->partial, ny1 * moment_blocks(dc) * 22)) ||
            (r = oalloc(c, w, w->planes, ny1 * 22)) || (r = oalloc(c, w, w->flag, 1)))
            return r;
        CK(cudaMemcpyAsync(cy, cosy.data(), cosy.size() * sizeof(double), cudaMemcpyHostToDevice, c->stream));
        CK(cudaMemcpyAsync(rxd, rx.data(), rx.size() * sizeof(double2), cudaMemcpyHostToDevice, c->stream));
        CK(cudaMemcpyAsync(rzd, rz.data(), rz.size() * sizeof(double2), cudaMemcpyHostToDevice, c->stream));
        CK(cudaMemcpyAsync(ryd, ry.data(), ry.size() * sizeof(double2), cudaMemcpyHostToDevice, c->stream));
        launch_cheb_tables(dc, cy, csyn, cana, c->stream);
        w->tc = c->t;
        w->tc.cosy = cy;
        w->tc.csyn = csyn;
        w->tc.cana = cana;
        w->tc.root_x = rxd;
        w->tc.root_z = rzd;
        w->tc.root_y = ryd;
        w->ccw = clenshaw_curtis(dc.NY2);
        CK(configure_transform_kernels(dc));
        CK(configure_cheb_kernels(dc));
        cudaError_t e = cudaSuccess;
        switch (lane_elems(d)) {
        case 1: e = configure_div_e<1>(d); break;
        case 2: e = configure_div_e<2>(d); break;
        case 4: e = configure_div_e<4>(d); break;
        case 8: e = configure_div_e<8>(d); break;
        default: e = cudaErrorInvalidValue;
        }
        CK(e);
        CK(cudaGetLastError());   // (limits are only ever raised: the fine-grid launches stay valid)
        // Chebyshev synthesis form on the coarse grid (four fields, as a statistics
        // sample): the faster of the matrix and FFT forms, timed here (cf. tune.cu)
        w->tc.yform = 0;
        Tables tf = w->tc;
        tf.yform = 3;
        if (ydct_available(dc, tf) && !std::getenv("CDNS_Y_TRANSFORM")) {
            cudaEvent_t a, b;
            CK(cudaEventCreate(&a));
            CK(cudaEventCreate(&b));
            float best[2] = {1e30f, 1e30f};
            for (int form = 0; form < 2; ++form) {
                const Tables &tt = form ? tf : w->tc;
                launch_ysynth(dc, tt, c->U[0], c->p, 3, 4, w->F, c->stream);   // warm-up
                for (int rep = 0; rep < 3; ++rep) {
                    CK(cudaEventRecord(a, c->stream));
                    launch_ysynth(dc, tt, c->U[0], c->p, 3, 4, w->F, c->stream);
                    CK(cudaEventRecord(b, c->stream));
                    CK(cudaEventSynchronize(b));
                    float ms = 0.f;
                    CK(cudaEventElapsedTime(&ms, a, b));
                    best[form] = std::min(best[form], ms);
                }
            }
            cudaEventDestroy(a);
            cudaEventDestroy(b);
            if (best[1] < best[0]) w->tc.yform = 1;
        } else if (const char *e = std::getenv("CDNS_Y_TRANSFORM")) {
            if (std::strcmp(e, "fft") == 0) w->tc.yform = 3;
        }
        CK(cudaGetLastError());
    }
    OutputWork *w = c->outw;
    if (!w->stats) {
        int r = oalloc(c, w, w->stats, 20 * (size_t)w->dc.ny2 + 2);
        if (r) return r;
    }
    if (snapshot && !w->phys) {
        const Dims &dc = w->dc;
        int r = oalloc(c, w, w->phys, 4 * (size_t)dc.NZ2 * dc.ny2 * dc.NX2);
        if (r) return r;
    }
    return CDNS_OK;
}

// Plane sums of the current state into w->planes (stream-ordered, no sync).
// check = true adds the divergence (sum 20) and the spectral finite check of
// a check step; a statistics sample needs neither and synthesises u, v, w, p
// straight from the state.
int enqueue_reduction(cdns_ctx *c, bool snapshot, bool check) {
    OutputWork *w = c->outw;
    const Dims &d = c->d, &dc = w->dc;
    cudaStream_t s = c->stream;
    CK(cudaMemsetAsync(w->flag, 0, sizeof(unsigned), s));
    if (check) {
        launch_divergence(d, c->t, c->U[c->cur], c->p, w->pd, w->flag, s);
        launch_ysynth(dc, w->tc, c->U[c->cur], w->pd, 3, 5, w->F, s);
    } else {
        launch_ysynth(dc, w->tc, c->U[c->cur], c->p, 3, 4, w->F, s);
    }
    const int nf = check ? 5 : 4;
    launch_z_backward(dc, w->pz, w->tc.root_z, w->F, w->G, nf, s, true);
    launch_x_moments(dc, w->px, w->tc.root_x, w->G, w->partial, snapshot ? w->phys : nullptr, nf, s);
    k_plane_finalize<<<dc.ny2, 32, 0, s>>>(moment_blocks(dc), w->partial, w->planes);
    CK(cudaGetLastError());
    return CDNS_OK;
}

}  // namespace
}  // namespace cdns

using namespace cdns;

extern "C" {

int cdns_output_reduce(cdns_ctx *c, int higher, double *plane_sums, double *diag, double *physical) {
    if (!c) return fail(CDNS_ERR_ARG, "null context");
    if (int r = require_whole(c)) return r;
    if (!c->have_velocity) return fail(CDNS_ERR_STATE, "cdns_output_reduce before cdns_set_velocity");
    DeviceGuard guard(c->device);
    int r = ensure_output(c, physical != nullptr);
    if (r || (r = enqueue_reduction(c, physical != nullptr, true))) return r;
    OutputWork *w = c->outw;
    const Dims &dc = w->dc;
    cudaStream_t s = c->stream;
    const int ny1 = dc.ny2;
    std::vector<double> pl((size_t)ny1 * 22);
    unsigned flag = 0;
    CK(cudaMemcpyAsync(pl.data(), w->planes, pl.size() * sizeof(double), cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(&flag, w->flag, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
    if (physical) {
        const size_t n = 4 * (size_t)dc.NZ2 * ny1 * dc.NX2;
        CK(cudaMemcpyAsync(physical, w->phys, n * sizeof(double), cudaMemcpyDeviceToHost, s));
    }
    CK(cudaStreamSynchronize(s));
    if (plane_sums) {
        for (int j = 0; j < ny1; ++j)
            for (int k = 0; k < 20; ++k)
                plane_sums[(size_t)j * 20 + k] = (higher || k < 7) ? pl[(size_t)j * 22 + k] : 0.0;
    }
    if (diag) {
        // Diagnostics::evaluate (src/sim/diagnostics.cpp:38-80)
        bool finite = flag == 0;
        const double inv_plane = 1.0 / ((double)dc.NX2 * (double)dc.NZ2);
        double ekt = 0.0, tke = 0.0, div_square = 0.0;
        for (int j = 0; j < ny1; ++j) {
            const double *sj = pl.data() + (size_t)j * 22;
            finite = finite && sj[21] == 1.0;
            ekt += sj[5];
            double variance = 0.0;
            for (int k = 0; k < 3; ++k) {
                const double mean = sj[k] * inv_plane;
                const double raw = sj[4 + k] * inv_plane - mean * mean;
                finite = finite && std::isfinite(raw);
                variance += std::max(0.0, raw);
            }
            tke += 0.5 * w->ccw[j] * variance;
            div_square += w->ccw[j] * inv_plane * sj[20];
        }
        const double l2 = std::sqrt(div_square);
        finite = finite && std::isfinite(ekt) && std::isfinite(tke) && std::isfinite(l2);
        diag[0] = ekt;
        diag[1] = tke;
        diag[2] = l2;
        diag[3] = finite ? 1.0 : 0.0;
    }
    return CDNS_OK;
}

int cdns_statistics_sample(cdns_ctx *c) {
    if (!c) return fail(CDNS_ERR_ARG, "null context");
    if (int r = require_whole(c)) return r;
    if (!c->have_velocity) return fail(CDNS_ERR_STATE, "cdns_statistics_sample before cdns_set_velocity");
    DeviceGuard guard(c->device);
    int r = ensure_output(c, false);
    if (r || (r = enqueue_reduction(c, false, false))) return r;
    OutputWork *w = c->outw;
    const Dims &dc = w->dc;
    const double scale = 1.0 / ((double)dc.NX2 * (double)dc.NZ2);
    k_stats_accumulate<<<(dc.ny2 + 127) / 128, 128, 0, c->stream>>>(dc.ny2, scale, w->count, w->planes, c->dpdx,
                                                                      w->stats);
    CK(cudaGetLastError());
    ++w->count;
    return CDNS_OK;
}

int cdns_statistics_read(cdns_ctx *c, long long *count, double *dp_means, double *means) {
    if (!c) return fail(CDNS_ERR_ARG, "null context");
    if (int r = require_whole(c)) return r;
    DeviceGuard guard(c->device);
    int r = ensure_output(c, false);
    if (r) return r;
    OutputWork *w = c->outw;
    const size_t n = 20 * (size_t)w->dc.ny2;
    std::vector<double> h(n + 2);
    CK(cudaMemcpyAsync(h.data(), w->stats, h.size() * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    if (count) *count = w->count;
    if (dp_means) {
        dp_means[0] = h[n];
        dp_means[1] = h[n + 1];
    }
    if (means) std::copy(h.begin(), h.begin() + n, means);
    return CDNS_OK;
}

int cdns_statistics_reset(cdns_ctx *c) {
    if (!c) return fail(CDNS_ERR_ARG, "null context");
    DeviceGuard guard(c->device);
    int r = ensure_output(c, false);
    if (r) return r;
    OutputWork *w = c->outw;
    CK(cudaMemsetAsync(w->stats, 0, (20 * (size_t)w->dc.ny2 + 2) * sizeof(double), c->stream));
    w->count = 0;
    return CDNS_OK;
}

int cdns_transform_coarse(cdns_ctx *c, int dir, const double *in, double *out) {
    if (!c || !in || !out) return fail(CDNS_ERR_ARG, "null argument");
    if (int r = require_whole(c)) return r;
    DeviceGuard guard(c->device);
    int r = ensure_output(c, true);
    if (r) return r;
    OutputWork *w = c->outw;
    const Dims &d = c->d, &dc = w->dc;
    cudaStream_t s = c->stream;
    const size_t nphys = (size_t)dc.NZ2 * dc.ny2 * dc.NX2;
    if (dir == 'B') {
        CK(cudaMemcpyAsync(w->pd, in, sizeof(double2) * d.Ns, cudaMemcpyHostToDevice, s));
        launch_ysynth(dc, w->tc, w->pd, nullptr, 1, 1, w->F, s);
        launch_z_backward(dc, w->pz, w->tc.root_z, w->F, w->G, 1, s, true);
        launch_x_c2r(dc, w->px, w->tc.root_x, w->G, w->phys, s, true);
        CK(cudaGetLastError());
        CK(cudaMemcpyAsync(out, w->phys, sizeof(double) * nphys, cudaMemcpyDeviceToHost, s));
    } else if (dir == 'F') {
        CK(cudaMemcpyAsync(w->phys, in, sizeof(double) * nphys, cudaMemcpyHostToDevice, s));
        launch_x_r2c(dc, w->px, w->tc.root_x, w->phys, w->G, s, true);
        launch_z_forward(dc, w->pz, w->tc.root_z, w->G, w->F, 1, s, true);
        launch_yanalysis(dc, w->tc, w->F, w->pd, 1, s);
        CK(cudaGetLastError());
        CK(cudaMemcpyAsync(out, w->pd, sizeof(double2) * d.Ns, cudaMemcpyDeviceToHost, s));
    } else {
        return fail(CDNS_ERR_ARG, "direction must be 'B' or 'F'");
    }
    CK(cudaStreamSynchronize(s));
    return CDNS_OK;
}

}  // extern "C"
