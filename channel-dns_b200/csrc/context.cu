// cdns context: device state, step orchestration (stream launches and CUDA
// graphs) and the extern "C" entry points declared in include/cdns.h.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "../../include/cdns.h"
#include "context.cuh"

using namespace cdns;

namespace {
thread_local std::string g_error;
}  // namespace

namespace cdns {
int fail(int code, const std::string &msg) {
    g_error = msg;
    return code;
}

// Records the calling thread's last error for cdns_last_error (used by
// entry points defined in other translation units).
int record_error(int code, const char *msg) {
    g_error = msg ? msg : "";
    return code;
}
}  // namespace cdns

namespace {
const char *kStageNames[kStages] = {"curl", "y_synthesis", "z_backward", "x_cross",
                                    "z_forward", "y_analysis", "solve"};
}  // namespace

namespace cdns {
bool plan_fft(int n, FftPlan &p) {
    p.n = n;
    p.nrad = 0;
    int m = n;
    auto push = [&](int r) {
        if (p.nrad >= 12) return false;
        p.radix[p.nrad++] = r;
        return true;
    };
    while (m % 4 == 0) { if (!push(4)) return false; m /= 4; }
    while (m % 2 == 0) { if (!push(2)) return false; m /= 2; }
    for (int q = 3; m > 1; q += 2) {
        while (m % q == 0) {
            if (q > 13 || !push(q)) return false;
            m /= q;
        }
    }
    return true;
}
}  // namespace cdns


namespace {
int upload(cdns_ctx *c, void *dst, const void *src, size_t b) {
    CK(cudaMemcpyAsync(dst, src, b, cudaMemcpyHostToDevice, c->stream));
    return CDNS_OK;
}

}  // namespace

namespace cdns {
void step_coefficients(int it, double dt, double re, double &a0, double &a1, double &b0, double &b1,
                       double &g) {
    // src/sim/simulation.cpp:36-45
    const int eff = it < 3 ? it : 2;
    a0 = (double)eff / dt;
    a1 = (double)(1 - eff) / (2.0 * dt);
    b0 = (double)eff;
    b1 = (double)(1 - eff);
    g = (a0 + a1) * re;
}

void enqueue_nonlinear(cdns_ctx *c, const double2 *u, double2 *N, bool prof, int step_slot, double2 *G_fp64) {
    const Dims &d = c->d;
    cudaStream_t s = c->stream;
    auto mark = [&](int stage) {
        if (prof) cudaEventRecord(c->ev[(size_t)step_slot * (kStages + 1) + stage], s);
    };
    mark(0);
    launch_curl(d, c->t, u, c->om, c->bw, c->pp.Re, s);
    mark(1);
    if (c->mixed) {
        float2 *F = reinterpret_cast<float2 *>(c->F), *G = reinterpret_cast<float2 *>(c->G);
        float2 *H = reinterpret_cast<float2 *>(c->H);
        launch_ysynth(d, c->t, u, c->om, 3, 6, F, c->mean, s);
        mark(2);
        launch_z_backward(d, c->t.root_z, F, G, 6, s);
        mark(3);
        launch_x_cross(d, c->t.root_x, G, H, c->mean, s);
        mark(4);
        launch_z_forward(d, c->t.root_z, H, F, 3, s);
        mark(5);
        launch_yanalysis(d, c->t, F, N, 3, s);
        launch_mean_products(d, c->t, c->mean, N, s);
        mark(6);
        return;
    }
    double2 *G = G_fp64 ? G_fp64 : c->G;
    launch_ysynth(d, c->t, u, c->om, 3, 6, c->F, s);
    mark(2);
    launch_z_backward(d, c->pz, c->t.root_z, c->F, G, 6, s);
    mark(3);
    launch_x_cross(d, c->px, c->t.root_x, G, c->H, s);
    mark(4);
    launch_z_forward(d, c->pz, c->t.root_z, c->H, c->F, 3, s);
    mark(5);
    launch_yanalysis(d, c->t, c->F, N, 3, s);
    mark(6);
}

}  // namespace cdns

namespace cdns {
void enqueue_solve(cdns_ctx *c, double a0, double a1, double b0, double b1, double g_v) {
    const int k = c->cur;
    StepArgs a{};
    a.u = c->U[k];
    a.u_prev = c->U[1 - k];
    a.N = c->Nb[k];
    a.N_prev = c->Nb[1 - k];
    a.bw = c->bw;
    a.B_prev = c->Bb[1 - k];
    a.B_new = c->Bb[k];
    a.bc_v = c->bc_v;
    a.u_out = c->U[1 - k];
    a.p_out = c->p;
    a.dpdx = c->dpdx;
    a.err = c->err;
    a.a0 = a0;
    a.a1 = a1;
    a.b0 = b0;
    a.b1 = b1;
    launch_step_solve(c->d, c->t, c->pp, g_v, c->st, a, c->stream);
}

int require_whole(const cdns_ctx *c) {
    if (c && c->pen) return fail(CDNS_ERR_STATE, "a pencil rank context holds one kx block: use cdns_pencil_stage");
    return CDNS_OK;
}
}  // namespace cdns

namespace {
void enqueue_step_body(cdns_ctx *c, double a0, double a1, double b0, double b1, double g_v,
                       bool prof, int slot) {
    enqueue_nonlinear(c, c->U[c->cur], c->Nb[c->cur], prof, slot);
    enqueue_solve(c, a0, a1, b0, b1, g_v);
    if (prof) cudaEventRecord(c->ev[(size_t)slot * (kStages + 1) + kStages], c->stream);
}

}  // namespace

namespace cdns {
int do_setup(cdns_ctx *c, double g_v) {
    if (c->g_setup == g_v) return CDNS_OK;  // deterministic: same g gives the same state
    setup_solver(c->d, c->t, c->pp, g_v, c->st, nullptr, c->stream);
    CK(cudaGetLastError());
    c->g_setup = g_v;
    return CDNS_OK;
}

}  // namespace cdns

namespace cdns {
int one_step(cdns_ctx *c, int it) {
    if (!c->have_velocity) return fail(CDNS_ERR_STATE, "cdns_step before cdns_set_velocity");
    if (it < 1) return fail(CDNS_ERR_ARG, "iteration must be >= 1");
    double a0, a1, b0, b1, g;
    step_coefficients(it, c->DT, c->pp.Re, a0, a1, b0, b1, g);
    // EqSolvePV::setup runs at it = 1, 2 (src/sim/simulation.cpp:176-177); later
    // steps reuse the it = 2 state, whose g equals theirs.  Re-running setup
    // whenever the stored g differs keeps that invariant after cdns_solve.
    {
        int r = do_setup(c, g);
        if (r) return r;
    }
    if (c->prof) {
        if (c->prof_steps >= kMaxProfSteps) return fail(CDNS_ERR_STATE, "profiling window full");
        enqueue_step_body(c, a0, a1, b0, b1, g, true, c->prof_steps);
        c->prof_steps++;
    } else if (it >= 3) {
        cudaGraphExec_t &ge = c->graph[c->cur];
        if (!ge) {
            cudaGraph_t graph;
            CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
            enqueue_step_body(c, a0, a1, b0, b1, g, false, 0);
            CK(cudaStreamEndCapture(c->stream, &graph));
            CK(cudaGraphInstantiate(&ge, graph, 0));
            CK(cudaGraphDestroy(graph));
        }
        CK(cudaGraphLaunch(ge, c->stream));
    } else {
        enqueue_step_body(c, a0, a1, b0, b1, g, false, 0);
    }
    CK(cudaGetLastError());
    c->cur = 1 - c->cur;
    return CDNS_OK;
}

}  // namespace cdns

namespace {
// cdns_create's body; ranks > 1 (or ranks = 1 through cdns_pencil_create)
// makes rank `rank` of a pencil decomposition: the spectral state of one kx
// block plus the y-slab stage buffers (pencil.cu).
int create_context(const cdns_mesh_desc *m, const cdns_params *p, int precision, int device, int ranks,
                   int rank, cdns_ctx **out) {
    if (!m || !p || !out) return fail(CDNS_ERR_ARG, "null argument");
    *out = nullptr;
    if (precision != CDNS_PRECISION_FP64 && precision != CDNS_PRECISION_MIXED)
        return fail(CDNS_ERR_ARG, "unsupported precision mode");
    if (ranks > 0 && precision != CDNS_PRECISION_FP64)
        return fail(CDNS_ERR_ARG, "pencil ranks run the FP64 step");
    if (m->NYS < 4 || m->NXS < 0 || m->NZS < 0 || m->NY2 < m->NYS || m->NY2 < 2 ||
        m->NX2 < 2 * m->NXS || m->NZ2 < 2 * m->NZS || m->NX2 < 1 || m->NZ2 < 1 ||
        !(m->XL > 0) || !(m->ZL > 0))
        return fail(CDNS_ERR_ARG, "invalid mesh: need NYS>=4, NY2>=NYS, NX2>=2 NXS, NZ2>=2 NZS");
    // the column solve keeps a column's NYS+1 coefficients in one warp's registers
    if (m->NYS > 255) return fail(CDNS_ERR_ARG, "invalid mesh: NYS must be at most 255");
    if (!(p->DT > 0.0) || !(p->Re > 0.0)) return fail(CDNS_ERR_ARG, "DT and Re must be positive");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
        return fail(CDNS_ERR_CUDA, "no CUDA device available");
    if (device < 0 || device >= ndev) return fail(CDNS_ERR_ARG, "bad device index");
    DeviceGuard guard(device);
    cdns_ctx *c = new (std::nothrow) cdns_ctx();
    if (!c) return fail(CDNS_ERR_NOMEM, "host allocation failed");
    c->device = device;
    c->mesh = *m;
    Dims &d = c->d;
    d.NX2 = m->NX2; d.NY2 = m->NY2; d.NZ2 = m->NZ2;
    d.NXS = m->NXS; d.NYS = m->NYS; d.NZS = m->NZS;
    d.nkx = m->NXS + 1; d.nkz = 2 * m->NZS + 1; d.ncy = m->NYS + 1; d.ny2 = m->NY2 + 1;
    d.kx0 = 0;
    if (ranks > 0) {
        int j0, nj;
        if (int r = pencil_blocks(*m, ranks, rank, d.kx0, d.nkx, j0, nj)) {
            delete c;
            return r;
        }
    }
    d.ncol = d.nkx * d.nkz;
    d.zc = d.kx0 == 0 ? d.NZS * d.nkx : -1;
    d.nyh = m->NY2 / 2 + 1;
    d.Ns = (long long)d.nkz * d.ncy * d.nkx;
    if (!plan_fft(d.NX2, c->px) || !plan_fft(d.NZ2, c->pz)) {
        delete c;
        return fail(CDNS_ERR_ARG, "NX2/NZ2 must factor into primes <= 13");
    }
    // step solve tiles [4][ncy][8] complex; Stockham z/x FFT blocks of up to 17 and 12 lines
    const size_t smem_solve = 16 * 4 * (size_t)d.ncy * 8;
    if (smem_solve > 220 * 1024 || (size_t)16 * d.NZ2 * 35 > 220 * 1024 ||
        (size_t)16 * d.NX2 * 25 > 220 * 1024) {
        delete c;
        return fail(CDNS_ERR_ARG, "mesh exceeds the shared-memory tiling limits");
    }
    if (precision == CDNS_PRECISION_MIXED && !register_forms(d)) {
        delete c;
        return fail(CDNS_ERR_ARG, "mixed precision needs NX2 and NZ2 in {32, 48, 64, 72, 96, 128, 144, 192, 196}");
    }
    c->mixed = precision == CDNS_PRECISION_MIXED;
    d.fcol = c->mixed ? d.ncol + (d.ncol & 1) : d.ncol;
    // physics parameters (src/core/params.cpp:296-307)
    PhysParams &pp = c->pp;
    pp.Re = p->Re; pp.G_pre = p->G_pre; pp.a_pre0 = p->a_pre0; pp.b_pre0 = p->b_pre0;
    for (int i = 0; i < 3; ++i) { pp.a_V[i] = p->a_V[i]; pp.b_V[i] = p->b_V[i]; }
    pp.grad_pre = p->INDEX_GRAD_PRE;
    const double pi = std::acos(-1.0);
    const double th = p->THETA * pi / 180.0;
    if (p->INDEX_GRAD_PRE == 1) {
        pp.gx = -std::cos(th); pp.gz = -std::sin(th); pp.qxm = pp.qzm = 0.0;
    } else {
        pp.qxm = std::cos(th); pp.qzm = std::sin(th); pp.gx = pp.gz = 0.0;
    }
    c->DT = p->DT;
    int r = 0;
    auto bail = [&](int code) { cdns_destroy(c); return code; };
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess)
        return bail(fail(CDNS_ERR_CUDA, "stream creation failed"));
    // ---- tables (src/fft/transforms.cpp:71-108) ----
    std::vector<double> wavx(d.nkx), wavz(d.nkz), WL(d.ncy, 0.0), WD(d.ncy, 0.0), WR(d.ncy, 0.0),
        cosy(2 * (size_t)d.NY2);
    const double alx = 2.0 * pi / m->XL, alz = 2.0 * pi / m->ZL;
    for (int k = 0; k < d.nkx; ++k) wavx[k] = (d.kx0 + k) * alx;
    for (int k = -d.NZS; k <= d.NZS; ++k) wavz[k + d.NZS] = k * alz;
    const int n = d.NYS;
    for (int iy = n; iy >= 2; --iy) {
        WL[iy] = 1.0 / (4.0 * iy * (iy - 1));
        WD[iy] = -1.0 / (2.0 * (iy * iy - 1));
        WR[iy] = 1.0 / (4.0 * iy * (iy + 1));
    }
    WL[2] = 2.0 * WL[2];
    for (int iy = n - 1; iy <= n; ++iy) WD[iy] = 0.0;
    for (int iy = n - 3; iy <= n; ++iy) WR[iy] = 0.0;
    const long double pil = 3.141592653589793238462643383279502884L;
    for (int mm = 0; mm < 2 * d.NY2; ++mm) {
        if (2 * mm == d.NY2 || 2 * mm == 3 * d.NY2) cosy[mm] = 0.0;
        else cosy[mm] = (double)cosl(pil * (long double)mm / (long double)d.NY2);
    }
    auto roots = [&](int nn) {
        std::vector<double2> rr(nn);
        for (int k = 0; k < nn; ++k) {
            const long double a = 2.0L * pil * (long double)k / (long double)nn;
            rr[k] = make_double2((double)cosl(a), (double)(-sinl(a)));
        }
        return rr;
    };
    const auto rx = roots(d.NX2), rz = roots(d.NZ2), ry = roots(d.NY2);
    double *tab = nullptr;
    // every table starts on a 256-byte boundary (double2 tables need 16)
    auto rup = [](size_t n) { return (n + 31) / 32 * 32; };
    const size_t ntab = rup(d.nkx) + rup(d.nkz) + 3 * rup(d.ncy) + rup(cosy.size()) +
                        rup(2 * (size_t)d.NX2) + rup(2 * (size_t)d.NZ2) + rup(2 * (size_t)d.NY2);
    if ((r = c->alloc(tab, ntab))) return bail(r);
    size_t o = 0;
    auto put = [&](const void *src, size_t count) {
        double *dst = tab + o;
        o += rup(count);
        return std::make_pair(dst, upload(c, dst, src, count * sizeof(double)));
    };
    auto pw = put(wavx.data(), wavx.size()); c->t.wavx = pw.first;
    auto pz = put(wavz.data(), wavz.size()); c->t.wavz = pz.first;
    auto pl = put(WL.data(), WL.size()); c->t.WL = pl.first;
    auto pd = put(WD.data(), WD.size()); c->t.WD = pd.first;
    auto pr = put(WR.data(), WR.size()); c->t.WR = pr.first;
    auto pc = put(cosy.data(), cosy.size()); c->t.cosy = pc.first;
    auto px = put(rx.data(), 2 * rx.size()); c->t.root_x = reinterpret_cast<const double2 *>(px.first);
    auto pzz = put(rz.data(), 2 * rz.size()); c->t.root_z = reinterpret_cast<const double2 *>(pzz.first);
    auto pyy = put(ry.data(), 2 * ry.size()); c->t.root_y = reinterpret_cast<const double2 *>(pyy.first);

    if (pw.second || pz.second || pl.second || pd.second || pr.second || pc.second || px.second || pzz.second ||
        pyy.second)
        return bail(CDNS_ERR_CUDA);
    {
        size_t nsyn, nana;
        cheb_table_sizes(d, &nsyn, &nana);
        double *csyn = nullptr, *cana = nullptr;
        if ((r = c->alloc(csyn, nsyn)) || (r = c->alloc(cana, nana))) return bail(r);
        launch_cheb_tables(d, c->t.cosy, csyn, cana, c->stream);
        c->t.csyn = csyn;
        c->t.cana = cana;
    }
    // ---- state and workspaces ----
    const size_t Ns = (size_t)d.Ns, nc = d.ncol;
    const size_t fbuf = 6 * (size_t)d.ny2 * nc;
    const size_t gbuf = 6 * (size_t)d.ny2 * d.NZ2 * d.nkx;
    const size_t hbuf = 3 * (size_t)d.ny2 * d.NZ2 * d.nkx;
    if ((r = c->alloc(c->U[0], 3 * Ns)) || (r = c->alloc(c->U[1], 3 * Ns)) ||
        (r = c->alloc(c->Nb[0], 3 * Ns)) || (r = c->alloc(c->Nb[1], 3 * Ns)) ||
        (r = c->alloc(c->Bb[0], 2 * nc)) || (r = c->alloc(c->Bb[1], 2 * nc)) ||
        (r = c->alloc(c->p, Ns)) || (r = c->alloc(c->bw, 2 * nc)) || (r = c->alloc(c->bc_v, 6 * nc)) ||
        (r = c->alloc(c->bc_p, 2 * nc)) || (r = c->alloc(c->F, fbuf)) || (r = c->alloc(c->G, gbuf)) ||
        (r = c->alloc(c->H, hbuf)) || (r = c->alloc(c->aux, 3 * Ns)) || (r = c->alloc(c->aux2, 3 * Ns)) ||
        (r = c->alloc(c->zero3, 3 * Ns)) || (r = c->alloc(c->om, 3 * Ns)) ||
        (r = c->alloc(c->mean, 6 * (size_t)d.ny2)) ||
        (r = c->alloc(c->phys, (size_t)d.NZ2 * d.ny2 * d.NX2)) || (r = c->alloc(c->dpdx, 2)) ||
        (r = c->alloc(c->err, 1)))
        return bail(r);
    SolverState &st = c->st;
    if ((r = c->alloc(st.wn_p, nc)) || (r = c->alloc(st.wn_v, nc)) || (r = c->alloc(st.ad_p, Ns)) ||
        (r = c->alloc(st.ad_v, Ns)) || (r = c->alloc(st.p_inf, 2 * Ns)) || (r = c->alloc(st.v_inf, 6 * Ns)) ||
        (r = c->alloc(st.inf_div, 4 * nc)) || (r = c->alloc(st.p_b, Ns)) || (r = c->alloc(st.v_b, 3 * Ns)) ||
        (r = c->alloc(st.sigma0, 2 * nc)) || (r = c->alloc(st.unit, 2 * (size_t)d.ncy + 2)))
        return bail(r);
    cudaError_t e = configure_transform_kernels(d);
    if (e == cudaSuccess) e = configure_cheb_kernels(d);
    if (e == cudaSuccess) e = configure_solver_kernels(d);
    if (e != cudaSuccess) return bail(fail(CDNS_ERR_CUDA, cudaGetErrorString(e)));
    // velocity_boundary (src/sim/initial_bc.cpp:95-101): v = V_Microblow0 on the zero mode
    std::vector<double2> bc(6 * nc, make_double2(0, 0));
    if (d.zc >= 0) {
        bc[(2 * 1 + 0) * nc + d.zc] = make_double2(p->V_Microblow0, 0.0);
        bc[(2 * 1 + 1) * nc + d.zc] = make_double2(p->V_Microblow0, 0.0);
    }
    if ((r = upload(c, c->bc_v, bc.data(), bc.size() * sizeof(double2)))) return bail(r);
    if (ranks > 0 && (r = pencil_init(c, ranks, rank))) return bail(r);
    if ((r = tune_context(c, false))) return bail(r);
    if (cudaStreamSynchronize(c->stream) != cudaSuccess) return bail(fail(CDNS_ERR_CUDA, "sync"));
    *out = c;
    return CDNS_OK;
}
}  // namespace

extern "C" {

int cdns_create(const cdns_mesh_desc *m, const cdns_params *p, int precision, int device,
                cdns_ctx **out) {
    return create_context(m, p, precision, device, 0, 0, out);
}

int cdns_pencil_create(const cdns_mesh_desc *m, const cdns_params *p, int ranks, int rank, int device,
                       cdns_ctx **out) {
    if (ranks < 1) return fail(CDNS_ERR_ARG, "ranks must be >= 1");
    return create_context(m, p, CDNS_PRECISION_FP64, device, ranks, rank, out);
}

int cdns_destroy(cdns_ctx *c) {
    if (!c) return CDNS_OK;
    DeviceGuard guard(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    for (auto &g : c->graph)
        if (g) cudaGraphExecDestroy(g);
    for (auto ev : c->ev) cudaEventDestroy(ev);
    adjoint_release(c->adj);
    output_release(c->outw);
    pencil_release(c->pen);
    for (void *p : c->allocs) cudaFree(p);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
    return CDNS_OK;
}

int cdns_set_velocity_device(cdns_ctx *c, const double *v) {
    if (!c || !v) return fail(CDNS_ERR_ARG, "null argument");
    DeviceGuard guard(c->device);
    const Dims &d = c->d;
    c->cur = 0;
    launch_deinterleave(reinterpret_cast<const double2 *>(v), c->U[0], d.Ns, 3, c->stream);
    CK(cudaMemsetAsync(c->U[1], 0, sizeof(double2) * 3 * d.Ns, c->stream));
    CK(cudaMemsetAsync(c->Nb[0], 0, sizeof(double2) * 3 * d.Ns, c->stream));
    CK(cudaMemsetAsync(c->Nb[1], 0, sizeof(double2) * 3 * d.Ns, c->stream));
    CK(cudaMemsetAsync(c->Bb[0], 0, sizeof(double2) * 2 * d.ncol, c->stream));
    CK(cudaMemsetAsync(c->Bb[1], 0, sizeof(double2) * 2 * d.ncol, c->stream));
    CK(cudaGetLastError());
    c->have_velocity = true;
    return CDNS_OK;
}

int cdns_set_velocity(cdns_ctx *c, const double *v) {
    if (!c || !v) return fail(CDNS_ERR_ARG, "null argument");
    DeviceGuard guard(c->device);
    CK(cudaMemcpyAsync(c->aux, v, sizeof(double2) * 3 * c->d.Ns, cudaMemcpyHostToDevice, c->stream));
    int r = cdns_set_velocity_device(c, reinterpret_cast<const double *>(c->aux));
    if (r) return r;
    CK(cudaStreamSynchronize(c->stream));
    return CDNS_OK;
}

int cdns_update_velocity(cdns_ctx *c, const double *v) {
    if (!c || !v) return fail(CDNS_ERR_ARG, "null argument");
    if (int r = require_whole(c)) return r;
    if (!c->have_velocity) return fail(CDNS_ERR_STATE, "cdns_update_velocity before cdns_set_velocity");
    DeviceGuard guard(c->device);
    CK(cudaMemcpyAsync(c->aux, v, sizeof(double2) * 3 * c->d.Ns, cudaMemcpyHostToDevice, c->stream));
    // the current slot only: u_prev, N_prev and B_prev of the multistep history stay
    launch_deinterleave(reinterpret_cast<const double2 *>(c->aux), c->U[c->cur], c->d.Ns, 3, c->stream);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(c->stream));
    return CDNS_OK;
}

int cdns_get_velocity_device(cdns_ctx *c, double *v) {
    if (!c || !v) return fail(CDNS_ERR_ARG, "null argument");
    if (!c->have_velocity) return fail(CDNS_ERR_STATE, "no velocity set");
    DeviceGuard guard(c->device);
    launch_interleave(c->U[c->cur], reinterpret_cast<double2 *>(v), c->d.Ns, 3, c->stream);
    CK(cudaGetLastError());
    return CDNS_OK;
}

int cdns_get_velocity(cdns_ctx *c, double *v) {
    if (!c || !v) return fail(CDNS_ERR_ARG, "null argument");
    int r = cdns_get_velocity_device(c, reinterpret_cast<double *>(c->aux2));
    if (r) return r;
    DeviceGuard guard(c->device);
    CK(cudaMemcpyAsync(v, c->aux2, sizeof(double2) * 3 * c->d.Ns, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return CDNS_OK;
}

int cdns_get_pressure(cdns_ctx *c, double *p) {
    if (!c || !p) return fail(CDNS_ERR_ARG, "null argument");
    DeviceGuard guard(c->device);
    CK(cudaMemcpyAsync(p, c->p, sizeof(double2) * c->d.Ns, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return CDNS_OK;
}

int cdns_set_pressure(cdns_ctx *c, const double *p) {
    if (!c || !p) return fail(CDNS_ERR_ARG, "null argument");
    DeviceGuard guard(c->device);
    CK(cudaMemcpyAsync(c->p, p, sizeof(double2) * c->d.Ns, cudaMemcpyHostToDevice, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return CDNS_OK;
}

int cdns_set_velocity_bc(cdns_ctx *c, const double *bc) {
    if (!c || !bc) return fail(CDNS_ERR_ARG, "null argument");
    DeviceGuard guard(c->device);
    const Dims &d = c->d;
    const size_t nc = d.ncol;
    std::vector<double2> v(6 * nc);
    const double2 *src = reinterpret_cast<const double2 *>(bc);
    for (int kz = 0; kz < d.nkz; ++kz)
        for (int w = 0; w < 2; ++w)
            for (int kx = 0; kx < d.nkx; ++kx)
                for (int comp = 0; comp < 3; ++comp)
                    v[(2 * comp + w) * nc + (size_t)kz * d.nkx + kx] =
                        src[(((size_t)kz * 2 + w) * d.nkx + kx) * 3 + comp];
    CK(cudaMemcpyAsync(c->bc_v, v.data(), v.size() * sizeof(double2), cudaMemcpyHostToDevice, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return CDNS_OK;
}

int cdns_step(cdns_ctx *c, int iteration) {
    if (!c) return fail(CDNS_ERR_ARG, "null context");
    if (int r = require_whole(c)) return r;
    DeviceGuard guard(c->device);
    return one_step(c, iteration);
}

int cdns_run(cdns_ctx *c, int first, int nsteps) {
    if (!c) return fail(CDNS_ERR_ARG, "null context");
    if (int r = require_whole(c)) return r;
    if (nsteps < 0) return fail(CDNS_ERR_ARG, "negative step count");
    DeviceGuard guard(c->device);
    for (int i = 0; i < nsteps; ++i) {
        int r = one_step(c, first + i);
        if (r) return r;
    }
    return CDNS_OK;
}

int cdns_synchronize(cdns_ctx *c) {
    if (!c) return fail(CDNS_ERR_ARG, "null context");
    DeviceGuard guard(c->device);
    CK(cudaStreamSynchronize(c->stream));
    unsigned e = 0;
    CK(cudaMemcpyAsync(&e, c->err, sizeof(unsigned), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    if (e) {
        CK(cudaMemsetAsync(c->err, 0, sizeof(unsigned), c->stream));
        CK(cudaStreamSynchronize(c->stream));
        if (e & ERR_NONFINITE) return fail(CDNS_ERR_NONFINITE, "non-finite value in the step output");
        return fail(CDNS_ERR_PIVOT, "zero or non-finite tau pivot or flow response");
    }
    return CDNS_OK;
}

int cdns_get_dpdx(cdns_ctx *c, double out[2]) {
    if (!c || !out) return fail(CDNS_ERR_ARG, "null argument");
    DeviceGuard guard(c->device);
    CK(cudaMemcpyAsync(out, c->dpdx, 2 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return CDNS_OK;
}

int cdns_nonlinear(cdns_ctx *c, const double *velocity, double *nl, double *pbc) {
    if (!c || !velocity || !nl) return fail(CDNS_ERR_ARG, "null argument");
    if (int r = require_whole(c)) return r;
    DeviceGuard guard(c->device);
    const Dims &d = c->d;
    CK(cudaMemcpyAsync(c->aux2, velocity, sizeof(double2) * 3 * d.Ns, cudaMemcpyHostToDevice, c->stream));
    launch_deinterleave(c->aux2, c->aux, d.Ns, 3, c->stream);
    enqueue_nonlinear(c, c->aux, c->aux2, false, 0);
    launch_pressure_bc(d, c->aux2, c->bw, c->bc_p, c->stream);
    launch_interleave(c->aux2, c->aux, d.Ns, 3, c->stream);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(nl, c->aux, sizeof(double2) * 3 * d.Ns, cudaMemcpyDeviceToHost, c->stream));
    std::vector<double2> b(2 * (size_t)d.ncol);
    CK(cudaMemcpyAsync(b.data(), c->bc_p, b.size() * sizeof(double2), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    if (pbc) {
        double2 *o = reinterpret_cast<double2 *>(pbc);
        for (int kz = 0; kz < d.nkz; ++kz)
            for (int w = 0; w < 2; ++w)
                for (int kx = 0; kx < d.nkx; ++kx)
                    o[((size_t)kz * 2 + w) * d.nkx + kx] = b[(size_t)w * d.ncol + (size_t)kz * d.nkx + kx];
    }
    return CDNS_OK;
}

int cdns_transform_fine(cdns_ctx *c, int dir, const double *in, double *out) {
    if (!c || !in || !out) return fail(CDNS_ERR_ARG, "null argument");
    if (int r = require_whole(c)) return r;
    DeviceGuard guard(c->device);
    const Dims &d = c->d;
    const size_t nphys = (size_t)d.NZ2 * d.ny2 * d.NX2;
    if (dir == 'B') {
        CK(cudaMemcpyAsync(c->aux, in, sizeof(double2) * d.Ns, cudaMemcpyHostToDevice, c->stream));
        launch_ysynth(d, c->t, c->aux, nullptr, 1, 1, c->F, c->stream);
        launch_z_backward(d, c->pz, c->t.root_z, c->F, c->G, 1, c->stream);
        launch_x_c2r(d, c->px, c->t.root_x, c->G, c->phys, c->stream);
        CK(cudaGetLastError());
        CK(cudaMemcpyAsync(out, c->phys, sizeof(double) * nphys, cudaMemcpyDeviceToHost, c->stream));
    } else if (dir == 'F') {
        CK(cudaMemcpyAsync(c->phys, in, sizeof(double) * nphys, cudaMemcpyHostToDevice, c->stream));
        launch_x_r2c(d, c->px, c->t.root_x, c->phys, c->H, c->stream);
        launch_z_forward(d, c->pz, c->t.root_z, c->H, c->F, 1, c->stream);
        launch_yanalysis(d, c->t, c->F, c->aux, 1, c->stream);
        CK(cudaGetLastError());
        CK(cudaMemcpyAsync(out, c->aux, sizeof(double2) * d.Ns, cudaMemcpyDeviceToHost, c->stream));
    } else {
        return fail(CDNS_ERR_ARG, "direction must be 'B' or 'F'");
    }
    CK(cudaStreamSynchronize(c->stream));
    return CDNS_OK;
}

int cdns_solve(cdns_ctx *c, double g, const double *rhs, const double *pbc, const double *vbc,
               double *pressure, double *velocity, double *units) {
    if (!c || !rhs || !pbc || !vbc || !pressure || !velocity) return fail(CDNS_ERR_ARG, "null argument");
    DeviceGuard guard(c->device);
    const Dims &d = c->d;
    const size_t nc = d.ncol;
    int r = do_setup(c, g);
    if (r) return r;
    // velocity BC and pressure BC into solver layouts
    std::vector<double2> bv(6 * nc), bp(2 * nc);
    const double2 *sv = reinterpret_cast<const double2 *>(vbc);
    const double2 *sp = reinterpret_cast<const double2 *>(pbc);
    for (int kz = 0; kz < d.nkz; ++kz)
        for (int w = 0; w < 2; ++w)
            for (int kx = 0; kx < d.nkx; ++kx) {
                const size_t col = (size_t)kz * d.nkx + kx;
                bp[w * nc + col] = sp[((size_t)kz * 2 + w) * d.nkx + kx];
                for (int comp = 0; comp < 3; ++comp)
                    bv[(2 * comp + w) * nc + col] = sv[(((size_t)kz * 2 + w) * d.nkx + kx) * 3 + comp];
            }
    double2 *dbv = c->G, *dbp = c->G + 6 * nc;
    CK(cudaMemcpyAsync(dbv, bv.data(), bv.size() * sizeof(double2), cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(dbp, bp.data(), bp.size() * sizeof(double2), cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(c->aux2, rhs, sizeof(double2) * 3 * d.Ns, cudaMemcpyHostToDevice, c->stream));
    launch_deinterleave(c->aux2, c->aux, d.Ns, 3, c->stream);
    const double2 *zero = c->zero3;  // zeros for the unused history terms
    StepArgs a{};
    a.u = c->aux;
    a.u_prev = zero;
    a.N = zero;
    a.N_prev = zero;
    a.bw = c->bw;
    a.B_prev = c->bc_p;
    a.B_new = c->bc_p;
    a.bc_v = dbv;
    a.bc_p = dbp;
    a.u_out = c->aux2;
    a.p_out = c->F;
    a.dpdx = c->dpdx;
    a.err = c->err;
    a.a0 = 1.0;
    a.solve_only = 1;
    launch_step_solve(d, c->t, c->pp, g, c->st, a, c->stream);
    launch_interleave(c->aux2, c->aux, d.Ns, 3, c->stream);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(velocity, c->aux, sizeof(double2) * 3 * d.Ns, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaMemcpyAsync(pressure, c->F, sizeof(double2) * d.Ns, cudaMemcpyDeviceToHost, c->stream));
    if (units) CK(cudaMemcpyAsync(units, c->st.unit, sizeof(double) * 2 * d.ncy, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return CDNS_OK;
}

int cdns_profile_begin(cdns_ctx *c) {
    if (!c) return fail(CDNS_ERR_ARG, "null context");
    if (int r = require_whole(c)) return r;
    DeviceGuard guard(c->device);
    if (c->ev.empty()) {
        c->ev.resize((size_t)kMaxProfSteps * (kStages + 1));
        for (auto &e : c->ev) CK(cudaEventCreate(&e));
    }
    c->prof = true;
    c->prof_steps = 0;
    return CDNS_OK;
}

int cdns_profile_end(cdns_ctx *c, double *stage_ms, int *nsteps) {
    if (!c || !stage_ms) return fail(CDNS_ERR_ARG, "null argument");
    DeviceGuard guard(c->device);
    CK(cudaStreamSynchronize(c->stream));
    for (int s = 0; s < kStages; ++s) stage_ms[s] = 0.0;
    for (int i = 0; i < c->prof_steps; ++i)
        for (int s = 0; s < kStages; ++s) {
            float ms = 0.f;
            CK(cudaEventElapsedTime(&ms, c->ev[(size_t)i * (kStages + 1) + s],
                                    c->ev[(size_t)i * (kStages + 1) + s + 1]));
            stage_ms[s] += ms;
        }
    if (nsteps) *nsteps = c->prof_steps;
    c->prof = false;
    c->prof_steps = 0;
    return CDNS_OK;
}

int cdns_stage_count(void) { return kStages; }
const char *cdns_stage_name(int s) { return (s >= 0 && s < kStages) ? kStageNames[s] : ""; }

int cdns_debug_copy(cdns_ctx *c, int which, double *out, size_t count) {
    if (!c || !out) return fail(CDNS_ERR_ARG, "null argument");
    DeviceGuard guard(c->device);
    const Dims &d = c->d;
    const void *src = nullptr;
    size_t n = 0;
    switch (which) {
    case 0: src = c->F; n = 6 * (size_t)d.ny2 * d.ncol; break;
    case 1: src = c->G; n = 6 * (size_t)d.ny2 * d.NZ2 * d.nkx; break;
    case 2: src = c->H; n = 3 * (size_t)d.ny2 * d.NZ2 * d.nkx; break;
    case 3: src = c->bw; n = 2 * (size_t)d.ncol; break;
    case 4: {
        if (count < 7) return fail(CDNS_ERR_ARG, "debug buffer too small");
        CK(cudaStreamSynchronize(c->stream));
        auto nonfinite = [&](const void *p, size_t ndbl, double &out) -> int {
            std::vector<double> h(ndbl);
            CK(cudaMemcpyAsync(h.data(), p, ndbl * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
            CK(cudaStreamSynchronize(c->stream));
            size_t k = 0;
            for (double v : h) k += !std::isfinite(v);
            out = (double)k;
            return CDNS_OK;
        };
        const SolverState &st = c->st;
        const size_t Ns = (size_t)d.Ns, nc = d.ncol;
        int r;
        if ((r = nonfinite(st.ad_p, Ns, out[0])) || (r = nonfinite(st.ad_v, Ns, out[1])) ||
            (r = nonfinite(st.inf_div, 8 * nc, out[2])) || (r = nonfinite(st.sigma0, 4 * nc, out[3])) ||
            (r = nonfinite(st.p_inf, 2 * Ns, out[4])) || (r = nonfinite(st.v_b, 3 * Ns, out[5])) ||
            (r = nonfinite(st.unit, 2 * (size_t)d.ncy + 2, out[6])))
            return r;
        return CDNS_OK;
    }
    case 5: src = c->st.inf_div; n = 4 * (size_t)d.ncol; break;
    case 6:
    case 7: {
        // stored by their nonzero parts: returned as complex values
        n = (which == 6 ? 6 : 2) * (size_t)d.Ns;
        if (count < 2 * n) return fail(CDNS_ERR_ARG, "debug buffer too small");
        std::vector<double> h(n);
        CK(cudaMemcpyAsync(h.data(), which == 6 ? c->st.v_inf : c->st.p_inf, n * sizeof(double),
                           cudaMemcpyDeviceToHost, c->stream));
        CK(cudaStreamSynchronize(c->stream));
        for (size_t i = 0; i < n; ++i) {
            const int comp = which == 6 ? (int)((i / (size_t)d.Ns) % 3) : 1;
            out[2 * i] = inf_imag(comp) ? 0.0 : h[i];
            out[2 * i + 1] = inf_imag(comp) ? h[i] : 0.0;
        }
        return CDNS_OK;
    }
    case 8: src = c->st.sigma0; n = 2 * (size_t)d.ncol; break;
    case 9: src = c->st.wn_p; n = (size_t)d.ncol; break;   // wn_p then wn_v as [2][ncol] doubles
    default: return fail(CDNS_ERR_ARG, "unknown debug buffer");
    }
    if (count < 2 * n) return fail(CDNS_ERR_ARG, "debug buffer too small");
    if (c->mixed && which <= 2) {
        // FP32 stage buffers: widen on the host (F rows are padded to fcol columns)
        const size_t row = which == 0 ? (size_t)d.ncol : n, prow = which == 0 ? (size_t)d.fcol : n;
        const size_t rows = n / row;
        std::vector<float2> h(rows * prow);
        CK(cudaMemcpyAsync(h.data(), src, h.size() * sizeof(float2), cudaMemcpyDeviceToHost, c->stream));
        CK(cudaStreamSynchronize(c->stream));
        for (size_t r = 0; r < rows; ++r)
            for (size_t i = 0; i < row; ++i) {
                out[2 * (r * row + i)] = h[r * prow + i].x;
                out[2 * (r * row + i) + 1] = h[r * prow + i].y;
            }
        return CDNS_OK;
    }
    if (which == 9) {
        CK(cudaMemcpyAsync(out, c->st.wn_p, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
        CK(cudaMemcpyAsync(out + n, c->st.wn_v, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
        CK(cudaStreamSynchronize(c->stream));
        return CDNS_OK;
    }
    CK(cudaMemcpyAsync(out, src, n * sizeof(double2), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return CDNS_OK;
}

int cdns_get_stream(cdns_ctx *c, void **stream) {
    if (!c || !stream) return fail(CDNS_ERR_ARG, "null argument");
    *stream = (void *)c->stream;
    return CDNS_OK;
}

int cdns_device_bytes(cdns_ctx *c, size_t *b) {
    if (!c || !b) return fail(CDNS_ERR_ARG, "null argument");
    *b = c->bytes + adjoint_bytes(c->adj) + output_bytes(c->outw);
    return CDNS_OK;
}

int cdns_last_error(char *buf, size_t len) {
    if (!buf || !len) return CDNS_ERR_ARG;
    std::snprintf(buf, len, "%s", g_error.c_str());
    return CDNS_OK;
}

const char *cdns_version(void) { return "cdns-b200 0.4 (sm_100a, fp64 + mixed fp32/fp64, batch, discrete adjoint, pencil ranks)"; }

}  // extern "C"

// ---------------------------------------------------------------------------
// Ensemble batch: independent channels (each a full context with its own
// stream, state and graphs) whose steady steps (it >= 3) are captured into
// one CUDA graph: a fork event on the batch stream, every member's step body
// on its own stream as a parallel branch, and a join back to the batch
// stream.  Steps 1 and 2 (setup) run member by member on the member streams.
// ---------------------------------------------------------------------------
struct cdns_batch {
    int device = 0;
    std::vector<cdns_ctx *> members;
    cudaStream_t stream = nullptr;
    cudaEvent_t fork = nullptr, done = nullptr;
    std::vector<cudaEvent_t> join;
    cudaGraphExec_t graph[2] = {nullptr, nullptr};
};

namespace {
// batch stream waits for the members' pending work; members wait for the batch
int batch_order_members_before(cdns_batch *b) {
    for (size_t i = 0; i < b->members.size(); ++i) {
        CK(cudaEventRecord(b->join[i], b->members[i]->stream));
        CK(cudaStreamWaitEvent(b->stream, b->join[i], 0));
    }
    return CDNS_OK;
}
int batch_order_members_after(cdns_batch *b) {
    CK(cudaEventRecord(b->done, b->stream));
    for (cdns_ctx *m : b->members) CK(cudaStreamWaitEvent(m->stream, b->done, 0));
    return CDNS_OK;
}

int batch_step(cdns_batch *b, int it) {
    bool direct = it < 3;
    for (cdns_ctx *m : b->members) {
        if (!m->have_velocity) return fail(CDNS_ERR_STATE, "batch step before every member has a velocity");
        direct = direct || m->prof || m->cur != b->members[0]->cur;
    }
    if (direct) {
        for (cdns_ctx *m : b->members) {
            int r = one_step(m, it);
            if (r) return r;
        }
        return CDNS_OK;
    }
    cudaGraphExec_t &ge = b->graph[b->members[0]->cur];
    if (!ge) {
        cudaGraph_t graph;
        CK(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
        CK(cudaEventRecord(b->fork, b->stream));
        // branches captured largest member first (more spectral values first), so
        // that the long launches start early and the small members fill in
        std::vector<size_t> order(b->members.size());
        for (size_t i = 0; i < order.size(); ++i) order[i] = i;
        std::stable_sort(order.begin(), order.end(), [&](size_t x, size_t y) {
            return b->members[x]->d.Ns > b->members[y]->d.Ns;
        });
        for (size_t i : order) {
            cdns_ctx *m = b->members[i];
            double a0, a1, b0, b1, g;
            step_coefficients(it, m->DT, m->pp.Re, a0, a1, b0, b1, g);
            CK(cudaStreamWaitEvent(m->stream, b->fork, 0));
            enqueue_step_body(m, a0, a1, b0, b1, g, false, 0);
            CK(cudaEventRecord(b->join[i], m->stream));
            CK(cudaStreamWaitEvent(b->stream, b->join[i], 0));
        }
        CK(cudaStreamEndCapture(b->stream, &graph));
        CK(cudaGraphInstantiate(&ge, graph, 0));
        CK(cudaGraphDestroy(graph));
    }
    int r = batch_order_members_before(b);
    if (r) return r;
    CK(cudaGraphLaunch(ge, b->stream));
    r = batch_order_members_after(b);
    if (r) return r;
    for (cdns_ctx *m : b->members) m->cur = 1 - m->cur;
    return CDNS_OK;
}
}  // namespace

extern "C" {

int cdns_batch_create(int n, const cdns_mesh_desc *meshes, const cdns_params *params, int precision, int device,
                      cdns_batch **out) {
    if (!out || n <= 0 || !meshes || !params) return fail(CDNS_ERR_ARG, "bad batch arguments");
    *out = nullptr;
    cdns_batch *b = new (std::nothrow) cdns_batch();
    if (!b) return fail(CDNS_ERR_NOMEM, "host allocation failed");
    b->device = device;
    auto bail = [&](int code) { cdns_batch_destroy(b); return code; };
    for (int i = 0; i < n; ++i) {
        cdns_ctx *m = nullptr;
        int r = cdns_create(&meshes[i], &params[i], precision, device, &m);
        if (r) return bail(r);
        b->members.push_back(m);
    }
    DeviceGuard guard(device);
    if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&b->done, cudaEventDisableTiming) != cudaSuccess)
        return bail(fail(CDNS_ERR_CUDA, "batch stream/event creation failed"));
    b->join.resize(n, nullptr);
    for (auto &e : b->join)
        if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess)
            return bail(fail(CDNS_ERR_CUDA, "batch event creation failed"));
    *out = b;
    return CDNS_OK;
}

int cdns_batch_destroy(cdns_batch *b) {
    if (!b) return CDNS_OK;
    {
        DeviceGuard guard(b->device);
        if (b->stream) cudaStreamSynchronize(b->stream);
        for (auto &g : b->graph)
            if (g) cudaGraphExecDestroy(g);
        for (auto e : b->join)
            if (e) cudaEventDestroy(e);
        if (b->fork) cudaEventDestroy(b->fork);
        if (b->done) cudaEventDestroy(b->done);
        if (b->stream) cudaStreamDestroy(b->stream);
    }
    for (cdns_ctx *m : b->members) cdns_destroy(m);
    delete b;
    return CDNS_OK;
}

int cdns_batch_size(cdns_batch *b, int *n) {
    if (!b || !n) return fail(CDNS_ERR_ARG, "null argument");
    *n = (int)b->members.size();
    return CDNS_OK;
}

int cdns_batch_member(cdns_batch *b, int i, cdns_ctx **ctx) {
    if (!b || !ctx) return fail(CDNS_ERR_ARG, "null argument");
    if (i < 0 || i >= (int)b->members.size()) return fail(CDNS_ERR_ARG, "member index out of range");
    *ctx = b->members[i];
    return CDNS_OK;
}

int cdns_batch_run(cdns_batch *b, int first, int nsteps) {
    if (!b) return fail(CDNS_ERR_ARG, "null batch");
    if (nsteps < 0 || first < 1) return fail(CDNS_ERR_ARG, "bad iteration range");
    DeviceGuard guard(b->device);
    for (int i = 0; i < nsteps; ++i) {
        int r = batch_step(b, first + i);
        if (r) return r;
    }
    return CDNS_OK;
}

int cdns_batch_synchronize(cdns_batch *b) {
    if (!b) return fail(CDNS_ERR_ARG, "null batch");
    DeviceGuard guard(b->device);
    CK(cudaStreamSynchronize(b->stream));
    int first_error = CDNS_OK;
    std::string msg;
    for (size_t i = 0; i < b->members.size(); ++i) {
        int r = cdns_synchronize(b->members[i]);
        if (r && !first_error) {
            first_error = r;
            msg = "member " + std::to_string(i) + ": " + g_error;
        }
    }
    if (first_error) return fail(first_error, msg);
    return CDNS_OK;
}

int cdns_batch_stream(cdns_batch *b, void **stream) {
    if (!b || !stream) return fail(CDNS_ERR_ARG, "null argument");
    *stream = (void *)b->stream;
    return CDNS_OK;
}

}  // extern "C"
