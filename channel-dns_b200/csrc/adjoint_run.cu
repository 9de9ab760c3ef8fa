// Discrete adjoint of the channel-dns step: orchestration and the extern "C"
// entry points cdns_adjoint_run, cdns_solve_adjoint, cdns_nonlinear_adjoint.
//
// Forward step s (iteration it = s, coefficients a0, a1, b0, b1, g of
// src/sim/simulation.cpp:36-45):
//   N^{s-1}, bw = NL(u^{s-1}),  B^{s-1} = bw + wall sums of N_y^{s-1}
//   R = a0 u^{s-1} + a1 u^{s-2} + b0 N^{s-1} + b1 N^{s-2}
//   (p^s, u^s) = Solve_g(R, b0 B^{s-1} + b1 B^{s-2}, bc_v)
// Reverse step s (s = nsteps .. 1), every product transposed:
//   lR, lBc, lbc_v += Solve_g^T(lu^s)          (+ the objective seed)
//   lu^{s-1} += a0 lR,  lu^{s-2} = a1 lR,  lN^{s-1} += b0 lR,  lN^{s-2} = b1 lR
//   lbw = lB^{s-1} + b0 lBc,  lB^{s-2} = b1 lBc, lN_y^{s-1} += wall sums^T(lbw)
//   lu^{s-1} += NL'(u^{s-1})^T (lN^{s-1}, lbw)
// Three rotating slots suffice for each adjoint history (indexed by parity).
// The forward sweep stores the multistep state (u^s, u^{s-1}, N^{s-1},
// B^{s-1}) every checkpoint_interval steps; the reverse sweep restores each
// interval, recomputes it once keeping the z-physical fields of u and omega
// of every step (the linearisation point of u x omega), and runs its reverse
// steps.  The last interval keeps those fields from the forward sweep and is
// not recomputed; the recomputation of interval i-1 (context stream) runs
// concurrently with the reverse steps of interval i (a second stream), the
// two alternating between two slot sets.  Iteration 1 (g of the first-order
// start) has its own solver state.
#include <algorithm>
#include <cstring>

#include "context.cuh"

namespace cdns {

struct AdjointWork {
    std::vector<void *> allocs;
    size_t bytes = 0;
    double *csyn_t = nullptr, *cana_t = nullptr;   // transposed Chebyshev tables
    SolverState st1{};                              // solver state of iteration 1
    double g1 = NAN;
    double2 *lU[2] = {nullptr, nullptr}, *lN[2] = {nullptr, nullptr}, *lB[2] = {nullptr, nullptr};
    double2 *lR = nullptr, *lBc = nullptr, *lbw = nullptr, *lbcv = nullptr, *l6 = nullptr;
    double2 *ck = nullptr;    // checkpoints [nck][9 Ns + 2 ncol]
    size_t nck = 0;
    double2 *gs = nullptr;    // z-physical fields of two intervals [2][k][6][NY2+1][NZ2][NXS+1]
    size_t ngs = 0;
    double *jbuf = nullptr;   // objective per step
    size_t nj = 0;
    double2 *AF = nullptr, *AG = nullptr;   // stage scratch of the reverse steps
    cudaStream_t rs = nullptr;              // reverse-step stream (recomputation runs on the context's)
    cudaEvent_t ev_rec[2] = {nullptr, nullptr}, ev_rev[2] = {nullptr, nullptr}, ev_fwd = nullptr,
                ev_done = nullptr;
};

void adjoint_release(AdjointWork *w) {
    if (!w) return;
    if (w->rs) cudaStreamSynchronize(w->rs);
    for (cudaEvent_t e : {w->ev_rec[0], w->ev_rec[1], w->ev_rev[0], w->ev_rev[1], w->ev_fwd, w->ev_done})
        if (e) cudaEventDestroy(e);
    if (w->rs) cudaStreamDestroy(w->rs);
    for (void *p : w->allocs) cudaFree(p);
    if (w->ck) cudaFree(w->ck);
    if (w->gs) cudaFree(w->gs);
    if (w->jbuf) cudaFree(w->jbuf);
    delete w;
}

size_t adjoint_bytes(const AdjointWork *w) { return w ? w->bytes : 0; }

namespace {

size_t ck_size(const Dims &d) { return 9 * (size_t)d.Ns + 2 * (size_t)d.ncol; }
size_t gs_size(const Dims &d) { return 6 * (size_t)d.ny2 * d.NZ2 * d.nkx; }

template <typename T> int dalloc(cdns_ctx *c, AdjointWork *w, T *&p, size_t n) {
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

// Growable buffer: reallocated (contents dropped) when more is needed.
template <typename T> int grow(cdns_ctx *c, AdjointWork *w, T *&p, size_t &have, size_t need, size_t unit) {
    if (need <= have) return CDNS_OK;
    CK(cudaStreamSynchronize(c->stream));
    if (p) {
        cudaFree(p);
        w->bytes -= sizeof(T) * have * unit;
        p = nullptr;
        have = 0;
    }
    void *q = nullptr;
    cudaError_t e = cudaMalloc(&q, sizeof(T) * need * unit);
    if (e != cudaSuccess) return fail(CDNS_ERR_NOMEM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
    p = static_cast<T *>(q);
    have = need;
    w->bytes += sizeof(T) * need * unit;
    return CDNS_OK;
}

int check_adjoint_mesh(const cdns_ctx *c) {
    const Dims &d = c->d;
    if (c->mixed) return fail(CDNS_ERR_ARG, "the adjoint needs the FP64 precision mode");
    if (!(d.NX2 > 2 * d.NXS && d.NZ2 > 2 * d.NZS && d.NY2 > d.NYS))
        return fail(CDNS_ERR_ARG, "the adjoint needs a dealiased mesh (NX2 > 2 NXS, NZ2 > 2 NZS, NY2 > NYS)");
    return CDNS_OK;
}

int ensure_work(cdns_ctx *c, size_t nck, size_t ngs, size_t nj) {
    const Dims &d = c->d;
    if (!c->adj) {
        AdjointWork *w = new AdjointWork;
        c->adj = w;
        const size_t Ns = (size_t)d.Ns, nc = d.ncol;
        size_t nsyn, nana;
        cheb_table_sizes(d, &nsyn, &nana);
        SolverState &st = w->st1;
        int r = 0;
        if ((r = dalloc(c, w, w->csyn_t, nsyn)) || (r = dalloc(c, w, w->cana_t, nana)) ||
            (r = dalloc(c, w, st.wn_p, nc)) || (r = dalloc(c, w, st.wn_v, nc)) || (r = dalloc(c, w, st.ad_p, Ns)) ||
            (r = dalloc(c, w, st.ad_v, Ns)) || (r = dalloc(c, w, st.p_inf, 2 * Ns)) ||
            (r = dalloc(c, w, st.v_inf, 6 * Ns)) || (r = dalloc(c, w, st.inf_div, 4 * nc)) ||
            (r = dalloc(c, w, st.p_b, Ns)) || (r = dalloc(c, w, st.v_b, 3 * Ns)) ||
            (r = dalloc(c, w, st.sigma0, 2 * nc)) || (r = dalloc(c, w, st.unit, 2 * (size_t)d.ncy + 2)) ||
            (r = dalloc(c, w, w->lU[0], 3 * Ns)) || (r = dalloc(c, w, w->lU[1], 3 * Ns)) ||
            (r = dalloc(c, w, w->lN[0], 3 * Ns)) || (r = dalloc(c, w, w->lN[1], 3 * Ns)) ||
            (r = dalloc(c, w, w->lB[0], 2 * nc)) || (r = dalloc(c, w, w->lB[1], 2 * nc)) ||
            (r = dalloc(c, w, w->lR, 3 * Ns)) || (r = dalloc(c, w, w->lBc, 2 * nc)) ||
            (r = dalloc(c, w, w->lbw, 2 * nc)) || (r = dalloc(c, w, w->lbcv, 6 * nc)) ||
            (r = dalloc(c, w, w->l6, 6 * Ns)) || (r = dalloc(c, w, w->AF, 6 * (size_t)d.ny2 * d.fcol)) ||
            (r = dalloc(c, w, w->AG, gs_size(d))))
            return r;
        CK(cudaStreamCreateWithFlags(&w->rs, cudaStreamNonBlocking));
        for (cudaEvent_t *e : {&w->ev_rec[0], &w->ev_rec[1], &w->ev_rev[0], &w->ev_rev[1], &w->ev_fwd, &w->ev_done})
            CK(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
        launch_cheb_tables_adjoint(d, c->t.cosy, w->csyn_t, w->cana_t, c->stream);
        CK(configure_adjoint_kernels(d));
        CK(cudaGetLastError());
    }
    AdjointWork *w = c->adj;
    int r = 0;
    if ((r = grow(c, w, w->ck, w->nck, nck, ck_size(d))) || (r = grow(c, w, w->gs, w->ngs, ngs, gs_size(d))) ||
        (r = grow(c, w, w->jbuf, w->nj, nj, 1)))
        return r;
    return CDNS_OK;
}

// Multistep state before the next step: U[cur], U[1-cur], Nb[1-cur], Bb[1-cur].
int save_checkpoint(cdns_ctx *c, size_t i) {
    const Dims &d = c->d;
    const size_t n3 = 3 * (size_t)d.Ns;
    double2 *b = c->adj->ck + i * ck_size(d);
    const int k = c->cur;
    CK(cudaMemcpyAsync(b, c->U[k], n3 * sizeof(double2), cudaMemcpyDeviceToDevice, c->stream));
    CK(cudaMemcpyAsync(b + n3, c->U[1 - k], n3 * sizeof(double2), cudaMemcpyDeviceToDevice, c->stream));
    CK(cudaMemcpyAsync(b + 2 * n3, c->Nb[1 - k], n3 * sizeof(double2), cudaMemcpyDeviceToDevice, c->stream));
    CK(cudaMemcpyAsync(b + 3 * n3, c->Bb[1 - k], 2 * (size_t)d.ncol * sizeof(double2), cudaMemcpyDeviceToDevice,
                       c->stream));
    return CDNS_OK;
}
int load_checkpoint(cdns_ctx *c, size_t i) {
    const Dims &d = c->d;
    const size_t n3 = 3 * (size_t)d.Ns;
    const double2 *b = c->adj->ck + i * ck_size(d);
    c->cur = 0;
    CK(cudaMemcpyAsync(c->U[0], b, n3 * sizeof(double2), cudaMemcpyDeviceToDevice, c->stream));
    CK(cudaMemcpyAsync(c->U[1], b + n3, n3 * sizeof(double2), cudaMemcpyDeviceToDevice, c->stream));
    CK(cudaMemcpyAsync(c->Nb[1], b + 2 * n3, n3 * sizeof(double2), cudaMemcpyDeviceToDevice, c->stream));
    CK(cudaMemcpyAsync(c->Bb[1], b + 3 * n3, 2 * (size_t)d.ncol * sizeof(double2), cudaMemcpyDeviceToDevice,
                       c->stream));
    return CDNS_OK;
}

// One forward step (the body of cdns_step) with an explicit solver state and
// z-physical buffer; solve = false stops once G holds the z-physical fields
// of u and omega (the linearisation point the reverse step needs).
void forward_step(cdns_ctx *c, int it, const SolverState &st, double2 *G, bool solve) {
    double a0, a1, b0, b1, g;
    step_coefficients(it, c->DT, c->pp.Re, a0, a1, b0, b1, g);
    const int k = c->cur;
    const Dims &d = c->d;
    if (!solve) {
        launch_curl(d, c->t, c->U[k], c->om, nullptr, c->pp.Re, c->stream);
        launch_ysynth(d, c->t, c->U[k], c->om, 3, 6, c->F, c->stream);
        launch_z_backward(d, c->pz, c->t.root_z, c->F, G, 6, c->stream);
        return;
    }
    enqueue_nonlinear(c, c->U[k], c->Nb[k], false, 0, G);
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
    launch_step_solve(c->d, c->t, c->pp, g, st, a, c->stream);
    c->cur = 1 - k;
}

// lu += NL'(u)^T (lN, lbw) about the z-physical fields G6 of u and omega:
// transposed analysis -> transposed z analysis -> transposed x stage ->
// transposed z synthesis -> transposed synthesis -> transposed curl, on
// stream s with the adjoint's own stage scratch.
void nonlinear_adjoint(cdns_ctx *c, const double2 *G6, const double2 *lN, const double2 *lbw, double2 *lu,
                       cudaStream_t s) {
    const Dims &d = c->d;
    AdjointWork *w = c->adj;
    Tables ta = c->t;
    ta.csyn = w->csyn_t;   // includes 1/(NX2 NZ2): the transposed x and z analysis scalings
    ta.yform = 0;          // the transposed tables run in the matrix form
    // the transposed analysis has the synthesis' structure and the transposed
    // synthesis the analysis': each takes the FFT form where the forward does
    if (!((c->t.yform & 2) && launch_ydct_adjoint_analysis(d, c->t, lN, 3, w->AF, s)))
        launch_ysynth(d, ta, lN, nullptr, 3, 3, w->AF, s);
    launch_z_backward(d, c->pz, c->t.root_z, w->AF, w->AG, 3, s);
    launch_x_adjoint(d, c->px, c->t.root_x, G6, w->AG, s);
    // transposed z synthesis = NZ2 x the (1/NZ2-scaled) forward z transform
    launch_z_forward(d, c->pz, c->t.root_z, w->AG, w->AF, 6, s);
    if (!((c->t.yform & 1) && launch_ydct_adjoint_synthesis(d, c->t, w->AF, 6, w->l6, (double)d.NZ2, s)))
        launch_yanalysis_scaled(d, w->cana_t, w->AF, w->l6, 6, (double)d.NZ2, s);
    launch_curl_adjoint(d, c->t, w->l6, lbw, lu, c->pp.Re, s);
}

void to_wall_layout(const Dims &d, const double2 *src, int ncomp, double2 *dst) {
    // [ncomp][2][ncol] -> [kz][2][kx][ncomp]
    const size_t nc = d.ncol;
    for (int kz = 0; kz < d.nkz; ++kz)
        for (int w = 0; w < 2; ++w)
            for (int kx = 0; kx < d.nkx; ++kx)
                for (int comp = 0; comp < ncomp; ++comp)
                    dst[(((size_t)kz * 2 + w) * d.nkx + kx) * ncomp + comp] =
                        src[(2 * (size_t)comp + w) * nc + (size_t)kz * d.nkx + kx];
}

}  // namespace
}  // namespace cdns

using namespace cdns;

extern "C" {

int cdns_adjoint_run(cdns_ctx *c, int nsteps, int kck, int objective, const double *weights,
                     const double *control, double *J, double *grad_u, double *grad_bc) {
    if (!c) return fail(CDNS_ERR_ARG, "null context");
    if (int r = require_whole(c)) return r;
    if (nsteps < 1 || kck < 1) return fail(CDNS_ERR_ARG, "nsteps and checkpoint_interval must be >= 1");
    if (objective != CDNS_OBJECTIVE_WALL_SHEAR && objective != CDNS_OBJECTIVE_PROJECTION)
        return fail(CDNS_ERR_ARG, "unknown objective");
    const bool shear = objective == CDNS_OBJECTIVE_WALL_SHEAR;
    if (!shear && !weights) return fail(CDNS_ERR_ARG, "the projection objective needs weights");
    int r = check_adjoint_mesh(c);
    if (r) return r;
    if (c->pp.grad_pre != 1)
        return fail(CDNS_ERR_ARG, "the adjoint supports INDEX_GRAD_PRE = 1 (fixed pressure gradient) only");
    if (!c->have_velocity) return fail(CDNS_ERR_STATE, "cdns_adjoint_run before cdns_set_velocity");
    DeviceGuard guard(c->device);
    if (control && (r = cdns_set_velocity_bc(c, control))) return r;
    const Dims &d = c->d;
    cudaStream_t s = c->stream;
    const bool grad = grad_u || grad_bc;
    const int nseg = (nsteps + kck - 1) / kck;
    if ((r = ensure_work(c, grad ? nseg + 1 : 0, grad ? (size_t)kck * (nseg > 1 ? 2 : 1) : 0, nsteps))) return r;
    AdjointWork *w = c->adj;
    double a0, a1, b0, b1, g1, g2;
    step_coefficients(1, c->DT, c->pp.Re, a0, a1, b0, b1, g1);
    step_coefficients(2, c->DT, c->pp.Re, a0, a1, b0, b1, g2);
    if (!(w->g1 == g1)) {
        setup_solver(d, c->t, c->pp, g1, w->st1, nullptr, s);
        CK(cudaGetLastError());
        w->g1 = g1;
    }
    if ((r = do_setup(c, g2))) return r;
    auto state_for = [&](int it) -> const SolverState & { return it == 1 ? w->st1 : c->st; };
    // ---- forward sweep (the last interval keeps its z-physical fields) ----
    const size_t gsz = gs_size(d);
    const int s_last = (nseg - 1) * kck;
    // z-physical slot of iteration it in interval seg (two sets, alternating)
    auto slot = [&](int seg, int it) { return w->gs + ((size_t)(seg & 1) * kck + (it - seg * kck - 1)) * gsz; };
    for (int it = 1; it <= nsteps; ++it) {
        if (grad && (it - 1) % kck == 0 && (r = save_checkpoint(c, (size_t)(it - 1) / kck))) return r;
        if (it >= 3 && !(grad && it > s_last)) {
            // steady steps into the context's own buffers: its captured step graphs
            if ((r = one_step(c, it))) return r;
        } else {
            double2 *G = (grad && it > s_last) ? slot(nseg - 1, it) : c->G;
            forward_step(c, it, state_for(it), G, true);
        }
        if (shear) launch_wall_shear(d, c->U[c->cur], c->pp.Re, w->jbuf + it - 1, s);
    }
    CK(cudaGetLastError());
    const size_t n3 = 3 * (size_t)d.Ns, nc = d.ncol;
    double Jp = 0.0;
    if (!shear) {
        // J = Re <w, u^nsteps>, in a fixed order on the host
        std::vector<double> hu(2 * n3);
        launch_interleave(c->U[c->cur], c->aux, d.Ns, 3, s);
        CK(cudaGetLastError());
        CK(cudaMemcpyAsync(hu.data(), c->aux, n3 * sizeof(double2), cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        for (size_t i = 0; i < 2 * n3; ++i) Jp += weights[i] * hu[i];
    }
    if (grad) {
        if ((r = save_checkpoint(c, (size_t)nseg))) return r;
        for (int i = 0; i < 2; ++i) {
            CK(cudaMemsetAsync(w->lU[i], 0, n3 * sizeof(double2), s));
            CK(cudaMemsetAsync(w->lN[i], 0, n3 * sizeof(double2), s));
            CK(cudaMemsetAsync(w->lB[i], 0, 2 * nc * sizeof(double2), s));
        }
        CK(cudaMemsetAsync(w->lbcv, 0, 6 * nc * sizeof(double2), s));
        if (!shear) {
            // terminal seed: lu^nsteps = w
            CK(cudaMemcpyAsync(c->aux2, weights, n3 * sizeof(double2), cudaMemcpyHostToDevice, s));
            launch_deinterleave(c->aux2, w->lU[nsteps & 1], d.Ns, 3, s);
        }
        const double seed = shear ? -1.0 / ((double)nsteps * c->pp.Re) : 0.0;
        // ---- reverse sweep: the reverse steps of interval seg run on the
        // reverse stream while the context stream recomputes interval seg - 1
        // from its checkpoint into the other slot set ----
        cudaStream_t rs = w->rs;
        CK(cudaEventRecord(w->ev_fwd, s));
        CK(cudaStreamWaitEvent(rs, w->ev_fwd, 0));
        for (int seg = nseg - 1; seg >= 0; --seg) {
            if (seg >= 1) {
                const int ps = seg - 1, p0 = ps * kck, p1 = std::min(p0 + kck, nsteps);
                if (seg + 1 <= nseg - 1) CK(cudaStreamWaitEvent(s, w->ev_rev[ps & 1], 0));
                if ((r = load_checkpoint(c, (size_t)ps))) return r;
                for (int it = p0 + 1; it <= p1; ++it) forward_step(c, it, state_for(it), slot(ps, it), it < p1);
                CK(cudaEventRecord(w->ev_rec[ps & 1], s));
            }
            const int s0 = seg * kck, s1 = std::min(s0 + kck, nsteps);
            if (seg < nseg - 1) CK(cudaStreamWaitEvent(rs, w->ev_rec[seg & 1], 0));
            for (int it = s1; it > s0; --it) {
                double g;
                step_coefficients(it, c->DT, c->pp.Re, a0, a1, b0, b1, g);
                const int cu = it & 1, pv = (it - 1) & 1;
                launch_solve_adjoint_step(d, c->t, c->pp, g, state_for(it), w->lU[cu], seed, a0, a1, b0, b1,
                                          w->lU[pv], w->lU[cu], w->lN[pv], w->lN[cu], w->lB[pv], w->lbw,
                                          w->lB[cu], w->lBc, w->lbcv, rs);
                nonlinear_adjoint(c, slot(seg, it), w->lN[pv], w->lbw, w->lU[pv], rs);
            }
            CK(cudaEventRecord(w->ev_rev[seg & 1], rs));
            CK(cudaGetLastError());
        }
        CK(cudaEventRecord(w->ev_done, rs));
        CK(cudaStreamWaitEvent(s, w->ev_done, 0));
        if (grad_u) {
            launch_interleave(w->lU[0], c->aux, d.Ns, 3, s);
            CK(cudaGetLastError());
            CK(cudaMemcpyAsync(grad_u, c->aux, n3 * sizeof(double2), cudaMemcpyDeviceToHost, s));
        }
        std::vector<double2> hb(grad_bc ? 6 * nc : 0);
        if (grad_bc) CK(cudaMemcpyAsync(hb.data(), w->lbcv, hb.size() * sizeof(double2), cudaMemcpyDeviceToHost, s));
        if ((r = load_checkpoint(c, (size_t)nseg))) return r;   // the state after nsteps
        CK(cudaStreamSynchronize(s));
        if (grad_bc) to_wall_layout(d, hb.data(), 3, reinterpret_cast<double2 *>(grad_bc));
    }
    std::vector<double> hj(shear ? nsteps : 0);
    if (shear) CK(cudaMemcpyAsync(hj.data(), w->jbuf, nsteps * sizeof(double), cudaMemcpyDeviceToHost, s));
    if ((r = cdns_synchronize(c))) return r;
    if (J) {
        double acc = 0.0;
        for (double v : hj) acc += v;
        *J = shear ? acc / (double)nsteps : Jp;
    }
    return CDNS_OK;
}

int cdns_solve_adjoint(cdns_ctx *c, double g, const double *lp, const double *lv, double *lrhs, double *lpbc,
                       double *lvbc) {
    if (!c || !lv || !lrhs || !lpbc || !lvbc) return fail(CDNS_ERR_ARG, "null argument");
    if (int r = require_whole(c)) return r;
    DeviceGuard guard(c->device);
    const Dims &d = c->d;
    cudaStream_t s = c->stream;
    int r = do_setup(c, g);
    if (r || (r = ensure_work(c, 0, 0, 0))) return r;
    AdjointWork *w = c->adj;
    const size_t Ns = (size_t)d.Ns, nc = d.ncol;
    if (lp) CK(cudaMemcpyAsync(c->F, lp, Ns * sizeof(double2), cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(c->aux2, lv, 3 * Ns * sizeof(double2), cudaMemcpyHostToDevice, s));
    launch_deinterleave(c->aux2, c->aux, d.Ns, 3, s);
    CK(cudaMemsetAsync(w->lbcv, 0, 6 * nc * sizeof(double2), s));
    launch_solve_adjoint(d, c->t, c->pp, g, c->st, lp ? c->F : nullptr, c->aux, w->lR, w->lBc, w->lbcv, 1, 0.0, s);
    launch_interleave(w->lR, c->aux2, d.Ns, 3, s);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(lrhs, c->aux2, 3 * Ns * sizeof(double2), cudaMemcpyDeviceToHost, s));
    std::vector<double2> hp(2 * nc), hv(6 * nc);
    CK(cudaMemcpyAsync(hp.data(), w->lBc, hp.size() * sizeof(double2), cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(hv.data(), w->lbcv, hv.size() * sizeof(double2), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    to_wall_layout(d, hp.data(), 1, reinterpret_cast<double2 *>(lpbc));
    to_wall_layout(d, hv.data(), 3, reinterpret_cast<double2 *>(lvbc));
    return CDNS_OK;
}

int cdns_nonlinear_adjoint(cdns_ctx *c, const double *velocity, const double *lN, const double *lpbc,
                           double *lu) {
    if (!c || !velocity || !lN || !lu) return fail(CDNS_ERR_ARG, "null argument");
    if (int r = require_whole(c)) return r;
    int r = check_adjoint_mesh(c);
    if (r) return r;
    DeviceGuard guard(c->device);
    const Dims &d = c->d;
    cudaStream_t s = c->stream;
    if ((r = ensure_work(c, 0, 1, 0))) return r;
    AdjointWork *w = c->adj;
    const size_t Ns = (size_t)d.Ns, nc = d.ncol;
    CK(cudaMemcpyAsync(c->aux2, velocity, 3 * Ns * sizeof(double2), cudaMemcpyHostToDevice, s));
    launch_deinterleave(c->aux2, c->aux, d.Ns, 3, s);
    enqueue_nonlinear(c, c->aux, w->lR, false, 0, w->gs);
    CK(cudaMemcpyAsync(c->aux2, lN, 3 * Ns * sizeof(double2), cudaMemcpyHostToDevice, s));
    launch_deinterleave(c->aux2, w->lN[0], d.Ns, 3, s);
    std::vector<double2> hb(2 * nc, make_double2(0.0, 0.0));
    if (lpbc) {
        const double2 *src = reinterpret_cast<const double2 *>(lpbc);
        for (int kz = 0; kz < d.nkz; ++kz)
            for (int wall = 0; wall < 2; ++wall)
                for (int kx = 0; kx < d.nkx; ++kx)
                    hb[(size_t)wall * nc + (size_t)kz * d.nkx + kx] = src[((size_t)kz * 2 + wall) * d.nkx + kx];
    }
    CK(cudaMemcpyAsync(w->lbw, hb.data(), hb.size() * sizeof(double2), cudaMemcpyHostToDevice, s));
    launch_pressure_bc_adjoint(d, w->lbw, w->lN[0], s);
    CK(cudaMemsetAsync(w->lU[0], 0, 3 * Ns * sizeof(double2), s));
    nonlinear_adjoint(c, w->gs, w->lN[0], w->lbw, w->lU[0], s);
    launch_interleave(w->lU[0], c->aux2, d.Ns, 3, s);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(lu, c->aux2, 3 * Ns * sizeof(double2), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    return CDNS_OK;
}

}  // extern "C"
