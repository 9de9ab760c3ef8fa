// Per-(kz, kx) Chebyshev-tau pressure/velocity solve of the channel-dns step
// (EqSolvePV, src/solver/eqsolve_pv.cpp) for sm_100a.
//
// One block owns TC consecutive spectral columns.  Coalesced block-wide
// passes stage each column's inputs in shared memory ([y][column] layout)
// and stream the precomputed influence / B-problem fields on write-back; the
// sequential y recurrences run two threads per column, because every tau
// recurrence (src/solver/eqsolve_pv.cpp:64-128) and every Chebyshev
// derivative recurrence (src/solver/vector_ops.cpp:17-25) couples only
// coefficients of one parity.  All arithmetic is FP64 in the reference's
// operation order.
#include "cdns_kernels.cuh"

namespace cdns {

namespace {
constexpr int TC = 8;          // spectral columns per block
constexpr int kThreads = 128;

enum Mode { MODE_STEP = 0, MODE_BASE = 1, MODE_COUPLED = 2 };

struct SolveArgs {
    double p_a, p_b;           // pressure wall condition a P + b dP/dn
    double2 bcp_top, bcp_bot;  // constant pressure wall data (setup problems)
    double2 *p_out;            // [Ns]
    double2 *v_out;            // [3][Ns]
    double2 *divb_out;         // [2][ncol] raw wall divergence (MODE_BASE)
    StepArgs step;             // MODE_STEP only
};

__device__ inline double tau_func(double a, double b, int y) {
    const int q = y & 1;
    if (a == 0.0 && b == 0.0) return (double)((1 - q) * y * y + q);
    return a + b * y * y;
}

// Chebyshev derivative coefficients of parity `par`:
// d_k = d_{k+2} + 2(k+1) f_{k+1}, d_NYS = 0, d_0 halved.
__device__ void deriv_chain(int par, int ny, const double2 *f, double2 *dout, int st) {
    int k = ((ny & 1) == par) ? ny : ny - 1;
    double2 dd = mk(0.0, 0.0);
    if (k == ny) {
        dout[(long long)ny * st] = dd;
        k -= 2;
    }
    for (; k >= 0; k -= 2) {
        dd = cadd(dd, cscale((double)(2 * (k + 1)), f[(long long)(k + 1) * st]));
        if (k == 0) dd = cscale(0.5, dd);
        dout[(long long)k * st] = dd;
    }
}

// One parity of the column tau solve of (D^2 - k^2 - g) f = r with
// a f + b f' = (lower, upper) at y = (+1, -1)  (src/solver/eqsolve_pv.cpp:64-128).
// Returns false if a pivot is zero or not finite.
__device__ bool tau_chain(int par, int ny, double g, double a, double b, bool zero_col,
                          double2 lower, double2 upper, double w, const double2 *r, double2 *out,
                          const double *ad, int st, const double *WL, const double *WD,
                          const double *WR) {
    const bool normalize = g == 0.0 && a == 0.0 && zero_col;
    double2 r0 = r[0];
    if (normalize && par == 0) {
        double2 corr = mk(0.0, 0.0);
        for (int y = 2; y <= ny; y += 2) corr = cadd(corr, cdivr(r[(long long)y * st], (double)(y * y - 1)));
        if (b != 0.0) corr = cadd(corr, cdivr(cadd(lower, upper), 2.0 * b));
        r0 = corr;
    }
#define RR(yy) ((yy) == 0 ? r0 : r[(long long)(yy) * st])
#define OUT(yy) out[(long long)(yy) * st]
#define AD(yy) ad[(long long)(yy) * st]
    if (par == 0) OUT(0) = cdivr(cadd(lower, upper), 2.0);
    else OUT(1) = cdivr(csub(lower, upper), 2.0);
    for (int y = 2 + par; y <= ny - 2; y += 2)
        OUT(y) = cadd(cadd(cscale(WL[y], RR(y - 2)), cscale(WD[y], RR(y))), cscale(WR[y], RR(y + 2)));
    if (((ny - 1) & 1) == par) OUT(ny - 1) = cadd(cscale(WL[ny - 1], RR(ny - 3)), cscale(WD[ny - 1], RR(ny - 1)));
    if ((ny & 1) == par) OUT(ny) = cadd(cscale(WL[ny], RR(ny - 2)), cscale(WD[ny], RR(ny)));
    int ys = ny - 2;
    if ((ys & 1) != par) ys -= 1;
    for (int y = ys; y >= 2; y -= 2) OUT(y) = csub(OUT(y), cscale((WR[y] * w) * AD(y + 2), OUT(y + 2)));
    double ad01 = tau_func(a, b, ((ny & 1) == par) ? ny : ny - 1);
    double2 o0 = OUT(par);
    for (int y = ys; y >= par; y -= 2) {
        o0 = csub(o0, cscale(ad01 * AD(y + 2), OUT(y + 2)));
        ad01 = tau_func(a, b, y) - ((WL[y + 2] * w) * ad01) * AD(y + 2);
    }
    if (normalize && par == 0) {
        o0 = mk(0.0, 0.0);
        ad01 = 1.0;
    }
    const bool ok = isfinite(ad01) && ad01 != 0.0;
    OUT(par) = cdivr(o0, ad01);
    for (int y = 2 + par; y <= ny; y += 2) OUT(y) = cscale(AD(y), csub(OUT(y), cscale(WL[y] * w, OUT(y - 2))));
#undef RR
#undef OUT
#undef AD
    return ok;
}

template <int MODE>
__global__ void __launch_bounds__(kThreads)
k_solve(Dims d, Tables t, PhysParams pp, double g_v, SolverState st, SolveArgs A) {
    extern __shared__ double2 sm2[];
    const int ncy = d.ncy, ny = d.NYS, nkx = d.nkx;
    const int S = ncy * TC;
    double2 *rv = sm2;            // [3][ncy][TC]
    double2 *pc = rv + 3 * S;     // [ncy][TC]
    double2 *dyb = pc + S;
    double2 *fo = dyb + S;
    double *adp = reinterpret_cast<double *>(fo + S);
    double *adv = adp + S;
    double *sWL = adv + S;
    double *sWD = sWL + ncy;
    double *sWR = sWD + ncy;
    __shared__ double2 s_lo[TC], s_up[TC], s_c0[TC], s_c1[TC], s_sig[2][TC];
    __shared__ double s_dp[2];

    const int col0 = blockIdx.x * TC;
    const int tid = threadIdx.x;
    for (int i = tid; i < ncy; i += blockDim.x) {
        sWL[i] = t.WL[i];
        sWD[i] = t.WD[i];
        sWR[i] = t.WR[i];
    }
    // ---- phase A: stage inputs -------------------------------------------
    for (int i = tid; i < S; i += blockDim.x) {
        const int y = i / TC, l = i - (i / TC) * TC;
        const int col = col0 + l;
        if (col < d.ncol) {
            const int kzi = col / nkx, kx = col - (col / nkx) * nkx;
            const long long off = ((long long)kzi * ncy + y) * nkx + kx;
            adp[i] = st.ad_p[off];
            adv[i] = st.ad_v[off];
            if (MODE == MODE_STEP) {
                const StepArgs &s = A.step;
                for (int c = 0; c < 3; ++c) {
                    const long long o = c * d.Ns + off;
                    // R = a0 u + a1 u_prev + b0 N + b1 N_prev (src/sim/simulation.cpp:151-158)
                    const double2 R = cadd(cadd(cadd(cscale(s.a0, s.u[o]), cscale(s.a1, s.u_prev[o])),
                                                cscale(s.b0, s.N[o])),
                                           cscale(s.b1, s.N_prev[o]));
                    rv[c * S + i] = R;
                }
                fo[i] = s.N[d.Ns + off];
            } else {
                for (int c = 0; c < 3; ++c) rv[c * S + i] = mk(0, 0);
                double rp = 0.0;
                if (MODE == MODE_COUPLED) {
                    // B-problem pressure RHS (src/solver/eqsolve_pv.cpp:452-461)
                    if (y == 0) rp = (double)(ny - 1);
                    else if (y < ny) rp = (double)(2 * (ny - ((y + 1) % 2)));
                }
                dyb[i] = mk(rp, 0.0);
            }
        } else {
            adp[i] = 1.0;
            adv[i] = 1.0;
            for (int c = 0; c < 3; ++c) rv[c * S + i] = mk(0, 0);
            dyb[i] = mk(0, 0);
            fo[i] = mk(0, 0);
        }
        pc[i] = mk(0, 0);
    }
    __syncthreads();

    // ---- phase B: recurrences, two threads (parities) per column ----------
    if (tid < 2 * TC) {
        const unsigned mask = 0x0000ffffu;
        const int l = tid >> 1, par = tid & 1;
        const int col = col0 + l;
        const bool active = col < d.ncol;
        const int kzi = active ? col / nkx : 0;
        const int kx = active ? col - kzi * nkx : 0;
        const double ax = t.wavx[kx], az = t.wavz[kzi];
        const bool zero_col = active && kzi == d.NZS && kx == 0;
        double2 tail0 = mk(0, 0), tail1 = mk(0, 0);
        bool ok = true;
        if (active && par == 0) {
            if (MODE == MODE_STEP && A.step.bc_p) {
                s_lo[l] = A.step.bc_p[col];
                s_up[l] = A.step.bc_p[d.ncol + col];
            } else if (MODE == MODE_STEP) {
                const StepArgs &s = A.step;
                double2 st_ = mk(0, 0), sb_ = mk(0, 0);
                for (int y = 0; y <= ny; ++y) {
                    const double2 n1 = fo[y * TC + l];
                    st_ = cadd(st_, n1);
                    sb_ = (y & 1) ? cadd(sb_, n1) : csub(sb_, n1);
                }
                const double2 bt = cadd(s.bw[col], st_);
                const double2 bb = cadd(s.bw[d.ncol + col], sb_);
                s.B_new[col] = bt;
                s.B_new[d.ncol + col] = bb;
                // combined wall data b0 B + b1 B_prev (src/sim/simulation.cpp:146-150)
                s_lo[l] = cadd(cscale(s.b0, bt), cscale(s.b1, s.B_prev[col]));
                s_up[l] = cadd(cscale(s.b0, bb), cscale(s.b1, s.B_prev[d.ncol + col]));
            } else {
                s_lo[l] = A.bcp_top;
                s_up[l] = A.bcp_bot;
            }
        }
        __syncwarp(mask);
        const double2 lower = s_lo[l], upper = s_up[l];
        if (MODE == MODE_STEP && active) {
            // fused divergence of the RHS (src/solver/eqsolve_pv.cpp:340-357)
            deriv_chain(par, ny, rv + S + l, dyb + l, TC);
            for (int y = par; y <= ny; y += 2) {
                const int k = y * TC + l;
                dyb[k] = cadd(cadd(fderiv(ax, rv[k]), dyb[k]), fderiv(az, rv[2 * S + k]));
            }
        }
        __syncwarp(mask);
        if (active) {
            ok &= tau_chain(par, ny, pp.G_pre, A.p_a, A.p_b, zero_col, lower, upper,
                            st.wn_p[col], dyb + l, pc + l, adp + l, TC, sWL, sWD, sWR);
        }
        __syncwarp(mask);
        if (active) {
            if (par == 0) {
                tail0 = rv[S + ny * TC + l];
                tail1 = rv[S + (ny - 1) * TC + l];
            }
            deriv_chain(par, ny, pc + l, dyb + l, TC);
        }
        __syncwarp(mask);
        if (active) {
            const double wv = st.wn_v[col];
            for (int c = 0; c < 3; ++c) {
                double2 *rc = rv + c * S + l;
                for (int y = par; y <= ny; y += 2) {
                    const int k = y * TC;
                    const double2 grad = (c == 0) ? fderiv(ax, pc[k + l])
                                         : (c == 1) ? dyb[k + l] : fderiv(az, pc[k + l]);
                    fo[k + l] = cscale(pp.Re, csub(grad, rc[k]));
                }
                double2 blo = mk(0, 0), bup = mk(0, 0);
                if (MODE == MODE_STEP) {
                    blo = A.step.bc_v[(2 * c) * d.ncol + col];
                    bup = A.step.bc_v[(2 * c + 1) * d.ncol + col];
                }
                ok &= tau_chain(par, ny, g_v, pp.a_V[c], pp.b_V[c], zero_col, blo, bup, wv,
                                fo + l, rc, adv + l, TC, sWL, sWD, sWR);
            }
        }
        __syncwarp(mask);
        if (active && par == 0) {
            // wall divergence by endpoint sums (src/solver/eqsolve_pv.cpp:397-406)
            double2 div0 = mk(0, 0), div1 = mk(0, 0);
            for (int y = 0; y <= ny; ++y) {
                const int k = y * TC + l;
                const double2 tang = cadd(fderiv(ax, rv[k]), fderiv(az, rv[2 * S + k]));
                const double2 nrm = cscale((double)(y * y), rv[S + k]);
                div0 = cadd(div0, cadd(tang, nrm));
                div1 = (y & 1) ? cadd(div1, cadd(mk(-tang.x, -tang.y), nrm)) : cadd(div1, csub(tang, nrm));
            }
            if (MODE == MODE_BASE) {
                A.divb_out[col] = div0;
                A.divb_out[d.ncol + col] = div1;
                s_c0[l] = mk(0, 0);
                s_c1[l] = mk(0, 0);
            } else {
                const double2 i00 = st.inf_div[col], i01 = st.inf_div[d.ncol + col];
                const double2 i10 = st.inf_div[2 * d.ncol + col], i11 = st.inf_div[3 * d.ncol + col];
                const double2 c0 = csub(cmul(div1, i10), cmul(div0, i11));
                const double2 c1 = csub(cmul(div0, i01), cmul(div1, i00));
                s_c0[l] = c0;
                s_c1[l] = c1;
                if (MODE == MODE_STEP) {
                    // sigma correction (src/solver/eqsolve_pv.cpp:413-429)
                    const long long base = (long long)kzi * ncy * nkx + kx;
                    const long long oN = base + (long long)ny * nkx;
                    const long long oN1 = base + (long long)(ny - 1) * nkx;
                    const double2 *PI0 = st.p_inf, *PI1 = st.p_inf + d.Ns;
                    const double2 *VI0 = st.v_inf + d.Ns, *VI1 = st.v_inf + 4 * d.Ns;  // component 1
                    const double2 ptop = cadd(pc[ny * TC + l], cadd(cmul(c0, PI0[oN]), cmul(c1, PI1[oN])));
                    const double2 vt0 = cadd(rv[S + ny * TC + l], cadd(cmul(c0, VI0[oN]), cmul(c1, VI1[oN])));
                    const double2 vt1 = cadd(rv[S + (ny - 1) * TC + l], cadd(cmul(c0, VI0[oN1]), cmul(c1, VI1[oN1])));
                    const double wv = st.wn_v[col];
                    const double2 n0 = csub(cscale(-wv, vt0), cscale(pp.Re, tail0));
                    const double2 n1 = cadd(cscale(-wv, vt1),
                                            cscale(pp.Re, csub(cscale(2.0 * ny, ptop), tail1)));
                    s_sig[0][l] = cdiv(n0, st.sigma0[col]);
                    s_sig[1][l] = cdiv(n1, st.sigma0[d.ncol + col]);
                }
            }
        }
        if (!ok && active) {
            unsigned *err = (MODE == MODE_STEP) ? A.step.err : nullptr;
            if (err) atomicOr(err, ERR_PIVOT);
        }
    }
    __syncthreads();

    // ---- phase C: corrections and single write-back -----------------------
    const int zero_col = d.NZS * nkx;
    bool bad = false;
    for (int i = tid; i < S; i += blockDim.x) {
        const int y = i / TC, l = i - (i / TC) * TC;
        const int col = col0 + l;
        if (col >= d.ncol) continue;
        const int kzi = col / nkx, kx = col - (col / nkx) * nkx;
        const long long off = ((long long)kzi * ncy + y) * nkx + kx;
        const int q = (y + 1) & 1;
        double2 p = pc[i];
        double2 v[3] = {rv[i], rv[S + i], rv[2 * S + i]};
        if (MODE != MODE_BASE) {
            const double2 c0 = s_c0[l], c1 = s_c1[l];
            p = cadd(p, cadd(cmul(c0, st.p_inf[off]), cmul(c1, st.p_inf[d.Ns + off])));
            if (MODE == MODE_STEP) p = cadd(p, cmul(s_sig[q][l], st.p_b[off]));
            for (int c = 0; c < 3; ++c) {
                v[c] = cadd(v[c], cadd(cmul(c0, st.v_inf[c * d.Ns + off]),
                                       cmul(c1, st.v_inf[(3 + c) * d.Ns + off])));
                if (MODE == MODE_STEP)
                    v[c] = cadd(v[c], cmul(s_sig[c == 1 ? 1 - q : q][l], st.v_b[c * d.Ns + off]));
            }
        }
        if (MODE == MODE_STEP && !A.step.solve_only && col == zero_col) {
            // correct_zero_mode (src/solver/timestepper.cpp:60-68)
            v[1] = (y == 0) ? cscale(0.5, cadd(A.step.bc_v[2 * d.ncol + col], A.step.bc_v[3 * d.ncol + col]))
                            : mk(0.0, 0.0);
        }
        if (MODE == MODE_STEP) {
            bad |= !(isfinite(p.x) && isfinite(p.y));
            for (int c = 0; c < 3; ++c) bad |= !(isfinite(v[c].x) && isfinite(v[c].y));
        }
        A.p_out[off] = p;
        for (int c = 0; c < 3; ++c) A.v_out[c * d.Ns + off] = v[c];
    }
    if (MODE == MODE_STEP && bad) atomicOr(A.step.err, ERR_NONFINITE);
    if (MODE == MODE_STEP && !A.step.solve_only && zero_col >= col0 && zero_col < col0 + TC) {
        // correct_flow (src/sim/simulation.cpp:111-140), single-rank branch
        __syncthreads();
        const long long zoff = (long long)d.NZS * ncy * nkx;  // (kz=0, y=0, kx=0)
        if (tid == 0) {
            const double *uu = st.unit;
            const double qxu = uu[2 * ncy], qzu = uu[2 * ncy + 1];
            double dpdx, dpdz;
            if (pp.grad_pre == 1) {
                dpdx = pp.gx;
                dpdz = pp.gz;
            } else {
                double qx = 0.0, qz = 0.0;
                for (int y = 0; y <= ny; y += 2) {
                    qx -= A.v_out[zoff + (long long)y * nkx].x / (double)(y * y - 1);
                    qz -= A.v_out[2 * d.Ns + zoff + (long long)y * nkx].x / (double)(y * y - 1);
                }
                if (!isfinite(qxu) || qxu == 0.0 || !isfinite(qzu) || qzu == 0.0)
                    atomicOr(A.step.err, ERR_PIVOT);
                dpdx = (pp.qxm - qx) / qxu;
                dpdz = (pp.qzm - qz) / qzu;
            }
            s_dp[0] = dpdx;
            s_dp[1] = dpdz;
            A.step.dpdx[0] = dpdx;
            A.step.dpdx[1] = dpdz;
        }
        __syncthreads();
        for (int y = tid; y <= ny; y += blockDim.x) {
            A.v_out[zoff + (long long)y * nkx].x += s_dp[0] * st.unit[y];
            A.v_out[2 * d.Ns + zoff + (long long)y * nkx].x += s_dp[1] * st.unit[ncy + y];
        }
    }
}

size_t solve_smem(const Dims &d) {
    const size_t S = (size_t)d.ncy * TC;
    return sizeof(double2) * 6 * S + sizeof(double) * (2 * S + 3 * (size_t)d.ncy);
}

// EqSolvePV::build_wn_ad (src/solver/eqsolve_pv.cpp:148-168), one thread per column.
__global__ void k_wn_ad(Dims d, Tables t, double g, double *wn, double *ad) {
    const int col = blockIdx.x * blockDim.x + threadIdx.x;
    if (col >= d.ncol) return;
    const int kzi = col / d.nkx, kx = col - (col / d.nkx) * d.nkx;
    const double ax = t.wavx[kx], az = t.wavz[kzi];
    const double w = -((ax * ax + az * az) + g);
    wn[col] = w;
    const int n = d.NYS;
    double *A = ad + (long long)kzi * d.ncy * d.nkx + kx;
    const long long s = d.nkx;
    A[0] = 0.0;
    A[s] = 0.0;
    A[n * s] = 1.0 / (1.0 + t.WD[n] * w);
    A[(n - 1) * s] = 1.0 / (1.0 + t.WD[n - 1] * w);
    for (int y = n - 2; y >= 2; --y) {
        const double fc = t.WR[y] * t.WL[y + 2];
        const double den = 1.0 + (t.WD[y] - (fc * w) * A[(y + 2) * s]) * w;
        A[y * s] = 1.0 / den;
    }
}

// Influence normalisation (src/solver/eqsolve_pv.cpp:282-302).
__global__ void k_inf_normalize(Dims d, double a_v1, double2 *inf_div) {
    const int col = blockIdx.x * blockDim.x + threadIdx.x;
    if (col >= d.ncol) return;
    double2 *I = inf_div;
    const int nc = d.ncol;
    const double2 i00 = I[col], i01 = I[nc + col], i10 = I[2 * nc + col], i11 = I[3 * nc + col];
    double2 den = csub(cmul(i00, i11), cmul(i01, i10));
    const bool root = (col == d.NZS * d.nkx);
    if (root) den = (a_v1 == 0.0) ? mk(1.0, 0.0) : cdiv(mk(0.25, 0.0), i00);
    if (root) {
        I[col] = den;
        I[nc + col] = mk(0, 0);
        I[2 * nc + col] = den;
        I[3 * nc + col] = mk(0, 0);
    } else {
        I[col] = cdiv(i00, den);
        I[nc + col] = cdiv(i01, den);
        I[2 * nc + col] = cdiv(i10, den);
        I[3 * nc + col] = cdiv(i11, den);
    }
}

// sigma0 denominators (src/solver/eqsolve_pv.cpp:466-476).
__global__ void k_sigma0(Dims d, double re, const double *wn_v, const double2 *p_b,
                         const double2 *v_b, double2 *sigma0) {
    const int col = blockIdx.x * blockDim.x + threadIdx.x;
    if (col >= d.ncol) return;
    const int kzi = col / d.nkx, kx = col - (col / d.nkx) * d.nkx;
    const long long base = (long long)kzi * d.ncy * d.nkx + kx;
    const int n = d.NYS;
    const double w = wn_v[col];
    const double2 vbn = v_b[d.Ns + base + (long long)n * d.nkx];
    const double2 vbn1 = v_b[d.Ns + base + (long long)(n - 1) * d.nkx];
    const double2 pbn = p_b[base + (long long)n * d.nkx];
    sigma0[col] = mk(re + w * vbn.x, w * vbn.y);
    double2 s1 = csub(mk(re + w * vbn1.x, w * vbn1.y), cscale(re * (2.0 * n), pbn));
    if (col == d.NZS * d.nkx) s1 = mk(1.0, 0.0);
    sigma0[d.ncol + col] = s1;
}

// Unit pressure-gradient responses of the zero mode
// (src/solver/eqsolve_pv.cpp:479-493): two threads (parities), one column.
__global__ void k_unit_response(Dims d, Tables t, PhysParams pp, double g_v, const double *ad_v,
                                double *unit) {
    extern __shared__ double2 su[];
    const int ncy = d.ncy, ny = d.NYS;
    double2 *r = su;
    double2 *o = r + ncy;
    double *ad = reinterpret_cast<double *>(o + ncy);
    double *WL = ad + ncy, *WD = WL + ncy, *WR = WD + ncy;
    const int par = threadIdx.x;
    const long long zc = (long long)d.NZS * ncy * d.nkx;
    for (int y = par; y < ncy; y += 2) {
        r[y] = mk(y == 0 ? pp.Re : 0.0, 0.0);
        ad[y] = ad_v[zc + (long long)y * d.nkx];
        WL[y] = t.WL[y];
        WD[y] = t.WD[y];
        WR[y] = t.WR[y];
    }
    __syncthreads();
    const double w = -((0.0 + 0.0) + g_v);
    for (int pass = 0; pass < 2; ++pass) {
        const int c = pass == 0 ? 0 : 2;
        tau_chain(par, ny, g_v, pp.a_V[c], pp.b_V[c], true, mk(0, 0), mk(0, 0), w, r, o, ad, 1, WL,
                  WD, WR);
        __syncthreads();
        if (par == 0) {
            double q = 0.0;
            for (int y = 0; y <= ny; y += 2) q -= o[y].x / (double)(y * y - 1);
            unit[2 * ncy + pass] = q;
            for (int y = 0; y <= ny; ++y) unit[pass * ncy + y] = o[y].x;
        }
        __syncthreads();
    }
}
__global__ void k_pressure_bc(Dims d, const double2 *N, const double2 *bw, double2 *B) {
    const int col = blockIdx.x * blockDim.x + threadIdx.x;
    if (col >= d.ncol) return;
    const int kzi = col / d.nkx, kx = col - (col / d.nkx) * d.nkx;
    const double2 *Ny = N + d.Ns + (long long)kzi * d.ncy * d.nkx + kx;
    double2 st_ = mk(0, 0), sb_ = mk(0, 0);
    for (int y = 0; y <= d.NYS; ++y) {
        const double2 n1 = Ny[(long long)y * d.nkx];
        st_ = cadd(st_, n1);
        sb_ = (y & 1) ? cadd(sb_, n1) : csub(sb_, n1);
    }
    B[col] = cadd(bw[col], st_);
    B[d.ncol + col] = cadd(bw[d.ncol + col], sb_);
}
}  // namespace

void launch_pressure_bc(const Dims &d, const double2 *N, const double2 *bw, double2 *B,
                        cudaStream_t s) {
    k_pressure_bc<<<(d.ncol + 127) / 128, 128, 0, s>>>(d, N, bw, B);
}

cudaError_t configure_solver_kernels(const Dims &d) {
    const int sm = (int)solve_smem(d);
    cudaError_t e = cudaFuncSetAttribute(k_solve<MODE_STEP>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(k_solve<MODE_BASE>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(k_solve<MODE_COUPLED>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
}

void setup_solver(const Dims &d, const Tables &t, const PhysParams &pp, double g_v, SolverState &st,
                  double2 *, cudaStream_t s) {
    const int nb = (d.ncol + 127) / 128;
    k_wn_ad<<<nb, 128, 0, s>>>(d, t, pp.G_pre, st.wn_p, st.ad_p);
    k_wn_ad<<<nb, 128, 0, s>>>(d, t, g_v, st.wn_v, st.ad_v);
    const int blocks = (d.ncol + TC - 1) / TC;
    const size_t sm = solve_smem(d);
    // influence responses: pressure Dirichlet data (1,0) and (0,1)
    for (int i = 0; i < 2; ++i) {
        SolveArgs A{};
        A.p_a = 1.0;
        A.p_b = 0.0;
        A.bcp_top = mk((double)(1 - i), 0.0);
        A.bcp_bot = mk((double)i, 0.0);
        A.p_out = st.p_inf + (long long)i * d.Ns;
        A.v_out = st.v_inf + (long long)i * 3 * d.Ns;
        A.divb_out = st.inf_div + (long long)i * 2 * d.ncol;
        k_solve<MODE_BASE><<<blocks, kThreads, sm, s>>>(d, t, pp, g_v, st, A);
    }
    k_inf_normalize<<<nb, 128, 0, s>>>(d, pp.a_V[1], st.inf_div);
    {
        SolveArgs A{};
        A.p_a = 1.0;
        A.p_b = 0.0;
        A.p_out = st.p_b;
        A.v_out = st.v_b;
        k_solve<MODE_COUPLED><<<blocks, kThreads, sm, s>>>(d, t, pp, g_v, st, A);
    }
    k_sigma0<<<nb, 128, 0, s>>>(d, pp.Re, st.wn_v, st.p_b, st.v_b, st.sigma0);
    const size_t smu = sizeof(double2) * 2 * d.ncy + sizeof(double) * 4 * d.ncy;
    k_unit_response<<<1, 2, smu, s>>>(d, t, pp, g_v, st.ad_v, st.unit);
}

void launch_step_solve(const Dims &d, const Tables &t, const PhysParams &pp, double g_v,
                       const SolverState &st, const StepArgs &a, cudaStream_t s) {
    SolveArgs A{};
    A.p_a = pp.a_pre0;
    A.p_b = pp.b_pre0;
    A.p_out = a.p_out;
    A.v_out = a.u_out;
    A.step = a;
    const int blocks = (d.ncol + TC - 1) / TC;
    k_solve<MODE_STEP><<<blocks, kThreads, solve_smem(d), s>>>(d, t, pp, g_v, st, A);
}

}  // namespace cdns
