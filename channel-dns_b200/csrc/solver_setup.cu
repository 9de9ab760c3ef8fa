// Precomputation of the column solver (EqSolvePV::setup,
// src/solver/eqsolve_pv.cpp:148-168, 266-303, 452-493) for sm_100a.
//
// The setup problems run in the reference's sequential operation order, two
// threads (the two y parities) per column over shared-memory columns.  Their
// results enter the step through differences that cancel: the second sigma
// denominator Re + w v_b(n-1) - 2 n Re p_b(n) of the lowest wavenumbers is
// about 1e-6 of its terms, so round-off of the B-problem differs from the
// reference's by 1e-9 relative after that cancellation unless the B-problem is
// computed in the same order.  Setup runs at steps 1 and 2 only.
//
// Outputs: the pivots ad_p, ad_v are stored column-major ([col][y]), read by
// the step solve's column warps; the influence / B-problem fields are planar
// ([kz][y][kx]), read by its coalesced correction pass.
#include "cdns_kernels.cuh"

namespace cdns {

namespace {
constexpr int TC = 4;          // spectral columns per block
constexpr int kThreads = 64;

enum SetupMode { MODE_BASE = 1, MODE_COUPLED = 2 };

struct SetupArgs {
    double2 bcp_top, bcp_bot;  // constant pressure wall data
    double *p_out;             // [Ns] planar, real
    double *v_out;             // [3][Ns] planar, parts as inf_imag(c)
    double2 *divb_out;         // [2][ncol] raw wall divergence (MODE_BASE)
};

__device__ inline double tau_func(double a, double b, int y) {
    const int q = y & 1;
    if (a == 0.0 && b == 0.0) return (double)((1 - q) * y * y + q);
    return a + b * y * y;
}

// Chebyshev derivative coefficients of parity `par` (src/solver/vector_ops.cpp:17-25):
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

// Setup column solve: pressure tau with constant wall data (MODE_BASE) or the
// B-problem right-hand side (MODE_COUPLED), velocity taus of Re grad P, wall
// divergence, and for MODE_COUPLED the influence correction
// (src/solver/eqsolve_pv.cpp:241-264, 311-450 without sigma).
//
// Only the columns kz <= 0 are solved.  Column -kz has the same k^2, so the
// same pivots and pressure; its right-hand sides differ only by the sign of
// the kz derivative, and every operation is linear with the rounding of a
// negated operand negated, so its solution is this column's with w negated,
// bit for bit, and its wall divergences are equal.  Both columns are written.
template <int MODE>
__global__ void __launch_bounds__(kThreads)
k_setup_solve(Dims d, Tables t, PhysParams pp, double g_v, SolverState st, SetupArgs A) {
    extern __shared__ double2 sm2[];
    if (MODE == MODE_BASE && blockIdx.y == 1) {
        // the second influence response: pressure data (0, 1), its own outputs
        A.bcp_top = mk(0.0, 0.0);
        A.bcp_bot = mk(1.0, 0.0);
        A.p_out += d.Ns;
        A.v_out += 3 * d.Ns;
        A.divb_out += 2 * d.ncol;
    }
    const int ncy = d.ncy, ny = d.NYS, nkx = d.nkx;
    const int nhalf = (d.NZS + 1) * nkx;   // columns kz <= 0 (kz index 0 .. NZS)
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
    __shared__ double2 s_c0[TC], s_c1[TC];

    const int col0 = blockIdx.x * TC;
    const int tid = threadIdx.x;
    for (int i = tid; i < ncy; i += blockDim.x) {
        sWL[i] = t.WL[i];
        sWD[i] = t.WD[i];
        sWR[i] = t.WR[i];
    }
    for (int i = tid; i < S; i += blockDim.x) {
        const int y = i / TC, l = i - (i / TC) * TC;
        const int col = col0 + l;
        double rp = 0.0;
        if (col < nhalf) {
            const long long cm = (long long)col * ncy + y;
            adp[i] = st.ad_p[cm];
            adv[i] = st.ad_v[cm];
            if (MODE == MODE_COUPLED) {
                // B-problem pressure RHS (src/solver/eqsolve_pv.cpp:452-461)
                if (y == 0) rp = (double)(ny - 1);
                else if (y < ny) rp = (double)(2 * (ny - ((y + 1) % 2)));
            }
        } else {
            adp[i] = 1.0;
            adv[i] = 1.0;
        }
        for (int c = 0; c < 3; ++c) rv[c * S + i] = mk(0, 0);
        dyb[i] = mk(rp, 0.0);
        fo[i] = mk(0, 0);
        pc[i] = mk(0, 0);
    }
    __syncthreads();

    if (tid < 2 * TC) {
        const unsigned mask = (1u << (2 * TC)) - 1u;
        const int l = tid >> 1, par = tid & 1;
        const int col = col0 + l;
        const bool active = col < nhalf;
        const int kzi = active ? col / nkx : 0;
        const int kx = active ? col - kzi * nkx : 0;
        const double ax = t.wavx[kx], az = t.wavz[kzi];
        const bool zero_col = active && col == d.zc;
        if (active)
            tau_chain(par, ny, pp.G_pre, 1.0, 0.0, zero_col, A.bcp_top, A.bcp_bot, st.wn_p[col], dyb + l,
                      pc + l, adp + l, TC, sWL, sWD, sWR);
        __syncwarp(mask);
        if (active) deriv_chain(par, ny, pc + l, dyb + l, TC);
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
                tau_chain(par, ny, g_v, pp.a_V[c], pp.b_V[c], zero_col, mk(0, 0), mk(0, 0), wv, fo + l, rc,
                          adv + l, TC, sWL, sWD, sWR);
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
                const int mir = (2 * d.NZS - kzi) * nkx + kx;   // column -kz
                A.divb_out[col] = div0;
                A.divb_out[d.ncol + col] = div1;
                A.divb_out[mir] = div0;
                A.divb_out[d.ncol + mir] = div1;
                s_c0[l] = mk(0, 0);
                s_c1[l] = mk(0, 0);
            } else {
                const double2 i00 = st.inf_div[col], i01 = st.inf_div[d.ncol + col];
                const double2 i10 = st.inf_div[2 * d.ncol + col], i11 = st.inf_div[3 * d.ncol + col];
                s_c0[l] = csub(cmul(div1, i10), cmul(div0, i11));
                s_c1[l] = csub(cmul(div0, i01), cmul(div1, i00));
            }
        }
    }
    __syncthreads();

    for (int i = tid; i < S; i += blockDim.x) {
        const int y = i / TC, l = i - (i / TC) * TC;
        const int col = col0 + l;
        if (col >= nhalf) continue;
        const int kzi = col / nkx, kx = col - (col / nkx) * nkx;
        const long long cm = ((long long)kzi * ncy + y) * nkx + kx;   // planar
        double2 p = pc[i];
        double2 v[3] = {rv[i], rv[S + i], rv[2 * S + i]};
        if (MODE == MODE_COUPLED) {
            const double2 c0 = s_c0[l], c1 = s_c1[l];
            p = cadd(p, cadd(cmul(c0, inf_value(st.p_inf[cm], false)), cmul(c1, inf_value(st.p_inf[d.Ns + cm], false))));
            for (int c = 0; c < 3; ++c)
                v[c] = cadd(v[c], cadd(cmul(c0, inf_value(st.v_inf[c * d.Ns + cm], inf_imag(c))),
                                       cmul(c1, inf_value(st.v_inf[(3 + c) * d.Ns + cm], inf_imag(c)))));
        }
        // the nonzero parts (the other parts are exact zeros)
        const double pv = p.x, vv[3] = {v[0].y, v[1].x, v[2].y};
        A.p_out[cm] = pv;
        for (int c = 0; c < 3; ++c) A.v_out[c * d.Ns + cm] = vv[c];
        const int kzm = 2 * d.NZS - kzi;
        if (kzm != kzi) {
            const long long mm = ((long long)kzm * ncy + y) * nkx + kx;
            A.p_out[mm] = pv;
            A.v_out[mm] = vv[0];
            A.v_out[d.Ns + mm] = vv[1];
            A.v_out[2 * d.Ns + mm] = -vv[2];
        }
    }
}

size_t setup_smem(const Dims &d) {
    const size_t S = (size_t)d.ncy * TC;
    return sizeof(double2) * 6 * S + sizeof(double) * (2 * S + 3 * (size_t)d.ncy);
}

// EqSolvePV::build_wn_ad (src/solver/eqsolve_pv.cpp:148-168), one thread per column;
// blockIdx.y = 0: the pressure operator (g = G_pre), 1: the velocity operator (g_v).
__global__ void k_wn_ad(Dims d, Tables t, double g_p, double g_v, double *wn_p, double *ad_p, double *wn_v,
                        double *ad_v) {
    const int col = blockIdx.x * blockDim.x + threadIdx.x;
    if (col >= d.ncol) return;
    const bool vel = blockIdx.y == 1;
    const double g = vel ? g_v : g_p;
    double *wn = vel ? wn_v : wn_p, *ad = vel ? ad_v : ad_p;
    const int kzi = col / d.nkx, kx = col - (col / d.nkx) * d.nkx;
    const double ax = t.wavx[kx], az = t.wavz[kzi];
    const double w = -((ax * ax + az * az) + g);
    wn[col] = w;
    const int n = d.NYS;
    double *A = ad + (long long)col * d.ncy;
    A[0] = 0.0;
    A[1] = 0.0;
    A[n] = 1.0 / (1.0 + t.WD[n] * w);
    A[n - 1] = 1.0 / (1.0 + t.WD[n - 1] * w);
    for (int y = n - 2; y >= 2; --y) {
        const double fc = t.WR[y] * t.WL[y + 2];
        const double den = 1.0 + (t.WD[y] - (fc * w) * A[y + 2]) * w;
        A[y] = 1.0 / den;
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
    const bool root = (col == d.zc);
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
__global__ void k_sigma0(Dims d, double re, const double *wn_v, const double *p_b,
                         const double *v_b, double2 *sigma0) {
    const int col = blockIdx.x * blockDim.x + threadIdx.x;
    if (col >= d.ncol) return;
    const int kzi = col / d.nkx, kx = col - (col / d.nkx) * d.nkx;
    const int n = d.NYS;
    const long long on = ((long long)kzi * d.ncy + n) * d.nkx + kx;   // planar (kz, n, kx)
    const double w = wn_v[col];
    const double2 vbn = inf_value(v_b[d.Ns + on], false);
    const double2 vbn1 = inf_value(v_b[d.Ns + on - d.nkx], false);
    const double2 pbn = inf_value(p_b[on], false);
    sigma0[col] = mk(re + w * vbn.x, w * vbn.y);
    double2 s1 = csub(mk(re + w * vbn1.x, w * vbn1.y), cscale(re * (2.0 * n), pbn));
    if (col == d.zc) s1 = mk(1.0, 0.0);
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
    const long long zc = (long long)d.zc * ncy;
    for (int y = par; y < ncy; y += 2) {
        r[y] = mk(y == 0 ? pp.Re : 0.0, 0.0);
        ad[y] = ad_v[zc + y];
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
}  // namespace

cudaError_t configure_setup_kernels(const Dims &d) {
    const int sm = (int)setup_smem(d);
    cudaError_t e = raise_smem(k_setup_solve<MODE_BASE>, sm);
    if (e != cudaSuccess) return e;
    return raise_smem(k_setup_solve<MODE_COUPLED>, sm);
}

void setup_solver(const Dims &d, const Tables &t, const PhysParams &pp, double g_v, SolverState &st,
                  double2 *, cudaStream_t s) {
    const int nb = (d.ncol + 127) / 128;
    k_wn_ad<<<dim3(nb, 2), 128, 0, s>>>(d, t, pp.G_pre, g_v, st.wn_p, st.ad_p, st.wn_v, st.ad_v);
    const int blocks = ((d.NZS + 1) * d.nkx + TC - 1) / TC;   // columns kz <= 0
    const size_t sm = setup_smem(d);
    // influence responses: pressure Dirichlet data (1,0) and (0,1), in one launch
    // (blockIdx.y = the response)
    {
        SetupArgs A{};
        A.bcp_top = mk(1.0, 0.0);
        A.bcp_bot = mk(0.0, 0.0);
        A.p_out = st.p_inf;
        A.v_out = st.v_inf;
        A.divb_out = st.inf_div;
        k_setup_solve<MODE_BASE><<<dim3(blocks, 2), kThreads, sm, s>>>(d, t, pp, g_v, st, A);
    }
    k_inf_normalize<<<nb, 128, 0, s>>>(d, pp.a_V[1], st.inf_div);
    {
        SetupArgs A{};
        A.p_out = st.p_b;
        A.v_out = st.v_b;
        k_setup_solve<MODE_COUPLED><<<blocks, kThreads, sm, s>>>(d, t, pp, g_v, st, A);
    }
    k_sigma0<<<nb, 128, 0, s>>>(d, pp.Re, st.wn_v, st.p_b, st.v_b, st.sigma0);
    // the zero mode's unit responses (correct_flow): only where that column is held
    const size_t smu = sizeof(double2) * 2 * d.ncy + sizeof(double) * 4 * d.ncy;
    if (d.zc >= 0) k_unit_response<<<1, 2, smu, s>>>(d, t, pp, g_v, st.ad_v, st.unit);
}

}  // namespace cdns
