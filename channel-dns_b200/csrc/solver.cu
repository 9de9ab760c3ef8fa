// Per-(kz, kx) Chebyshev-tau pressure/velocity solve of the channel-dns step
// (EqSolvePV, src/solver/eqsolve_pv.cpp) for sm_100a.
//
// One warp owns one spectral column (kz, kx) and keeps all its y coefficients
// in registers.  Lane L = 2h + p holds, for every field, the coefficients of
// parity p at y = 2(E h + e) + p, e = 0..E-1 (E = ceil((NYS+1)/32) rounded up
// to 1, 2, 4 or 8).  Every tau recurrence (src/solver/eqsolve_pv.cpp:64-128)
// and every Chebyshev derivative recurrence (src/solver/vector_ops.cpp:17-25)
// couples only coefficients of one parity, so each becomes a first-order
// affine recurrence along the 16 lanes of that parity: a sequential pass over
// a lane's E coefficients, a 4-level shuffle scan over the lanes, and a
// carry-in.  Wall sums are shuffle reductions.  This reassociates the
// reference's sequential sums and recurrences; the results agree with the
// sequential order to round-off (tested against the oracle at 1e-10).
//
// The step solve reads the spectral state in its planar [kz][y][kx] layout
// through swizzled shared-memory tiles (a block of TC warps owns TC
// consecutive columns, so every global access is a coalesced row of TC
// columns).  The warps leave the uncorrected solution in the tiles together
// with four coefficients per column; the influence-matrix and sigma
// corrections then run over the block as one coalesced elementwise pass over
// the planar influence and B-problem fields (solver_setup.cu).  The tau
// pivots are stored column-major ([col][y]) and read by each warp directly.
#include "cdns_kernels.cuh"
#include "warp_columns.cuh"

namespace cdns {

namespace {
constexpr int TC = kColsPerBlock;     // columns (warps) per block
constexpr int kThreads = 32 * TC;

struct SolveArgs {
    double p_a, p_b;           // pressure wall condition a P + b dP/dn
    double2 *p_out;            // [Ns] planar
    double2 *v_out;            // [3][Ns] planar
    StepArgs step;
};


// Tau solve of (D^2 - k^2 - g) f = r with a f + b f' = (lower, upper) at
// y = (+1, -1), both parities at once (src/solver/eqsolve_pv.cpp:64-128).
// r must be zero beyond ny.  Returns false in a lane whose parity's pivot is
// zero or not finite.
template <int E>
__device__ bool tau_warp(int ny, double g, double a, double b, bool zero_col, double2 lower,
                         double2 upper, double w, const double2 (&r)[E], double2 (&out)[E],
                         const double (&ad)[E], const double *__restrict__ WL,
                         const double *__restrict__ WD, const double *__restrict__ WR) {
    const int L = lane_id(), p = L & 1;
    const bool normalize = g == 0.0 && a == 0.0 && zero_col;
    const int top = ((ny & 1) == p) ? ny : ny - 1;
    double2 rr[E];
#pragma unroll
    for (int e = 0; e < E; ++e) rr[e] = r[e];
    if (normalize) {
        // the even chain of the singular zero column is closed by the mean
        // (eqsolve_pv.cpp:71-79): r_0 <- sum_{y>=2 even} r_y/(y^2-1) + (lo+up)/(2b)
        double2 part = mk(0.0, 0.0);
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const int y = ycoef<E>(e);
            if (p == 0 && y >= 2 && y <= ny) part = cadd(part, cdivr(r[e], (double)(y * y - 1)));
        }
        part = sum_parity(part);
        if (b != 0.0) part = cadd(part, cdivr(cadd(lower, upper), 2.0 * b));
        if (L == 0) rr[0] = part;
    }
    // three-term combination of the rhs
    double2 rm2_0 = shfl2_up(rr[E - 1], 2);
    double2 rp2_l = shfl2_down(rr[0], 2);
    if (L + 2 >= 32) rp2_l = mk(0.0, 0.0);
    double2 X[E];
#pragma unroll
    for (int e = 0; e < E; ++e) {
        const int y = ycoef<E>(e);
        const double2 rm2 = e > 0 ? rr[(e + E - 1) % E] : rm2_0;
        const double2 rp2 = e + 1 < E ? rr[(e + 1) % E] : rp2_l;
        if (y > ny) X[e] = mk(0.0, 0.0);
        else if (y == p) X[e] = (p == 0) ? cdivr(cadd(lower, upper), 2.0) : cdivr(csub(lower, upper), 2.0);
        else if (y >= ny - 1) X[e] = cadd(cscale(WL[y], rm2), cscale(WD[y], rr[e]));
        else X[e] = cadd(cadd(cscale(WL[y], rm2), cscale(WD[y], rr[e])), cscale(WR[y], rp2));
    }
    // pivots one step up the chain, AD(y + 2)
    double adn_l = __shfl_down_sync(kFull, ad[0], 2);
    if (L + 2 >= 32) adn_l = 0.0;
    // backward sweep X_y -= (WR_y w AD_{y+2}) X_{y+2} for 2 <= y <= top - 2
    double A[E];
#pragma unroll
    for (int e = 0; e < E; ++e) {
        const int y = ycoef<E>(e);
        const double adn = e + 1 < E ? ad[(e + 1) % E] : adn_l;
        A[e] = (y >= 2 && y <= top - 2) ? -((WR[y] * w) * adn) : 0.0;
    }
    affine_suffix<E>(A, X);
    // pivot chain ad01_j = tau(j) - (WL_{j+2} w ad01_{j+2}) AD_{j+2}, ad01_top = tau(top)
    double Aa[E], Ba[E];
#pragma unroll
    for (int e = 0; e < E; ++e) {
        const int y = ycoef<E>(e);
        const double adn = e + 1 < E ? ad[(e + 1) % E] : adn_l;
        if (y > top) {
            Aa[e] = 0.0;
            Ba[e] = 0.0;
        } else if (y == top) {
            Aa[e] = 0.0;
            Ba[e] = tau_func(a, b, y);
        } else {
            Aa[e] = -((WL[y + 2] * w) * adn);
            Ba[e] = tau_func(a, b, y);
        }
    }
    affine_suffix<E>(Aa, Ba);
    // o0 = X_par - sum_{j = par+2..top} ad01_j AD_j X_j ; pivot ad01_par
    double2 s = mk(0.0, 0.0);
#pragma unroll
    for (int e = 0; e < E; ++e) {
        const int y = ycoef<E>(e);
        if (y >= p + 2 && y <= top) s = cadd(s, cscale(Ba[e] * ad[e], X[e]));
    }
    s = sum_parity(s);
    double2 o0 = csub(shfl2(X[0], p), s);
    double piv = __shfl_sync(kFull, Ba[0], p);
    if (normalize && p == 0) {
        o0 = mk(0.0, 0.0);
        piv = 1.0;
    }
    const bool ok = isfinite(piv) && piv != 0.0;
    const double2 zpar = cdivr(o0, piv);
    // forward sweep Z_y = AD_y (X_y - WL_y w Z_{y-2})
#pragma unroll
    for (int e = 0; e < E; ++e) {
        const int y = ycoef<E>(e);
        if (y == p) {
            A[e] = 0.0;
            X[e] = zpar;
        } else if (y <= ny) {
            A[e] = -(ad[e] * (WL[y] * w));
            X[e] = cscale(ad[e], X[e]);
        } else {
            A[e] = 0.0;
            X[e] = mk(0.0, 0.0);
        }
    }
    affine_prefix<E>(A, X);
#pragma unroll
    for (int e = 0; e < E; ++e) out[e] = ycoef<E>(e) <= ny ? X[e] : mk(0.0, 0.0);
    return ok;
}

template <int E>
__global__ void __launch_bounds__(kThreads, E <= 4 ? 2 : 1)
k_solve(Dims d, Tables t, PhysParams pp, double g_v, SolverState st, SolveArgs A) {
    extern __shared__ double2 tile[];   // [4][ncy][TC]
    __shared__ double2 s_c0[TC], s_c1[TC], s_sg[2][TC];   // per-column correction coefficients
    const int ncy = d.ncy, ny = d.NYS, nkx = d.nkx, ncol = d.ncol;
    const int S = ncy * TC;
    const int col0 = blockIdx.x * TC;
    const int tid = threadIdx.x;
    const int w = tid >> 5;
    const int L = tid & 31, p = L & 1;
    const int col = col0 + w;
    const StepArgs &s = A.step;

    // ---- stage R = a0 u + a1 u_prev + b0 N + b1 N_prev and N_y -------------
#pragma unroll 2
    for (int i = tid; i < S; i += kThreads) {
        const int y = i / TC, l = i - (i / TC) * TC;
        const int c2 = col0 + l;
        if (c2 < ncol) {
            const int kzi = c2 / nkx, kx = c2 - (c2 / nkx) * nkx;
            const long long off = ((long long)kzi * ncy + y) * nkx + kx;
            const int sl = tile_slot<E>(y, l);
            double2 nv[3];
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                const long long o = c * d.Ns + off;
                nv[c] = s.N[o];
                // R (src/sim/simulation.cpp:151-158)
                tile[c * S + sl] = cadd(cadd(cadd(cscale(s.a0, s.u[o]), cscale(s.a1, s.u_prev[o])),
                                             cscale(s.b0, nv[c])),
                                        cscale(s.b1, s.N_prev[o]));
            }
            tile[3 * S + sl] = nv[1];
        }
    }
    __syncthreads();

    if (col < ncol) {
        const int kzi = col / nkx, kx = col - kzi * nkx;
        const double ax = t.wavx[kx], az = t.wavz[kzi];
        const bool zero_col = col == d.zc;
        const long long cm = (long long)col * ncy;   // column-major base
        bool pivot_fail = false;
        double2 pv[E], v0[E], v1[E], v2[E], dy[E];
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const int y = ycoef<E>(e);
            if (y <= ny) {
                const int sl = tile_slot<E>(y, w);
                v0[e] = tile[sl];
                v1[e] = tile[S + sl];
                v2[e] = tile[2 * S + sl];
                dy[e] = tile[3 * S + sl];
            } else {
                v0[e] = v1[e] = v2[e] = dy[e] = mk(0.0, 0.0);
            }
        }
        double2 lower, upper;
        if (s.bc_p) {
            lower = s.bc_p[col];
            upper = s.bc_p[ncol + col];
        } else {
            // pressure wall data (src/solver/eqsolve_pv.cpp:322-337)
            double2 st_ = mk(0, 0), sb_ = mk(0, 0);
#pragma unroll
            for (int e = 0; e < E; ++e) {
                st_ = cadd(st_, dy[e]);
                sb_ = p ? cadd(sb_, dy[e]) : csub(sb_, dy[e]);
            }
            st_ = sum_warp(st_);
            sb_ = sum_warp(sb_);
            const double2 bt = cadd(s.bw[col], st_);
            const double2 bb = cadd(s.bw[ncol + col], sb_);
            if (L == 0) {
                s.B_new[col] = bt;
                s.B_new[ncol + col] = bb;
            }
            // combined wall data b0 B + b1 B_prev (src/sim/simulation.cpp:146-150)
            lower = cadd(cscale(s.b0, bt), cscale(s.b1, s.B_prev[col]));
            upper = cadd(cscale(s.b0, bb), cscale(s.b1, s.B_prev[ncol + col]));
        }
        // divergence of R (src/solver/eqsolve_pv.cpp:340-357)
        deriv_warp<E>(ny, v1, dy);
#pragma unroll
        for (int e = 0; e < E; ++e)
            if (ycoef<E>(e) <= ny) dy[e] = cadd(cadd(fderiv(ax, v0[e]), dy[e]), fderiv(az, v2[e]));
        // pressure
        double ad[E];
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const int y = ycoef<E>(e);
            ad[e] = y <= ny ? st.ad_p[cm + y] : 0.0;
        }
        pivot_fail |= !tau_warp<E>(ny, pp.G_pre, A.p_a, A.p_b, zero_col, lower, upper, st.wn_p[col], dy, pv,
                                   ad, t.WL, t.WD, t.WR);
        const double2 tail0 = elem<E>(v1, ny), tail1 = elem<E>(v1, ny - 1);
        // velocity: Re (grad P - R) (src/solver/eqsolve_pv.cpp:359-395)
        deriv_warp<E>(ny, pv, dy);
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const int y = ycoef<E>(e);
            ad[e] = y <= ny ? st.ad_v[cm + y] : 0.0;
        }
        const double wv = st.wn_v[col];
        auto velocity = [&](int c, double2(&vc)[E]) {
            double2 f[E];
#pragma unroll
            for (int e = 0; e < E; ++e) {
                const double2 grad = (c == 0) ? fderiv(ax, pv[e]) : (c == 1) ? dy[e] : fderiv(az, pv[e]);
                f[e] = ycoef<E>(e) <= ny ? cscale(pp.Re, csub(grad, vc[e])) : mk(0.0, 0.0);
            }
            const double2 blo = s.bc_v[(2 * c) * ncol + col], bup = s.bc_v[(2 * c + 1) * ncol + col];
            pivot_fail |= !tau_warp<E>(ny, g_v, pp.a_V[c], pp.b_V[c], zero_col, blo, bup, wv, f, vc, ad,
                                       t.WL, t.WD, t.WR);
        };
        velocity(0, v0);
        velocity(1, v1);
        velocity(2, v2);
        // wall divergence by endpoint sums (src/solver/eqsolve_pv.cpp:397-406)
        double2 div0 = mk(0, 0), div1 = mk(0, 0);
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const int y = ycoef<E>(e);
            const double2 tang = cadd(fderiv(ax, v0[e]), fderiv(az, v2[e]));
            const double2 nrm = cscale((double)(y * y), v1[e]);
            div0 = cadd(div0, cadd(tang, nrm));
            div1 = p ? cadd(div1, cadd(mk(-tang.x, -tang.y), nrm)) : cadd(div1, csub(tang, nrm));
        }
        div0 = sum_warp(div0);
        div1 = sum_warp(div1);
        // influence and sigma coefficients (src/solver/eqsolve_pv.cpp:408-429)
        const double2 i00 = st.inf_div[col], i01 = st.inf_div[ncol + col];
        const double2 i10 = st.inf_div[2 * ncol + col], i11 = st.inf_div[3 * ncol + col];
        const double2 c0 = csub(cmul(div1, i10), cmul(div0, i11));
        const double2 c1 = csub(cmul(div0, i01), cmul(div1, i00));
        const long long o_n = ((long long)kzi * ncy + ny) * nkx + kx, o_n1 = o_n - nkx;
        const double2 ptop = cadd(elem<E>(pv, ny), cadd(inf_mul(c0, st.p_inf[o_n], false),
                                                        inf_mul(c1, st.p_inf[d.Ns + o_n], false)));
        const double2 vt0 = cadd(elem<E>(v1, ny), cadd(inf_mul(c0, st.v_inf[d.Ns + o_n], false),
                                                       inf_mul(c1, st.v_inf[4 * d.Ns + o_n], false)));
        const double2 vt1 = cadd(elem<E>(v1, ny - 1), cadd(inf_mul(c0, st.v_inf[d.Ns + o_n1], false),
                                                           inf_mul(c1, st.v_inf[4 * d.Ns + o_n1], false)));
        const double2 n0 = csub(cscale(-wv, vt0), cscale(pp.Re, tail0));
        const double2 n1 = cadd(cscale(-wv, vt1), cscale(pp.Re, csub(cscale(2.0 * ny, ptop), tail1)));
        if (L == 0) {
            s_c0[w] = c0;
            s_c1[w] = c1;
            s_sg[0][w] = cdiv(n0, st.sigma0[col]);
            s_sg[1][w] = cdiv(n1, st.sigma0[ncol + col]);
        }
        // uncorrected solution into the tile (each warp rewrites only its own column's slots)
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const int y = ycoef<E>(e);
            if (y > ny) continue;
            const int sl = tile_slot<E>(y, w);
            tile[sl] = pv[e];
            tile[S + sl] = v0[e];
            tile[2 * S + sl] = v1[e];
            tile[3 * S + sl] = v2[e];
        }
        if (__any_sync(kFull, pivot_fail) && L == 0) atomicOr(s.err, ERR_PIVOT);
    }
    __syncthreads();

    // ---- influence and sigma corrections, coalesced over the block --------
    // odd-y coefficients take sigma_0 for p, u, w and sigma_1 for v; even-y the reverse
    const int zc = d.zc;   // the (kz, kx) = (0, 0) column (-1: not on this rank)
    const bool fix_zero = !s.solve_only && zc >= col0 && zc < col0 + TC;
    bool bad = false;
    for (int i = tid; i < S; i += kThreads) {
        const int y = i / TC, l = i - (i / TC) * TC;
        const int c2 = col0 + l;
        if (c2 >= ncol) continue;
        const int kzi = c2 / nkx, kx = c2 - (c2 / nkx) * nkx;
        const long long off = ((long long)kzi * ncy + y) * nkx + kx;
        const int sl = tile_slot<E>(y, l);
        const double2 c0 = s_c0[l], c1 = s_c1[l];
        const double2 sq = s_sg[(y + 1) & 1][l], sv = s_sg[y & 1][l];
        double2 pr = cadd(tile[sl], cadd(inf_mul(c0, st.p_inf[off], false), inf_mul(c1, st.p_inf[d.Ns + off], false)));
        pr = cadd(pr, inf_mul(sq, st.p_b[off], false));
        double2 v[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            v[c] = cadd(tile[(1 + c) * S + sl], cadd(inf_mul(c0, st.v_inf[c * d.Ns + off], inf_imag(c)),
                                                     inf_mul(c1, st.v_inf[(3 + c) * d.Ns + off], inf_imag(c))));
            v[c] = cadd(v[c], inf_mul(c == 1 ? sv : sq, st.v_b[c * d.Ns + off], inf_imag(c)));
        }
        if (fix_zero && c2 == zc) {
            tile[sl] = pr;
#pragma unroll
            for (int c = 0; c < 3; ++c) tile[(1 + c) * S + sl] = v[c];
            continue;
        }
        bad |= !(isfinite(pr.x) && isfinite(pr.y) && isfinite(v[0].x) && isfinite(v[0].y) && isfinite(v[1].x) &&
                 isfinite(v[1].y) && isfinite(v[2].x) && isfinite(v[2].y));
        A.p_out[off] = pr;
#pragma unroll
        for (int c = 0; c < 3; ++c) A.v_out[c * d.Ns + off] = v[c];
    }
    if (fix_zero) {
        __syncthreads();
        if (w == zc - col0) {
            const int kzi = d.NZS;
            double2 pz[E], u0[E], u1[E], u2[E];
#pragma unroll
            for (int e = 0; e < E; ++e) {
                const int y = ycoef<E>(e);
                const int sl = tile_slot<E>(y <= ny ? y : 0, w);
                pz[e] = tile[sl];
                u0[e] = tile[S + sl];
                u2[e] = tile[3 * S + sl];
            }
            // correct_zero_mode (src/solver/timestepper.cpp:60-68)
            const double2 v1w = cscale(0.5, cadd(s.bc_v[2 * ncol + zc], s.bc_v[3 * ncol + zc]));
#pragma unroll
            for (int e = 0; e < E; ++e) u1[e] = ycoef<E>(e) == 0 ? v1w : mk(0.0, 0.0);
            // correct_flow (src/sim/simulation.cpp:111-140), single-rank branch
            const double *uu = st.unit;
            double dpdx, dpdz;
            bool pfail = false;
            if (pp.grad_pre == 1) {
                dpdx = pp.gx;
                dpdz = pp.gz;
            } else {
                double qx = 0.0, qz = 0.0;
#pragma unroll
                for (int e = 0; e < E; ++e) {
                    const int y = ycoef<E>(e);
                    if (p == 0 && y <= ny) {
                        qx += u0[e].x / (double)(y * y - 1);
                        qz += u2[e].x / (double)(y * y - 1);
                    }
                }
                qx = -sum_warp(qx);
                qz = -sum_warp(qz);
                const double qxu = uu[2 * ncy], qzu = uu[2 * ncy + 1];
                pfail = !isfinite(qxu) || qxu == 0.0 || !isfinite(qzu) || qzu == 0.0;
                dpdx = (pp.qxm - qx) / qxu;
                dpdz = (pp.qzm - qz) / qzu;
            }
            if (L == 0) {
                s.dpdx[0] = dpdx;
                s.dpdx[1] = dpdz;
                if (pfail) atomicOr(s.err, ERR_PIVOT);
            }
#pragma unroll
            for (int e = 0; e < E; ++e) {
                const int y = ycoef<E>(e);
                if (y > ny) continue;
                u0[e].x += dpdx * uu[y];
                u2[e].x += dpdz * uu[ncy + y];
                bad |= !(isfinite(pz[e].x) && isfinite(pz[e].y) && isfinite(u0[e].x) && isfinite(u0[e].y) &&
                         isfinite(u1[e].x) && isfinite(u1[e].y) && isfinite(u2[e].x) && isfinite(u2[e].y));
                const long long off = ((long long)kzi * ncy + y) * nkx;
                A.p_out[off] = pz[e];
                A.v_out[off] = u0[e];
                A.v_out[d.Ns + off] = u1[e];
                A.v_out[2 * d.Ns + off] = u2[e];
            }
        }
    }
    if (__any_sync(kFull, bad) && L == 0) atomicOr(s.err, ERR_NONFINITE);
}

size_t solve_smem(const Dims &d) { return sizeof(double2) * 4 * (size_t)d.ncy * TC; }

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

template <int E>
cudaError_t configure_e(const Dims &d) {
    return raise_smem(k_solve<E>, (int)solve_smem(d));
}

template <int E>
void step_e(const Dims &d, const Tables &t, const PhysParams &pp, double g_v, const SolverState &st,
            const SolveArgs &A, cudaStream_t s) {
    const int blocks = (d.ncol + TC - 1) / TC;
    k_solve<E><<<blocks, kThreads, solve_smem(d), s>>>(d, t, pp, g_v, st, A);
}
}  // namespace

void launch_pressure_bc(const Dims &d, const double2 *N, const double2 *bw, double2 *B,
                        cudaStream_t s) {
    k_pressure_bc<<<(d.ncol + 127) / 128, 128, 0, s>>>(d, N, bw, B);
}

cudaError_t configure_solver_kernels(const Dims &d) {
    cudaError_t e = configure_setup_kernels(d);
    if (e != cudaSuccess) return e;
    switch (lane_elems(d)) {
    case 1: return configure_e<1>(d);
    case 2: return configure_e<2>(d);
    case 4: return configure_e<4>(d);
    case 8: return configure_e<8>(d);
    default: return cudaErrorInvalidValue;   // more than 256 Chebyshev coefficients
    }
}

void launch_step_solve(const Dims &d, const Tables &t, const PhysParams &pp, double g_v,
                       const SolverState &st, const StepArgs &a, cudaStream_t s) {
    SolveArgs A{};
    A.p_a = pp.a_pre0;
    A.p_b = pp.b_pre0;
    A.p_out = a.p_out;
    A.v_out = a.u_out;
    A.step = a;
    switch (lane_elems(d)) {
    case 1: step_e<1>(d, t, pp, g_v, st, A, s); break;
    case 2: step_e<2>(d, t, pp, g_v, st, A, s); break;
    case 4: step_e<4>(d, t, pp, g_v, st, A, s); break;
    case 8: step_e<8>(d, t, pp, g_v, st, A, s); break;
    default: break;
    }
}

}  // namespace cdns
