// Discrete adjoint of the channel-dns step (FP64) for sm_100a.
//
// Every forward stage is linear except u x omega, so the adjoint of a step is
// the transposes of its linear stages in reverse order plus the linearised
// product.  This file holds the transposes of the column solve (k_solve in
// solver.cu): the same warp-per-column layout, with every recurrence run in
// the opposite direction (a prefix scan becomes a suffix scan and vice
// versa) and the influence / sigma corrections turned into per-column
// reductions.  Transposes are with respect to the real inner product
// Re sum conj(a) b over the stored spectral arrays, so a product by a complex
// constant c transposes to a product by conj(c).
#include <algorithm>

#include "cdns_kernels.cuh"
#include "warp_columns.cuh"

namespace cdns {

namespace {
constexpr int TC = kColsPerBlock;
constexpr int kThreads = 32 * TC;

__device__ __forceinline__ double2 cmulc(double2 a, double2 b) { return cmul(cconj(a), b); }   // conj(a) b
// conj(a) b for an influence value a stored by its nonzero part (inf_imag)
__device__ __forceinline__ double2 cmulc_inf(double part, bool imag, double2 b) { return cmulc(inf_value(part, imag), b); }

// Transpose of the Chebyshev derivative d_k = sum_{j>k, j-k odd} 2 j f_j,
// d_0 halved, d_NYS = 0: lf_j = 2 j sum_{k<j, k=j-1 mod 2} g_k, g_0 = ld_0 / 2.
template <int E> __device__ __forceinline__ void deriv_T(int ny, const double2 (&ld)[E], double2 (&lf)[E]) {
    const int L = lane_id(), p = L & 1;
    double2 P[E];
#pragma unroll
    for (int e = 0; e < E; ++e) {
        const int y = ycoef<E>(e);
        P[e] = y < ny ? (y == 0 ? cscale(0.5, ld[e]) : ld[e]) : mk(0.0, 0.0);
    }
    prefix_sum<E>(P);
    // value at y - 1 (the neighbour of opposite parity)
    double2 a[E];
#pragma unroll
    for (int e = 0; e < E; ++e) a[e] = shfl2_xor(P[e], 1);
    double2 c = shfl2_up(P[E - 1], 1);
    if (L == 0) c = mk(0.0, 0.0);
#pragma unroll
    for (int e = 0; e < E; ++e) {
        const int y = ycoef<E>(e);
        const double2 prev = (p == 1) ? a[e] : (e > 0 ? a[(e + E - 1) % E] : c);
        lf[e] = (y >= 1 && y <= ny) ? cscale((double)(2 * y), prev) : mk(0.0, 0.0);
    }
}

// Transpose of tau_warp (solver.cu): given the adjoint lz of the tau
// solution, the adjoints of its right-hand side (lr) and of its wall data.
template <int E>
__device__ void tau_adj(int ny, double g, double a, double b, bool zero_col, double w, const double2 (&lz)[E],
                        double2 (&lr)[E], double2 &llower, double2 &lupper, const double (&ad)[E],
                        const double *__restrict__ WL, const double *__restrict__ WD,
                        const double *__restrict__ WR) {
    const int L = lane_id(), p = L & 1;
    const bool normalize = g == 0.0 && a == 0.0 && zero_col;
    const int top = ((ny & 1) == p) ? ny : ny - 1;
    double adn_l = __shfl_down_sync(kFull, ad[0], 2);
    if (L + 2 >= 32) adn_l = 0.0;
    // forward coefficients: backward sweep A_b, pivot chain ad01, forward sweep A_f
    double Ab[E], Aa[E], Ba[E], Af[E];
#pragma unroll
    for (int e = 0; e < E; ++e) {
        const int y = ycoef<E>(e);
        const double adn = e + 1 < E ? ad[(e + 1) % E] : adn_l;
        Ab[e] = (y >= 2 && y <= top - 2) ? -((WR[y] * w) * adn) : 0.0;
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
        Af[e] = (y == p || y > ny) ? 0.0 : -(ad[e] * (WL[y] * w));
    }
    affine_suffix<E>(Aa, Ba);   // Ba = ad01
    double piv = __shfl_sync(kFull, Ba[0], p);
    if (normalize && p == 0) piv = 1.0;
    // 1. forward sweep Z_y = B_y + Af_y Z_{y-2}: transpose lB_y = lZ_y + Af_{y+2} lB_{y+2}
    double An[E];
    double af_l = __shfl_down_sync(kFull, Af[0], 2);
    if (L + 2 >= 32) af_l = 0.0;
    double2 lB[E];
#pragma unroll
    for (int e = 0; e < E; ++e) {
        const int y = ycoef<E>(e);
        An[e] = y <= ny ? (e + 1 < E ? Af[(e + 1) % E] : af_l) : 0.0;
        lB[e] = y <= ny ? lz[e] : mk(0.0, 0.0);
    }
    affine_suffix<E>(An, lB);
    // 2. B_p = zpar, B_y = AD_y X_y
    const double2 lzpar = shfl2(lB[0], p);
    double2 lX[E];
#pragma unroll
    for (int e = 0; e < E; ++e) {
        const int y = ycoef<E>(e);
        lX[e] = (y != p && y <= ny) ? cscale(ad[e], lB[e]) : mk(0.0, 0.0);
    }
    // 3-4. zpar = o0 / piv, o0 = X_p - sum_{p+2 <= y <= top} ad01_y AD_y X_y
    double2 lo0 = cdivr(lzpar, piv);
    if (normalize && p == 0) lo0 = mk(0.0, 0.0);
#pragma unroll
    for (int e = 0; e < E; ++e) {
        const int y = ycoef<E>(e);
        if (y >= p + 2 && y <= top) lX[e] = csub(lX[e], cscale(Ba[e] * ad[e], lo0));
        if (y == p) lX[e] = cadd(lX[e], lo0);
    }
    // 5. backward sweep X_y = X0_y + Ab_y X_{y+2}: transpose lX0_y = lX_y + Ab_{y-2} lX0_{y-2}
    double ab_f = __shfl_up_sync(kFull, Ab[E - 1], 2);
    if (L < 2) ab_f = 0.0;
#pragma unroll
    for (int e = 0; e < E; ++e) An[e] = e > 0 ? Ab[(e + E - 1) % E] : ab_f;
    affine_prefix<E>(An, lX);   // lX = lX0
    // 6. three-term combination and the wall-data rows
    const double2 lx00 = shfl2(lX[0], 0), lx01 = shfl2(lX[0], 1);
    llower = cscale(0.5, cadd(lx00, lx01));
    lupper = cscale(0.5, csub(lx00, lx01));
    double2 tw[E], uL[E], vR[E];
#pragma unroll
    for (int e = 0; e < E; ++e) {
        const int y = ycoef<E>(e);
        tw[e] = (y != p && y <= ny) ? lX[e] : mk(0.0, 0.0);
        uL[e] = (y != p && y <= ny) ? cscale(WL[y], tw[e]) : mk(0.0, 0.0);
        vR[e] = (y != p && y <= ny - 2) ? cscale(WR[y], tw[e]) : mk(0.0, 0.0);
    }
    double2 u_l = shfl2_down(uL[0], 2);
    if (L + 2 >= 32) u_l = mk(0.0, 0.0);
    double2 v_f = shfl2_up(vR[E - 1], 2);
    if (L < 2) v_f = mk(0.0, 0.0);
#pragma unroll
    for (int e = 0; e < E; ++e) {
        const int y = ycoef<E>(e);
        const double2 up = e + 1 < E ? uL[(e + 1) % E] : u_l;   // WL_{y+2} lX0_{y+2}
        const double2 dn = e > 0 ? vR[(e + E - 1) % E] : v_f;  // WR_{y-2} lX0_{y-2}
        lr[e] = y <= ny ? cadd(cadd(y != p ? cscale(WD[y], tw[e]) : mk(0.0, 0.0), up), dn) : mk(0.0, 0.0);
    }
    // 7. the singular zero column's closed even chain: r_0 <- sum r_y/(y^2-1) + (lo+up)/(2b)
    if (normalize) {
        const double2 lpart = shfl2(lr[0], 0);
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const int y = ycoef<E>(e);
            if (y == 0) lr[e] = mk(0.0, 0.0);
            else if (p == 0 && y <= ny) lr[e] = cadd(lr[e], cdivr(lpart, (double)(y * y - 1)));
        }
        if (b != 0.0) {
            const double2 lb = cdivr(lpart, 2.0 * b);
            llower = cadd(llower, lb);
            lupper = cadd(lupper, lb);
        }
    }
}

struct AdjArgs {
    double p_a, p_b;
    const double2 *lp;        // [Ns] adjoint of the pressure (may be null)
    const double2 *lv;        // [3][Ns] adjoint of the new velocity
    double2 *lR;              // [3][Ns] adjoint of the right-hand side R
    double2 *lBc;             // [2][ncol] adjoint of the pressure wall data
    double2 *lbcv;            // [3][2][ncol] adjoint of the velocity wall data (accumulated)
    int solve_only;           // 1: no zero-mode overwrite (cdns_solve)
    double seed;              // objective seed on the mean profile (0: none)
    // Reverse-step bookkeeping in place of the lR output (acc != 0), for
    // R = a0 u^{s-1} + a1 u^{s-2} + b0 N^{s-1} + b1 N^{s-2} and wall data
    // b0 B^{s-1} + b1 B^{s-2} (B = bw + wall sums of N_y):
    //   lu1 += a0 lR, lu2 = a1 lR, lN1 += b0 lR (+ wall sums^T(lbw) in y),
    //   lN2 = b1 lR, lbw = lB1 + b0 lBc, lB2 = b1 lBc.
    int acc;
    double a0, a1, b0, b1;
    double2 *lu1, *lu2, *lN1, *lN2, *lbw, *lB2;
    const double2 *lB1;
};

template <int E>
__global__ void __launch_bounds__(kThreads, E <= 2 ? 2 : 1)
k_solve_adj(Dims d, Tables t, PhysParams pp, double g_v, SolverState st, AdjArgs A) {
    extern __shared__ double2 tile[];   // [4][ncy][TC]
    __shared__ double2 red[TC][TC][4];  // [warp][column][lc0, lc1, lsg0, lsg1]
    __shared__ double2 s_zbc;           // zero mode: adjoint of the mean wall v
    __shared__ double2 s_bw[TC][2];     // per column: complete lbw (top, bottom)
    const int ncy = d.ncy, ny = d.NYS, nkx = d.nkx, ncol = d.ncol;
    const long long Ns = d.Ns;
    const int S = ncy * TC;
    const int col0 = blockIdx.x * TC;
    const int tid = threadIdx.x, w = tid >> 5, L = tid & 31, p = L & 1;
    const int zc = d.zc;
    const bool zero_mode = !A.solve_only;

    // ---- correction pass transposed: coalesced loads, per-column sums ------
    // (a thread's elements all belong to column l = tid % TC)
    double2 acc[4] = {mk(0, 0), mk(0, 0), mk(0, 0), mk(0, 0)};
    if (tid == 0) s_zbc = mk(0.0, 0.0);
    __syncthreads();
    for (int i = tid; i < S; i += kThreads) {
        const int y = i / TC, l = i - (i / TC) * TC;
        const int c2 = col0 + l;
        if (c2 >= ncol) continue;
        const int kzi = c2 / nkx, kx = c2 - (c2 / nkx) * nkx;
        const long long off = ((long long)kzi * ncy + y) * nkx + kx;
        const int sl = tile_slot<E>(y, l);
        const double2 lp = A.lp ? A.lp[off] : mk(0.0, 0.0);
        double2 lv[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) lv[c] = A.lv[c * Ns + off];
        if (zero_mode && c2 == zc) {
            // correct_zero_mode overwrote v: only the mean wall v at y = 0 carries an adjoint
            if (y == 0) s_zbc = cscale(0.5, lv[1]);
            lv[1] = mk(0.0, 0.0);
            // wall shear objective: d/dRe(u_y) of seed * sum_{y even} y^2 Re(u_y)
            if ((y & 1) == 0) lv[0].x += A.seed * (double)(y * y);
        }
        tile[sl] = lp;
#pragma unroll
        for (int c = 0; c < 3; ++c) tile[(1 + c) * S + sl] = lv[c];
        acc[0] = cadd(acc[0], cmulc_inf(st.p_inf[off], false, lp));
        acc[1] = cadd(acc[1], cmulc_inf(st.p_inf[Ns + off], false, lp));
        const int qi = (y + 1) & 1, vi = y & 1;
        double2 sq = cmulc_inf(st.p_b[off], false, lp);
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            acc[0] = cadd(acc[0], cmulc_inf(st.v_inf[c * Ns + off], inf_imag(c), lv[c]));
            acc[1] = cadd(acc[1], cmulc_inf(st.v_inf[(3 + c) * Ns + off], inf_imag(c), lv[c]));
            if (c != 1) sq = cadd(sq, cmulc_inf(st.v_b[c * Ns + off], inf_imag(c), lv[c]));
        }
        acc[2 + qi] = cadd(acc[2 + qi], sq);
        acc[2 + vi] = cadd(acc[2 + vi], cmulc_inf(st.v_b[Ns + off], false, lv[1]));
    }
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        acc[k] = cadd(acc[k], shfl2_xor(acc[k], 8));
        acc[k] = cadd(acc[k], shfl2_xor(acc[k], 16));
        if (L < TC) red[w][L][k] = acc[k];
    }
    __syncthreads();

    const int col = col0 + w;
    if (col < ncol) {
        const int kzi = col / nkx, kx = col - kzi * nkx;
        const double ax = t.wavx[kx], az = t.wavz[kzi];
        const bool zero_col = col == d.zc;
        const long long cm = (long long)col * ncy;
        double2 lc0 = mk(0, 0), lc1 = mk(0, 0), lsg0 = mk(0, 0), lsg1 = mk(0, 0);
#pragma unroll
        for (int q = 0; q < TC; ++q) {
            lc0 = cadd(lc0, red[q][w][0]);
            lc1 = cadd(lc1, red[q][w][1]);
            lsg0 = cadd(lsg0, red[q][w][2]);
            lsg1 = cadd(lsg1, red[q][w][3]);
        }
        double2 lpv[E], lv0[E], lv1[E], lv2[E];
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const int y = ycoef<E>(e);
            if (y <= ny) {
                const int sl = tile_slot<E>(y, w);
                lpv[e] = tile[sl];
                lv0[e] = tile[S + sl];
                lv1[e] = tile[2 * S + sl];
                lv2[e] = tile[3 * S + sl];
            } else {
                lpv[e] = lv0[e] = lv1[e] = lv2[e] = mk(0.0, 0.0);
            }
        }
        // sigma: sg = n / sigma0, n0 = -w vt0 - Re tail0, n1 = -w vt1 + Re (2 ny ptop - tail1)
        const double wv = st.wn_v[col];
        const double2 ln0 = cdiv(lsg0, cconj(st.sigma0[col]));
        const double2 ln1 = cdiv(lsg1, cconj(st.sigma0[ncol + col]));
        const double2 lvt0 = cscale(-wv, ln0), lvt1 = cscale(-wv, ln1);
        const double2 ltail0 = cscale(-pp.Re, ln0), ltail1 = cscale(-pp.Re, ln1);
        const double2 lptop = cscale(pp.Re * 2.0 * ny, ln1);
        const long long o_n = ((long long)kzi * ncy + ny) * nkx + kx, o_n1 = o_n - nkx;
        lc0 = cadd(lc0, cadd(cmulc_inf(st.p_inf[o_n], false, lptop),
                             cadd(cmulc_inf(st.v_inf[Ns + o_n], false, lvt0), cmulc_inf(st.v_inf[Ns + o_n1], false, lvt1))));
        lc1 = cadd(lc1, cadd(cmulc_inf(st.p_inf[Ns + o_n], false, lptop),
                             cadd(cmulc_inf(st.v_inf[4 * Ns + o_n], false, lvt0), cmulc_inf(st.v_inf[4 * Ns + o_n1], false, lvt1))));
        // c0 = div1 i10 - div0 i11, c1 = div0 i01 - div1 i00
        const double2 i00 = st.inf_div[col], i01 = st.inf_div[ncol + col];
        const double2 i10 = st.inf_div[2 * ncol + col], i11 = st.inf_div[3 * ncol + col];
        const double2 ldiv1 = csub(cmulc(i10, lc0), cmulc(i00, lc1));
        const double2 ldiv0 = csub(cmulc(i01, lc1), cmulc(i11, lc0));
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const int y = ycoef<E>(e);
            if (y > ny) continue;
            if (y == ny) {
                lpv[e] = cadd(lpv[e], lptop);
                lv1[e] = cadd(lv1[e], lvt0);
            }
            if (y == ny - 1) lv1[e] = cadd(lv1[e], lvt1);
            // wall divergence: tang = i ax v0 + i az v2, nrm = y^2 v1
            const double2 ltang = p ? csub(ldiv0, ldiv1) : cadd(ldiv0, ldiv1);
            const double2 lnrm = p ? cadd(ldiv0, ldiv1) : csub(ldiv0, ldiv1);
            lv0[e] = cadd(lv0[e], fderiv(-ax, ltang));
            lv2[e] = cadd(lv2[e], fderiv(-az, ltang));
            lv1[e] = cadd(lv1[e], cscale((double)(y * y), lnrm));
        }
        // velocity taus: f_c = Re (grad_c P - R_c)
        double ad[E];
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const int y = ycoef<E>(e);
            ad[e] = y <= ny ? st.ad_v[cm + y] : 0.0;
        }
        double2 lR0[E], lR1[E], lR2[E], ldpy[E];
        double2 lblo[3], lbup[3];
        auto velocity = [&](int c, const double2(&lvc)[E], double2(&lRc)[E]) {
            double2 lf[E];
            tau_adj<E>(ny, g_v, pp.a_V[c], pp.b_V[c], zero_col, wv, lvc, lf, lblo[c], lbup[c], ad, t.WL, t.WD,
                       t.WR);
#pragma unroll
            for (int e = 0; e < E; ++e) {
                const double2 lg = cscale(pp.Re, lf[e]);
                lRc[e] = cscale(-1.0, lg);
                if (c == 0) lpv[e] = cadd(lpv[e], fderiv(-ax, lg));
                if (c == 1) ldpy[e] = lg;
                if (c == 2) lpv[e] = cadd(lpv[e], fderiv(-az, lg));
            }
        };
        velocity(0, lv0, lR0);
        velocity(1, lv1, lR1);
        velocity(2, lv2, lR2);
        // dP/dy
        double2 tmp[E];
        deriv_T<E>(ny, ldpy, tmp);
#pragma unroll
        for (int e = 0; e < E; ++e) lpv[e] = cadd(lpv[e], tmp[e]);
        // tails of R_1 in the sigma numerators
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const int y = ycoef<E>(e);
            if (y == ny) lR1[e] = cadd(lR1[e], ltail0);
            if (y == ny - 1) lR1[e] = cadd(lR1[e], ltail1);
        }
        // pressure tau and the divergence of R
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const int y = ycoef<E>(e);
            ad[e] = y <= ny ? st.ad_p[cm + y] : 0.0;
        }
        double2 ldy[E], llo, lup;
        tau_adj<E>(ny, pp.G_pre, A.p_a, A.p_b, zero_col, st.wn_p[col], lpv, ldy, llo, lup, ad, t.WL, t.WD, t.WR);
        deriv_T<E>(ny, ldy, tmp);
#pragma unroll
        for (int e = 0; e < E; ++e) {
            lR0[e] = cadd(lR0[e], fderiv(-ax, ldy[e]));
            lR1[e] = cadd(lR1[e], tmp[e]);
            lR2[e] = cadd(lR2[e], fderiv(-az, ldy[e]));
        }
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const int y = ycoef<E>(e);
            if (y > ny) continue;
            const int sl = tile_slot<E>(y, w);
            tile[S + sl] = lR0[e];
            tile[2 * S + sl] = lR1[e];
            tile[3 * S + sl] = lR2[e];
        }
        if (L == 0) {
            A.lBc[col] = llo;
            A.lBc[ncol + col] = lup;
            if (A.acc) {
                const double2 bt = cadd(A.lB1[col], cscale(A.b0, llo));
                const double2 bb = cadd(A.lB1[ncol + col], cscale(A.b0, lup));
                A.lbw[col] = bt;
                A.lbw[ncol + col] = bb;
                A.lB2[col] = cscale(A.b1, llo);
                A.lB2[ncol + col] = cscale(A.b1, lup);
                s_bw[w][0] = bt;
                s_bw[w][1] = bb;
            }
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                double2 lo = lblo[c], up = lbup[c];
                if (c == 1 && zero_mode && col == zc) {
                    lo = cadd(lo, s_zbc);
                    up = cadd(up, s_zbc);
                }
                A.lbcv[(2 * c) * ncol + col] = cadd(A.lbcv[(2 * c) * ncol + col], lo);
                A.lbcv[(2 * c + 1) * ncol + col] = cadd(A.lbcv[(2 * c + 1) * ncol + col], up);
            }
        }
    }
    __syncthreads();
    for (int i = tid; i < S; i += kThreads) {
        const int y = i / TC, l = i - (i / TC) * TC;
        const int c2 = col0 + l;
        if (c2 >= ncol) continue;
        const int kzi = c2 / nkx, kx = c2 - (c2 / nkx) * nkx;
        const long long off = ((long long)kzi * ncy + y) * nkx + kx;
        const int sl = tile_slot<E>(y, l);
        if (!A.acc) {
#pragma unroll
            for (int c = 0; c < 3; ++c) A.lR[c * Ns + off] = tile[(1 + c) * S + sl];
            continue;
        }
        const double2 bt = s_bw[l][0], bb = s_bw[l][1];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const long long o = c * Ns + off;
            const double2 r = tile[(1 + c) * S + sl];
            A.lu1[o] = cadd(A.lu1[o], cscale(A.a0, r));
            A.lu2[o] = cscale(A.a1, r);
            double2 nn = cadd(A.lN1[o], cscale(A.b0, r));
            if (c == 1) nn = cadd(nn, (y & 1) ? cadd(bt, bb) : csub(bt, bb));
            A.lN1[o] = nn;
            A.lN2[o] = cscale(A.b1, r);
        }
    }
}

size_t solve_adj_smem(const Dims &d) { return sizeof(double2) * 4 * (size_t)d.ncy * TC; }

template <int E> cudaError_t configure_adj_e(const Dims &d) { return raise_smem(k_solve_adj<E>, solve_adj_smem(d)); }

template <int E>
void solve_adj_e(const Dims &d, const Tables &t, const PhysParams &pp, double g_v, const SolverState &st,
                 const AdjArgs &A, cudaStream_t s) {
    k_solve_adj<E><<<(d.ncol + TC - 1) / TC, kThreads, solve_adj_smem(d), s>>>(d, t, pp, g_v, st, A);
}
}  // namespace

static cudaError_t configure_solve_adjoint(const Dims &d) {
    switch (lane_elems(d)) {
    case 1: return configure_adj_e<1>(d);
    case 2: return configure_adj_e<2>(d);
    case 4: return configure_adj_e<4>(d);
    case 8: return configure_adj_e<8>(d);
    default: return cudaErrorInvalidValue;
    }
}

static void solve_adj_dispatch(const Dims &d, const Tables &t, const PhysParams &pp, double g_v,
                               const SolverState &st, const AdjArgs &A, cudaStream_t s) {
    switch (lane_elems(d)) {
    case 1: solve_adj_e<1>(d, t, pp, g_v, st, A, s); break;
    case 2: solve_adj_e<2>(d, t, pp, g_v, st, A, s); break;
    case 4: solve_adj_e<4>(d, t, pp, g_v, st, A, s); break;
    case 8: solve_adj_e<8>(d, t, pp, g_v, st, A, s); break;
    default: break;
    }
}

void launch_solve_adjoint_step(const Dims &d, const Tables &t, const PhysParams &pp, double g_v,
                               const SolverState &st, const double2 *lv, double seed, double a0, double a1,
                               double b0, double b1, double2 *lu1, double2 *lu2, double2 *lN1, double2 *lN2,
                               const double2 *lB1, double2 *lbw, double2 *lB2, double2 *lBc, double2 *lbcv,
                               cudaStream_t s) {
    AdjArgs A{};
    A.p_a = pp.a_pre0;
    A.p_b = pp.b_pre0;
    A.lv = lv;
    A.lBc = lBc;
    A.lbcv = lbcv;
    A.seed = seed;
    A.acc = 1;
    A.a0 = a0;
    A.a1 = a1;
    A.b0 = b0;
    A.b1 = b1;
    A.lu1 = lu1;
    A.lu2 = lu2;
    A.lN1 = lN1;
    A.lN2 = lN2;
    A.lB1 = lB1;
    A.lbw = lbw;
    A.lB2 = lB2;
    solve_adj_dispatch(d, t, pp, g_v, st, A, s);
}

void launch_solve_adjoint(const Dims &d, const Tables &t, const PhysParams &pp, double g_v, const SolverState &st,
                          const double2 *lp, const double2 *lv, double2 *lR, double2 *lBc, double2 *lbcv,
                          int solve_only, double seed, cudaStream_t s) {
    AdjArgs A{};
    A.seed = seed;
    A.p_a = pp.a_pre0;
    A.p_b = pp.b_pre0;
    A.lp = lp;
    A.lv = lv;
    A.lR = lR;
    A.lBc = lBc;
    A.lbcv = lbcv;
    A.solve_only = solve_only;
    solve_adj_dispatch(d, t, pp, g_v, st, A, s);
}


// ---------------------------------------------------------------------------
// Transpose of the spectral curl and of its pressure-wall sums (k_curl in
// chebyshev.cu): with om_x = Dw - i kz v, om_y = i kz u - i kx w,
// om_z = i kx v - Du and bw = sum_y (i kx/Re om_z - i kz/Re om_x) s_y,
//   lu = -i kz lom_y - D^T lom_z,  lv = i kz lom_x - i kx lom_z,
//   lw = D^T lom_x + i kx lom_y,
// after lom_x += i kz/Re lwall, lom_z -= i kx/Re lwall, lwall_y = lbw_top +
// s_y lbw_bottom (s_y = +1 for odd y, -1 for even y).  The direct part
// lS[0..2] (the velocity fields of the synthesis) is added too:
//   lu_out += lS[0..2] + curl^T(lS[3..5], lbw).
// ---------------------------------------------------------------------------
namespace {
template <int E>
__global__ void __launch_bounds__(32 * kColsPerBlock)
k_curl_adj(Dims d, Tables t, const double2 *__restrict__ lS, const double2 *__restrict__ lbw,
           double2 *__restrict__ lu, double re) {
    extern __shared__ double2 tile[];   // [3][ncy][kColsPerBlock]
    const int ncy = d.ncy, ny = d.NYS, nkx = d.nkx, ncol = d.ncol;
    const int S = ncy * kColsPerBlock;
    const int col0 = blockIdx.x * kColsPerBlock;
    const int tid = threadIdx.x, w = tid >> 5, L = tid & 31, p = L & 1;
    for (int i = tid; i < S; i += blockDim.x) {
        const int y = i / kColsPerBlock, l = i - (i / kColsPerBlock) * kColsPerBlock;
        const int c2 = col0 + l;
        if (c2 >= ncol) continue;
        const int kzi = c2 / nkx, kx = c2 - (c2 / nkx) * nkx;
        const long long off = ((long long)kzi * ncy + y) * nkx + kx;
        const int sl = tile_slot<E>(y, l);
#pragma unroll
        for (int c = 0; c < 3; ++c) tile[c * S + sl] = lS[(3 + c) * d.Ns + off];
    }
    __syncthreads();
    const int col = col0 + w;
    if (col < ncol) {
        const int kzi = col / nkx, kx = col - kzi * nkx;
        const double ax = t.wavx[kx], az = t.wavz[kzi];
        const double axr = ax / re, azr = az / re;
        const double2 lbt = lbw ? lbw[col] : mk(0.0, 0.0), lbb = lbw ? lbw[ncol + col] : mk(0.0, 0.0);
        double2 lox[E], loy[E], loz[E];
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const int y = ycoef<E>(e);
            if (y <= ny) {
                const int sl = tile_slot<E>(y, w);
                const double2 lwall = p ? cadd(lbt, lbb) : csub(lbt, lbb);
                lox[e] = cadd(tile[sl], fderiv(azr, lwall));
                loy[e] = tile[S + sl];
                loz[e] = cadd(tile[2 * S + sl], fderiv(-axr, lwall));
            } else {
                lox[e] = loy[e] = loz[e] = mk(0.0, 0.0);
            }
        }
        double2 dx[E], dz[E];
        deriv_T<E>(ny, lox, dx);
        deriv_T<E>(ny, loz, dz);
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const int y = ycoef<E>(e);
            if (y > ny) continue;
            const int sl = tile_slot<E>(y, w);
            tile[sl] = csub(fderiv(-az, loy[e]), dz[e]);
            tile[S + sl] = cadd(fderiv(az, lox[e]), fderiv(-ax, loz[e]));
            tile[2 * S + sl] = cadd(dx[e], fderiv(ax, loy[e]));
        }
    }
    __syncthreads();
    for (int i = tid; i < S; i += blockDim.x) {
        const int y = i / kColsPerBlock, l = i - (i / kColsPerBlock) * kColsPerBlock;
        const int c2 = col0 + l;
        if (c2 >= ncol) continue;
        const int kzi = c2 / nkx, kx = c2 - (c2 / nkx) * nkx;
        const long long off = ((long long)kzi * ncy + y) * nkx + kx;
        const int sl = tile_slot<E>(y, l);
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const long long o = c * d.Ns + off;
            lu[o] = cadd(lu[o], cadd(lS[o], tile[c * S + sl]));
        }
    }
}

size_t curl_adj_smem(const Dims &d) { return sizeof(double2) * 3 * (size_t)d.ncy * kColsPerBlock; }

// lN_y += the transposed wall sums of lB (standalone nonlinear adjoint).
__global__ void k_pressure_bc_adj(Dims d, const double2 *__restrict__ lB, double2 *__restrict__ lN) {
    const long long ncol = d.ncol;
    for (long long off = blockIdx.x * (long long)blockDim.x + threadIdx.x; off < d.Ns;
         off += (long long)gridDim.x * blockDim.x) {
        const int kx = (int)(off % d.nkx);
        const long long q = off / d.nkx;
        const int y = (int)(q % d.ncy), kzi = (int)(q / d.ncy);
        const long long col = (long long)kzi * d.nkx + kx;
        const double2 bt = lB[col], bb = lB[ncol + col];
        lN[d.Ns + off] = cadd(lN[d.Ns + off], (y & 1) ? cadd(bt, bb) : csub(bt, bb));
    }
}

// Time-step value of the wall-shear objective: -(1/Re) sum_{y even} y^2 Re u_y
// of the streamwise mean profile, i.e. (dU/dy(-1) - dU/dy(+1)) / (2 Re).
__global__ void k_wall_shear(Dims d, const double2 *__restrict__ u, double re, double *__restrict__ out) {
    const int L = threadIdx.x;
    double acc = 0.0;
    for (int y = 2 * L; y <= d.NYS; y += 64) {
        const long long off = ((long long)d.NZS * d.ncy + y) * d.nkx;
        acc += (double)(y * y) * u[off].x;
    }
    acc = sum_warp(acc);
    if (L == 0) *out = -acc / re;
}
}  // namespace

cudaError_t configure_adjoint_kernels(const Dims &d) {
    cudaError_t e = configure_solve_adjoint(d);
    if (e != cudaSuccess) return e;
    const int sm = (int)curl_adj_smem(d);
    switch (lane_elems(d)) {
    case 1: return raise_smem(k_curl_adj<1>, sm);
    case 2: return raise_smem(k_curl_adj<2>, sm);
    case 4: return raise_smem(k_curl_adj<4>, sm);
    case 8: return raise_smem(k_curl_adj<8>, sm);
    default: return cudaErrorInvalidValue;
    }
}

void launch_curl_adjoint(const Dims &d, const Tables &t, const double2 *lS, const double2 *lbw, double2 *lu,
                         double re, cudaStream_t s) {
    const int blocks = (d.ncol + kColsPerBlock - 1) / kColsPerBlock;
    const size_t sm = curl_adj_smem(d);
    switch (lane_elems(d)) {
    case 1: k_curl_adj<1><<<blocks, 32 * kColsPerBlock, sm, s>>>(d, t, lS, lbw, lu, re); break;
    case 2: k_curl_adj<2><<<blocks, 32 * kColsPerBlock, sm, s>>>(d, t, lS, lbw, lu, re); break;
    case 4: k_curl_adj<4><<<blocks, 32 * kColsPerBlock, sm, s>>>(d, t, lS, lbw, lu, re); break;
    case 8: k_curl_adj<8><<<blocks, 32 * kColsPerBlock, sm, s>>>(d, t, lS, lbw, lu, re); break;
    default: break;
    }
}

static int grid_for(long long n) { return (int)std::min<long long>((n + 255) / 256, 148LL * 16); }

void launch_pressure_bc_adjoint(const Dims &d, const double2 *lB, double2 *lN, cudaStream_t s) {
    k_pressure_bc_adj<<<grid_for(d.Ns), 256, 0, s>>>(d, lB, lN);
}

void launch_wall_shear(const Dims &d, const double2 *u, double re, double *out, cudaStream_t s) {
    k_wall_shear<<<1, 32, 0, s>>>(d, u, re, out);
}

}  // namespace cdns
