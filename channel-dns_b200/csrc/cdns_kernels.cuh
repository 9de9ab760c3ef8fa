// Launch wrappers shared between the kernel translation units and the
// context code.
#pragma once

#include "cdns_common.cuh"

namespace cdns {

// ---- chebyshev.cu ----
void cheb_table_sizes(const Dims &d, size_t *nsyn, size_t *nana);
// cana may be null (synthesis matrix only)
void launch_cheb_tables(const Dims &d, const double *cosy, double *csyn, double *cana, cudaStream_t s);
cudaError_t configure_cheb_kernels(const Dims &d);
// vorticity om[3][Ns] of u[3][Ns] and its pressure-wall sums bw[2][ncol] (bw may be null)
void launch_curl(const Dims &d, const Tables &t, const double2 *u, double2 *om, double2 *bw, double re,
                 cudaStream_t s);
// F[f][j][col] of nf spectral fields: f < nsplit from src0, the others from src1
void launch_ysynth(const Dims &d, const Tables &t, const double2 *src0, const double2 *src1, int nsplit,
                   int nf, double2 *F, cudaStream_t s);
void launch_yanalysis(const Dims &d, const Tables &t, const double2 *F, double2 *S, int nf, cudaStream_t s);
// FP32 stage buffers (mixed precision): synthesis written, analysis read as
// float2.  The (kz, kx) = (0, 0) mean profiles stay FP64 in mean[6][NY2+1]
// (zero in F); launch_mean_products adds their mean x mean product to N.
void launch_ysynth(const Dims &d, const Tables &t, const double2 *src0, const double2 *src1, int nsplit,
                   int nf, float2 *F, double *mean, cudaStream_t s);
void launch_mean_products(const Dims &d, const Tables &t, const double *mean, double2 *S, cudaStream_t s);
void launch_yanalysis(const Dims &d, const Tables &t, const float2 *F, double2 *S, int nf, cudaStream_t s);
// Discrete adjoint: tables of the transposed analysis (synthesis layout) and
// transposed synthesis (analysis layout); analysis with a custom table and
// one output scale for every coefficient.
void launch_cheb_tables_adjoint(const Dims &d, const double *cosy, double *csyn_t, double *cana_t,
                                cudaStream_t s);
void launch_yanalysis_scaled(const Dims &d, const double *cana, const double2 *F, double2 *S, int nf,
                             double scale, cudaStream_t s);

// ---- transforms.cu ----
cudaError_t configure_transform_kernels(const Dims &d);
// coarse = true: the coarse-grid conventions of a full spectrum's Nyquist
// modes (channel_xyzfft) instead of the fine grid's (channel_xyzfft2).
void launch_z_backward(const Dims &d, const FftPlan &P, const double2 *roots, const double2 *F,
                       double2 *G, int nf, cudaStream_t s, bool coarse = false);
void launch_x_cross(const Dims &d, const FftPlan &P, const double2 *roots, const double2 *G,
                    double2 *H, cudaStream_t s);
void launch_z_forward(const Dims &d, const FftPlan &P, const double2 *roots, const double2 *H,
                      double2 *F, int nf, cudaStream_t s, bool coarse = false);
void launch_x_c2r(const Dims &d, const FftPlan &P, const double2 *roots, const double2 *G,
                  double *phys, cudaStream_t s, bool coarse = false);
// FP32 stage buffers (mixed precision); only meshes with register_forms(d)
bool register_forms(const Dims &d);
void launch_z_backward(const Dims &d, const double2 *roots, const float2 *F, float2 *G, int nf, cudaStream_t s);
// mean: FP64 mean profiles [6][NY2+1] added to the FP32 fluctuations in the products
void launch_x_cross(const Dims &d, const double2 *roots, const float2 *G, float2 *H, const double *mean,
                    cudaStream_t s);
void launch_z_forward(const Dims &d, const double2 *roots, const float2 *H, float2 *F, int nf, cudaStream_t s);
void launch_x_r2c(const Dims &d, const FftPlan &P, const double2 *roots, const double *phys,
                  double2 *H, cudaStream_t s, bool coarse = false);
// Every pencil rank's y-physical column buffer as seen from one rank: rank q
// holds the kx block [kx0_q, kx0_q + nkx_q) in the layout [f][NY2+1][2NZS+1][nkx_q],
// so line kx of the whole spectrum is col[kx] = &F_q[kx - kx0_q] with row stride
// width[kx] = nkx_q.  The pointers are device pointers valid in this process.
struct PeerCols {
    double2 *const *col;   // [NXS+1]
    const int *width;      // [NXS+1]
    int ny2;               // NY2 + 1: every rank's buffer holds all y points
    int j0;                // first y point of this rank's slab
};
// The z transforms of a pencil rank's y slab (ds: every kx, ny2 = the slab's
// points) with the exchange fused in: the synthesis of the six fields reads
// the slab's rows from every rank's columns, the analysis of the three fields
// writes them back there.  Register forms of NZ2 only (false otherwise).
bool launch_z_backward_peers(const Dims &ds, const double2 *roots, const PeerCols &pc, double2 *G,
                             cudaStream_t s);
bool launch_z_forward_peers(const Dims &ds, const double2 *roots, const double2 *H, const PeerCols &pc,
                            cudaStream_t s);
// Chebyshev synthesis (ana = false: spectral src0/src1 as in launch_ysynth ->
// F) or analysis (ana = true: F in src0 -> spectral) in the FFT (DCT-I) form;
// false if NY2 has no register split (the caller takes the matrix form).
bool ydct_available(const Dims &d, const Tables &t);
bool launch_ydct(const Dims &d, const Tables &t, const double2 *src0, const double2 *src1, int nsplit, int nf,
                 double2 *out, bool ana, cudaStream_t s);
// The same for FP32 stage buffers: the synthesis keeps the (kz, kx) = (0, 0)
// column in FP64 (mean[f][j]) and writes zeros there; the analysis applies
// the 1 / (NX2 NZ2) the FP32 z and x analyses leave out.
bool launch_ydct_synthesis_fp32(const Dims &d, const Tables &t, const double2 *src0, const double2 *src1,
                                int nsplit, int nf, float2 *F, double *mean, cudaStream_t s);
bool launch_ydct_analysis_fp32(const Dims &d, const Tables &t, const float2 *F, double2 *S, int nf,
                               cudaStream_t s);
// Transposes of the analysis and of the synthesis (discrete adjoint) in the
// FFT form: the products of k_cheb_tables_adjoint's csyn_t and cana_t tables.
bool launch_ydct_adjoint_analysis(const Dims &d, const Tables &t, const double2 *lS, int nf, double2 *F,
                                  cudaStream_t s);
bool launch_ydct_adjoint_synthesis(const Dims &d, const Tables &t, const double2 *F, int nf, double2 *S,
                                   double scale, cudaStream_t s);
// Output reduction, x stage on the coarse grid (Dims of the coarse grid):
// c2r of G[nf] (u, v, w, p and, if nf = 5, div), per-point moments summed per
// block into partial[NY+1][moment_blocks][22]; phys (may be null) receives u, v, w, p.
int moment_blocks(const Dims &d);
void launch_x_moments(const Dims &d, const FftPlan &P, const double2 *roots, const double2 *G, double *partial,
                      double *phys, int nf, cudaStream_t s);
// Transpose of x_cross about the forward fields G[6]: L[0..2] = lH in, L[0..5] = lG out.
void launch_x_adjoint(const Dims &d, const FftPlan &P, const double2 *roots, const double2 *G, double2 *L,
                      cudaStream_t s);

// ---- solver.cu ----
// Precomputed solver state (EqSolvePV members, src/solver/eqsolve_pv.hpp:60-76).
struct SolverState {
    double *wn_p, *wn_v;        // [ncol]
    double *ad_p, *ad_v;        // [ncol][ncy] (column-major)
    // Influence and B-problem fields, planar, each stored by its one nonzero
    // part: the pressure and v are real, u and w purely imaginary (real wall
    // data and real operators; i kx, i kz enter only through the gradient), so
    // the other part is an exact zero and is not kept (inf_part).
    double *p_inf;              // [2][Ns]
    double *v_inf;              // [2][3][Ns]
    double2 *inf_div;           // [2 (response)][2 (wall)][ncol]
    double *p_b;                // [Ns]
    double *v_b;                // [3][Ns]
    double2 *sigma0;            // [2][ncol]
    double *unit;               // [2][ncy] u_dpdx_unit, w_dpdz_unit ; [2*ncy..] qx, qz
};

// Velocity component c of an influence or B-problem field: imaginary for u
// and w (c = 0, 2), real for v (c = 1).
__host__ __device__ inline bool inf_imag(int c) { return c != 1; }
// The complex value of a stored part; c * value without the products by the
// exact zero (cmul with a zero part gives the same bits for finite c).
__device__ inline double2 inf_value(double part, bool imag) { return imag ? mk(0.0, part) : mk(part, 0.0); }
__device__ inline double2 inf_mul(double2 c, double part, bool imag) {
    return imag ? fderiv(part, c) : cscale(part, c);
}

struct PhysParams {
    double Re, G_pre, a_pre0, b_pre0;
    double a_V[3], b_V[3];
    int grad_pre;               // INDEX_GRAD_PRE
    double gx, gz;              // GRAD_PRE_X/Z
    double qxm, qzm;            // QXmean/QZmean
};

struct StepArgs {
    const double2 *u, *u_prev, *N, *N_prev;   // planar 3-component spectral fields
    const double2 *bw;          // [2][ncol] vorticity part of the wall condition
    const double2 *B_prev;      // [2][ncol]
    double2 *B_new;             // [2][ncol]
    const double2 *bc_v;        // [3][2][ncol]
    double2 *u_out;             // [3][Ns]
    double2 *p_out;             // [Ns]
    double *dpdx;               // [2]
    unsigned *err;
    double a0, a1, b0, b1;
    const double2 *bc_p;        // if set: pressure wall data [2][ncol] used as is
    int solve_only;             // 1: solve_modes alone (no zero-mode / flow correction)
};

// ---- solver_setup.cu ----
cudaError_t configure_setup_kernels(const Dims &d);
void setup_solver(const Dims &d, const Tables &t, const PhysParams &pp, double g_v,
                  SolverState &st, double2 *scratch, cudaStream_t s);

// ---- solver.cu ----
void launch_step_solve(const Dims &d, const Tables &t, const PhysParams &pp, double g_v,
                       const SolverState &st, const StepArgs &a, cudaStream_t s);
cudaError_t configure_solver_kernels(const Dims &d);
// Pressure wall data of a standalone nonlinear evaluation: B = bw + endpoint sums of N_y.
void launch_pressure_bc(const Dims &d, const double2 *N, const double2 *bw, double2 *B,
                        cudaStream_t s);

// ---- adjoint.cu ----
cudaError_t configure_adjoint_kernels(const Dims &d);
// Transpose of the column solve: lp (may be null) and lv[3][Ns] of the
// solution -> lR[3][Ns], lBc[2][ncol] (pressure wall data), lbcv[3][2][ncol]
// += (velocity wall data).  solve_only = 0 adds the zero-mode overwrite and
// the wall-shear seed.
void launch_solve_adjoint(const Dims &d, const Tables &t, const PhysParams &pp, double g_v, const SolverState &st,
                          const double2 *lp, const double2 *lv, double2 *lR, double2 *lBc, double2 *lbcv,
                          int solve_only, double seed, cudaStream_t s);
// lu[3][Ns] += lS[0..2] + curl^T(lS[3..5], lbw[2][ncol]) (lbw may be null)
void launch_curl_adjoint(const Dims &d, const Tables &t, const double2 *lS, const double2 *lbw, double2 *lu,
                         double re, cudaStream_t s);
// Reverse step s of the time stepping: the solve transpose of lv = lu^s
// (+ the wall-shear seed) with the multistep bookkeeping fused:
//   lu1 += a0 lR, lu2 = a1 lR, lN1 += b0 lR + wall sums^T(lbw), lN2 = b1 lR,
//   lbw = lB1 + b0 lBc, lB2 = b1 lBc, lbcv += the velocity wall data adjoint.
void launch_solve_adjoint_step(const Dims &d, const Tables &t, const PhysParams &pp, double g_v,
                               const SolverState &st, const double2 *lv, double seed, double a0, double a1,
                               double b0, double b1, double2 *lu1, double2 *lu2, double2 *lN1, double2 *lN2,
                               const double2 *lB1, double2 *lbw, double2 *lB2, double2 *lBc, double2 *lbcv,
                               cudaStream_t s);
void launch_pressure_bc_adjoint(const Dims &d, const double2 *lB, double2 *lN, cudaStream_t s);
void launch_wall_shear(const Dims &d, const double2 *u, double re, double *out, cudaStream_t s);

// ---- context.cu ----
int record_error(int code, const char *msg);

// ---- layout.cu ----
void launch_deinterleave(const double2 *src, double2 *dst, long long n, int nc, cudaStream_t s);
void launch_interleave(const double2 *src, double2 *dst, long long n, int nc, cudaStream_t s);

}  // namespace cdns
