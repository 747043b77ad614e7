// Internal declarations shared by the CUDA translation units of librayleigh_b200.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <string>
#include <vector>

#include "../../include/rayleigh_b200.h"
#include "ozaki.h"

namespace ra {

// ---------------------------------------------------------------------------
// Sizes and index maps
// ---------------------------------------------------------------------------
//  L    = l_max + 1  (number of m values, and of l values)
//  n_lm = L (L + 1) / 2
//  "lm"  index : l-major, m ascending      lm(l, m) = l (l + 1) / 2 + m
//  "row" index : m-major, parity sorted    row(m, l) = off(m) + (l - m even ? (l - m)/2 : ne(m) + (l - m - 1)/2)
//                off(m) = m L - m (m - 1) / 2,  ne(m) = (L - m + 1) / 2
struct Dims {
    int L, lmax, nr, nth, nth2, nphi;
    long nlm;
    int rda;          // 1-based dealiasing index of the Chebyshev grid: coefficients n >= rda-1 are zero
    int kc;           // number of retained Chebyshev coefficients = rda - 1
};

__host__ __device__ inline long lm_index(int l, int m) { return (long)l * (l + 1) / 2 + m; }
__host__ __device__ inline long m_off(int m, int L) { return (long)m * L - (long)m * (m - 1) / 2; }
__host__ __device__ inline int n_even(int m, int L) { return (L - m + 1) / 2; }
__host__ __device__ inline int n_odd(int m, int L) { return (L - m) / 2; }
__host__ __device__ inline long row_index(int m, int l, int L) {
    int d = l - m;
    return m_off(m, L) + ((d & 1) ? (n_even(m, L) + (d - 1) / 2) : (d / 2));
}

// Number of grid outputs of the Chebyshev synthesis and the layout of the
// post-solve grid buffer g[o][lm][ri][r]:
//   0 W  1 W'  2 W''  3 W'''  4 P  5 P'  6 T  7 T'  8 T''  9 Z  10 Z'  11 Z''
enum { G_W0, G_W1, G_W2, G_W3, G_P0, G_P1, G_T0, G_T1, G_T2, G_Z0, G_Z1, G_Z2, NG };
// RHS terms of Post_Solve (Add_Derivative calls, Sphere_Spectral_Space.F90:285-389):
// (equation, grid source).  coef[l][slot][r].
enum { EQ_W = 0, EQ_P = 1, EQ_T = 2, EQ_Z = 3 };
constexpr int NSLOT = 16;
struct Slot { int eq, g; };
constexpr Slot kSlots[NSLOT] = {
    {EQ_W, G_W0}, {EQ_W, G_W1}, {EQ_W, G_W2}, {EQ_W, G_P1}, {EQ_W, G_T0},
    {EQ_P, G_W0}, {EQ_P, G_W1}, {EQ_P, G_W2}, {EQ_P, G_W3}, {EQ_P, G_P0},
    {EQ_T, G_T0}, {EQ_T, G_T1}, {EQ_T, G_T2},
    {EQ_Z, G_Z0}, {EQ_Z, G_Z1}, {EQ_Z, G_Z2}};

// Spectral forward-leg fields after Post_Solve (s2a, 7 fields; P is not carried
// because the hydrodynamic non-output step never transforms it):
enum { S_W, S_T, S_Z, S_W1, S_T1, S_Z1, S_W2, NS2A };
// Fields of the inverse Legendre transform (p2a, 11 fields).  s2a11 and p2a
// keep the fields of one radius together ([..][r][field][re, im]), in an order
// that puts the fields each physical-space FFT batch reads next to each other:
// {DVRDT, DVTDR, VR, VT}, {VR, VT, VP, DVRDR}, {VP, DVPDR, OMR, DTDR}, {DTDT, T}.
enum { A_DVRDT, A_DVTDR, A_VR, A_VT, A_VP, A_DVRDR, A_DVPDR, A_OMR, A_DTDR, A_DTDT, A_T, NP2A };
// Return-leg fields (p2b / s2b / ab): W P T Z; p2b and s2b are [..][r][field][re, im]
constexpr int NP2B = 4;

// The magnetic (dynamo) equation set adds, behind the hydrodynamic fields:
//  grids of the Chebyshev synthesis: C C' C'' A A' A'' (g[12..17])
enum { G_C0 = NG, G_C1, G_C2, G_A0, G_A1, G_A2, NG_MAG };
//  spectral fields of rlm_spacea's magnetic part, s2am[row][f][r][re, im]
enum { SM_C, SM_A, SM_C1, SM_A1, SM_C2, NS2AM };
//  inverse-transform fields (Compute_BandCurlB, Sphere_Hybrid_Space.F90:357-435):
//  B_r, (curl B)_r, and r sin(theta) times (curl B)_theta, (curl B)_phi, B_theta, B_phi
enum { A_BR = NP2A, A_CBR, A_CBT, A_CBP, A_BT, A_BP, NP2A_MAG };
//  return-leg fields in the reference's slots (Fields.F90:365-368): EMF_theta in C's,
//  EMF_r in A's, EMF_phi after them
enum { B_EMFT = NP2B, B_EMFR, B_EMFP, NP2B_MAG };
//  Post_Solve coefficients of the C and A equations, coef_mag[l][slot][r]
enum { MS_C0, MS_C2, MS_A0, MS_A1, MS_A2, NMSLOT };

struct Radial {
    std::vector<double> radius, delta_r, density, dlnrho, buoy, dpdr_w, pdwdr, nu, kappa;
    std::vector<double> int_w;   // radial integration weights (a volume average over the shell)
    double coriolis;
    std::vector<double> eta;     // magnetic diffusivity (magnetism)
    double lorentz = 0.0;        // Lorentz_Coeff
    double rmin = 0.0, rmax = 0.0;
    double fd_dr = 0.0;          // the uniform spacing of the finite-difference grid
    // the rest of the reference state and of the transport profiles (anelastic terms)
    std::vector<double> d2lnrho, temperature, dlnT, dlnu, dlnkappa, dlneta;
    // Compute_Diffusion_Coefs (PDE_Coefficients.F90:2032-2098)
    std::vector<double> w_diff0, w_diff1, dw_diff0, dw_diff1, dw_diff2, s_diff1, z_diff0, z_diff1, a_diff1;
    // viscous_heating_coeff, ohmic_heating_coeff (zero when the term is off)
    std::vector<double> visc_heat, ohm_heat;
    bool heating = false;        // either heating term is on
};

struct GemmTile { int item, mt, nt, par; };

// One batch of per-l systems for the block substitution (k_solve.cu): M in
// block-substitution form [count][n][n], row permutations [count][n],
// right-hand sides and solutions as columns of n doubles.
struct LuSys {
    const double* M;
    const int* perm;
    const double* rhs;
    double* sol;
    int n;
};
// where a tile's right-hand-side columns are: the step's equation-set layout
// (2 (l+1) columns from l (l+1)/2 on), the identity (explicit inverse), or a
// fixed number of columns per l ([l][ncols][n])
enum { LU_MODE_STEP = 0, LU_MODE_INVERSE = 1, LU_MODE_FIXED = 2 };
struct LuWork {
    int* d_status = nullptr;
    double* d_inv = nullptr;   // inverses of the diagonal blocks
    int cap_n = 0, cap_count = 0;
};

// One batched split-precision product of the step (RA_PREC_MIXED): digit
// buffers of its operands, the per-product descriptors, the tile list and the
// per-step split jobs.
struct MixedPlan {
    int8_t *d_adig = nullptr, *d_bdig = nullptr;
    int *d_ea = nullptr, *d_eb = nullptr;
    OzProblem* d_probs = nullptr;
    int* d_tiles = nullptr;
    int ntiles = 0;
    OzSplitJob* d_jobs = nullptr;
    int njobs = 0, max_rows = 0, kinds = 0;
    OzSplitJob* d_setup_jobs = nullptr;   // splits of the constant operand, rerun when it changes
    int nsetup_jobs = 0, setup_max_rows = 0, setup_kinds = 0;
};

// A split-product plan of the device-resident unit transform (ra_transform_dev) for one
// direction, with the operands it was built for.
struct UnitPlan {
    MixedPlan plan;
    bool built = false;
    const double* in = nullptr;
    double* out = nullptr;
    int ncol = 0;
};

struct Ctx {
    ra_config cfg;
    Dims d;
    std::string err;
    cudaStream_t stream = nullptr;
    int device = 0;
    double dt = 0, old_dt = 0;
    int iteration = 1;
    bool have_state = false;
    long launches = 0;
    bool mag = false;                                 // the magnetic equation set (C, A)
    // RA_PREC_MIXED solves by split products of the explicit inverses; with the cgs
    // polytrope (reference_type 2) its matrices are too badly conditioned for an explicit
    // inverse, and in the finite-difference mode the grid-space inverse of the W-P-T system
    // has entries whose products cancel (W within 8.7e-9 of the oracle after 20 steps, against
    // 1.1e-10 through the LU factors): both solve by the FP64 block substitution
    bool mixed_solve = false;
    bool custom_reference = false;                    // radial profiles given by ra_set_reference
    UnitPlan unit_inv, unit_fwd;                      // ra_transform_dev's split-product plans
    int nfa = NP2A, nfb = NP2B, ng = NG;              // fields of s2a11/p2a, of p2b/s2b, grids (more with mag)

    Radial rad;
    std::vector<double> costheta_h;     // Gauss-Legendre nodes (double)
    std::vector<double> cheb_D;         // [4][nr][nr] dcheby(r, n, d) with scalings
    double deriv_scaling = 1.0;

    // device constants
    double *d_Ptab = nullptr, *d_iPtab = nullptr;     // [row][nth2]
    double *d_D = nullptr;                            // [4][nr][nr]
    double *d_Dpar = nullptr;                         // [4][2][nr/2][(kc+1)/2] parity planes of D, r < nr/2
    double *d_Dfd = nullptr;                          // finite differences: I, D1, D2, D3, D1 D1 in bands:
    int fd_w = 0;                                     //   [5][nr][1 + fd_w] = first column, fd_w coefficients
    double *d_coef = nullptr;                         // [L][NSLOT][nr]
    double *d_radial = nullptr;                       // packed radial profiles (see kRadial*)
    double *d_costh = nullptr;                        // [nth] cos, then sin, csc, cot
    double *d_twid = nullptr;                         // [nth] complex exp(2 pi i k / nphi)
    double *d_twp = nullptr;                          // per-pass twiddles of the in-place phi FFT
    bool physics3_ok = false;                         // n_theta has a physical-space kernel with the last pass in registers
    int physics_form = 0;                             // 0/2: that kernel (2 / 1 CTAs per SM), 1: all passes in shared memory
    double *d_Awpt = nullptr, *d_Az = nullptr;        // LU factors in block-substitution form [L][3nr][3nr], [L][nr][nr]
    int *d_perm_wpt = nullptr, *d_perm_z = nullptr;   // row permutations of the factors [L][3nr], [L][nr]
    int *d_skip_z = nullptr;                          // [L]: 1 where Z is not solved for (l = 0)
    double *d_Ainv_wpt = nullptr, *d_Ainv_z = nullptr;   // RA_PREC_MIXED: (A_l^-1)^T, rows = columns of A_l^-1
    int solve_nc = 32, solve_nc_z = 32;               // right-hand-side columns per substitution CTA (W-P-T, Z)
    int n_inv_sol_tiles = 0, n_inv_sol_tiles_z = 0, n_solve_tiles_z = 0;
    int *d_inv_sol_tiles = nullptr, *d_inv_sol_tiles_z = nullptr;   // tile lists of the explicit inverses (mixed form)
    int* d_solve_tiles_z = nullptr;                   // the Z system's substitution tiles
    int *d_ltiles = nullptr;                          // LT tile lists
    int n_inv_tiles = 0, n_fwd_tiles = 0, n_cheb_tiles = 0, n_solve_tiles = 0;
    int *d_inv_tiles = nullptr, *d_fwd_tiles = nullptr, *d_cheb_tiles = nullptr, *d_solve_tiles = nullptr;

    // device state and step buffers
    double *d_sol_wpt = nullptr, *d_sol_z = nullptr;  // [lm][2][3nr], [lm][2][nr]
    double *d_rhs_wpt = nullptr, *d_rhs_z = nullptr;
    double *d_ab = nullptr;                           // [4][lm][2][nr]
    double *d_g = nullptr;                            // [NG][lm][2][nr]
    double *d_s2a = nullptr;                          // [row][NS2A][nr][2]
    double *d_s2a11 = nullptr;                        // [row][NP2A][nr][2]
    double *d_p2a = nullptr;                          // [m][par][nth2][NP2A][nr][2]  E, O
    double *d_p2b = nullptr;                          // [m][par][nth2][4][nr][2]     f_even, f_odd
    double *d_s2b = nullptr;                          // [row][4][nr][2]
    unsigned long long *d_cfl = nullptr;              // CFL max (double bits)
    int *d_status = nullptr;                          // device error word (RA_STATUS_* bits)
    int matrices_loaded = 0;                          // ra_load_matrices: bit 0 W-P-T, bit 1 Z (until ra_factor)
    double *d_bcval = nullptr;                        // caller's boundary values [eq][lm][re/im][top/bottom], or none
    double *d_kew = nullptr;                          // [nth] theta weights / n_phi, then [nr] radial weights
    double *d_ke_rows = nullptr;                      // [nth][nr] kinetic-energy shares, then the sum
    double *d_kaz = nullptr;                          // [nth] 1 / n_phi (azimuthal averages)
    // magnetic equation set
    double *d_sol_c = nullptr, *d_sol_a = nullptr;    // [lm][2][nr] poloidal / toroidal potentials
    double *d_rhs_c = nullptr, *d_rhs_a = nullptr;
    double *d_Ac = nullptr, *d_Aa = nullptr;          // LU factors [L][nr][nr]
    double *d_Ainv_c = nullptr, *d_Ainv_a = nullptr;  // RA_PREC_MIXED: transposed inverses, as for Z
    int *d_perm_c = nullptr, *d_perm_a = nullptr;
    double *d_coef_mag = nullptr;                     // [L][NMSLOT][nr]
    double *d_s2am = nullptr;                         // [row][NS2AM][nr][2]
    double *d_xemf = nullptr;                         // [lm][2][nr] the term Finalize_EMF differentiates
    double *d_Memf = nullptr;                         // [nr][nr] grid -> d/dr on the grid (dealiased)

    MixedPlan mx_inv, mx_fwd, mx_solve;               // RA_PREC_MIXED Legendre transforms, implicit solve
    LuWork lu_work;                                   // factorisation scratch

    cudaGraph_t graph = nullptr;
    cudaGraphExec_t graph_exec = nullptr;
    long graph_launches = 0;                          // kernels in one replay of the step graph
    double graph_old_ab = 0, graph_new_ab = 0;
    // ra_step_adaptive's device-side CFL control: a graph whose conditional WHILE node replays
    // the steady step followed by Adjust_TimeStep until dt changes or the count is reached
    cudaGraph_t adapt_graph = nullptr;
    cudaGraphExec_t adapt_exec = nullptr;
    ra_dt_controls adapt_ctl{};
    double adapt_new_ab = 0, adapt_old_ab = 0;
    long adapt_launches = 0;
    int* d_adapt = nullptr;          // [0] steps done, [1] steps wanted, [2] dt changed
    double* d_adapt_dt = nullptr;    // [0] the steps' dt, [1] the next dt, [2] the last CFL cargo
};

// bits of the device error word
constexpr int RA_STATUS_TIMEOUT = 1;     // a bounded pipeline wait of a split-precision product ran out
constexpr int RA_STATUS_NONFINITE = 2;   // a NaN/Inf reached the right-hand side of the implicit solve

// radial profile packing in d_radial: index k * nr + r
enum { R_RADIUS, R_OVER_R, R_DELTA_R, R_DENSITY, R_DLNRHO, R_OVER_RHOR, R_OVER_RHORSQ, R_DRHO_TERM, R_TWO_OVER_R,
       R_OVER_RSQ, R_VISC_HEAT, R_OHM_HEAT, R_RHO_T, R_COUNT };   // R_RHO_T: rho T of the reference state

// ---- kernels / launchers (defined in the .cu files) ----
void launch_plm(Ctx& c, const double* d_x, const double* d_w);
void launch_lt_inverse(Ctx& c, const double* s2, double* p2, int ncol);
void launch_lt_forward(Ctx& c, const double* p2, double* s2, int ncol);
void launch_cheb_synthesis(Ctx& c);
void launch_post_assemble(Ctx& c, double old_ab);
void launch_rlm_a(Ctx& c);
void launch_physics(Ctx& c);
void launch_kinetic_energy(Ctx& c, bool magnetic = false);
// one diagnostic quantity on the phi grid at up to MAXL radial levels
// A diagnostic quantity's buffer-field sum: sum over j < nt of c x field (d/dphi where dphi,
// times the theta factor th: 0 none, 1 csc, 2 cot, 3 csc cot, 4 csc^2, and the radial factor
// rad: 0 none, 1 1/r, 2 r, 3 r dlnrho + 2), of the part mpart (0 the field, 1 its
// fluctuations, m > 0, 2 its azimuthal mean, m = 0); nt = 0: the constant 1.
struct DiagTerm { int field, dphi, th, rad; double c; };
struct DiagCombo { int nt, mpart; DiagTerm t[4]; };

struct SliceSpec {
    static constexpr int MAXL = 64;
    int field, dphi, csc, nl;   // p2a field, d/dphi, times 1/sin(theta), levels in this launch
    int pressure;               // formed with the P grid in T's place (pressure quantities)
    int orad;                   // times 1/r (the r sin(theta) B_theta, B_phi fields)
    int mpart;                  // 0 the field, 1 its fluctuating part (m > 0), 2 its azimuthal mean
    // nprod > 0: coef x sum over i < nprod of a[i] b[i] (b[i] = a[i] where bsame[i], the
    // constant 1 where b[i].nt = 0), coef 0: one, 1: rho(r) / 2, 2: cval, 3: rho(r) T(r),
    // 4: (rho(r) T(r))^2, 5: rho(r) (field, dphi, csc, orad and mpart then unused)
    int nprod, bsame[3], coef;
    double cval;
    DiagCombo a[3], b[3];
    int level[MAXL];            // radial indices
};
void launch_shell_slice(Ctx& c, const SliceSpec& S, double* out);
void launch_shell_moments(Ctx& c, const SliceSpec& S, double* rows, double* out);
void launch_azimuthal_average(Ctx& c, const SliceSpec& S, double* rows);
void launch_spectra_rows(Ctx& c, const SliceSpec& S, int slot0, double* p2b);
void launch_spectra_gather(Ctx& c, const double* s2, int nslots, double* out);
void launch_equatorial_slice(Ctx& c, const SliceSpec& S, double* out);
void launch_meridional_slice(Ctx& c, const SliceSpec& S, double* out);
void launch_pressure_to_s2a(Ctx& c);
void launch_global_average(Ctx& c, const SliceSpec& S, double* rows, double* mean, double* out);
// point-probe index lists (radial, theta, phi grid indices)
struct ProbeSet {
    static constexpr int MAXP = 64;
    int nr, ntheta, nphi;
    int r[MAXP], theta[MAXP], phi[MAXP];
};
void launch_point_probes(Ctx& c, const SliceSpec& S, const ProbeSet& Q, double* out);
// tables the launches read, built at set-up (never inside a graph capture)
void physics_prepare(Ctx& c);
bool physics_form1_supported(int n_theta);
void lt_forward_prepare(Ctx& c);
void solve_prepare(Ctx& c);
void launch_rlm_b(Ctx& c, double new_ab);
void launch_post_assemble_mag(Ctx& c, double old_ab);
void launch_rlm_b_mag(Ctx& c, double new_ab);
void launch_solve_mag(Ctx& c);
void launch_solve(Ctx& c);
void factor_matrices(Ctx& c);
void rebuild_solve_tiles(Ctx& c);   // LU of the loaded per-l matrices (+ explicit inverses in the mixed form)
// k_solve.cu
int lu_nc_for(int n);
void lu_workspace(LuWork& w, int n, int count);
void lu_workspace_free(LuWork& w);
int lu_factor_batch(cudaStream_t st, LuWork& w, double* d_mats, int* d_perm, int n, int count, const int* d_skip,
                    long* launches);
void launch_lu_solve(cudaStream_t st, const int* d_tiles, int ntiles, const LuSys& sys, int mode, int ncols_fixed,
                     int nc);
void lu_append_tiles(std::vector<int>& t, int sys, int L, const std::vector<int>& ncols_of_l, int nc);
void launch_lu_refine(cudaStream_t st, const int* d_tiles, int ntiles, const LuSys& s, const float* d_mf,
                      const double* d_a, int ncols, int* d_iters);
void launch_to_float(cudaStream_t st, const double* in, float* out, long count);
int lu_refine_tile_cols();
void launch_fft_rows(Ctx& c, double* d_x, long howmany, int inverse);
void launch_cheb_columns(Ctx& c, const double* d_in, double* d_out, long ncols, int mode, int order);
void mixed_setup(Ctx& c);
void mixed_release(Ctx& c);
void launch_lt_inverse_mixed(Ctx& c);
void launch_lt_unit_mixed(Ctx& c, int inverse, const double* in, double* out, int ncol);
void transform_dev(Ctx& c, int direction, int precision, double* spec, double* grid, double* work, int nfr,
                   double* stage_ms);
void launch_lt_forward_mixed(Ctx& c);
void launch_solve_mixed(Ctx& c);
void mixed_resplit_solve(Ctx& c);

#define RA_CUDA(call)                                                             \
    do {                                                                          \
        cudaError_t e_ = (call);                                                  \
        if (e_ != cudaSuccess) {                                                  \
            throw ra::CudaError(e_, #call, __FILE__, __LINE__);                   \
        }                                                                         \
    } while (0)

struct CudaError {
    cudaError_t code;
    std::string what;
    CudaError(cudaError_t e, const char* call, const char* file, int line) : code(e) {
        what = std::string(call) + " failed at " + file + ":" + std::to_string(line) + ": " + cudaGetErrorString(e);
    }
};

struct SingularError {   // a zero pivot in a per-l matrix: RA_ERR_SINGULAR
    std::string what;
    explicit SingularError(std::string w) : what(std::move(w)) {}
};

struct NonFiniteError {   // RA_ERR_NONFINITE
    std::string what;
    explicit NonFiniteError(std::string w) : what(std::move(w)) {}
};

struct ArgError {
    std::string what;
    explicit ArgError(std::string w) : what(std::move(w)) {}
};

struct StateError {   // a call out of order: RA_ERR_STATE
    std::string what;
    explicit StateError(std::string w) : what(std::move(w)) {}
};

}  // namespace ra

// the opaque handle of the C ABI
struct ra_ctx {
    ra::Ctx c;
};
