/*
 * rayleigh_b200.h -- C ABI of the B200 (sm_100a) implementation of Rayleigh's
 * per-timestep spectral-transform + implicit-solve path.
 *
 * Every entry point returns 0 on success and a negative RA_ERR_* code on
 * failure; ra_last_error() gives the message.  A context owns all device
 * buffers; calls on one context are not thread-safe and run on the
 * context's CUDA stream.  Host pointers are plain double arrays in the
 * reference's Fortran layouts (described per call, written here with the
 * fastest index first).
 *
 * The entry points replace the Fortran module procedures that the
 * reference's main loop calls (paths inside geodynamics/Rayleigh 1.2.0):
 *   Post_Solve              src/Physics/Sphere_Spectral_Space.F90:178
 *   rlm_spacea              src/Physics/Sphere_Hybrid_Space.F90:64
 *   physical_space          src/Physics/Sphere_Physical_Space.F90:98
 *   rlm_spaceb              src/Physics/Sphere_Hybrid_Space.F90:127
 *   AdvanceTime             src/Physics/Sphere_Spectral_Space.F90:415
 *   Reset_Linear_Equations  src/Physics/Sphere_Linear_Terms.F90:67
 * and, for unit-level parity, the math-layer calls
 *   Legendre_Transform      src/Math_Layer/Legendre_Transforms.F90:37-40 (StP_4d_dgp2 :968, PtS_4d_dgpv3 :1077)
 *   FFT_To_Physical/Spectral src/Math_Layer/Fourier_Transform.F90:25-35 (c2r :142, r2c :100)
 *   Cheby_Grid%to_spectral/from_spectral/d_by_dr_cp
 *                           src/Math_Layer/Chebyshev_Polynomials.F90:375,450,560
 */
#ifndef RAYLEIGH_B200_H
#define RAYLEIGH_B200_H

#ifdef __cplusplus
extern "C" {
#endif

#define RA_OK               0
#define RA_ERR_ARG         -1   /* invalid argument or unsupported configuration */
#define RA_ERR_CUDA        -2   /* a CUDA runtime call failed */
#define RA_ERR_SINGULAR    -3   /* a zero or non-finite pivot in a per-l implicit matrix (DGETRF INFO > 0) */
#define RA_ERR_NOMEM       -4   /* device allocation failed */
#define RA_ERR_STATE       -5   /* call out of order (e.g. step before put_state) */
#define RA_ERR_NONFINITE   -6   /* NaN/Inf in an input, or reaching the implicit solve during a step */

#define RA_PREC_FP64   0        /* every product in FP64 */
#define RA_PREC_MIXED  1        /* split-precision tensor-core products, FP64 state */

typedef struct ra_ctx ra_ctx;

/* Problem description: the namelist values the path reads
 * (ProblemSize_Namelist, Physical_Controls, Temporal_Controls,
 *  Boundary_Conditions, Reference_Namelist, Transport_Namelist). */
typedef struct ra_config {
    int    n_r;              /* Chebyshev collocation points (even), one domain */
    int    l_max;            /* maximum spherical-harmonic degree */
    int    n_theta;          /* 0 -> 3(l_max+1)/2 (ProblemSize.F90:444-450) */
    double aspect_ratio;     /* r_min / r_max */
    double shell_depth;      /* r_max - r_min */
    double rayleigh;         /* Rayleigh_Number (buoyancy = Ra/Pr (r/r_o)^gravity_power) */
    double ekman;
    double prandtl;
    double magnetic_prandtl;
    double gravity_power;
    int    rotation;         /* Coriolis terms on/off */
    int    magnetism;        /* 1: the dynamo equation set (C, A potentials, Lorentz force, EMF;
                                insulating boundaries); needs n_theta <= 768 */
    int    no_slip_top, no_slip_bottom;    /* else stress-free */
    int    fix_tvar_top, fix_tvar_bottom;  /* else fixed dT/dr */
    double t_top, t_bottom, dtdr_top, dtdr_bottom;
    double dt;               /* time step (fixed; ra_set_dt changes it) */
    double alpha_implicit;   /* Crank-Nicolson weight, 0.5 */
    int    precision;        /* RA_PREC_FP64 or RA_PREC_MIXED */
    int    use_graph;        /* capture the steady AB2 step as a CUDA graph */
    int    device;           /* CUDA device ordinal */
    int    autotune;         /* 0: built-in kernel choices; 1: time the candidate kernels of each
                                tunable stage at set-up on this device and keep the fastest */
    /* Reference state (Reference_Namelist, PDE_Coefficients.F90:84-160, 216-257) */
    int    reference_type;   /* 1: Boussinesq (Constant_Reference, :335-435); 2: dimensional (cgs)
                                polytrope (Polytropic_Reference, :925-1051); 3: nondimensional
                                polytrope (Polytropic_ReferenceND, :437-537).  Types 2 and 3 are
                                anelastic; their heating terms need n_theta <= 768 */
    double poly_n;           /* polytropic index (types 2, 3) */
    double poly_nrho;        /* density scale heights across the shell (types 2, 3) */
    double poly_mass;        /* interior mass, g (type 2; gravity G M / r^2) */
    double poly_rho_i;       /* density at the inner radius, g/cm^3 (type 2) */
    double pressure_specific_heat;   /* c_P (type 2) */
    double angular_velocity; /* frame rotation rate, rad/s (type 2; Coriolis 2 Omega) */
    double modified_rayleigh;        /* Modified_Rayleigh_Number (type 3) */
    /* Transport_Namelist (:186-207): type 1 constant, 2 x_top (rho / rho_top)^power.  The tops
       are read for reference_type 2; types 1 and 3 set them (1, 1/Pr, 1/Pm; Ek, Ek/Pr, Ek/Pm) */
    int    nu_type, kappa_type, eta_type;
    double nu_power, kappa_power, eta_power;
    double nu_top, kappa_top, eta_top;
    /* Controls.F90:64-65, both on by default; Constant_Reference turns both off */
    int    viscous_heating, ohmic_heating;
    /* Numerical_Controls: 1 Chebyshev collocation (default); 0 finite differences on the
       uniform grid (ProblemSize.F90:607-618) with the default 5-point stencils
       (Finite_Difference.F90:464-689); the state then holds grid values */
    int    chebyshev;
} ra_config;

/* Fills *cfg with the defaults of the reference (Controls.F90, PDE_Coefficients.F90). */
int ra_default_config(ra_config* cfg);

/* Creates a context: builds the grids, the P_l^m tables (on the device),
 * the radial coefficient profiles, the per-l implicit matrices and their LU
 * factors (Reset_Linear_Equations).  A singular matrix returns RA_ERR_SINGULAR.  Replaces Main_Initialization's grid,
 * Legendre and linear-system set-up (src/Physics/Main.F90:71-117). */
int ra_create(ra_ctx** ctx, const ra_config* cfg);
int ra_destroy(ra_ctx* ctx);
int ra_last_error(const ra_ctx* ctx, char* msg, int len);

/* Sizes of the state arrays: n_lm = (l_max+1)(l_max+2)/2 (l-major, m ascending). */
int ra_sizes(const ra_ctx* ctx, long* n_lm, int* n_r, int* n_theta, int* n_phi);

/* CFL time-step control (Adjust_TimeStep, Sphere_Hybrid_Space.F90:604-649; the
 * Temporal_Controls namelist values, Controls.F90:113-115, ClockInfo.F90:27). */
typedef struct ra_dt_controls {
    double cflmin, cflmax;      /* 0.4, 0.6 */
    double max_time_step;       /* 1.0 */
    double min_time_step;       /* 1e-13 */
    double min_dt_change;       /* 0.1: a decrease is at least this fraction */
} ra_dt_controls;
int ra_default_dt_controls(ra_dt_controls* ctl);
/* The dt Adjust_TimeStep chooses after a step of size dt whose CFL cargo (the
 * value ra_step returns: the largest squared inverse crossing time) is cfl;
 * host arithmetic only.  RA_ERR_NONFINITE when it falls below min_time_step. */
int ra_next_dt(const ra_dt_controls* ctl, double dt, double cfl, double* new_dt);
/* nsteps steps with that control: after each step the next dt is chosen from
 * its CFL cargo and, when it changes, the implicit matrices are rebuilt and
 * factored (Reset_Linear_Equations) before the next step.  *dt_out receives the
 * dt of the next step, *dt_changes how many changes were made (either may be NULL). */
int ra_step_adaptive(ra_ctx* ctx, int nsteps, const ra_dt_controls* ctl, double* dt_out, int* dt_changes);

/* New time step: Reset_Linear_Equations (Sphere_Linear_Terms.F90:67-76):
 * rebuild LHS = I - alpha dt L with boundary rows and factor it per l on the
 * device (LU with partial pivoting, LU_Decompose_full, Linear_Solve.F90:1028-1036).
 * Replaces any matrices loaded with ra_load_matrices. */
int ra_set_dt(ra_ctx* ctx, double dt);

/* The driver's own implicit system, for runs whose matrices the library does
 * not assemble itself (other reference states, custom coefficients):
 * Load_Linear_Coefficients + Set_Boundary_Conditions output
 * (Sphere_Linear_Terms.F90:196-1100), replacing the context's matrices of
 * one system:
 *   sys 0: the linked W-P-T system, lhs(3 n_r, 3 n_r, l_max + 1)
 *   sys 1: Z,                       lhs(  n_r,   n_r, l_max + 1)
 *   sys 2: C, sys 3: A (magnetism), lhs(  n_r,   n_r, l_max + 1); their coefs are
 *          coefs(n_r, 2, l_max + 1) = (C,C,0) (C,C,2) and coefs(n_r, 3, l_max + 1) =
 *          (A,A,0) (A,A,1) (A,A,2); l = 0 has no magnetic equation (its matrix is ignored)
 * each lhs(:, :, l) = equation_set(l, eq)%lhs in Fortran (column-major) order,
 * rows/columns ordered W, P, T blocks of n_r.  coefs (may be NULL) replaces
 * the explicit Post_Solve coefficients of the system's equations
 * (equation_set(l, eq)%coefs(var)%data(:, dorder), Linear_Solve.F90:494-539)
 * as coefs(n_r, 16, l_max + 1), the 16 slots being (eq, var, dorder) =
 *   (W,W,0) (W,W,1) (W,W,2) (W,P,1) (W,T,0) (P,W,0) (P,W,1) (P,W,2) (P,W,3)
 *   (P,P,0) (T,T,0) (T,T,1) (T,T,2) (Z,Z,0) (Z,Z,1) (Z,Z,2)
 * (sys 0 reads the W, P, T slots, sys 1 the Z slots).  Non-finite entries
 * return RA_ERR_NONFINITE.  The matrices take effect at ra_factor. */
int ra_load_matrices(ra_ctx* ctx, int sys, const double* lhs, const double* coefs);
/* The library's own assembly of those matrices for a configuration, on the
 * host only (no device is used): lhs(n, n, nl) of l = l0 .. l0+nl-1 in the
 * layout ra_load_matrices takes, and (if coefs is not NULL) coefs(n_r, 16, nl).
 * Either output may be NULL. */
int ra_build_matrices(const ra_config* cfg, int sys, int l0, int nl, double* lhs, double* coefs);
/* LU_Decompose_Matrices (Linear_Solve.F90:459-480) of the loaded matrices of
 * all systems (both, or the four with magnetism), which belong to time step dt (the AB2 factors use it).
 * RA_ERR_SINGULAR names the system and l of a zero pivot. */
int ra_factor(ra_ctx* ctx, double dt);
/* bc_values(2 [top, bottom], 2 [re, im], n_lm, 4 [W, P, T, Z]) of
 * BoundaryConditions.F90:364-531, written into the boundary rows of the
 * right-hand sides by Apply_Boundary_Mask (Linear_Solve.F90:401-418); (l, m)
 * in this library's l-major order.  NULL restores the built-in values (zero,
 * except the fixed T or dT/dr of l = 0). */
int ra_set_bc_mask(ra_ctx* ctx, const double* bc_values);
/* The driver's own reference state for the explicit terms, for reference states the
 * library does not restate (reference_type 4 and 5, custom files, Augment_Reference;
 * PDE_Coefficients.F90:216-257): per radius (n_r, the collocation order, outer radius
 * first) ref%density and ref%dlnrho (the density weights of rlm_spacea's velocity,
 * Sphere_Hybrid_Space.F90:44-62, 240-350, and of the momentum terms), the
 * viscous_heating_coeff and ohmic_heating_coeff of the entropy equation
 * (Sphere_Physical_Space.F90:337-466; NULL: the term is off; ohmic needs magnetism) and
 * ref%Coriolis_Coeff, ref%Lorentz_Coeff.  The implicit terms are the driver's too: load
 * its matrices with ra_load_matrices and factor them with ra_factor; ra_set_dt and a dt
 * change in ra_step_adaptive then return RA_ERR_STATE.  Non-finite entries return
 * RA_ERR_NONFINITE, a density <= 0 RA_ERR_ARG. */
int ra_set_reference(ra_ctx* ctx, const double* density, const double* dlnrho, const double* viscous_heating_coeff,
                     const double* ohmic_heating_coeff, double coriolis_coeff, double lorentz_coeff);

/* State exchange in the equation-set RHS layout (Linear_Solve.F90:355-386):
 *   wpt[3 n_r][2][n_lm]  W, P, T Chebyshev coefficients of the linked l-block
 *   z  [  n_r][2][n_lm]  Z coefficients
 *   ab [n_r][2][n_lm][4] Adams-Bashforth term p1b (W, P, T, Z RHS); may be NULL (zero)
 * iteration: the reference's iteration counter (1 = Euler first step). */
int ra_put_state(ra_ctx* ctx, const double* wpt, const double* z, const double* ab, int iteration);
int ra_get_state(ra_ctx* ctx, double* wpt, double* z, double* ab);
/* The magnetic part of the state (contexts created with magnetism = 1), in the
 * same layout: the equation-set RHS of the C (poloidal) and A (toroidal)
 * equations (ceq, aeq; Fields.F90:86-88, Linear_Solve.F90:355-386)
 *   c [n_r][2][n_lm], a [n_r][2][n_lm]  Chebyshev coefficients
 *   ab[n_r][2][n_lm][2]                 their Adams-Bashforth terms (C, A); may be NULL (zero)
 * Independent of ra_put_state (either order); a magnetic context whose
 * magnetic state was never put starts from C = A = 0. */
int ra_put_magnetic_state(ra_ctx* ctx, const double* c, const double* a, const double* ab);
int ra_get_magnetic_state(ra_ctx* ctx, double* c, double* a, double* ab);
/* Checkpoint files in the reference's format (Write_Checkpoint / Read_Checkpoint,
 * Checkpointing.F90:143-801, version 2): a directory holding one file per field
 * (W P T Z, C A with magnetism, their AB terms WAB ..., boundary_conditions) and
 * grid_etc (endian tag 314, version, n_r, grid type: 2 Chebyshev, 1 finite differences,
 * l_max, dt, new_dt, radius, elapsed time, iteration).  A field file is n_r (l_max+1)(l_max+2) float64: the
 * real parts, then the imaginary parts, one chunk per radial index, each chunk
 * the (l, m) pairs m-major with l fastest.  ra_write_checkpoint writes the
 * context's state (its last completed iteration, the last and the next dt)
 * into dir (created if missing); ra_read_checkpoint puts a checkpoint of the
 * same grid and grid type (no interpolation: RA_ERR_ARG otherwise) into the context, rebuilds
 * the implicit matrices if its next dt differs, and continues from the
 * following iteration.  The field helpers convert one field between the state
 * layout (n_r, 2, n_lm) and a file; they use no device. */
int ra_write_checkpoint(ra_ctx* ctx, const char* dir, double elapsed_time);
int ra_read_checkpoint(ra_ctx* ctx, const char* dir, int* iteration, double* elapsed_time);
int ra_checkpoint_write_field(const char* path, int n_r, int l_max, const double* field);
int ra_checkpoint_read_field(const char* path, int n_r, int l_max, double* field);

/* The same for one rank's slice of the modes (the (l, m) pairs a rank of the
 * reference holds, Load_Balance.F90:357-368): l_of[i], m_of[i] name mode i of
 * the slice, whose arrays are the rank's own equation-set layout
 *   wpt[3 n_r][2][nmodes], z[n_r][2][nmodes], ab[n_r][2][nmodes][4]
 * (Fortran order; ab may be NULL = zero).  A driver that gathers its ranks'
 * slices puts each one (in any order) before stepping; modes not put keep
 * their previous values.  Non-finite input returns RA_ERR_NONFINITE. */
int ra_put_state_modes(ra_ctx* ctx, int nmodes, const int* l_of, const int* m_of, const double* wpt, const double* z,
                       const double* ab, int iteration);
int ra_get_state_modes(ra_ctx* ctx, int nmodes, const int* l_of, const int* m_of, double* wpt, double* z,
                       double* ab);

/* One full step, the five stage calls of Main_Loop_Sphere
 * (Sphere_Driver.F90:305-328) at the current dt, nsteps times.  cfl (may be
 * NULL) receives the CFL cargo global_msgs(1) of the last step
 * (Sphere_Physical_Space.F90:784-813). */
int ra_step(ra_ctx* ctx, int nsteps, double* cfl);

/* The stages, for a driver that interleaves its own work between them. */
int ra_post_solve(ra_ctx* ctx);                 /* Post_Solve + Transpose_1a2a */
int ra_rlm_a(ra_ctx* ctx);                      /* rlm_spacea + StP Legendre + Transpose_2a3a */
int ra_physical(ra_ctx* ctx, double* cfl);      /* physical_space: FFTs, NL terms, CFL, 3b2b */
int ra_rlm_b(ra_ctx* ctx);                      /* PtS Legendre + rlm_spaceb + Transpose_2b1b */
int ra_advance(ra_ctx* ctx);                    /* AdvanceTime: AB term, BCs, Implicit_Solve */

/* Benchmark_Checkup's volume-averaged kinetic energy of the current state
 * (Benchmarking.F90:645-656, 733-736): 0.5 rho |u|^2 on the physical grid,
 * averaged over phi, over theta with the Gauss-Legendre weights / 2
 * (Spherical_IO.F90:1350-1391) and over radius with the Chebyshev integration
 * weights (Spherical_IO.F90:1436-1470, Chebyshev_Polynomials.F90:165-194).
 * Runs the stages that form the velocity on the grid (Post_Solve through the
 * inverse Legendre transform; they only assign their outputs, so the next
 * ra_step is unchanged) and a reduction on the device; *ke receives the sum. */
int ra_kinetic_energy(ra_ctx* ctx, double* ke);
/* The magnetic energy of the benchmark report (magnetism only; Benchmarking.F90:689-696, 846):
 * the volume average of |B|^2 (the same weights as the kinetic energy) times 1 / (2 Ek Pm). */
int ra_magnetic_energy(ra_ctx* ctx, double* me);

/* Shell slices of the current state (Shell_Slices output, Spherical_IO.F90):
 * each quantity of quantities[0..nq) on the full theta-phi grid at the radial
 * indices levels[0..nlev) (0-based grid indices, 0 = outer boundary), into
 * out(n_phi, n_theta, nlev, nq) (Fortran order; phi fastest, theta in the
 * grid's order).  Quantity codes are the reference's output codes
 * (velocity_field_codes.F, vorticity_field_codes.F, thermal_field_codes.F) of values the
 * physical-space buffer holds: */
#define RA_Q_V_R            1
#define RA_Q_V_THETA        2
#define RA_Q_V_PHI          3
#define RA_Q_DV_R_DR       10
#define RA_Q_DV_THETA_DR   11
#define RA_Q_DV_PHI_DR     12
#define RA_Q_DV_R_DT       19
#define RA_Q_DV_THETA_DT   20   /* formed as Compute_dvtheta_by_dtheta, Compute_dvphi_by_dtheta do */
#define RA_Q_DV_PHI_DT     21
#define RA_Q_DV_R_DP       28
#define RA_Q_DV_THETA_DP   29
#define RA_Q_DV_PHI_DP     30
#define RA_Q_VORT_R       301   /* l(l+1) Z / (rho r^2), the radial vorticity */
#define RA_Q_VORT_THETA   302   /* (csc dv_r/dphi - v_phi) / r - dv_phi/dr */
#define RA_Q_VORT_PHI     303   /* dv_theta/dr + (v_theta - dv_r/dtheta) / r */
#define RA_Q_ENTROPY      501
#define RA_Q_PRESSURE     502   /* formed with the P grid in T's place; the pressure codes need reference_type 1 */
#define RA_Q_ENTROPY_DR   507
#define RA_Q_PRESSURE_DR  508
#define RA_Q_ENTROPY_DTHETA 513
#define RA_Q_ENTROPY_DPHI 519
#define RA_Q_PRESSURE_DPHI 520
#define RA_Q_B_R          801   /* magnetism only (magnetic_field_codes.F) */
#define RA_Q_B_THETA      802
#define RA_Q_B_PHI        803
#define RA_Q_J_R         1001   /* magnetism only: the current density curl B (current_density_codes.F) */
#define RA_Q_J_THETA     1004
#define RA_Q_J_PHI       1007
/* The fluctuating part (the field minus its azimuthal mean: m > 0) and the azimuthal mean
 * (m = 0) of each quantity above, under the reference's codes: */
#define RA_Q_VP_R           4
#define RA_Q_VP_THETA       5
#define RA_Q_VP_PHI         6
#define RA_Q_VM_R           7
#define RA_Q_VM_THETA       8
#define RA_Q_VM_PHI         9
#define RA_Q_DVP_R_DR      13
#define RA_Q_DVP_THETA_DR  14
#define RA_Q_DVP_PHI_DR    15
#define RA_Q_DVM_R_DR      16
#define RA_Q_DVM_THETA_DR  17
#define RA_Q_DVM_PHI_DR    18
#define RA_Q_DVP_R_DT      22
#define RA_Q_DVM_R_DT      25
#define RA_Q_DVP_THETA_DT  23
#define RA_Q_DVP_PHI_DT    24
#define RA_Q_DVM_THETA_DT  26
#define RA_Q_DVM_PHI_DT    27
#define RA_Q_DVP_R_DP      31
#define RA_Q_DVP_THETA_DP  32
#define RA_Q_DVP_PHI_DP    33
#define RA_Q_DVM_R_DP      34   /* the mean of a phi derivative: zero */
#define RA_Q_DVM_THETA_DP  35
#define RA_Q_DVM_PHI_DP    36
#define RA_Q_VORTP_R      304
#define RA_Q_VORTM_R      307
#define RA_Q_VORTP_THETA  305
#define RA_Q_VORTP_PHI    306
#define RA_Q_VORTM_THETA  308
#define RA_Q_VORTM_PHI    309
#define RA_Q_ENTROPY_P    503
#define RA_Q_PRESSURE_P   504
#define RA_Q_ENTROPY_M    505
#define RA_Q_PRESSURE_M   506
#define RA_Q_ENTROPY_P_DR 509
#define RA_Q_PRESSURE_P_DR 510
#define RA_Q_ENTROPY_M_DR 511
#define RA_Q_PRESSURE_M_DR 512
#define RA_Q_ENTROPY_P_DTHETA 515
#define RA_Q_ENTROPY_M_DTHETA 517
#define RA_Q_ENTROPY_P_DPHI 521
#define RA_Q_PRESSURE_P_DPHI 522
#define RA_Q_ENTROPY_M_DPHI 523
#define RA_Q_PRESSURE_M_DPHI 524
#define RA_Q_BP_R         804
#define RA_Q_BP_THETA     805
#define RA_Q_BP_PHI       806
#define RA_Q_BM_R         807
#define RA_Q_BM_THETA     808
#define RA_Q_BM_PHI       809
#define RA_Q_JP_R        1002
#define RA_Q_JM_R        1003
#define RA_Q_JP_THETA    1005
#define RA_Q_JM_THETA    1006
#define RA_Q_JP_PHI      1008
#define RA_Q_JM_PHI      1009
/* Products (Diagnostics_Vorticity_Field.F90): enstrophy and its mean / fluctuating forms, the
 * squared vorticity components, the kinetic helicity v.omega by component and in total with
 * the (velocity, vorticity) part pairs pp, mm, mp, pm; with magnetism mean J . J': */
#define RA_Q_ENSTROPHY              310
#define RA_Q_ENSTROPHY_PM           311
#define RA_Q_ENSTROPHY_MM           312
#define RA_Q_ENSTROPHY_PP           313
#define RA_Q_VORT_R_SQ              314
#define RA_Q_VORT_THETA_SQ          315
#define RA_Q_VORT_PHI_SQ            316
#define RA_Q_VORTP_R_SQ             317
#define RA_Q_VORTP_THETA_SQ         318
#define RA_Q_VORTP_PHI_SQ           319
#define RA_Q_VORTM_R_SQ             320
#define RA_Q_VORTM_THETA_SQ         321
#define RA_Q_VORTM_PHI_SQ           322
#define RA_Q_KIN_HELICITY_R         324
#define RA_Q_KIN_HELICITY_THETA     325
#define RA_Q_KIN_HELICITY_PHI       326
#define RA_Q_KIN_HELICITY_PP_R      327
#define RA_Q_KIN_HELICITY_PP_THETA  328
#define RA_Q_KIN_HELICITY_PP_PHI    329
#define RA_Q_KIN_HELICITY_MM_R      330
#define RA_Q_KIN_HELICITY_MM_THETA  331
#define RA_Q_KIN_HELICITY_MM_PHI    332
#define RA_Q_KIN_HELICITY_MP_R      333
#define RA_Q_KIN_HELICITY_MP_THETA  334
#define RA_Q_KIN_HELICITY_MP_PHI    335
#define RA_Q_KIN_HELICITY_PM_R      336
#define RA_Q_KIN_HELICITY_PM_THETA  337
#define RA_Q_KIN_HELICITY_PM_PHI    338
#define RA_Q_KIN_HELICITY           339
#define RA_Q_KIN_HELICITY_PP        340
#define RA_Q_KIN_HELICITY_MM        341
#define RA_Q_KIN_HELICITY_MP        342
#define RA_Q_KIN_HELICITY_PM        343
#define RA_Q_JPM_SQ                1013
/* mass_flux_codes.F: rho v and its fluctuating and mean parts: */
#define RA_Q_RHOV_R                 201
#define RA_Q_RHOV_THETA             202
#define RA_Q_RHOV_PHI               203
#define RA_Q_RHOVP_R                204
#define RA_Q_RHOVP_THETA            205
#define RA_Q_RHOVP_PHI              206
#define RA_Q_RHOVM_R                207
#define RA_Q_RHOVM_THETA            208
#define RA_Q_RHOVM_PHI              209
/* thermal_energy_codes.F: rho T S of the reference state, its parts and their squares: */
#define RA_Q_THERMAL_ENERGY_FULL    701
#define RA_Q_THERMAL_ENERGY_P       702
#define RA_Q_THERMAL_ENERGY_M       703
#define RA_Q_THERMAL_ENERGY_SQ      707
#define RA_Q_THERMAL_ENERGYP_SQ     708
#define RA_Q_THERMAL_ENERGYM_SQ     709
/* with magnetism, the phi derivatives of B and their parts (the means are zero): */
#define RA_Q_DB_R_DP           828
#define RA_Q_DB_THETA_DP       829
#define RA_Q_DB_PHI_DP         830
#define RA_Q_DBP_R_DP          831
#define RA_Q_DBP_THETA_DP      832
#define RA_Q_DBP_PHI_DP        833
#define RA_Q_DBM_R_DP          834
#define RA_Q_DBM_THETA_DP      835
#define RA_Q_DBM_PHI_DP        836
/* Squares (Diagnostics_Energies.F90, Diagnostics_Current_Density.F90): 1/2 rho |v|^2 and its
 * parts, of the mean flow and of the fluctuations (kinetic_energy_codes.F), the same without
 * rho, J.J and its parts, and 1/2 Lorentz_Coeff |B|^2 likewise (magnetic_energy_codes.F): */
#define RA_Q_KINETIC_ENERGY     401
#define RA_Q_RADIAL_KE          402
#define RA_Q_THETA_KE           403
#define RA_Q_PHI_KE             404
#define RA_Q_MKINETIC_ENERGY    405
#define RA_Q_RADIAL_MKE         406
#define RA_Q_THETA_MKE          407
#define RA_Q_PHI_MKE            408
#define RA_Q_PKINETIC_ENERGY    409
#define RA_Q_RADIAL_PKE         410
#define RA_Q_THETA_PKE          411
#define RA_Q_PHI_PKE            412
#define RA_Q_VSQ                413
#define RA_Q_RADIAL_VSQ         414
#define RA_Q_THETA_VSQ          415
#define RA_Q_PHI_VSQ            416
#define RA_Q_MVSQ               417
#define RA_Q_RADIAL_MVSQ        418
#define RA_Q_THETA_MVSQ         419
#define RA_Q_PHI_MVSQ           420
#define RA_Q_PVSQ               421
#define RA_Q_RADIAL_PVSQ        422
#define RA_Q_THETA_PVSQ         423
#define RA_Q_PHI_PVSQ           424
#define RA_Q_J_SQ              1010
#define RA_Q_JP_SQ             1011
#define RA_Q_JM_SQ             1012
#define RA_Q_J_R_SQ            1014
#define RA_Q_JP_R_SQ           1015
#define RA_Q_JM_R_SQ           1016
#define RA_Q_J_THETA_SQ        1017
#define RA_Q_JP_THETA_SQ       1018
#define RA_Q_JM_THETA_SQ       1019
#define RA_Q_J_PHI_SQ          1020
#define RA_Q_JP_PHI_SQ         1021
#define RA_Q_JM_PHI_SQ         1022
#define RA_Q_MAGNETIC_ENERGY   1101
#define RA_Q_RADIAL_ME         1102
#define RA_Q_THETA_ME          1103
#define RA_Q_PHI_ME            1104
#define RA_Q_MMAGNETIC_ENERGY  1105
#define RA_Q_RADIAL_MME        1106
#define RA_Q_THETA_MME         1107
#define RA_Q_PHI_MME           1108
#define RA_Q_PMAGNETIC_ENERGY  1109
#define RA_Q_RADIAL_PME        1110
#define RA_Q_THETA_PME         1111
#define RA_Q_PHI_PME           1112
/* Runs the stages that form the fields on the grid (as ra_kinetic_energy);
 * another code, or a level outside 0 .. n_r-1, returns RA_ERR_ARG. */
int ra_shell_slices(ra_ctx* ctx, const int* quantities, int nq, const int* levels, int nlev, double* out);

/* Shell averages of the current state (Shell_Averages output, Spherical_IO.F90
 * Add_Quantity :548-575 with ComputeEll0 :1350-1391): for each quantity of
 * quantities[0..nq) (codes as above) and each radius, the mean over the sphere
 * (phi mean, Gauss-Legendre theta weights / 2) and the same average of
 * (q - mean)^2, ^3, ^4, into out(n_r, 4, nq) (Fortran order).  Runs the stages
 * that form the fields on the grid (as ra_kinetic_energy); unknown codes
 * return RA_ERR_ARG. */
int ra_shell_averages(ra_ctx* ctx, const int* quantities, int nq, double* out);

/* Azimuthal averages of the current state (AZ_Avgs output, Spherical_IO.F90
 * :477-481): the phi mean of each quantity at every (r, theta) point, into
 * out(n_r, n_theta, nq) (Fortran order; theta in the grid's order).  Codes and
 * errors as for ra_shell_slices. */
int ra_azimuthal_averages(ra_ctx* ctx, const int* quantities, int nq, double* out);

/* Shell spectra of the current state (Shell_Spectra output; Parallel_IO.F90
 * Spectral_Prep :973-1047): each quantity at the radial indices levels[0..nlev)
 * taken to (l, m) space by the unnormalised phi FFT and the forward Legendre
 * transform (FFT_To_Spectral, Legendre_Transform p2b -> s2b), into
 * out(l_max+1 [l], l_max+1 [m], 2 [re, im], nlev, nq) (Fortran order; zero for
 * l < m).  Codes, levels and errors as for ra_shell_slices. */
int ra_shell_spectra(ra_ctx* ctx, const int* quantities, int nq, const int* levels, int nlev, double* out);

/* Equatorial slices of the current state (Equatorial_Slices output,
 * Spherical_IO.F90:394-398: the mean of the theta rows n_theta/2 and
 * n_theta/2 + 1) at every radius, into out(n_phi, n_r, nq) (Fortran order).
 * Codes and errors as for ra_shell_slices. */
int ra_equatorial_slices(ra_ctx* ctx, const int* quantities, int nq, double* out);

/* Meridional slices of the current state (Meridional_Slices output,
 * Spherical_IO.F90:384-387, 467-473): each quantity at the phi indices
 * phi_indices[0..nphi_sel) (0-based, 0 .. n_phi-1) at every (r, theta), into
 * out(n_r, n_theta, nphi_sel, nq) (Fortran order).  Codes and errors as for
 * ra_shell_slices; an index outside 0 .. n_phi-1 returns RA_ERR_ARG. */
int ra_meridional_slices(ra_ctx* ctx, const int* quantities, int nq, const int* phi_indices, int nphi_sel,
                         double* out);

/* Global averages of the current state (G_Avgs output; Compute_Radial_Average,
 * Spherical_IO.F90:1436-1470): the volume average of each quantity (the
 * spherical means per radius weighted by the radial integration weights, as
 * in ra_kinetic_energy), into out[0..nq).  Codes and errors as for
 * ra_shell_slices. */
int ra_global_averages(ra_ctx* ctx, const int* quantities, int nq, double* out);

/* Point probes of the current state (Point_Probes output, Spherical_IO.F90:
 * 379-382): each quantity at the tensor product of the radial, theta and phi
 * grid indices (0-based; 1 .. 64 of each), into
 * out(nphi_p, ntheta_p, nr_p, nq) (Fortran order).  Codes as for
 * ra_shell_slices; an index out of range returns RA_ERR_ARG. */
int ra_point_probes(ra_ctx* ctx, const int* quantities, int nq, const int* r_idx, int nr_p, const int* theta_idx,
                    int ntheta_p, const int* phi_idx, int nphi_p, double* out);

/* Timed stepping for benchmarks: runs nsteps like ra_step (without graph
 * replay, so that CUDA events on the context's stream bracket every kernel)
 * and returns the elapsed device time of the whole region in *total_ms and,
 * if kernel_ms is not NULL, the summed time of each kernel of the step in
 * kernel_ms[0..nk) in the order of ra_kernel_name(). */
int ra_time_steps(ra_ctx* ctx, int nsteps, double* total_ms, double* kernel_ms, int nk);
/* ra_step (graph replays included) bracketed by CUDA events on the context's
 * stream: *total_ms receives the device time of the nsteps steps.  The
 * status check that ends ra_step (a host read of the device error word)
 * follows the closing event, so it is not part of the time. */
int ra_step_timed(ra_ctx* ctx, int nsteps, double* total_ms);
/* Number of kernels one step launches and their names (static strings). */
int ra_kernels_per_step(void);
const char* ra_kernel_name(int i);

/* Blocks until the context's stream is idle; returns the first device error. */
int ra_sync(ra_ctx* ctx);

/* ---- math-layer operators (host buffers in the reference layouts) ---- */

/* StP_4d_dgp2 (Legendre_Transforms.F90:968-1074).
 * s: concatenation over m = 0..l_max of s2a(m)%data(m:l_max, nr, 2, nf)
 * p: p2a(n_theta, nr*2*nf, l_max+1)  (nrhs = (r, re/im, field), r fastest) */
int ra_legendre_s2p(ra_ctx* ctx, const double* s, double* p, int nf, int nr);
/* PtS_4d_dgpv3 (Legendre_Transforms.F90:1077-1175): layouts as above, reversed. */
int ra_legendre_p2s(ra_ctx* ctx, const double* p, double* s, int nf, int nr);

/* c2r_ip4D_fftw / r2c_ip4D_fftw (Fourier_Transform.F90:100-183): in place on
 * x(n_phi+2, howmany), unnormalised, FFTW's packed (re, im) layout. */
int ra_fft_c2r(ra_ctx* ctx, double* x, long howmany);
/* Device-resident spherical-harmonic transforms of nfr complex columns (fields x radial
 * levels), operands in device memory (no host copies): direction 0 (spectral -> physical)
 * runs StP_4d_dgp2 (Legendre_Transforms.F90:968-1074) from d_spec into d_work, unfolds the
 * (theta, pi - theta) blocks into phi rows in d_grid and runs FFT_To_Physical's c2r
 * (Fourier_Transform.F90:142-183) in place; direction 1 (physical -> spectral) runs the r2c
 * in place on d_grid (overwriting it), folds into d_work and runs PtS_4d_dgpv3 (:1077-1175)
 * into d_spec.  precision RA_PREC_FP64 (FP64 tensor-core products) or RA_PREC_MIXED
 * (split int8 products; their plan is built on the first call with given operands).
 *   d_spec: [n_lm rows][nfr][re, im], rows m-major with the even l - m first (the row order
 *           of the ra_* device buffers: row(m, l) = off(m) + (l - m even ? (l - m)/2 :
 *           ne(m) + (l - m - 1)/2), off(m) = m L - m (m - 1)/2, ne(m) = (L - m + 1)/2)
 *   d_grid: [n_theta][nfr][n_phi + 2] real rows (Gauss-Legendre theta order)
 *   d_work: l_max + 1 times n_theta times nfr complex entries (the E/O or folded blocks)
 * stage_ms (may be NULL) receives the device times of [0] the Legendre product (with the
 * digit split), [1] the relayout and [2] the FFT.  The call first makes the context's stream
 * wait for the work queued on the legacy default stream (operands written there are
 * complete) and returns with its own work complete; operands written on other streams must
 * be complete before the call. */
int ra_transform_dev(ra_ctx* ctx, int direction, int precision, double* d_spec, double* d_grid, double* d_work,
                     int nfr, double* stage_ms);
int ra_fft_r2c(ra_ctx* ctx, double* x, long howmany);

/* Chebyshev_Polynomials.F90: To_Spectral4D (:375), From_Spectral4D (:450) and
 * Cheby_Deriv_Buffer_4D (:560) of order 1..3 on columns f(n_r, ncols).  A context
 * in the finite-difference mode returns RA_ERR_STATE. */
int ra_cheby_to_spectral(ra_ctx* ctx, const double* f, double* c, long ncols);
int ra_cheby_from_spectral(ra_ctx* ctx, const double* c, double* f, long ncols);
int ra_cheby_deriv(ra_ctx* ctx, const double* c, double* dc, int order, long ncols);

/* Split-precision product on the tensor cores, the engine of RA_PREC_MIXED:
 * C = A B with A (m x k) and B (k x n) row-major host arrays, C (m x n)
 * row-major; each operand is cut into 5 balanced base-256 int8 digits per
 * element (rows of A, columns of B scaled by powers of two) and the 15
 * leading digit products are accumulated exactly in int32 by tcgen05 before
 * an FP64 recombination (k <= 20000).
 * Replaces, for the parity tests, the DGEMM calls of Legendre_Transforms.F90:1028-1150. */
int ra_mixed_gemm(ra_ctx* ctx, const double* a, const double* b, double* c, int m, int n, int k);

/* Allocation-free form of ra_mixed_gemm, for callers that cannot allocate
 * device memory.  No counterpart in the reference.  a (m x k), b (k x n) and
 * c (m x n) are row-major DEVICE arrays on the current device; the work is
 * enqueued on `stream` (a cudaStream_t, NULL = legacy default stream) and the
 * call returns after it finished.  Scratch comes from one fixed 16 MiB
 * device array inside the library (about 5 (m + n) k bytes are needed;
 * larger products return RA_ERR_ARG with the needed size in msg).  Every
 * call looks up that array's address on the current device.  The call is
 * synchronous (it reads a status word back and waits for `stream`), so it
 * cannot be made on a stream that is being captured.  Calls that overlap in
 * time on one device race on the shared scratch.  msg (may be NULL) receives an error message of at most
 * msg_len bytes. */
int ra_mixed_gemm_noalloc(const double* a, const double* b, double* c, int m, int n, int k, void* stream,
                          char* msg, int msg_len);

/* ---- batched per-l solves on their own (no transform context) ----
 * LU_Decompose_full / LU_Solve_full (Linear_Solve.F90:1028-1036, 1088-1110)
 * for count matrices of order n (even, <= 1152) on one device. */
typedef struct ra_lu ra_lu;
#define RA_SOLVE_FP64    0   /* block substitution with the FP64 LU factors */
#define RA_SOLVE_REFINE  1   /* FP32 substitution + FP64 residuals, refined to FP64 accuracy */
int ra_lu_create(ra_lu** lu, int n, int count, int device);
int ra_lu_destroy(ra_lu* lu);
int ra_lu_last_error(const ra_lu* lu, char* msg, int len);
/* a(n, n, count): the matrices in Fortran (column-major) order.  Factors them
 * on the device (partial pivoting); ms (may be NULL) receives the device time
 * of the factorisation.  RA_ERR_SINGULAR names the first singular matrix,
 * RA_ERR_NONFINITE refuses NaN/Inf entries. */
int ra_lu_factor(ra_lu* lu, const double* a, double* ms);
/* x = A_l^-1 b for b(n, ncols, count) (Fortran order) in one launch.  iters
 * (may be NULL) receives, per matrix and per tile of columns
 * (ra_lu_tiles(lu, ncols, mode) entries, matrix-major), the refinement
 * iterations (1 in the FP64 form); ms the device time of the solve. */
int ra_lu_solve(ra_lu* lu, const double* b, double* x, int ncols, int mode, int* iters, double* ms);
int ra_lu_tiles(const ra_lu* lu, int ncols, int mode);

/* Radial grid of the context: radius(n_r), r(1) = r_max (Chebyshev_Polynomials.F90:168-200). */
int ra_radius(const ra_ctx* ctx, double* radius);
/* Gauss-Legendre nodes cos(theta) (n_theta) as used by the context. */
int ra_costheta(const ra_ctx* ctx, double* costheta);

/* Kernel choices of the tunable stages (the autotuner's knobs):
 *   "physics"   physical-space kernel: 1 every FFT pass in shared memory
 *               (n_theta <= 768); 0 the last (radix-3) pass and the
 *               nonlinear terms in registers, two CTAs per SM, 2 the same
 *               with one CTA per SM (n_theta 384, 768, 1536; the only
 *               kernel at 1536)
 *   "solve_nc"  right-hand-side columns per block-substitution CTA of the
 *               W-P-T system: 32 or 16 (32 only where its column block fits)
 * ra_get_choice reads a choice, ra_set_choice forces one (RA_ERR_ARG for an
 * unknown knob or value); the results do not depend on the choice beyond
 * rounding.  ra_autotune times every candidate on the context's buffers
 * (nreps launches each, CUDA events) and keeps the fastest; ms_out (may be
 * NULL) receives, per knob in the order above, the chosen candidate's time. */
int ra_get_choice(const ra_ctx* ctx, const char* knob, int* value);
int ra_set_choice(ra_ctx* ctx, const char* knob, int value);
int ra_autotune(ra_ctx* ctx, int nreps, double* ms_out);

/* Number of kernel launches issued by the last ra_step call (for accounting). */
long ra_launch_count(const ra_ctx* ctx);

/* Diagnostics: copies internal device buffer `which` (RA_BUF_*) to host
 * memory; n is the capacity of out in doubles, *n_out receives the size.
 * With out == NULL only the size is returned.  Used by the parity tests to
 * compare every stage of a step with the CPU restatement; the reference
 * exposes the same data as its Spherical_Buffer configurations. */
#define RA_BUF_GRID    0   /* [12][n_lm][2][n_r]  W, dW, d2W, d3W, P, dP, T, dT, d2T, Z, dZ, d2Z on the grid */
#define RA_BUF_S2A     1   /* [row][7][n_r][2]    after Post_Solve: W, T, Z, dW, dT, dZ, d2W */
#define RA_BUF_S2A11   2   /* [row][n_r][11][2]   after rlm_spacea; fields DVRDT, DVTDR, VR, VT, VP,
                                 DVRDR, DVPDR, OMR, DTDR, DTDT, T */
#define RA_BUF_P2A     3   /* [n_theta/2][m][2][n_r][11][2]  even-l / odd-l products E, O */
#define RA_BUF_P2B     4   /* [m][2][n_theta/2][n_r][4][2]   folded f_even, f_odd */
#define RA_BUF_S2B     5   /* [row][n_r][4][2]    */
#define RA_BUF_AB      6   /* [4][n_lm][2][n_r]   */
#define RA_BUF_RHS_WPT 7   /* [n_lm][2][3 n_r]    */
#define RA_BUF_RHS_Z   8   /* [n_lm][2][n_r]      */
#define RA_BUF_PTAB    9   /* [row][n_theta/2]    P_l^m (times 1/2 for m > 0) */
#define RA_BUF_IPTAB  10   /* [row][n_theta/2]    weighted P_l^m with the FFT normalisation */
/* with magnetism: RA_BUF_GRID adds C, dC, d2C, A, dA, d2A ([18]); RA_BUF_S2A11 and RA_BUF_P2A add
 * B_r, (curl B)_r, (curl B)_theta, (curl B)_phi, B_theta, B_phi ([17], the last four times
 * r sin(theta)); RA_BUF_P2B and RA_BUF_S2B add EMF_theta, EMF_r, EMF_phi ([7]; after rlm_spaceb
 * the C right-hand side, EMF_r and the term whose radial derivative completes the A one);
 * RA_BUF_AB holds [6] fields (W P T Z C A) */
#define RA_BUF_S2AM   11   /* [row][5][n_r][2]    magnetism: C, A, dC, dA, d2C after Post_Solve */
#define RA_BUF_RHS_C  12   /* [n_lm][2][n_r]      magnetism */
#define RA_BUF_RHS_A  13   /* [n_lm][2][n_r]      magnetism */
int ra_debug_buffer(ra_ctx* ctx, int which, double* out, long n, long* n_out);

#ifdef __cplusplus
}
#endif
#endif /* RAYLEIGH_B200_H */
