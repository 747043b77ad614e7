// C ABI, context set-up and step orchestration of librayleigh_b200.
//
// Set-up restates the reference's initialisation of the path:
//   grid sizes                 ProblemSize.F90:334-464
//   Gauss-Legendre nodes       Legendre_Polynomials.F90:332-393 (in long double)
//   Chebyshev grid/matrices    Chebyshev_Polynomials.F90:65-351
//   Boussinesq reference state PDE_Coefficients.F90:335-435
//   implicit matrices + BCs    Sphere_Linear_Terms.F90:196-1100, Linear_Solve.F90:494-539,1459-1522
// Host work here is configuration-time only (O(n_r^2 l_max) matrix entries);
// every per-step operation runs on the device.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>

#include "ra_internal.h"
#include "ozaki.h"

using namespace ra;


namespace ra {

static void check_config(const ra_config& cfg) {
    if (cfg.n_r < 8 || (cfg.n_r & 1)) throw ArgError("n_r must be even and >= 8");
    if (cfg.l_max < 3) throw ArgError("l_max must be >= 3");
    if (cfg.magnetism && !(cfg.magnetic_prandtl > 0)) throw ArgError("magnetic_prandtl must be positive");
    if (!(cfg.aspect_ratio > 0 && cfg.aspect_ratio < 1)) throw ArgError("aspect_ratio must lie in (0, 1)");
    if (!(cfg.shell_depth > 0)) throw ArgError("shell_depth must be positive");
    if (!(cfg.dt > 0)) throw ArgError("dt must be positive");
    if (cfg.precision != RA_PREC_FP64 && cfg.precision != RA_PREC_MIXED) throw ArgError("unknown precision mode");
    if (cfg.reference_type < 1 || cfg.reference_type > 3)
        throw ArgError("reference_type must be 1 (Boussinesq), 2 or 3 (polytropes)");
    if (cfg.reference_type >= 2 && !(cfg.poly_n > 0 && cfg.poly_nrho > 0))
        throw ArgError("a polytropic reference state needs poly_n > 0 and poly_nrho > 0");
    if (cfg.reference_type == 2 && !(cfg.poly_mass > 0 && cfg.poly_rho_i > 0 && cfg.pressure_specific_heat > 0 &&
                                     cfg.nu_top > 0 && cfg.kappa_top > 0 && (!cfg.magnetism || cfg.eta_top > 0)))
        throw ArgError("reference_type 2 needs poly_mass, poly_rho_i, pressure_specific_heat, nu_top, kappa_top "
                       "(and eta_top with magnetism) > 0");
    if (cfg.reference_type == 3 && !(cfg.modified_rayleigh > 0))
        throw ArgError("reference_type 3 needs modified_rayleigh > 0");
    for (int t : {cfg.nu_type, cfg.kappa_type, cfg.eta_type})
        if (t != 1 && t != 2) throw ArgError("transport types 1 (constant) and 2 (density power) are provided");
}

static Dims make_dims(const ra_config& cfg) {
    Dims d{};
    d.lmax = cfg.l_max;
    d.L = cfg.l_max + 1;
    d.nth = cfg.n_theta > 0 ? cfg.n_theta : (3 * (cfg.l_max + 1)) / 2;
    if (d.nth & 1) throw ArgError("n_theta must be even");
    if (d.nth < d.L) throw ArgError("n_theta must be >= l_max + 1");
    d.nth2 = d.nth / 2;
    d.nphi = 2 * d.nth;
    d.nr = cfg.n_r;
    d.nlm = (long)d.L * (d.L + 1) / 2;
    if (cfg.chebyshev) {
        d.rda = (2 * d.nr) / 3 + 1;
        d.kc = d.rda - 1;
    } else {   // finite differences: no dealiasing, boundary rows over every column
        d.rda = d.nr + 1;
        d.kc = d.nr;
    }
    return d;
}

// Find_Colocation + nth_legendre (Legendre_Polynomials.F90:332-393) in long double.
static void gauss_legendre(int n, std::vector<long double>& x, std::vector<long double>& w) {
    x.assign(n, 0.0L);
    w.assign(n, 0.0L);
    const long double PI = 3.141592653589793238462643383279502884L;
    const long double eps = 3e-14L;
    for (int i = 1; i <= (n + 1) / 2; ++i) {
        long double root = cosl(PI * (i - 0.25L) / (n + 0.5L));
        for (int it = 0; it < 100; ++it) {
            long double pn = 1.0L, pm1 = 0.0L;
            for (int j = 1; j <= n; ++j) {
                const long double pm2 = pm1;
                pm1 = pn;
                pn = ((2.0L * j - 1.0L) * root * pm1 - (j - 1.0L) * pm2) / j;
            }
            const long double dpn = n * (root * pn - pm1) / (root * root - 1.0L);
            const long double nw = root - pn / dpn;
            const long double del = fabsl(root - nw);
            root = nw;
            x[i - 1] = -root;
            x[n - i] = root;
            w[i - 1] = 2.0L / ((1.0L - root * root) * dpn * dpn);
            w[n - i] = w[i - 1];
            if (del <= eps) break;
        }
    }
}

// Chebyshev collocation grid and derivative matrices dcheby(r, n, d), d = 0..3
// (Chebyshev_Polynomials.F90:65-351; single domain, zeros of T_N).
static void chebyshev_setup(Ctx& c, double rmin, double rmax) {
    const int n = c.d.nr;
    c.rad.rmin = rmin;
    c.rad.rmax = rmax;
    std::vector<double> theta(n), x(n);
    const double dth = M_PI / n;
    double arg = dth * 0.5;
    for (int i = 0; i < n; ++i) {   // accumulated as in Gen_Colocation_Points
        theta[i] = arg;
        x[i] = cos(arg);
        arg = arg + dth;
    }
    std::vector<double> alpha((size_t)n * n, 0.0);
    alpha[(size_t)(n - 2) * n + (n - 1)] = 2.0 * (n - 1);
    for (int k = n - 3; k >= 0; --k) {
        alpha[(size_t)k * n + k + 1] = 2.0 * (k + 1);
        for (int j = 0; j < n; ++j) alpha[(size_t)k * n + j] += alpha[(size_t)(k + 2) * n + j];
    }
    c.cheb_D.assign((size_t)4 * n * n, 0.0);
    double* D0 = c.cheb_D.data();
    for (int r = 0; r < n; ++r)
        for (int k = 0; k < n; ++k) D0[(size_t)r * n + k] = cos(k * theta[r]);
    for (int r = 0; r < n; ++r) D0[(size_t)r * n] -= 0.5;
    for (int d = 1; d < 4; ++d) {
        const double* Dp = c.cheb_D.data() + (size_t)(d - 1) * n * n;
        double* Dd = c.cheb_D.data() + (size_t)d * n * n;
        for (int r = 0; r < n; ++r)
            for (int j = 0; j < n; ++j) {
                double s = 0.0;
                for (int i = 0; i < n; ++i) s += Dp[(size_t)r * n + i] * alpha[(size_t)i * n + j];
                Dd[(size_t)r * n + j] = s;
            }
    }
    const double xmin = x[n - 1], xmax = x[0];
    double scaling = (rmax - rmin) / (xmax - xmin);
    c.rad.radius.resize(n);
    for (int i = 0; i < n; ++i) c.rad.radius[i] = (x[i] - xmin) * scaling + rmin;
    // integration weights 3 pi scaling / ((r_o^3 - r_i^3) N) r^2 sqrt(1 - x^2), halved
    // at the two end points (Chebyshev_Polynomials.F90:165-194)
    const double int_scale = 3.0 * M_PI * scaling / ((rmax * rmax * rmax - rmin * rmin * rmin) * n);
    c.rad.int_w.resize(n);
    for (int i = 0; i < n; ++i)
        c.rad.int_w[i] = int_scale * c.rad.radius[i] * c.rad.radius[i] * sqrt(1.0 - x[i] * x[i]);
    c.rad.int_w[0] *= 0.5;
    c.rad.int_w[n - 1] *= 0.5;
    scaling = 1.0 / scaling;
    c.deriv_scaling = scaling;
    for (int d = 1; d < 4; ++d) {
        const double s = pow(scaling, d);
        double* Dd = c.cheb_D.data() + (size_t)d * n * n;
        for (size_t e = 0; e < (size_t)n * n; ++e) Dd[e] *= s;
    }
}

// One stencil of Generate_Coefs (Finite_Difference.F90:525-689): the weights of derivative
// order deriv at offsets dees (scaled by dmean) from the inverse of their Vandermonde matrix,
// each row times (j - 1)! / dmean^(j - 1).  Gauss-Jordan with partial pivoting on the small
// matrix (at most 5 x 5), in long double.
static std::vector<double> fd_weights(const std::vector<double>& dees, double dmean, int deriv) {
    const int n = (int)dees.size();
    std::vector<long double> a((size_t)n * 2 * n, 0.0L);
    for (int j = 0; j < n; ++j) {
        long double p = 1.0L;
        for (int k = 0; k < n; ++k) {
            a[(size_t)j * 2 * n + k] = p;
            p *= dees[j];
        }
        a[(size_t)j * 2 * n + n + j] = 1.0L;
    }
    for (int col = 0; col < n; ++col) {
        int piv = col;
        for (int i = col + 1; i < n; ++i)
            if (fabsl(a[(size_t)i * 2 * n + col]) > fabsl(a[(size_t)piv * 2 * n + col])) piv = i;
        if (a[(size_t)piv * 2 * n + col] == 0.0L) throw ArgError("finite-difference stencil is singular");
        if (piv != col)
            for (int k = 0; k < 2 * n; ++k) std::swap(a[(size_t)piv * 2 * n + k], a[(size_t)col * 2 * n + k]);
        const long double inv = 1.0L / a[(size_t)col * 2 * n + col];
        for (int k = 0; k < 2 * n; ++k) a[(size_t)col * 2 * n + k] *= inv;
        for (int i = 0; i < n; ++i)
            if (i != col) {
                const long double f = a[(size_t)i * 2 * n + col];
                if (f != 0.0L)
                    for (int k = 0; k < 2 * n; ++k) a[(size_t)i * 2 * n + k] -= f * a[(size_t)col * 2 * n + k];
            }
    }
    // row deriv of the inverse, times deriv! / dmean^deriv
    long double fact = 1.0L;
    for (int j = 2; j <= deriv; ++j) fact *= j;
    const long double sc = fact / powl((long double)dmean, deriv);
    std::vector<double> w(n);
    for (int k = 0; k < n; ++k) w[k] = (double)(a[(size_t)deriv * 2 * n + n + k] * sc);
    return w;
}

// Finite-difference radial mode (chebyshev = 0): the uniform grid (ProblemSize.F90:607-618),
// the derivative matrices D_d (d = 1..3) of the default 5-point stencils with one-sided
// boundary stencils of d + 2 points (Initialize_dcoefs and Generate_Coefs,
// Finite_Difference.F90:464-689; the rows d_by_dx3d3 and Load_Interior_RowsFD apply,
// :374-460, :717-777), D_0 = I, and Initialize_Derivatives' integration weights (:69-93).
static void fd_setup(Ctx& c, double rmin, double rmax) {
    const int n = c.d.nr, ns = 5, kd = 3, sc = 3;
    c.rad.rmin = rmin;
    c.rad.rmax = rmax;
    std::vector<double>& r = c.rad.radius;
    r.assign(n, 0.0);
    r[n - 1] = rmin;
    const double dr = 1.0 / (n - 1.0) * (rmax - rmin);
    for (int i = n - 2; i >= 0; --i) r[i] = dr + r[i + 1];
    c.rad.fd_dr = dr;
    c.cheb_D.assign((size_t)4 * n * n, 0.0);
    for (int i = 0; i < n; ++i) c.cheb_D[(size_t)i * n + i] = 1.0;
    for (int dd = 1; dd <= 3; ++dd) {
        double* D = c.cheb_D.data() + (size_t)dd * n * n;
        // interior rows (Fortran i = 2 .. n-1): the centred stencil clipped at the ends
        for (int i = 2; i <= n - 1; ++i) {
            const int jstart = std::max(1, sc - i + 1), jend = std::min(ns, (n - i) + sc);
            const int nxy = jend - jstart + 1;
            std::vector<double> dees(nxy);
            double dsum = 0.0;
            for (int j = jstart; j <= jend; ++j) {
                dees[j - jstart] = r[i + j - sc - 1] - r[i - 1];
                dsum += fabs(dees[j - jstart]);
            }
            dees[sc - jstart] = 0.0;
            const double dmean = dsum / (double)(nxy - 1);
            for (double& v : dees) v /= dmean;
            const std::vector<double> w = fd_weights(dees, dmean, dd);
            for (int j = jstart; j <= jend; ++j) {   // stencil point j -> column i + j - kd (1-based)
                const int col = i + j - kd - 1;
                D[(size_t)(i - 1) * n + col] = w[j - jstart];
            }
        }
        // the end points: one-sided stencils of dd + 2 points
        const int nxy = dd + 2;
        for (int side = 0; side < 2; ++side) {
            const int pt = side ? n : 1;
            std::vector<double> dees(nxy, 0.0);
            double dsum = 0.0;
            for (int j = (side ? 1 : 2); j <= (side ? nxy - 1 : nxy); ++j) {
                dees[j - 1] = side ? r[pt + (j - nxy) - 1] - r[pt - 1] : r[pt + j - 2] - r[pt - 1];
                dsum += dees[j - 1];
            }
            const double dmean = dsum / (double)(nxy - 1);
            for (double& v : dees) v /= dmean;
            const std::vector<double> w = fd_weights(dees, dmean, dd);
            for (int k = 0; k < nxy; ++k) {
                if (side) D[(size_t)(n - 1) * n + (n - nxy + k)] = w[k];
                else D[k] = w[k];
            }
        }
    }
    // integration weights (r_{i-1} - r_{i+1}) / 2 r_i^2, one-sided at the ends, normalised
    std::vector<double>& w = c.rad.int_w;
    w.assign(n, 0.0);
    for (int i = 1; i < n - 1; ++i) w[i] = (r[i - 1] - r[i + 1]) / 2.0 * r[i] * r[i];
    w[0] = (r[0] - r[1]) / 2.0 * r[0] * r[0];
    w[n - 1] = (r[n - 2] - r[n - 1]) / 2.0 * r[n - 1] * r[n - 1];
    double sum = 0.0;
    for (double v : w) sum += v;
    for (double& v : w) v /= sum;
    c.deriv_scaling = 1.0;
}

static void radial_setup(Ctx& c, double rmin, double rmax) {
    if (c.cfg.chebyshev)
        chebyshev_setup(c, rmin, rmax);
    else
        fd_setup(c, rmin, rmax);
}

// Reference state and transport coefficients (PDE_Coefficients.F90:216-257, 335-537, 925-1051,
// 1766-2098): Constant_Reference (Boussinesq), Polytropic_Reference (cgs) or
// Polytropic_ReferenceND, then Initialize_Diffusivity and Compute_Diffusion_Coefs.
static void reference_setup(Ctx& c) {
    const ra_config& cfg = c.cfg;
    const int n = c.d.nr;
    Radial& R = c.rad;
    const std::vector<double>& r = R.radius;
    const bool mag = cfg.magnetism != 0;
    R.delta_r.resize(n);
    R.delta_r[0] = r[0] - r[1];
    for (int i = 1; i < n; ++i) R.delta_r[i] = r[i - 1] - r[i];
    if (!cfg.chebyshev) R.delta_r.assign(n, R.fd_dr);   // Delta_r(:) = uniform_dr (ProblemSize.F90:613)
    R.density.assign(n, 1.0);
    R.dlnrho.assign(n, 0.0);
    R.d2lnrho.assign(n, 0.0);
    R.temperature.assign(n, 1.0);
    R.dlnT.assign(n, 0.0);
    R.buoy.resize(n);
    std::vector<double> visc_amp(n, 2.0), ohm_amp(n, 0.0);
    double pscaling = 1.0, nu_top, kappa_top, eta_top;
    bool visc = cfg.viscous_heating != 0, ohm = cfg.ohmic_heating != 0;
    if (cfg.reference_type == 1) {
        for (int i = 0; i < n; ++i) R.buoy[i] = (cfg.rayleigh / cfg.prandtl) * pow(r[i] / r[0], cfg.gravity_power);
        pscaling = cfg.rotation ? 1.0 / cfg.ekman : 1.0;
        R.coriolis = 2.0 / cfg.ekman;
        nu_top = 1.0;
        kappa_top = 1.0 / cfg.prandtl;
        // magnetism (:418-427): Lorentz_Coeff = 1 / (Pm Ek), eta = 1 / Pm
        R.lorentz = mag ? 1.0 / (cfg.magnetic_prandtl * cfg.ekman) : 0.0;
        eta_top = mag ? 1.0 / cfg.magnetic_prandtl : 0.0;
        std::fill(ohm_amp.begin(), ohm_amp.end(), R.lorentz);
        visc = ohm = false;   // Constant_Reference turns both heating terms off
    } else if (cfg.reference_type == 2) {
        const double G = 6.67e-8, pn = cfg.poly_n;
        const double ri = r[n - 1], ro = r[0], beta = ri / ro, dd = ro - ri;
        const double zeta0 = (beta + 1.0) / (beta * exp(cfg.poly_nrho / pn) + 1.0);
        const double c0 = (2.0 * zeta0 - beta - 1.0) / (1.0 - beta);
        const double c1 = (1.0 + beta) * (1.0 - zeta0) / ((1.0 - beta) * (1.0 - beta));
        std::vector<double> zeta(n);
        for (int i = 0; i < n; ++i) zeta[i] = c0 + c1 * dd / r[i];
        const double rho_c = cfg.poly_rho_i / pow(zeta[n - 1], pn);
        const double P_c = G * cfg.poly_mass * rho_c / ((pn + 1.0) * dd * c1);
        const double T_c = (pn + 1.0) * P_c / (cfg.pressure_specific_heat * rho_c);
        for (int i = 0; i < n; ++i) {
            const double gravity = G * cfg.poly_mass / (r[i] * r[i]);
            R.density[i] = rho_c * pow(zeta[i], pn);
            R.dlnrho[i] = -pn * c1 * dd / (zeta[i] * r[i] * r[i]);
            R.d2lnrho[i] = -R.dlnrho[i] * (2.0 / r[i] - c1 * dd / zeta[i] / (r[i] * r[i]));
            R.temperature[i] = T_c * zeta[i];
            R.dlnT[i] = -c1 * dd / (r[i] * r[i]) / zeta[i];
            R.buoy[i] = gravity / cfg.pressure_specific_heat * R.density[i];
            visc_amp[i] = 2.0 / R.temperature[i];
        }
        R.coriolis = 2.0 * cfg.angular_velocity;
        nu_top = cfg.nu_top;
        kappa_top = cfg.kappa_top;
        eta_top = cfg.eta_top;
        R.lorentz = mag ? 1.0 / (4.0 * M_PI) : 0.0;
        for (int i = 0; i < n; ++i) ohm_amp[i] = R.lorentz / R.density[i] / R.temperature[i];
    } else {   // 3: Polytropic_ReferenceND
        const double pn = cfg.poly_n, beta = cfg.aspect_ratio;
        const double diss = beta * (exp(cfg.poly_nrho / pn) - 1.0), dtmp = 1.0 / (1.0 - beta);
        const double rmax = R.rmax;
        for (int i = 0; i < n; ++i) {
            const double gravity = rmax * rmax / (r[i] * r[i]);
            R.temperature[i] = dtmp * diss * (dtmp / r[i] - 1.0) + 1.0;
            R.density[i] = pow(R.temperature[i], pn);
            R.buoy[i] = gravity * cfg.modified_rayleigh * R.density[i];
            R.dlnT[i] = -diss * gravity / R.temperature[i];
            R.dlnrho[i] = pn * R.dlnT[i];
            R.d2lnrho[i] = -pn * R.dlnT[i] * R.dlnT[i] + (pn / R.temperature[i]) * (2.0 * diss * gravity / r[i]);
            visc_amp[i] = 2.0 / R.temperature[i] * diss / cfg.modified_rayleigh;
        }
        R.coriolis = 2.0;
        nu_top = cfg.ekman;
        kappa_top = cfg.ekman / cfg.prandtl;
        R.lorentz = mag ? cfg.ekman / cfg.magnetic_prandtl : 0.0;
        eta_top = mag ? cfg.ekman / cfg.magnetic_prandtl : 0.0;
        const double otmp = diss * cfg.ekman * cfg.ekman /
                            (cfg.modified_rayleigh * cfg.magnetic_prandtl * cfg.magnetic_prandtl);
        for (int i = 0; i < n; ++i) ohm_amp[i] = mag ? otmp / R.density[i] / R.temperature[i] : 0.0;
    }
    R.dpdr_w.resize(n);
    R.pdwdr.resize(n);
    for (int i = 0; i < n; ++i) {
        R.dpdr_w[i] = R.density[i] * pscaling;
        R.pdwdr[i] = -1.0 * R.density[i] * pscaling;
    }
    // Initialize_Diffusivity / Vary_With_Density (:1906-1981)
    auto diffusivity = [&](double top, int type, double power, std::vector<double>& x, std::vector<double>& dlnx) {
        x.assign(n, top);
        dlnx.assign(n, 0.0);
        if (type == 2)
            for (int i = 0; i < n; ++i) {
                x[i] = top * pow(R.density[i] / R.density[0], power);
                dlnx[i] = power * R.dlnrho[i];
            }
    };
    diffusivity(nu_top, cfg.nu_type, cfg.nu_power, R.nu, R.dlnu);
    diffusivity(kappa_top, cfg.kappa_type, cfg.kappa_power, R.kappa, R.dlnkappa);
    if (mag)
        diffusivity(eta_top, cfg.eta_type, cfg.eta_power, R.eta, R.dlneta);
    else {
        R.eta.assign(n, 0.0);
        R.dlneta.assign(n, 0.0);
    }
    // viscous_heating_coeff = viscous_amp nu, ohmic_heating_coeff = ohmic_amp eta (:1822-1836)
    R.visc_heat.assign(n, 0.0);
    R.ohm_heat.assign(n, 0.0);
    for (int i = 0; i < n; ++i) {
        if (visc) R.visc_heat[i] = visc_amp[i] * R.nu[i];
        if (mag && ohm) R.ohm_heat[i] = ohm_amp[i] * R.eta[i];
    }
    R.heating = visc || (mag && ohm);
    // Compute_Diffusion_Coefs (:2032-2098)
    auto sz = [&](std::vector<double>& v) { v.assign(n, 0.0); };
    for (auto* v : {&R.w_diff0, &R.w_diff1, &R.dw_diff0, &R.dw_diff1, &R.dw_diff2, &R.s_diff1, &R.z_diff0,
                    &R.z_diff1, &R.a_diff1})
        sz(*v);
    for (int i = 0; i < n; ++i) {
        const double nu = R.nu[i], dlnu = R.dlnu[i], dlnrho = R.dlnrho[i], d2lnrho = R.d2lnrho[i], ri = r[i];
        R.w_diff0[i] = -nu * (4.0 / 3.0) * (dlnu * dlnrho + d2lnrho + dlnrho / ri + 3.0 * dlnu / ri);
        R.w_diff1[i] = nu * (2.0 * dlnu - dlnrho / 3.0);
        R.dw_diff2[i] = (dlnu - dlnrho) * nu;
        R.dw_diff1[i] = -(d2lnrho + 2.0 / ri * dlnrho + 2.0 / ri * dlnu + dlnu * dlnrho) * nu;
        R.dw_diff0[i] = -(2.0 * dlnrho / 3.0 + dlnu) * nu;
        R.s_diff1[i] = R.kappa[i] * (R.dlnkappa[i] + dlnrho + R.dlnT[i]);
        R.z_diff0[i] = -nu * (2.0 * dlnu / ri + dlnrho * dlnu + d2lnrho + 2.0 * dlnrho / ri);
        R.z_diff1[i] = nu * (dlnu - dlnrho);
        R.a_diff1[i] = R.eta[i] * R.dlneta[i];
    }
}

// The C (poloidal) and A (toroidal) systems of one l > 0 (Sphere_Linear_Terms.F90:473-499)
// with the insulating boundaries (:1041-1077): A = 0 at both; C matched to a potential
// field, dC/dr + l C / r = 0 at the top and dC/dr - (l + 1) C / r = 0 at the bottom.
// coefm[NMSLOT][nr]: the Post_Solve coefficients (C,C,0) (C,C,2) (A,A,0) (A,A,1) (A,A,2).
static void build_l_mag(const Ctx& c, int l, std::vector<double>& Cm, std::vector<double>& Am, double* coefm) {
    const int nr = c.d.nr, rda = c.d.rda;
    const double dt = c.dt, al = c.cfg.alpha_implicit;
    const double lf = -dt * al, rf = dt * (1.0 - al);
    const double* D = c.cheb_D.data();
    const std::vector<double>& r = c.rad.radius;
    const std::vector<double>& eta = c.rad.eta;
    Cm.assign((size_t)nr * nr, 0.0);
    Am.assign((size_t)nr * nr, 0.0);
    std::fill(coefm, coefm + (size_t)NMSLOT * nr, 0.0);
    if (l == 0) return;   // no magnetic equation at l = 0 (Sphere_Linear_Terms.F90:160-163)
    const double llp1 = (double)l * (l + 1);
    auto add = [&](std::vector<double>& M, int slot, int d, int i, double amp, bool stat) {
        if (slot >= 0) coefm[(size_t)slot * nr + i] += stat ? amp : amp * rf;
        const double fac = stat ? 1.0 : lf;
        const double* Dd = D + (size_t)d * nr * nr;
        for (int j = 0; j < nr; ++j) M[(size_t)i * nr + j] += amp * fac * Dd[(size_t)i * nr + j];
    };
    for (int i = 0; i < nr; ++i) {
        const double H = -llp1 / (r[i] * r[i]);
        add(Am, MS_A0, 0, i, 1.0, true);
        add(Am, MS_A0, 0, i, H * eta[i], false);
        add(Am, MS_A2, 2, i, 1.0 * eta[i], false);
        add(Am, MS_A1, 1, i, c.rad.a_diff1[i], false);   // A_Diffusion_Coefs_1
        add(Cm, MS_C0, 0, i, 1.0, true);
        add(Cm, MS_C0, 0, i, H * eta[i], false);
        add(Cm, MS_C2, 2, i, 1.0 * eta[i], false);
    }
    auto clear = [&](std::vector<double>& M, int row) {
        std::fill(M.begin() + (size_t)row * nr, M.begin() + (size_t)(row + 1) * nr, 0.0);
    };
    auto bc = [&](std::vector<double>& M, int row, int d, double amp) {
        const double* Dd = D + (size_t)d * nr * nr;
        for (int j = 0; j < rda - 1; ++j) M[(size_t)row * nr + j] += amp * Dd[(size_t)row * nr + j];
    };
    const int top = 0, bot = nr - 1;
    clear(Cm, top);
    clear(Cm, bot);
    clear(Am, top);
    clear(Am, bot);
    bc(Am, top, 0, 1.0);
    bc(Am, bot, 0, 1.0);
    bc(Cm, top, 1, 1.0);
    bc(Cm, top, 0, l / r[top]);
    bc(Cm, bot, 1, 1.0);
    bc(Cm, bot, 0, -(l + 1) / r[bot]);
}

// Finalize_EMF's radial operator (Sphere_Spectral_Space.F90:436-488, Chebyshev branch) as one
// matrix on the collocation grid: grid -> coefficients (To_Spectral4D) -> d/dr
// (Cheby_Deriv_Buffer_4D) -> dealias -> grid (From_Spectral4D), formed in long double.
static void emf_matrix(const Ctx& c, std::vector<double>& M) {
    const int n = c.d.nr, kc = c.d.kc;
    if (!c.cfg.chebyshev) {   // finite differences: d_by_dx of order 1 (Finalize_EMF's FD branch)
        M.assign(c.cheb_D.begin() + (size_t)n * n, c.cheb_D.begin() + (size_t)2 * n * n);
        return;
    }
    std::vector<long double> T((size_t)n * n), Dr((size_t)n * n, 0.0L);
    // To_Spectral4D: c_k = (2/N) sum_r f(r) cos(k theta_r), theta_r accumulated in double as
    // Gen_Colocation_Points does (Chebyshev_Polynomials.F90:233-244)
    std::vector<long double> th(n);
    const double dth = M_PI / n;
    double a = dth * 0.5;
    for (int i = 0; i < n; ++i) {
        th[i] = a;
        a = a + dth;
    }
    for (int k = 0; k < n; ++k)
        for (int i = 0; i < n; ++i) T[(size_t)k * n + i] = 2.0L / n * cosl(k * th[i]);
    // derivative recursion d_{N-1} = 0, d_{N-2} = 2 (N-1) c_{N-1}, d_i = d_{i+2} + 2 (i+1) c_{i+1}
    for (int k = n - 2; k >= 0; --k) {
        Dr[(size_t)k * n + k + 1] = 2.0L * (k + 1);
        if (k + 2 < n)
            for (int j = 0; j < n; ++j) Dr[(size_t)k * n + j] += Dr[(size_t)(k + 2) * n + j];
    }
    // grid value: sum_{k < kc} d_k cos(k theta_r) - d_0 / 2, times the derivative scaling
    M.assign((size_t)n * n, 0.0);
    std::vector<long double> DT((size_t)n * n, 0.0L);   // (Dr T)[k][i]
    for (int k = 0; k < kc; ++k)
        for (int j = 0; j < n; ++j) {
            const long double dkj = Dr[(size_t)k * n + j];
            if (dkj == 0.0L) continue;
            for (int i = 0; i < n; ++i) DT[(size_t)k * n + i] += dkj * T[(size_t)j * n + i];
        }
    const long double sc = (long double)c.deriv_scaling;
    for (int r = 0; r < n; ++r)
        for (int i = 0; i < n; ++i) {
            long double v = -0.5L * DT[i];
            for (int k = 0; k < kc; ++k) v += DT[(size_t)k * n + i] * cosl(k * th[r]);
            M[(size_t)r * n + i] = (double)(v * sc);
        }
}

// One l of the implicit system: LHS (row-major) and the Post_Solve RHS coefficients.
static void build_l(const Ctx& c, int l, std::vector<double>& A, std::vector<double>& Z, double* coef) {
    const int nr = c.d.nr, n3 = 3 * nr, rda = c.d.rda;
    const ra_config& cfg = c.cfg;
    const Radial& R = c.rad;
    const std::vector<double>& r = R.radius;
    const double dt = c.dt, al = cfg.alpha_implicit;
    const double lf = -dt * al, rf = dt * (1.0 - al);
    const double* D = c.cheb_D.data();
    A.assign((size_t)n3 * n3, 0.0);
    Z.assign((size_t)nr * nr, 0.0);
    std::fill(coef, coef + (size_t)NSLOT * nr, 0.0);
    // slot lookup for (eq, var, d); var/d given as the grid source
    auto slot_of = [&](int eq, int var, int d) -> int {
        static const int gsrc[4][4] = {{G_W0, G_W1, G_W2, G_W3}, {G_P0, G_P1, -1, -1},
                                       {G_T0, G_T1, G_T2, -1}, {G_Z0, G_Z1, G_Z2, -1}};
        const int gs = gsrc[var][d];
        for (int s = 0; s < NSLOT; ++s)
            if (kSlots[s].eq == eq && kSlots[s].g == gs) return s;
        return -1;
    };
    // Add_Implicit_Term: LHS += amp*(static ? 1 : lf)*D_d in rows of eq, columns of var;
    // Post_Solve coefficient += amp*(static ? 1 : rf)
    auto add = [&](int eq, int var, int d, const std::vector<double>& amp, bool stat) {
        const int s = slot_of(eq, var, d);
        if (s >= 0)
            for (int i = 0; i < nr; ++i) coef[(size_t)s * nr + i] += stat ? amp[i] : amp[i] * rf;
        const double fac = stat ? 1.0 : lf;
        const double* Dd = D + (size_t)d * nr * nr;
        if (eq == EQ_Z) {
            for (int i = 0; i < nr; ++i)
                for (int j = 0; j < nr; ++j) Z[(size_t)i * nr + j] += amp[i] * fac * Dd[(size_t)i * nr + j];
        } else {
            const int rb = eq * nr, cb = var * nr;
            for (int i = 0; i < nr; ++i)
                for (int j = 0; j < nr; ++j)
                    A[(size_t)(rb + i) * n3 + cb + j] += amp[i] * fac * Dd[(size_t)i * nr + j];
        }
    };
    std::vector<double> ones(nr, 1.0), v(nr);
    const double llp1 = (double)l * (l + 1);
    std::vector<double> H(nr);
    for (int i = 0; i < nr; ++i) H[i] = -llp1 / (r[i] * r[i]);
    auto vec = [&](auto f) {
        for (int i = 0; i < nr; ++i) v[i] = f(i);
        return v;
    };
    const int W_ = 0, P_ = 1, T_ = 2, Z_ = 3;
    if (l == 0) {
        add(EQ_T, T_, 0, ones, true);
        add(EQ_T, T_, 1, vec([&](int i) { return 2.0 / r[i] * R.kappa[i]; }), false);
        add(EQ_T, T_, 2, vec([&](int i) { return 1.0 * R.kappa[i]; }), false);
        add(EQ_T, T_, 1, R.s_diff1, false);
        add(EQ_P, T_, 0, vec([&](int i) { return -R.buoy[i]; }), true);
        add(EQ_P, P_, 1, R.dpdr_w, true);
        add(EQ_W, W_, 0, ones, true);
    } else {
        add(EQ_W, T_, 0, vec([&](int i) { return -R.buoy[i] / H[i]; }), false);
        add(EQ_W, P_, 1, vec([&](int i) { return R.dpdr_w[i] / H[i]; }), false);
        add(EQ_W, W_, 0, ones, true);
        add(EQ_W, W_, 0, vec([&](int i) { return H[i] * R.nu[i]; }), false);
        add(EQ_W, W_, 2, R.nu, false);
        add(EQ_W, W_, 0, R.w_diff0, false);
        add(EQ_W, W_, 1, R.w_diff1, false);
        add(EQ_P, P_, 0, R.pdwdr, false);
        add(EQ_P, W_, 1, ones, true);
        add(EQ_P, W_, 0, vec([&](int i) { return -R.nu[i] * H[i] * 2.0 / r[i]; }), false);
        add(EQ_P, W_, 1, vec([&](int i) { return H[i] * R.nu[i]; }), false);
        add(EQ_P, W_, 3, R.nu, false);
        add(EQ_P, W_, 0, vec([&](int i) { return R.dw_diff0[i] * H[i]; }), false);
        add(EQ_P, W_, 1, R.dw_diff1, false);
        add(EQ_P, W_, 2, R.dw_diff2, false);
        add(EQ_T, T_, 0, ones, true);
        add(EQ_T, T_, 0, vec([&](int i) { return H[i] * R.kappa[i]; }), false);
        add(EQ_T, T_, 1, vec([&](int i) { return 2.0 / r[i] * R.kappa[i]; }), false);
        add(EQ_T, T_, 2, R.kappa, false);
        add(EQ_T, T_, 1, R.s_diff1, false);
        add(EQ_Z, Z_, 0, ones, true);
        add(EQ_Z, Z_, 0, vec([&](int i) { return H[i] * R.nu[i]; }), false);
        add(EQ_Z, Z_, 2, R.nu, false);
        add(EQ_Z, Z_, 0, R.z_diff0, false);
        add(EQ_Z, Z_, 1, R.z_diff1, false);
    }
    // Set_Boundary_Conditions (Sphere_Linear_Terms.F90:539-1100):
    // clear boundary rows, then Load_Single_Row_Cheby over the dealiased columns
    auto clear = [&](std::vector<double>& M, int ncols, int row) {
        std::fill(M.begin() + (size_t)row * ncols, M.begin() + (size_t)(row + 1) * ncols, 0.0);
    };
    auto bc = [&](std::vector<double>& M, int ncols, int row, int col0, int d, double amp) {
        const double* Dd = D + (size_t)d * nr * nr;
        const int rr = row % nr;
        for (int j = 0; j < rda - 1; ++j) M[(size_t)row * ncols + col0 + j] += amp * Dd[(size_t)rr * nr + j];
    };
    const int top = 0, bot = nr - 1;
    if (l == 0) {
        clear(A, n3, nr + top);
        clear(A, n3, 2 * nr + top);
        clear(A, n3, 2 * nr + bot);
        bc(A, n3, 2 * nr + top, 2 * nr, cfg.fix_tvar_top ? 0 : 1, 1.0);
        bc(A, n3, 2 * nr + bot, 2 * nr, cfg.fix_tvar_bottom ? 0 : 1, 1.0);
        bc(A, n3, nr + top, nr, 0, 1.0);   // pressure node at the top
    } else {
        for (int rb = 0; rb < n3; rb += nr) {
            clear(A, n3, rb + top);
            clear(A, n3, rb + bot);
        }
        clear(Z, nr, top);
        clear(Z, nr, bot);
        bc(A, n3, 2 * nr + top, 2 * nr, cfg.fix_tvar_top ? 0 : 1, 1.0);
        bc(A, n3, 2 * nr + bot, 2 * nr, cfg.fix_tvar_bottom ? 0 : 1, 1.0);
        bc(A, n3, top, 0, 0, 1.0);   // impenetrable: W = 0
        bc(A, n3, bot, 0, 0, 1.0);
        if (cfg.no_slip_top) {
            bc(Z, nr, top, 0, 0, 1.0);
            bc(A, n3, nr + top, 0, 1, 1.0);
        } else {
            const double samp = -(2.0 / r[top] + R.dlnrho[top]);
            bc(A, n3, nr + top, 0, 2, 1.0);
            bc(A, n3, nr + top, 0, 1, samp);
            bc(Z, nr, top, 0, 1, 1.0);
            bc(Z, nr, top, 0, 0, samp);
        }
        if (cfg.no_slip_bottom) {
            bc(A, n3, nr + bot, 0, 1, 1.0);
            bc(Z, nr, bot, 0, 0, 1.0);
        } else {
            const double samp = -(2.0 / r[bot] + R.dlnrho[bot]);
            bc(A, n3, nr + bot, 0, 2, 1.0);
            bc(A, n3, nr + bot, 0, 1, samp);
            bc(Z, nr, bot, 0, 1, 1.0);
            bc(Z, nr, bot, 0, 0, samp);
        }
    }
}

// Reset_Linear_Equations: build every l, upload, invert on the device.
static void linear_setup(Ctx& c) {
    const int L = c.d.L, nr = c.d.nr, n3 = 3 * nr;
    std::vector<double> coef((size_t)L * NSLOT * nr);
    std::vector<double> Aall((size_t)L * n3 * n3), Zall((size_t)L * nr * nr);
    std::vector<double> A, Z;
    for (int l = 0; l < L; ++l) {
        build_l(c, l, A, Z, coef.data() + (size_t)l * NSLOT * nr);
        std::copy(A.begin(), A.end(), Aall.begin() + (size_t)l * n3 * n3);
        std::copy(Z.begin(), Z.end(), Zall.begin() + (size_t)l * nr * nr);
    }
    RA_CUDA(cudaMemcpyAsync(c.d_coef, coef.data(), coef.size() * sizeof(double), cudaMemcpyHostToDevice, c.stream));
    RA_CUDA(cudaMemcpyAsync(c.d_Awpt, Aall.data(), Aall.size() * sizeof(double), cudaMemcpyHostToDevice, c.stream));
    RA_CUDA(cudaMemcpyAsync(c.d_Az, Zall.data(), Zall.size() * sizeof(double), cudaMemcpyHostToDevice, c.stream));
    if (c.mag) {
        std::vector<double> cm((size_t)L * NMSLOT * nr), Call((size_t)L * nr * nr), Aall2((size_t)L * nr * nr);
        std::vector<double> Cm, Am;
        for (int l = 0; l < L; ++l) {
            build_l_mag(c, l, Cm, Am, cm.data() + (size_t)l * NMSLOT * nr);
            std::copy(Cm.begin(), Cm.end(), Call.begin() + (size_t)l * nr * nr);
            std::copy(Am.begin(), Am.end(), Aall2.begin() + (size_t)l * nr * nr);
        }
        RA_CUDA(cudaMemcpyAsync(c.d_coef_mag, cm.data(), cm.size() * sizeof(double), cudaMemcpyHostToDevice, c.stream));
        RA_CUDA(cudaMemcpyAsync(c.d_Ac, Call.data(), Call.size() * sizeof(double), cudaMemcpyHostToDevice, c.stream));
        RA_CUDA(cudaMemcpyAsync(c.d_Aa, Aall2.data(), Aall2.size() * sizeof(double), cudaMemcpyHostToDevice, c.stream));
        RA_CUDA(cudaStreamSynchronize(c.stream));   // the host vectors go out of scope
    }
    factor_matrices(c);
}

// The packed radial profiles the kernels read (R_* rows of n_r): the grid, the reference
// density and its log-derivative with rlm_spacea's over_rhor, over_rhorsq and drho_term
// (Sphere_Hybrid_Space.F90:44-62), and the heating coefficients.
static std::vector<double> radial_table(const Ctx& c) {
    const int nr = c.d.nr;
    std::vector<double> rp((size_t)R_COUNT * nr);
    for (int i = 0; i < nr; ++i) {
        const double r = c.rad.radius[i];
        const double oor = 1.0 / r;
        const double oor2 = 1.0 / (r * r);
        rp[R_RADIUS * nr + i] = r;
        rp[R_OVER_R * nr + i] = oor;
        rp[R_DELTA_R * nr + i] = c.rad.delta_r[i];
        rp[R_DENSITY * nr + i] = c.rad.density[i];
        rp[R_DLNRHO * nr + i] = c.rad.dlnrho[i];
        rp[R_OVER_RHOR * nr + i] = oor / c.rad.density[i];
        rp[R_OVER_RHORSQ * nr + i] = oor2 / c.rad.density[i];
        rp[R_DRHO_TERM * nr + i] = c.rad.dlnrho[i] + oor;
        rp[R_TWO_OVER_R * nr + i] = 2.0 / r;
        rp[R_OVER_RSQ * nr + i] = oor2;
        rp[R_VISC_HEAT * nr + i] = c.rad.visc_heat[i];
        rp[R_OHM_HEAT * nr + i] = c.rad.ohm_heat[i];
        rp[R_RHO_T * nr + i] = c.rad.density[i] * c.rad.temperature[i];
    }
    return rp;
}

template <class T>
static void dalloc(T*& p, size_t count) {
    cudaError_t e = cudaMalloc(&p, count * sizeof(T));
    if (e != cudaSuccess) throw CudaError(e, "cudaMalloc", __FILE__, __LINE__);
}

static void autotune(Ctx& c, int nreps, double* ms_out);

static void setup(Ctx& c) {
    const Dims& d = c.d;
    c.mag = c.cfg.magnetism != 0;
    c.mixed_solve = c.cfg.precision == RA_PREC_MIXED && c.cfg.reference_type != 2 && c.cfg.chebyshev;
    c.nfa = c.mag ? (int)NP2A_MAG : (int)NP2A;
    c.nfb = c.mag ? (int)NP2B_MAG : (int)NP2B;
    c.ng = c.mag ? (int)NG_MAG : (int)NG;
    RA_CUDA(cudaSetDevice(c.cfg.device));
    RA_CUDA(cudaStreamCreateWithFlags(&c.stream, cudaStreamNonBlocking));
    c.dt = c.cfg.dt;
    c.old_dt = c.cfg.dt;
    const double rmax = c.cfg.shell_depth / (1.0 - c.cfg.aspect_ratio);
    const double rmin = rmax * c.cfg.aspect_ratio;
    radial_setup(c, rmin, rmax);
    reference_setup(c);
    // horizontal grid
    std::vector<long double> xq, wq;
    gauss_legendre(d.nth, xq, wq);
    c.costheta_h.resize(d.nth);
    for (int i = 0; i < d.nth; ++i) c.costheta_h[i] = (double)xq[i];
    // [x hi | x lo | s hi | s lo] and [2 pi w hi | lo] for the table recurrence (double-double)
    std::vector<double> xs(4 * (size_t)d.nth2), w2(2 * (size_t)d.nth2);
    const long double PI = 3.141592653589793238462643383279502884L;
    for (int i = 0; i < d.nth2; ++i) {
        const long double x = xq[i], sn = sqrtl((1.0L - xq[i]) * (1.0L + xq[i])), w = 2.0L * PI * wq[i];
        xs[i] = (double)x;
        xs[d.nth2 + i] = (double)(x - (long double)xs[i]);
        xs[2 * d.nth2 + i] = (double)sn;
        xs[3 * d.nth2 + i] = (double)(sn - (long double)xs[2 * d.nth2 + i]);
        w2[i] = (double)w;
        w2[d.nth2 + i] = (double)(w - (long double)w2[i]);
    }
    // trig tables as the reference computes them in double (ProblemSize.F90:489-495)
    std::vector<double> trig(4 * (size_t)d.nth);
    for (int i = 0; i < d.nth; ++i) {
        const double ct = c.costheta_h[i];
        const double s2 = 1.0 - ct * ct;
        const double st = sqrt(s2);
        trig[i] = ct;
        trig[d.nth + i] = st;
        trig[2 * d.nth + i] = 1.0 / st;
        trig[3 * d.nth + i] = ct / st;
    }
    std::vector<double> twid(2 * (size_t)d.nth);
    for (int k = 0; k < d.nth; ++k) {
        const long double a = 2.0L * PI * k / (long double)d.nphi;
        twid[2 * k] = (double)cosl(a);
        twid[2 * k + 1] = (double)sinl(a);
    }
    // weights of the kinetic-energy diagnostic: theta (Gauss-Legendre / 2 / n_phi), then radius
    std::vector<double> kew((size_t)d.nth + d.nr);
    for (int i = 0; i < d.nth; ++i) kew[i] = (double)(wq[i] / 2.0L) / d.nphi;
    for (int i = 0; i < d.nr; ++i) kew[d.nth + i] = c.rad.int_w[i];
    // radial profiles
    const int nr = d.nr;
    const std::vector<double> rp = radial_table(c);
    // device buffers
    const long nlm = d.nlm;
    dalloc(c.d_Ptab, (size_t)nlm * d.nth2);
    dalloc(c.d_iPtab, (size_t)nlm * d.nth2);
    dalloc(c.d_D, c.cheb_D.size());
    dalloc(c.d_coef, (size_t)d.L * NSLOT * nr);
    dalloc(c.d_radial, rp.size());
    dalloc(c.d_costh, trig.size());
    dalloc(c.d_twid, twid.size());
    dalloc(c.d_Awpt, (size_t)d.L * 9 * nr * nr);
    dalloc(c.d_Az, (size_t)d.L * nr * nr);
    dalloc(c.d_perm_wpt, (size_t)d.L * 3 * nr);
    dalloc(c.d_perm_z, (size_t)d.L * nr);
    dalloc(c.d_skip_z, (size_t)d.L);
    {
        std::vector<int> skip(d.L, 0);
        skip[0] = 1;   // Z is not solved for at l = 0 (Sphere_Linear_Terms.F90:116-150)
        RA_CUDA(cudaMemcpyAsync(c.d_skip_z, skip.data(), skip.size() * sizeof(int), cudaMemcpyHostToDevice, c.stream));
        RA_CUDA(cudaStreamSynchronize(c.stream));
    }
    if (c.mixed_solve) {
        dalloc(c.d_Ainv_wpt, (size_t)d.L * 9 * nr * nr);
        dalloc(c.d_Ainv_z, (size_t)d.L * nr * nr);
    }
    dalloc(c.d_sol_wpt, (size_t)nlm * 2 * 3 * nr);
    dalloc(c.d_sol_z, (size_t)nlm * 2 * nr);
    dalloc(c.d_rhs_wpt, (size_t)nlm * 2 * 3 * nr);
    dalloc(c.d_rhs_z, (size_t)nlm * 2 * nr);
    const int nab = c.mag ? 6 : 4;   // AB history: W P T Z (C A)
    dalloc(c.d_ab, (size_t)nab * nlm * 2 * nr);
    // grids; the finite-difference mode adds the deriv_cluge plane behind them
    dalloc(c.d_g, (size_t)(c.ng + (c.cfg.chebyshev ? 0 : 1)) * nlm * 2 * nr);
    dalloc(c.d_s2a, (size_t)nlm * NS2A * 2 * nr);
    dalloc(c.d_s2a11, (size_t)nlm * c.nfa * 2 * nr);
    dalloc(c.d_p2a, (size_t)d.L * d.nth * c.nfa * 2 * nr);
    dalloc(c.d_p2b, (size_t)d.L * d.nth * c.nfb * 2 * nr);
    dalloc(c.d_s2b, (size_t)nlm * c.nfb * 2 * nr);
    if (c.mag) {
        const size_t plane = (size_t)nlm * 2 * nr;
        dalloc(c.d_sol_c, plane);
        dalloc(c.d_sol_a, plane);
        dalloc(c.d_rhs_c, plane);
        dalloc(c.d_rhs_a, plane);
        dalloc(c.d_xemf, plane);
        dalloc(c.d_s2am, (size_t)nlm * NS2AM * 2 * nr);
        dalloc(c.d_Ac, (size_t)d.L * nr * nr);
        dalloc(c.d_Aa, (size_t)d.L * nr * nr);
        if (c.mixed_solve) {
            dalloc(c.d_Ainv_c, (size_t)d.L * nr * nr);
            dalloc(c.d_Ainv_a, (size_t)d.L * nr * nr);
        }
        dalloc(c.d_perm_c, (size_t)d.L * nr);
        dalloc(c.d_perm_a, (size_t)d.L * nr);
        dalloc(c.d_coef_mag, (size_t)d.L * NMSLOT * nr);
        std::vector<double> M;
        emf_matrix(c, M);
        dalloc(c.d_Memf, M.size());
        RA_CUDA(cudaMemcpyAsync(c.d_Memf, M.data(), M.size() * sizeof(double), cudaMemcpyHostToDevice, c.stream));
        RA_CUDA(cudaMemsetAsync(c.d_sol_c, 0, plane * sizeof(double), c.stream));
        RA_CUDA(cudaMemsetAsync(c.d_sol_a, 0, plane * sizeof(double), c.stream));
        RA_CUDA(cudaStreamSynchronize(c.stream));
    }
    dalloc(c.d_cfl, 1);
    dalloc(c.d_status, 1);
    RA_CUDA(cudaMemsetAsync(c.d_status, 0, sizeof(int), c.stream));
    dalloc(c.d_kew, kew.size());
    {
        const std::vector<double> kaz((size_t)d.nth, 1.0 / d.nphi);
        dalloc(c.d_kaz, kaz.size());
        RA_CUDA(cudaMemcpyAsync(c.d_kaz, kaz.data(), kaz.size() * sizeof(double), cudaMemcpyHostToDevice, c.stream));
        RA_CUDA(cudaStreamSynchronize(c.stream));
    }
    dalloc(c.d_ke_rows, (size_t)d.nth * nr + 1);
    RA_CUDA(cudaMemcpyAsync(c.d_kew, kew.data(), kew.size() * sizeof(double), cudaMemcpyHostToDevice, c.stream));
    RA_CUDA(cudaMemsetAsync(c.d_ab, 0, (size_t)nab * nlm * 2 * nr * sizeof(double), c.stream));
    RA_CUDA(cudaMemsetAsync(c.d_sol_wpt, 0, (size_t)nlm * 2 * 3 * nr * sizeof(double), c.stream));
    RA_CUDA(cudaMemsetAsync(c.d_sol_z, 0, (size_t)nlm * 2 * nr * sizeof(double), c.stream));
    RA_CUDA(cudaMemcpyAsync(c.d_D, c.cheb_D.data(), c.cheb_D.size() * sizeof(double), cudaMemcpyHostToDevice, c.stream));
    {
        // parity planes of the synthesis matrices: Dpar[d][par][r][k'] = D_d(r, 2k' + par), r < nr/2, 2k'+par < kc
        const int nr2 = nr / 2, kh = (d.kc + 1) / 2;
        std::vector<double> dp((size_t)4 * 2 * nr2 * kh, 0.0);
        for (int dd = 0; dd < 4; ++dd)
            for (int par = 0; par < 2; ++par)
                for (int r = 0; r < nr2; ++r)
                    for (int k = 0; k < kh; ++k)
                        if (2 * k + par < d.kc)
                            dp[(((size_t)dd * 2 + par) * nr2 + r) * kh + k] =
                                c.cheb_D[((size_t)dd * nr + r) * nr + 2 * k + par];
        dalloc(c.d_Dpar, dp.size());
        RA_CUDA(cudaMemcpyAsync(c.d_Dpar, dp.data(), dp.size() * sizeof(double), cudaMemcpyHostToDevice, c.stream));
        RA_CUDA(cudaStreamSynchronize(c.stream));
    }
    if (!c.cfg.chebyshev) {
        // the finite-difference synthesis operators [I, D_1, D_2, D_3, D_1 D_1] as bands: each row's
        // nonzero stencil (Generate_Coefs' 5 points, one-sided at the ends; 9 for D_1 D_1) held as
        // its first column and fd_w coefficients, the first column moved left near the bottom
        // boundary so that the fd_w columns stay on the grid (the extra coefficients are zeros)
        const size_t nn = (size_t)nr * nr;
        std::vector<double> fdm(5 * nn, 0.0);
        std::copy(c.cheb_D.begin(), c.cheb_D.begin() + 4 * nn, fdm.begin());
        const double* D1 = c.cheb_D.data() + nn;
        for (int i = 0; i < nr; ++i)
            for (int j = 0; j < nr; ++j) {
                long double sum = 0.0L;
                for (int k = 0; k < nr; ++k) sum += (long double)D1[(size_t)i * nr + k] * D1[(size_t)k * nr + j];
                fdm[4 * nn + (size_t)i * nr + j] = (double)sum;
            }
        std::vector<int> lo(5 * (size_t)nr), hi(5 * (size_t)nr);
        int w = 1;
        for (size_t row = 0; row < 5 * (size_t)nr; ++row) {
            const double* m = fdm.data() + row * nr;
            int a = 0, b = -1;
            for (int j = 0; j < nr; ++j)
                if (m[j] != 0.0) {
                    if (b < 0) a = j;
                    b = j;
                }
            if (b < 0) a = b = 0;
            lo[row] = a;
            hi[row] = b;
            w = std::max(w, b - a + 1);
        }
        if (w > 16) throw ArgError("finite differences: a stencil wider than 16 points");
        c.fd_w = w;
        std::vector<double> band(5 * (size_t)nr * (w + 1), 0.0);
        for (size_t row = 0; row < 5 * (size_t)nr; ++row) {
            const int first = std::min(lo[row], nr - w);
            double* o = band.data() + row * (w + 1);
            o[0] = first;
            for (int j = lo[row]; j <= hi[row]; ++j) o[1 + j - first] = fdm[row * nr + j];
        }
        dalloc(c.d_Dfd, band.size());
        RA_CUDA(cudaMemcpyAsync(c.d_Dfd, band.data(), band.size() * sizeof(double), cudaMemcpyHostToDevice, c.stream));
        RA_CUDA(cudaStreamSynchronize(c.stream));
    }
    RA_CUDA(cudaMemcpyAsync(c.d_radial, rp.data(), rp.size() * sizeof(double), cudaMemcpyHostToDevice, c.stream));
    RA_CUDA(cudaMemcpyAsync(c.d_costh, trig.data(), trig.size() * sizeof(double), cudaMemcpyHostToDevice, c.stream));
    RA_CUDA(cudaMemcpyAsync(c.d_twid, twid.data(), twid.size() * sizeof(double), cudaMemcpyHostToDevice, c.stream));
    double *d_x = nullptr, *d_w = nullptr;
    dalloc(d_x, xs.size());
    dalloc(d_w, w2.size());
    RA_CUDA(cudaMemcpyAsync(d_x, xs.data(), xs.size() * sizeof(double), cudaMemcpyHostToDevice, c.stream));
    RA_CUDA(cudaMemcpyAsync(d_w, w2.data(), w2.size() * sizeof(double), cudaMemcpyHostToDevice, c.stream));
    launch_plm(c, d_x, d_w);
    RA_CUDA(cudaStreamSynchronize(c.stream));
    cudaFree(d_x);
    cudaFree(d_w);
    solve_prepare(c);
    linear_setup(c);
    physics_prepare(c);
    lt_forward_prepare(c);
    if (c.cfg.precision == RA_PREC_MIXED) mixed_setup(c);
    if (c.cfg.autotune) autotune(c, 3, nullptr);
}

static void release(Ctx& c) {
    mixed_release(c);
    if (c.graph_exec) cudaGraphExecDestroy(c.graph_exec);
    if (c.graph) cudaGraphDestroy(c.graph);
    if (c.adapt_exec) cudaGraphExecDestroy(c.adapt_exec);
    if (c.adapt_graph) cudaGraphDestroy(c.adapt_graph);
    if (c.d_adapt) cudaFree(c.d_adapt);
    if (c.d_adapt_dt) cudaFree(c.d_adapt_dt);
    lu_workspace_free(c.lu_work);
    double* bufs[] = {c.d_Ptab, c.d_iPtab, c.d_D, c.d_Dpar, c.d_Dfd, c.d_coef, c.d_radial, c.d_costh, c.d_twid, c.d_twp,
                      c.d_Awpt, c.d_Az,
                      c.d_Ainv_wpt, c.d_Ainv_z,
                      c.d_sol_wpt, c.d_sol_z, c.d_rhs_wpt, c.d_rhs_z, c.d_ab, c.d_g, c.d_s2a, c.d_s2a11,
                      c.d_p2a, c.d_p2b, c.d_s2b, c.d_kew, c.d_ke_rows, c.d_kaz, c.d_bcval,
                      c.d_sol_c, c.d_sol_a, c.d_rhs_c, c.d_rhs_a, c.d_Ac, c.d_Aa, c.d_coef_mag, c.d_s2am,
                      c.d_xemf, c.d_Memf, c.d_Ainv_c, c.d_Ainv_a};
    for (double* b : bufs)
        if (b) cudaFree(b);
    int* ibufs[] = {c.d_ltiles, c.d_inv_tiles, c.d_fwd_tiles, c.d_cheb_tiles, c.d_solve_tiles, c.d_status,
                    c.d_perm_wpt, c.d_perm_z, c.d_skip_z, c.d_inv_sol_tiles, c.d_inv_sol_tiles_z,
                    c.d_solve_tiles_z, c.d_perm_c, c.d_perm_a};
    for (int* b : ibufs)
        if (b) cudaFree(b);
    if (c.d_cfl) cudaFree(c.d_cfl);
    if (c.stream) cudaStreamDestroy(c.stream);
}

// AB2 factors (Sphere_Spectral_Space.F90:204-211)
static void ab_factors(const Ctx& c, double& new_ab, double& old_ab) {
    if (c.iteration == 1) {
        new_ab = c.dt;
        old_ab = 0.0;
    } else {
        new_ab = 0.5 * c.dt * (2.0 + c.dt / c.old_dt);
        old_ab = -0.5 * c.dt * c.dt / c.old_dt;
    }
}

// The eight stages of one step, in launch order (their names: kKernelNames).
constexpr int kNK = 8;
static void run_stage(Ctx& c, int k, double new_ab, double old_ab) {
    const bool mixed = c.cfg.precision == RA_PREC_MIXED;
    switch (k) {
        case 0: launch_cheb_synthesis(c); break;
        case 1:
            launch_post_assemble(c, old_ab);
            if (c.mag) launch_post_assemble_mag(c, old_ab);
            break;
        case 2:
            launch_rlm_a(c);   // with the magnetic fields when c.mag
            break;
        case 3:
            if (mixed)
                launch_lt_inverse_mixed(c);
            else
                launch_lt_inverse(c, c.d_s2a11, c.d_p2a, c.nfa * c.d.nr * 2);
            break;
        case 4:
            RA_CUDA(cudaMemsetAsync(c.d_cfl, 0, sizeof(unsigned long long), c.stream));
            launch_physics(c);
            break;
        case 5:
            if (mixed)
                launch_lt_forward_mixed(c);
            else
                launch_lt_forward(c, c.d_p2b, c.d_s2b, c.nfb * c.d.nr * 2);
            break;
        case 6:
            launch_rlm_b(c, new_ab);
            if (c.mag) launch_rlm_b_mag(c, new_ab);
            break;
        default:
            if (c.mixed_solve) {
                launch_solve_mixed(c);   // every system, C and A included
            } else {
                launch_solve(c);
                if (c.mag) launch_solve_mag(c);
            }
            break;
    }
}

static void enqueue_step(Ctx& c, double new_ab, double old_ab) {
    for (int k = 0; k < kNK; ++k) run_stage(c, k, new_ab, old_ab);
}

// the device error word: bounded tensor-core waits of the split-precision
// products, and non-finite values reaching the implicit solve's right-hand side
static void check_status(Ctx& c) {
    if (!c.d_status) return;
    int st = 0;
    RA_CUDA(cudaMemcpyAsync(&st, c.d_status, sizeof(int), cudaMemcpyDeviceToHost, c.stream));
    RA_CUDA(cudaStreamSynchronize(c.stream));
    if (st & RA_STATUS_TIMEOUT)
        throw CudaError(cudaErrorLaunchTimeout, "split-precision product (pipeline barrier wait timed out)", __FILE__,
                        __LINE__);
    if (st & RA_STATUS_NONFINITE)
        throw NonFiniteError("a NaN or Inf reached the right-hand side of the implicit solve (iteration " +
                             std::to_string(c.iteration - 1) + " or earlier); put a finite state to continue");
}

__global__ void nonfinite_scan_kernel(const double* __restrict__ x, long n, int* __restrict__ flag) {
    bool bad = false;
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
        bad |= !isfinite(x[i]);
    if (__syncthreads_or(bad) && threadIdx.x == 0) atomicOr(flag, RA_STATUS_NONFINITE);
}

static void scan_nonfinite(Ctx& c, const double* d_x, long n) {
    nonfinite_scan_kernel<<<1184, 256, 0, c.stream>>>(d_x, n, c.d_status);
    RA_CUDA(cudaGetLastError());
}

// Adjust_TimeStep (Sphere_Hybrid_Space.F90:604-649): cfl = the largest squared inverse crossing
// time of the step (the CFL cargo); the new dt applies from the next step.  The same arithmetic
// on the host (ra_next_dt) and in the adaptive step graph (dt_control_kernel).
__host__ __device__ inline double next_dt_value(const ra_dt_controls& ctl, double dt, double cfl) {
    double nd = dt;
    if (cfl > 0.0) {
        const double maxt = 1.0 / sqrt(cfl);
        if (dt < maxt * ctl.cflmin) {
            nd = fmin(ctl.cflmax * maxt, ctl.max_time_step);
        } else if (dt > maxt * ctl.cflmax) {
            nd = ctl.cflmax * maxt;
            if (nd > dt * (1.0 - ctl.min_dt_change)) nd = dt * (1.0 - ctl.min_dt_change);
        }
    }
    if (nd > ctl.max_time_step * 1.000001) nd = ctl.max_time_step;
    return nd;
}

// The last node of the adaptive loop's body: the next dt from this step's CFL cargo; the loop
// goes on while dt stays, the wanted count is not reached and no error was raised.
__global__ void dt_control_kernel(const unsigned long long* __restrict__ cfl_bits, int* ad, double* adt,
                                  const int* __restrict__ status, ra_dt_controls ctl, cudaGraphConditionalHandle h) {
    if (threadIdx.x != 0) return;
    const double cfl = __longlong_as_double((long long)*cfl_bits);
    const double dt = adt[0];
    const double nd = next_dt_value(ctl, dt, cfl);
    const int done = ad[0] + 1;
    ad[0] = done;
    adt[1] = nd;
    adt[2] = cfl;
    const int changed = nd != dt;
    ad[2] = changed;
    const bool go = !changed && done < ad[1] && !(nd < ctl.min_time_step) && *status == 0;
    cudaGraphSetConditional(h, go ? 1u : 0u);
}

static void enqueue_step(Ctx& c, double new_ab, double old_ab);

// The adaptive loop's graph for the steady step (AB2 factors of equal dt): a conditional WHILE
// node whose body is the step's kernels and dt_control_kernel, captured once per (dt, controls).
static void adaptive_graph(Ctx& c, const ra_dt_controls& ctl, double new_ab, double old_ab) {
    if (c.adapt_exec && !std::memcmp(&c.adapt_ctl, &ctl, sizeof(ctl)) && c.adapt_new_ab == new_ab &&
        c.adapt_old_ab == old_ab)
        return;
    if (c.adapt_exec) cudaGraphExecDestroy(c.adapt_exec);
    if (c.adapt_graph) cudaGraphDestroy(c.adapt_graph);
    c.adapt_exec = nullptr;
    c.adapt_graph = nullptr;
    if (!c.d_adapt) {
        RA_CUDA(cudaMalloc(&c.d_adapt, 4 * sizeof(int)));
        RA_CUDA(cudaMalloc(&c.d_adapt_dt, 3 * sizeof(double)));
    }
    cudaGraph_t g = nullptr;
    RA_CUDA(cudaGraphCreate(&g, 0));
    c.adapt_graph = g;
    cudaGraphConditionalHandle h;
    RA_CUDA(cudaGraphConditionalHandleCreate(&h, g, 1, cudaGraphCondAssignDefault));
    cudaGraphNodeParams p{};
    p.type = cudaGraphNodeTypeConditional;
    p.conditional.handle = h;
    p.conditional.type = cudaGraphCondTypeWhile;
    p.conditional.size = 1;
    cudaGraphNode_t node;
    RA_CUDA(cudaGraphAddNode(&node, g, nullptr, 0, &p));
    cudaGraph_t body = p.conditional.phGraph_out[0];
    const long before = c.launches;
    RA_CUDA(cudaStreamBeginCaptureToGraph(c.stream, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    enqueue_step(c, new_ab, old_ab);
    dt_control_kernel<<<1, 32, 0, c.stream>>>(c.d_cfl, c.d_adapt, c.d_adapt_dt, c.d_status, ctl, h);
    RA_CUDA(cudaGetLastError());
    RA_CUDA(cudaStreamEndCapture(c.stream, &body));
    c.adapt_launches = c.launches - before + 1;
    c.launches = before;
    RA_CUDA(cudaGraphInstantiate(&c.adapt_exec, g, 0));
    c.adapt_ctl = ctl;
    c.adapt_new_ab = new_ab;
    c.adapt_old_ab = old_ab;
}

static void run_steps(Ctx& c, int nsteps, double* cfl, bool check = true) {
    if (!c.have_state) throw ArgError("ra_put_state must be called before stepping");
    for (int s = 0; s < nsteps; ++s) {
        double new_ab, old_ab;
        ab_factors(c, new_ab, old_ab);
        const bool graphable = c.cfg.use_graph && c.iteration > 1;
        if (graphable) {
            if (c.graph_exec && (c.graph_new_ab != new_ab || c.graph_old_ab != old_ab)) {
                cudaGraphExecDestroy(c.graph_exec);
                cudaGraphDestroy(c.graph);
                c.graph_exec = nullptr;
                c.graph = nullptr;
            }
            if (!c.graph_exec) {
                const long before = c.launches;
                RA_CUDA(cudaStreamBeginCapture(c.stream, cudaStreamCaptureModeThreadLocal));
                enqueue_step(c, new_ab, old_ab);
                RA_CUDA(cudaStreamEndCapture(c.stream, &c.graph));
                RA_CUDA(cudaGraphInstantiate(&c.graph_exec, c.graph, 0));
                c.graph_new_ab = new_ab;
                c.graph_old_ab = old_ab;
                c.graph_launches = c.launches - before;
                c.launches = before;
            }
            RA_CUDA(cudaGraphLaunch(c.graph_exec, c.stream));
            c.launches += c.graph_launches;
        } else {
            enqueue_step(c, new_ab, old_ab);
        }
        c.old_dt = c.dt;
        ++c.iteration;
    }
    if (check) check_status(c);
    if (cfl) {
        unsigned long long bits = 0;
        RA_CUDA(cudaMemcpyAsync(&bits, c.d_cfl, sizeof(bits), cudaMemcpyDeviceToHost, c.stream));
        RA_CUDA(cudaStreamSynchronize(c.stream));
        double v;
        std::memcpy(&v, &bits, sizeof(v));
        *cfl = v;
    }
}

// Rank-local state exchange: the modes of one slice (a rank's (l, m) list,
// Load_Balance.F90:357-368) between the slice's own arrays (mode index
// slowest, the reference's equation_set rhs(N_r nlinks, 2, my_num_lm)) and
// the device state ([lm][re/im][k], lm = l (l + 1) / 2 + m).
__global__ void modes_scatter_kernel(const double* __restrict__ src, double* __restrict__ dst,
                                     const long* __restrict__ lm_of, int nmodes, int k, long state_plane,
                                     long slice_plane, int nplanes, int to_device) {
    const long total = (long)nplanes * nmodes * 2 * k;
    for (long e = (long)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (long)gridDim.x * blockDim.x) {
        const int i = (int)(e % (2L * k));
        const long rest = e / (2L * k);
        const int md = (int)(rest % nmodes);
        const int pl = (int)(rest / nmodes);
        const long so = pl * slice_plane + (long)md * 2 * k + i;
        const long dof = pl * state_plane + lm_of[md] * 2 * k + i;
        if (to_device)
            dst[dof] = src[so];   // src: the slice, dst: the state
        else
            dst[so] = src[dof];   // src: the state, dst: the slice
    }
}

// Batched transpose: out[b][i][j] = in[b][j][i] (n x n blocks), for the
// reference's column-major per-l matrices.
__global__ void transpose_batch_kernel(const double* __restrict__ in, double* __restrict__ out, int n) {
    __shared__ double tile[32][33];
    const size_t b = blockIdx.z;
    const int i0 = blockIdx.y * 32, j0 = blockIdx.x * 32;
    const double* src = in + b * n * n;
    double* dst = out + b * n * n;
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
        const int j = j0 + r, i = i0 + threadIdx.x;
        if (j < n && i < n) tile[r][threadIdx.x] = src[(size_t)j * n + i];
    }
    __syncthreads();
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
        const int i = i0 + r, j = j0 + threadIdx.x;
        if (i < n && j < n) dst[(size_t)i * n + j] = tile[threadIdx.x][r];
    }
}

static void scatter_launch(Ctx& c, const double* src, double* dst, const long* d_lm, int nmodes, int k,
                           long state_plane, long slice_plane, int np, bool to_device) {
    modes_scatter_kernel<<<1184, 256, 0, c.stream>>>(src, dst, d_lm, nmodes, k, state_plane, slice_plane, np,
                                                     to_device ? 1 : 0);
    RA_CUDA(cudaGetLastError());
}

static std::vector<long> mode_indices(const Ctx& c, int nmodes, const int* l_of, const int* m_of) {
    if (nmodes <= 0 || !l_of || !m_of) throw ArgError("a mode list needs nmodes > 0 and l, m arrays");
    std::vector<long> lm(nmodes);
    std::vector<char> seen(c.d.nlm, 0);
    for (int i = 0; i < nmodes; ++i) {
        const int l = l_of[i], m = m_of[i];
        if (l < 0 || l > c.d.lmax || m < 0 || m > l)
            throw ArgError("mode " + std::to_string(i) + " (l = " + std::to_string(l) + ", m = " + std::to_string(m) +
                           ") is outside 0 <= m <= l <= l_max");
        lm[i] = lm_index(l, m);
        if (seen[lm[i]]) throw ArgError("mode (l = " + std::to_string(l) + ", m = " + std::to_string(m) + ") repeated");
        seen[lm[i]] = 1;
    }
    return lm;
}

// moves one slice's W-P-T, Z and AB arrays to (to_device) or from the device state
static void move_modes(Ctx& c, int nmodes, const int* l_of, const int* m_of, const double* wpt_in, const double* z_in,
                       const double* ab_in, double* wpt_out, double* z_out, double* ab_out, bool to_device) {
    const std::vector<long> lm = mode_indices(c, nmodes, l_of, m_of);
    const int nr = c.d.nr;
    long* d_lm = nullptr;
    double* d_tmp = nullptr;
    const size_t nw = (size_t)nmodes * 2 * 3 * nr, nz = (size_t)nmodes * 2 * nr;
    RA_CUDA(cudaMalloc(&d_lm, lm.size() * sizeof(long)));
    cudaError_t e = cudaMalloc(&d_tmp, (nw + 5 * nz) * sizeof(double));
    if (e != cudaSuccess) {
        cudaFree(d_lm);
        throw CudaError(e, "cudaMalloc", __FILE__, __LINE__);
    }
    try {
        RA_CUDA(cudaMemcpyAsync(d_lm, lm.data(), lm.size() * sizeof(long), cudaMemcpyHostToDevice, c.stream));
        double* t_w = d_tmp;
        double* t_z = d_tmp + nw;
        double* t_ab = d_tmp + nw + nz;
        const long plane = c.d.nlm * 2L * nr;
        auto run = [&](const double* src, double* dst, int k, long state_plane, long slice_plane, int np) {
            scatter_launch(c, src, dst, d_lm, nmodes, k, state_plane, slice_plane, np, to_device);
        };
        if (to_device) {
            RA_CUDA(cudaMemcpyAsync(t_w, wpt_in, nw * sizeof(double), cudaMemcpyHostToDevice, c.stream));
            RA_CUDA(cudaMemcpyAsync(t_z, z_in, nz * sizeof(double), cudaMemcpyHostToDevice, c.stream));
            if (ab_in) RA_CUDA(cudaMemcpyAsync(t_ab, ab_in, 4 * nz * sizeof(double), cudaMemcpyHostToDevice, c.stream));
            else RA_CUDA(cudaMemsetAsync(t_ab, 0, 4 * nz * sizeof(double), c.stream));
            run(t_w, c.d_sol_wpt, 3 * nr, 0, 0, 1);
            run(t_z, c.d_sol_z, nr, 0, 0, 1);
            run(t_ab, c.d_ab, nr, plane, (long)nz, 4);
            RA_CUDA(cudaMemsetAsync(c.d_status, 0, sizeof(int), c.stream));
            scan_nonfinite(c, t_w, (long)(nw + 5 * nz));
        } else {
            run(c.d_sol_wpt, t_w, 3 * nr, 0, 0, 1);
            run(c.d_sol_z, t_z, nr, 0, 0, 1);
            run(c.d_ab, t_ab, nr, plane, (long)nz, 4);
            if (wpt_out) RA_CUDA(cudaMemcpyAsync(wpt_out, t_w, nw * sizeof(double), cudaMemcpyDeviceToHost, c.stream));
            if (z_out) RA_CUDA(cudaMemcpyAsync(z_out, t_z, nz * sizeof(double), cudaMemcpyDeviceToHost, c.stream));
            if (ab_out) RA_CUDA(cudaMemcpyAsync(ab_out, t_ab, 4 * nz * sizeof(double), cudaMemcpyDeviceToHost, c.stream));
        }
        RA_CUDA(cudaStreamSynchronize(c.stream));
    } catch (...) {
        cudaFree(d_lm);
        cudaFree(d_tmp);
        throw;
    }
    cudaFree(d_lm);
    cudaFree(d_tmp);
}

// ---- the autotuner: candidate kernels of the tunable stages ----
static std::vector<int> knob_candidates(const Ctx& c, int knob) {
    if (knob == 0) {   // physics
        std::vector<int> v;
        if (c.physics3_ok && !c.mag && !c.rad.heating) {   // the magnetic and heating terms exist in form 1 only
            v.push_back(0);
            v.push_back(2);
        }
        if (physics_form1_supported(c.d.nth)) v.push_back(1);
        return v;
    }
    std::vector<int> v;   // solve_nc
    if (lu_nc_for(3 * c.d.nr) == 32) v.push_back(32);
    v.push_back(16);
    return v;
}

static int knob_index(const char* knob) {
    if (!knob) return -1;
    if (!std::strcmp(knob, "physics")) return 0;
    if (!std::strcmp(knob, "solve_nc")) return 1;
    return -1;
}

static void drop_graph(Ctx& c) {
    if (c.graph_exec) cudaGraphExecDestroy(c.graph_exec);
    if (c.graph) cudaGraphDestroy(c.graph);
    c.graph_exec = nullptr;
    c.graph = nullptr;
    if (c.adapt_exec) cudaGraphExecDestroy(c.adapt_exec);
    if (c.adapt_graph) cudaGraphDestroy(c.adapt_graph);
    c.adapt_exec = nullptr;
    c.adapt_graph = nullptr;
}

static void set_knob(Ctx& c, int knob, int value) {
    const std::vector<int> cand = knob_candidates(c, knob);
    if (std::find(cand.begin(), cand.end(), value) == cand.end())
        throw ArgError("value " + std::to_string(value) + " is not a candidate of this knob for this configuration");
    if (knob == 0) {
        c.physics_form = value;
    } else if (value != c.solve_nc) {
        c.solve_nc = value;
        if (c.d_solve_tiles) cudaFree(c.d_solve_tiles);
        c.d_solve_tiles = nullptr;
        if (c.d_inv_sol_tiles) cudaFree(c.d_inv_sol_tiles);
        c.d_inv_sol_tiles = nullptr;
        rebuild_solve_tiles(c);
    }
    drop_graph(c);
}

// Times every candidate of each knob on the context's own buffers (the stage's
// kernel alone, nreps launches after one untimed launch) and keeps the fastest.
static void autotune(Ctx& c, int nreps, double* ms_out) {
    const size_t plane = (size_t)c.d.nlm * 2 * c.d.nr;
    if (!c.have_state) {   // give the stages finite inputs
        RA_CUDA(cudaMemsetAsync(c.d_p2a, 0, (size_t)c.d.L * c.d.nth * c.nfa * 2 * c.d.nr * sizeof(double), c.stream));
        RA_CUDA(cudaMemsetAsync(c.d_rhs_wpt, 0, 3 * plane * sizeof(double), c.stream));
        RA_CUDA(cudaMemsetAsync(c.d_rhs_z, 0, plane * sizeof(double), c.stream));
    }
    // the solve overwrites the state: park it in the grid buffer (rebuilt by every step)
    RA_CUDA(cudaMemcpyAsync(c.d_g, c.d_sol_wpt, 3 * plane * sizeof(double), cudaMemcpyDeviceToDevice, c.stream));
    RA_CUDA(cudaMemcpyAsync(c.d_g + 3 * plane, c.d_sol_z, plane * sizeof(double), cudaMemcpyDeviceToDevice, c.stream));
    cudaEvent_t e0, e1;
    RA_CUDA(cudaEventCreate(&e0));
    RA_CUDA(cudaEventCreate(&e1));
    for (int knob = 0; knob < 2; ++knob) {
        double best = 1e300;
        int best_v = -1;
        for (int v : knob_candidates(c, knob)) {
            set_knob(c, knob, v);
            auto run = [&] {
                if (knob == 0) {
                    RA_CUDA(cudaMemsetAsync(c.d_cfl, 0, sizeof(unsigned long long), c.stream));
                    launch_physics(c);
                } else {
                    if (c.mixed_solve) return;   // the mixed form solves by split products
                    launch_solve(c);
                }
            };
            run();
            RA_CUDA(cudaEventRecord(e0, c.stream));
            for (int i = 0; i < nreps; ++i) run();
            RA_CUDA(cudaEventRecord(e1, c.stream));
            RA_CUDA(cudaEventSynchronize(e1));
            float ms = 0.f;
            RA_CUDA(cudaEventElapsedTime(&ms, e0, e1));
            const double per = ms / std::max(1, nreps);
            if (per < best) {
                best = per;
                best_v = v;
            }
        }
        set_knob(c, knob, best_v);
        if (ms_out) ms_out[knob] = best;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    RA_CUDA(cudaMemcpyAsync(c.d_sol_wpt, c.d_g, 3 * plane * sizeof(double), cudaMemcpyDeviceToDevice, c.stream));
    RA_CUDA(cudaMemcpyAsync(c.d_sol_z, c.d_g + 3 * plane, plane * sizeof(double), cudaMemcpyDeviceToDevice, c.stream));
    RA_CUDA(cudaMemsetAsync(c.d_status, 0, sizeof(int), c.stream));
    RA_CUDA(cudaStreamSynchronize(c.stream));
}

}  // namespace ra

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
template <class F>
static int guarded(ra_ctx* ctx, F f) {
    try {
        // one process may hold contexts on several devices: make this context's current
        if (ctx && ctx->c.stream) RA_CUDA(cudaSetDevice(ctx->c.cfg.device));
        f();
        return RA_OK;
    } catch (const ArgError& e) {
        if (ctx) ctx->c.err = e.what;
        return RA_ERR_ARG;
    } catch (const SingularError& e) {
        if (ctx) ctx->c.err = e.what;
        return RA_ERR_SINGULAR;
    } catch (const NonFiniteError& e) {
        if (ctx) ctx->c.err = e.what;
        return RA_ERR_NONFINITE;
    } catch (const StateError& e) {
        if (ctx) ctx->c.err = e.what;
        return RA_ERR_STATE;
    } catch (const CudaError& e) {
        if (ctx) ctx->c.err = e.what;
        return e.code == cudaErrorMemoryAllocation ? RA_ERR_NOMEM : RA_ERR_CUDA;
    } catch (const std::bad_alloc&) {
        if (ctx) ctx->c.err = "host allocation failed";
        return RA_ERR_NOMEM;
    }
}

extern "C" {

int ra_default_config(ra_config* cfg) {
    if (!cfg) return RA_ERR_ARG;
    std::memset(cfg, 0, sizeof(*cfg));
    cfg->n_r = 48;
    cfg->l_max = 63;
    cfg->n_theta = 0;
    cfg->aspect_ratio = 0.35;
    cfg->shell_depth = 1.0;
    cfg->rayleigh = 1.0e5;
    cfg->ekman = 1.0e-3;
    cfg->prandtl = 1.0;
    cfg->magnetic_prandtl = 1.0;
    cfg->gravity_power = 1.0;
    cfg->rotation = 1;
    cfg->magnetism = 0;
    cfg->no_slip_top = cfg->no_slip_bottom = 1;
    cfg->fix_tvar_top = cfg->fix_tvar_bottom = 1;
    cfg->t_top = 0.0;
    cfg->t_bottom = 1.0;
    cfg->dt = 1.0e-4;
    cfg->alpha_implicit = 0.5;
    cfg->precision = RA_PREC_FP64;
    cfg->use_graph = 1;
    cfg->device = 0;
    cfg->autotune = 0;
    cfg->reference_type = 1;
    cfg->pressure_specific_heat = 1.0;
    cfg->angular_velocity = -1.0;
    cfg->modified_rayleigh = -1.0;
    cfg->nu_type = cfg->kappa_type = cfg->eta_type = 1;
    cfg->nu_top = cfg->kappa_top = cfg->eta_top = -1.0;
    cfg->viscous_heating = cfg->ohmic_heating = 1;
    cfg->chebyshev = 1;
    return RA_OK;
}

int ra_create(ra_ctx** out, const ra_config* cfg) {
    if (!out || !cfg) return RA_ERR_ARG;
    *out = nullptr;
    ra_ctx* ctx = new (std::nothrow) ra_ctx();
    if (!ctx) return RA_ERR_NOMEM;
    int rc = guarded(ctx, [&] {
        check_config(*cfg);
        ctx->c.cfg = *cfg;
        ctx->c.d = make_dims(*cfg);
        setup(ctx->c);
    });
    if (rc != RA_OK) {
        // keep the context so the caller can read the message, but free device memory
        release(ctx->c);
        Ctx fresh;
        fresh.err = ctx->c.err;
        ctx->c = fresh;
    }
    *out = ctx;
    return rc;
}

int ra_destroy(ra_ctx* ctx) {
    if (!ctx) return RA_OK;
    release(ctx->c);
    delete ctx;
    return RA_OK;
}

int ra_last_error(const ra_ctx* ctx, char* msg, int len) {
    if (!ctx || !msg || len <= 0) return RA_ERR_ARG;
    std::strncpy(msg, ctx->c.err.c_str(), (size_t)len - 1);
    msg[len - 1] = 0;
    return RA_OK;
}

int ra_sizes(const ra_ctx* ctx, long* n_lm, int* n_r, int* n_theta, int* n_phi) {
    if (!ctx || ctx->c.d.L == 0) return RA_ERR_STATE;
    if (n_lm) *n_lm = ctx->c.d.nlm;
    if (n_r) *n_r = ctx->c.d.nr;
    if (n_theta) *n_theta = ctx->c.d.nth;
    if (n_phi) *n_phi = ctx->c.d.nphi;
    return RA_OK;
}

int ra_set_dt(ra_ctx* ctx, double dt) {
    if (!ctx || ctx->c.d.L == 0) return RA_ERR_STATE;
    return guarded(ctx, [&] {
        if (!(dt > 0)) throw ArgError("dt must be positive");
        if (ctx->c.custom_reference)
            throw StateError("the reference state was set by ra_set_reference: load the matrices of the new dt "
                             "with ra_load_matrices and factor them with ra_factor");
        ctx->c.dt = dt;
        linear_setup(ctx->c);
        if (ctx->c.mixed_solve) mixed_resplit_solve(ctx->c);
    });
}

int ra_put_state(ra_ctx* ctx, const double* wpt, const double* z, const double* ab, int iteration) {
    if (!ctx || ctx->c.d.L == 0) return RA_ERR_STATE;
    if (!wpt || !z) return RA_ERR_ARG;
    return guarded(ctx, [&] {
        Ctx& c = ctx->c;
        const size_t nw = (size_t)c.d.nlm * 2 * 3 * c.d.nr, nz = (size_t)c.d.nlm * 2 * c.d.nr;
        RA_CUDA(cudaMemcpyAsync(c.d_sol_wpt, wpt, nw * sizeof(double), cudaMemcpyHostToDevice, c.stream));
        RA_CUDA(cudaMemcpyAsync(c.d_sol_z, z, nz * sizeof(double), cudaMemcpyHostToDevice, c.stream));
        if (ab) RA_CUDA(cudaMemcpyAsync(c.d_ab, ab, 4 * nz * sizeof(double), cudaMemcpyHostToDevice, c.stream));
        else RA_CUDA(cudaMemsetAsync(c.d_ab, 0, 4 * nz * sizeof(double), c.stream));
        // a new state clears the error word; non-finite input is refused
        RA_CUDA(cudaMemsetAsync(c.d_status, 0, sizeof(int), c.stream));
        scan_nonfinite(c, c.d_sol_wpt, (long)nw);
        scan_nonfinite(c, c.d_sol_z, (long)nz);
        if (ab) scan_nonfinite(c, c.d_ab, 4L * (long)nz);
        c.have_state = false;
        check_status(c);
        c.iteration = iteration > 0 ? iteration : 1;
        c.have_state = true;
    });
}

int ra_get_state(ra_ctx* ctx, double* wpt, double* z, double* ab) {
    if (!ctx || ctx->c.d.L == 0) return RA_ERR_STATE;
    return guarded(ctx, [&] {
        Ctx& c = ctx->c;
        const size_t nw = (size_t)c.d.nlm * 2 * 3 * c.d.nr, nz = (size_t)c.d.nlm * 2 * c.d.nr;
        if (wpt) RA_CUDA(cudaMemcpyAsync(wpt, c.d_sol_wpt, nw * sizeof(double), cudaMemcpyDeviceToHost, c.stream));
        if (z) RA_CUDA(cudaMemcpyAsync(z, c.d_sol_z, nz * sizeof(double), cudaMemcpyDeviceToHost, c.stream));
        if (ab) RA_CUDA(cudaMemcpyAsync(ab, c.d_ab, 4 * nz * sizeof(double), cudaMemcpyDeviceToHost, c.stream));
        RA_CUDA(cudaStreamSynchronize(c.stream));
    });
}

int ra_put_magnetic_state(ra_ctx* ctx, const double* cpol, const double* ator, const double* ab) {
    if (!ctx || ctx->c.d.L == 0) return RA_ERR_STATE;
    if (!cpol || !ator) return RA_ERR_ARG;
    return guarded(ctx, [&] {
        Ctx& c = ctx->c;
        if (!c.mag) throw ArgError("the context was created without magnetism");
        const size_t nz = (size_t)c.d.nlm * 2 * c.d.nr;
        double* ab_ca = c.d_ab + 4 * nz;   // AB history planes 4, 5: C, A
        RA_CUDA(cudaMemcpyAsync(c.d_sol_c, cpol, nz * sizeof(double), cudaMemcpyHostToDevice, c.stream));
        RA_CUDA(cudaMemcpyAsync(c.d_sol_a, ator, nz * sizeof(double), cudaMemcpyHostToDevice, c.stream));
        if (ab) RA_CUDA(cudaMemcpyAsync(ab_ca, ab, 2 * nz * sizeof(double), cudaMemcpyHostToDevice, c.stream));
        else RA_CUDA(cudaMemsetAsync(ab_ca, 0, 2 * nz * sizeof(double), c.stream));
        RA_CUDA(cudaMemsetAsync(c.d_status, 0, sizeof(int), c.stream));
        scan_nonfinite(c, c.d_sol_c, (long)nz);
        scan_nonfinite(c, c.d_sol_a, (long)nz);
        if (ab) scan_nonfinite(c, ab_ca, 2L * (long)nz);
        check_status(c);
    });
}

int ra_get_magnetic_state(ra_ctx* ctx, double* cpol, double* ator, double* ab) {
    if (!ctx || ctx->c.d.L == 0) return RA_ERR_STATE;
    return guarded(ctx, [&] {
        Ctx& c = ctx->c;
        if (!c.mag) throw ArgError("the context was created without magnetism");
        const size_t nz = (size_t)c.d.nlm * 2 * c.d.nr;
        if (cpol) RA_CUDA(cudaMemcpyAsync(cpol, c.d_sol_c, nz * sizeof(double), cudaMemcpyDeviceToHost, c.stream));
        if (ator) RA_CUDA(cudaMemcpyAsync(ator, c.d_sol_a, nz * sizeof(double), cudaMemcpyDeviceToHost, c.stream));
        if (ab) RA_CUDA(cudaMemcpyAsync(ab, c.d_ab + 4 * nz, 2 * nz * sizeof(double), cudaMemcpyDeviceToHost, c.stream));
        RA_CUDA(cudaStreamSynchronize(c.stream));
    });
}

int ra_put_state_modes(ra_ctx* ctx, int nmodes, const int* l_of, const int* m_of, const double* wpt, const double* z,
                       const double* ab, int iteration) {
    if (!ctx || ctx->c.d.L == 0) return RA_ERR_STATE;
    if (!wpt || !z) return RA_ERR_ARG;
    return guarded(ctx, [&] {
        Ctx& c = ctx->c;
        c.have_state = false;
        move_modes(c, nmodes, l_of, m_of, wpt, z, ab, nullptr, nullptr, nullptr, true);
        check_status(c);
        c.iteration = iteration > 0 ? iteration : 1;
        c.have_state = true;
    });
}

int ra_get_state_modes(ra_ctx* ctx, int nmodes, const int* l_of, const int* m_of, double* wpt, double* z, double* ab) {
    if (!ctx || ctx->c.d.L == 0) return RA_ERR_STATE;
    return guarded(ctx, [&] {
        move_modes(ctx->c, nmodes, l_of, m_of, nullptr, nullptr, nullptr, wpt, z, ab, false);
    });
}

int ra_build_matrices(const ra_config* cfg, int sys, int l0, int nl, double* lhs, double* coefs) {
    if (!cfg || sys < 0 || sys > 3 || nl < 1 || l0 < 0 || l0 + nl - 1 > cfg->l_max || (!lhs && !coefs))
        return RA_ERR_ARG;
    if (sys >= 2 && !cfg->magnetism) return RA_ERR_ARG;
    try {   // host only: the library's own Load_Linear_Coefficients + Set_Boundary_Conditions
        Ctx c;
        check_config(*cfg);
        c.cfg = *cfg;
        c.d = make_dims(*cfg);
        c.dt = cfg->dt;
        const double rmax = cfg->shell_depth / (1.0 - cfg->aspect_ratio);
        radial_setup(c, rmax * cfg->aspect_ratio, rmax);
        reference_setup(c);
        const int nr = c.d.nr, n = sys ? nr : 3 * nr;
        std::vector<double> A, Z, cf((size_t)NSLOT * nr), cm((size_t)NMSLOT * nr);
        // coefficient slots of the magnetic systems: C (C,C,0) (C,C,2); A (A,A,0) (A,A,1) (A,A,2)
        static const int kMagSlots[2][3] = {{MS_C0, MS_C2, -1}, {MS_A0, MS_A1, MS_A2}};
        for (int i = 0; i < nl; ++i) {
            const std::vector<double>* M;
            if (sys < 2) {
                build_l(c, l0 + i, A, Z, cf.data());
                M = sys ? &Z : &A;
            } else {
                build_l_mag(c, l0 + i, Z, A, cm.data());   // Z: C, A: A
                M = sys == 2 ? &Z : &A;
            }
            if (lhs) {
                double* out = lhs + (size_t)i * n * n;   // column-major
                for (int r = 0; r < n; ++r)
                    for (int k = 0; k < n; ++k) out[(size_t)k * n + r] = (*M)[(size_t)r * n + k];
            }
            if (coefs && sys < 2) std::copy(cf.begin(), cf.end(), coefs + (size_t)i * NSLOT * nr);
            if (coefs && sys >= 2) {
                const int ns = sys == 2 ? 2 : 3;
                for (int q = 0; q < ns; ++q)
                    std::copy(cm.begin() + (size_t)kMagSlots[sys - 2][q] * nr,
                              cm.begin() + (size_t)(kMagSlots[sys - 2][q] + 1) * nr,
                              coefs + ((size_t)i * ns + q) * nr);
            }
        }
        return RA_OK;
    } catch (const ArgError&) {
        return RA_ERR_ARG;
    } catch (const std::bad_alloc&) {
        return RA_ERR_NOMEM;
    }
}

int ra_load_matrices(ra_ctx* ctx, int sys, const double* lhs, const double* coefs) {
    if (!ctx || ctx->c.d.L == 0) return RA_ERR_STATE;
    return guarded(ctx, [&] {
        Ctx& c = ctx->c;
        if (sys < 0 || sys > 3) throw ArgError("sys must be 0 (linked W-P-T), 1 (Z), 2 (C) or 3 (A)");
        if (sys >= 2 && !c.mag) throw ArgError("systems 2 (C) and 3 (A) exist with magnetism only");
        if (!lhs && !coefs) throw ArgError("nothing to load");
        const int L = c.d.L, nr = c.d.nr, n = sys ? nr : 3 * nr;
        double* const dst = sys == 0 ? c.d_Awpt : sys == 1 ? c.d_Az : sys == 2 ? c.d_Ac : c.d_Aa;
        if (lhs) {
            const size_t cnt = (size_t)L * n * n;
            for (size_t i = 0; i < cnt; ++i)
                if (!std::isfinite(lhs[i]))
                    throw NonFiniteError("lhs entry " + std::to_string(i) + " is not finite");
            double* tmp = nullptr;
            RA_CUDA(cudaMalloc(&tmp, cnt * sizeof(double)));
            cudaError_t e = cudaMemcpyAsync(tmp, lhs, cnt * sizeof(double), cudaMemcpyHostToDevice, c.stream);
            if (e == cudaSuccess) {
                dim3 grid((n + 31) / 32, (n + 31) / 32, L);
                transpose_batch_kernel<<<grid, dim3(32, 8), 0, c.stream>>>(tmp, dst, n);
                e = cudaGetLastError();
            }
            if (e == cudaSuccess) e = cudaStreamSynchronize(c.stream);
            cudaFree(tmp);
            if (e != cudaSuccess) throw CudaError(e, "ra_load_matrices upload", __FILE__, __LINE__);
            c.matrices_loaded |= 1 << sys;
        }
        if (coefs && sys >= 2) {
            // coefs(n_r, 2 | 3 slots, l): C (C,C,0) (C,C,2); A (A,A,0) (A,A,1) (A,A,2)
            static const int kMagSlots[2][3] = {{MS_C0, MS_C2, -1}, {MS_A0, MS_A1, MS_A2}};
            const int ns = sys == 2 ? 2 : 3;
            std::vector<double> h((size_t)L * NMSLOT * nr);
            RA_CUDA(cudaMemcpy(h.data(), c.d_coef_mag, h.size() * sizeof(double), cudaMemcpyDeviceToHost));
            for (int l = 0; l < L; ++l)
                for (int q = 0; q < ns; ++q)
                    for (int r = 0; r < nr; ++r) {
                        const double v = coefs[((size_t)l * ns + q) * nr + r];
                        if (!std::isfinite(v)) throw NonFiniteError("coefs entry is not finite");
                        h[((size_t)l * NMSLOT + kMagSlots[sys - 2][q]) * nr + r] = v;
                    }
            RA_CUDA(cudaMemcpy(c.d_coef_mag, h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice));
        } else if (coefs) {
            // coefs(n_r, 16 slots, l) of this system's equations: slots of other equations are kept
            std::vector<double> h((size_t)L * NSLOT * nr);
            RA_CUDA(cudaMemcpy(h.data(), c.d_coef, h.size() * sizeof(double), cudaMemcpyDeviceToHost));
            for (int l = 0; l < L; ++l)
                for (int sl = 0; sl < NSLOT; ++sl) {
                    if ((kSlots[sl].eq == EQ_Z) != (sys == 1)) continue;
                    for (int r = 0; r < nr; ++r) {
                        const double v = coefs[((size_t)l * NSLOT + sl) * nr + r];
                        if (!std::isfinite(v)) throw NonFiniteError("coefs entry is not finite");
                        h[((size_t)l * NSLOT + sl) * nr + r] = v;
                    }
                }
            RA_CUDA(cudaMemcpy(c.d_coef, h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice));
        }
    });
}

int ra_factor(ra_ctx* ctx, double dt) {
    if (!ctx || ctx->c.d.L == 0) return RA_ERR_STATE;
    return guarded(ctx, [&] {
        Ctx& c = ctx->c;
        if (!(dt > 0)) throw ArgError("dt must be positive");
        const int need = c.mag ? 15 : 3;
        if (c.matrices_loaded != need)
            throw ArgError(c.mag ? "ra_factor needs the four systems (W-P-T, Z, C, A) loaded by ra_load_matrices"
                                 : "ra_factor needs both systems loaded by ra_load_matrices");
        c.dt = dt;
        factor_matrices(c);
        if (c.mixed_solve) mixed_resplit_solve(c);
        c.matrices_loaded = 0;
    });
}

int ra_set_bc_mask(ra_ctx* ctx, const double* bc_values) {
    if (!ctx || ctx->c.d.L == 0) return RA_ERR_STATE;
    return guarded(ctx, [&] {
        Ctx& c = ctx->c;
        drop_graph(c);   // the captured steps hold the old pointer
        if (!bc_values) {
            if (c.d_bcval) cudaFree(c.d_bcval);
            c.d_bcval = nullptr;
            return;
        }
        const size_t cnt = (size_t)4 * c.d.nlm * 4;
        for (size_t i = 0; i < cnt; ++i)
            if (!std::isfinite(bc_values[i])) throw NonFiniteError("bc_values entry is not finite");
        if (!c.d_bcval) dalloc(c.d_bcval, cnt);
        RA_CUDA(cudaMemcpyAsync(c.d_bcval, bc_values, cnt * sizeof(double), cudaMemcpyHostToDevice, c.stream));
        RA_CUDA(cudaStreamSynchronize(c.stream));
    });
}

int ra_set_reference(ra_ctx* ctx, const double* density, const double* dlnrho, const double* viscous_heating_coeff,
                     const double* ohmic_heating_coeff, double coriolis_coeff, double lorentz_coeff) {
    if (!ctx || ctx->c.d.L == 0) return RA_ERR_STATE;
    if (!density || !dlnrho) return RA_ERR_ARG;
    return guarded(ctx, [&] {
        Ctx& c = ctx->c;
        const int n = c.d.nr;
        auto check = [&](const double* v, const char* what, bool positive) {
            if (!v) return;
            for (int i = 0; i < n; ++i) {
                if (!std::isfinite(v[i])) throw NonFiniteError(std::string(what) + " is not finite");
                if (positive && !(v[i] > 0)) throw ArgError(std::string(what) + " must be positive");
            }
        };
        check(density, "density", true);
        check(dlnrho, "dlnrho", false);
        check(viscous_heating_coeff, "viscous_heating_coeff", false);
        check(ohmic_heating_coeff, "ohmic_heating_coeff", false);
        if (!std::isfinite(coriolis_coeff) || !std::isfinite(lorentz_coeff))
            throw NonFiniteError("coriolis_coeff / lorentz_coeff is not finite");
        if (ohmic_heating_coeff && !c.mag) throw ArgError("ohmic heating needs magnetism");
        Radial& R = c.rad;
        R.density.assign(density, density + n);
        R.dlnrho.assign(dlnrho, dlnrho + n);
        R.visc_heat.assign(n, 0.0);
        R.ohm_heat.assign(n, 0.0);
        bool heat = false;
        for (int i = 0; i < n; ++i) {
            if (viscous_heating_coeff) R.visc_heat[i] = viscous_heating_coeff[i];
            if (ohmic_heating_coeff) R.ohm_heat[i] = ohmic_heating_coeff[i];
            heat = heat || R.visc_heat[i] != 0.0 || R.ohm_heat[i] != 0.0;
        }
        if (heat && !physics_form1_supported(c.d.nth))
            throw ArgError("viscous / ohmic heating needs n_theta in 24..768 (2^a or 3*2^a)");
        R.heating = heat;
        if (heat || c.mag) c.physics_form = 1;   // the form with the heating and magnetic terms
        R.coriolis = coriolis_coeff;
        if (c.mag) R.lorentz = lorentz_coeff;
        c.custom_reference = true;
        const std::vector<double> rp = radial_table(c);
        RA_CUDA(cudaMemcpyAsync(c.d_radial, rp.data(), rp.size() * sizeof(double), cudaMemcpyHostToDevice,
                                c.stream));
        RA_CUDA(cudaStreamSynchronize(c.stream));
        drop_graph(c);   // the captured step holds the old Coriolis and Lorentz coefficients
    });
}

int ra_step_timed(ra_ctx* ctx, int nsteps, double* total_ms) {
    if (!ctx || ctx->c.d.L == 0) return RA_ERR_STATE;
    if (nsteps < 1 || !total_ms) return RA_ERR_ARG;
    int rc = guarded(ctx, [&] {
        Ctx& c = ctx->c;
        cudaEvent_t e0, e1;
        RA_CUDA(cudaEventCreate(&e0));
        RA_CUDA(cudaEventCreate(&e1));
        c.launches = 0;
        RA_CUDA(cudaEventRecord(e0, c.stream));
        run_steps(c, nsteps, nullptr, false);   // graph replays from the second step on (use_graph)
        RA_CUDA(cudaEventRecord(e1, c.stream));
        RA_CUDA(cudaEventSynchronize(e1));
        check_status(c);
        float ms = 0.f;
        RA_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        *total_ms = ms;
    });
    if (rc == RA_ERR_ARG && !ctx->c.have_state) return RA_ERR_STATE;
    return rc;
}

int ra_get_choice(const ra_ctx* ctx, const char* knob, int* value) {
    if (!ctx || ctx->c.d.L == 0) return RA_ERR_STATE;
    const int k = knob_index(knob);
    if (k < 0 || !value) return RA_ERR_ARG;
    *value = k == 0 ? ctx->c.physics_form : ctx->c.solve_nc;
    return RA_OK;
}

int ra_set_choice(ra_ctx* ctx, const char* knob, int value) {
    if (!ctx || ctx->c.d.L == 0) return RA_ERR_STATE;
    return guarded(ctx, [&] {
        const int k = knob_index(knob);
        if (k < 0) throw ArgError(std::string("unknown knob ") + (knob ? knob : "(null)"));
        set_knob(ctx->c, k, value);
    });
}

int ra_autotune(ra_ctx* ctx, int nreps, double* ms_out) {
    if (!ctx || ctx->c.d.L == 0) return RA_ERR_STATE;
    return guarded(ctx, [&] { autotune(ctx->c, std::max(1, nreps), ms_out); });
}

int ra_step(ra_ctx* ctx, int nsteps, double* cfl) {
    if (!ctx || ctx->c.d.L == 0) return RA_ERR_STATE;
    if (nsteps < 0) return RA_ERR_ARG;
    int rc = guarded(ctx, [&] {
        ctx->c.launches = 0;
        run_steps(ctx->c, nsteps, cfl);
    });
    if (rc == RA_ERR_ARG && !ctx->c.have_state) return RA_ERR_STATE;
    return rc;
}

int ra_post_solve(ra_ctx* ctx) {
    if (!ctx || !ctx->c.have_state) return RA_ERR_STATE;
    return guarded(ctx, [&] {
        double n, o;
        ab_factors(ctx->c, n, o);
        run_stage(ctx->c, 0, n, o);
        run_stage(ctx->c, 1, n, o);
    });
}

int ra_rlm_a(ra_ctx* ctx) {
    if (!ctx || !ctx->c.have_state) return RA_ERR_STATE;
    return guarded(ctx, [&] {
        run_stage(ctx->c, 2, 0.0, 0.0);
        run_stage(ctx->c, 3, 0.0, 0.0);
    });
}

int ra_physical(ra_ctx* ctx, double* cfl) {
    if (!ctx || !ctx->c.have_state) return RA_ERR_STATE;
    return guarded(ctx, [&] {
        Ctx& c = ctx->c;
        run_stage(c, 4, 0.0, 0.0);
        if (cfl) {
            unsigned long long bits = 0;
            RA_CUDA(cudaMemcpyAsync(&bits, c.d_cfl, sizeof(bits), cudaMemcpyDeviceToHost, c.stream));
            RA_CUDA(cudaStreamSynchronize(c.stream));
            std::memcpy(cfl, &bits, sizeof(double));
        }
    });
}

// The stages that form the fields on the physical grid (p2a) from the current
// state; they only assign their outputs, so the next ra_step is unchanged.
// With pressure, the P and dP/dr grids take the places of T and dT/dr before
// rlm_spacea, so that the T and dT/dr slots of p2a hold P and dP/dr.
static void form_grid_fields(Ctx& c, bool pressure) {
    double n, o;
    ab_factors(c, n, o);
    run_stage(c, 0, n, o);
    run_stage(c, 1, n, o);
    if (pressure) launch_pressure_to_s2a(c);
    run_stage(c, 2, n, o);
    run_stage(c, 3, n, o);
}

static void need_phase(Ctx& c, int& phase, const SliceSpec& S) {
    if (phase != S.pressure) {
        form_grid_fields(c, S.pressure != 0);
        phase = S.pressure;
    }
}

int ra_magnetic_energy(ra_ctx* ctx, double* me) {
    if (!ctx || !ctx->c.have_state) return RA_ERR_STATE;
    if (!me) return RA_ERR_ARG;
    return guarded(ctx, [&] {
        Ctx& c = ctx->c;
        if (!c.mag) throw ArgError("the magnetic energy needs a context created with magnetism");
        form_grid_fields(c, false);
        launch_kinetic_energy(c, true);
        double v = 0.0;
        RA_CUDA(cudaMemcpyAsync(&v, c.d_ke_rows + (size_t)c.d.nth * c.d.nr, sizeof(double), cudaMemcpyDeviceToHost,
                                c.stream));
        RA_CUDA(cudaStreamSynchronize(c.stream));
        check_status(c);
        // mag_factor of the benchmark report (Benchmarking.F90:392, 846): 1 / (2 Ek Pm)
        *me = v / (2.0 * c.cfg.ekman * c.cfg.magnetic_prandtl);
    });
}

int ra_next_dt(const ra_dt_controls* ctl, double dt, double cfl, double* new_dt) {
    if (!ctl || !new_dt || !(dt > 0)) return RA_ERR_ARG;
    const double nd = next_dt_value(*ctl, dt, cfl);
    *new_dt = nd;
    return nd < ctl->min_time_step ? RA_ERR_NONFINITE : RA_OK;
}

int ra_default_dt_controls(ra_dt_controls* ctl) {
    if (!ctl) return RA_ERR_ARG;
    ctl->cflmin = 0.4;        // Controls.F90:113-115, ClockInfo.F90:27
    ctl->cflmax = 0.6;
    ctl->max_time_step = 1.0;
    ctl->min_time_step = 1.0e-13;
    ctl->min_dt_change = 0.1;
    return RA_OK;
}

int ra_step_adaptive(ra_ctx* ctx, int nsteps, const ra_dt_controls* ctl, double* dt_out, int* dt_changes) {
    if (!ctx || ctx->c.d.L == 0) return RA_ERR_STATE;
    if (!ctl || nsteps < 0) return RA_ERR_ARG;
    int changes = 0;
    const int rc = guarded(ctx, [&] {
        Ctx& c = ctx->c;
        if (!c.have_state) throw ArgError("ra_put_state must be called before stepping");
        auto change_dt = [&](double nd) {   // Reset_Linear_Equations before the next step
            if (nd < ctl->min_time_step)
                throw NonFiniteError("the time step became smaller than min_time_step (" + std::to_string(nd) + ")");
            if (nd == c.dt) return;
            if (c.custom_reference) throw StateError("a dt change needs the driver's matrices after ra_set_reference");
            c.dt = nd;
            linear_setup(c);
            if (c.mixed_solve) mixed_resplit_solve(c);
            ++changes;
        };
        int s = 0;
        while (s < nsteps) {
            double new_ab, old_ab;
            ab_factors(c, new_ab, old_ab);
            if (!c.cfg.use_graph || c.iteration == 1 || c.old_dt != c.dt || nsteps - s < 2) {
                // one step on the host's control: the first (Euler) step, the first after a dt
                // change (unequal AB2 factors), or a last single step
                double cfl = 0.0;
                run_steps(c, 1, &cfl);
                ++s;
                change_dt(next_dt_value(*ctl, c.dt, cfl));
                continue;
            }
            // the steady steps on the device's control: the loop graph runs until dt changes
            adaptive_graph(c, *ctl, new_ab, old_ab);
            int ad[4] = {0, nsteps - s, 0, 0};
            double adt[3] = {c.dt, c.dt, 0.0};
            RA_CUDA(cudaMemcpyAsync(c.d_adapt, ad, sizeof(ad), cudaMemcpyHostToDevice, c.stream));
            RA_CUDA(cudaMemcpyAsync(c.d_adapt_dt, adt, sizeof(adt), cudaMemcpyHostToDevice, c.stream));
            RA_CUDA(cudaGraphLaunch(c.adapt_exec, c.stream));
            RA_CUDA(cudaMemcpyAsync(ad, c.d_adapt, sizeof(ad), cudaMemcpyDeviceToHost, c.stream));
            RA_CUDA(cudaMemcpyAsync(adt, c.d_adapt_dt, sizeof(adt), cudaMemcpyDeviceToHost, c.stream));
            RA_CUDA(cudaStreamSynchronize(c.stream));
            const int done = ad[0];
            if (done < 1 || done > nsteps - s) throw ArgError("adaptive step loop: bad step count");
            c.launches += (long)done * c.adapt_launches;
            c.iteration += done;
            c.old_dt = c.dt;
            s += done;
            check_status(c);
            change_dt(adt[1]);
        }
    });
    if (dt_out) *dt_out = ctx->c.dt;
    if (dt_changes) *dt_changes = changes;
    return rc;
}

int ra_kinetic_energy(ra_ctx* ctx, double* ke) {
    if (!ctx || !ctx->c.have_state) return RA_ERR_STATE;
    if (!ke) return RA_ERR_ARG;
    return guarded(ctx, [&] {
        Ctx& c = ctx->c;
        form_grid_fields(c, false);
        launch_kinetic_energy(c);
        RA_CUDA(cudaMemcpyAsync(ke, c.d_ke_rows + (size_t)c.d.nth * c.d.nr, sizeof(double), cudaMemcpyDeviceToHost,
                                c.stream));
        RA_CUDA(cudaStreamSynchronize(c.stream));
        check_status(c);
    });
}

// Diagnostic quantity codes of the reference's output system (velocity_field_codes.F,
// vorticity_field_codes.F, thermal_field_codes.F: voffset = 0, vort_off = 300,
// pt_off = 500) that are values of the physical-space buffer, and where each
// comes from in p2a.  vort_r, which Diagnostics_Vorticity_Field.F90:89-93 forms
// as (dv_phi/dtheta + cot v_phi - csc dv_theta/dphi) / r, is the spectral
// l(l+1) Z / r^2 here: the same band-limited field, equal up to rounding.
// With magnetism, magnetic_field_codes.F (boffset = 800): B_r, B_theta, B_phi and their phi
// derivatives (828-830, d/dphi in the spectrum as for the velocity), the B_theta, B_phi ones
// formed from the r sin(theta) B_theta, B_phi fields the step transforms (rsintheta_div), and
// current_density_codes.F (joffset = boffset + 200): J_r, J_theta, J_phi, the curl of B as
// Compute_J_Components reads it (Diagnostics_Current_Density.F90), the last two likewise.
struct QuantitySource { int code, field, dphi, csc, pressure, orad; };
static const QuantitySource kQuantities[] = {
    {1, A_VR, 0, 0, 0, 0},     {2, A_VT, 0, 1, 0, 0},     {3, A_VP, 0, 1, 0, 0},     {10, A_DVRDR, 0, 0, 0, 0},
    {11, A_DVTDR, 0, 1, 0, 0}, {12, A_DVPDR, 0, 1, 0, 0}, {19, A_DVRDT, 0, 1, 0, 0}, {28, A_VR, 1, 0, 0, 0},
    {29, A_VT, 1, 1, 0, 0},    {30, A_VP, 1, 1, 0, 0},    {501, A_T, 0, 0, 0, 0},    {507, A_DTDR, 0, 0, 0, 0},
    {513, A_DTDT, 0, 1, 0, 0}, {519, A_T, 1, 0, 0, 0},
    {301, A_OMR, 0, 0, 0, 0},  // vort_r: l(l+1) Z / r^2, the radial vorticity of the Boussinesq velocity
    {502, A_T, 0, 0, 1, 0},    // pressure, formed in T's place
    {508, A_DTDR, 0, 0, 1, 0}, // d pressure / dr, in dT/dr's place
    {520, A_T, 1, 0, 1, 0},    // d pressure / d phi
    {801, A_BR, 0, 0, 0, 0},   {802, A_BT, 0, 1, 0, 1},   {803, A_BP, 0, 1, 0, 1},
    {1001, A_CBR, 0, 0, 0, 0}, {1004, A_CBT, 0, 1, 0, 1}, {1007, A_CBP, 0, 1, 0, 1},
    {828, A_BR, 1, 0, 0, 0},   {829, A_BT, 1, 1, 0, 1},   {830, A_BP, 1, 1, 0, 1},   // dB/dphi
};

// The fluctuating (m > 0) and azimuthal-mean (m = 0) codes of each quantity above, as the
// reference numbers them (velocity_field_codes.F: vp_r = v_r + 3, vm_r = v_r + 6, ...;
// thermal_field_codes.F: entropy_p = entropy + 2, entropy_m = entropy + 4, ...;
// vorticity_field_codes.F, magnetic_field_codes.F; current_density_codes.F: jp_r = j_r + 1,
// jm_r = j_r + 2).  Diagnostics_Base forms them from the buffer minus, or as, its phi average
// (fbuffer, m0_values); here the m = 0 term of the spectrum is dropped or kept alone.
struct QuantityParts { int full, fluct, mean; };
static const QuantityParts kParts[] = {
    {1, 4, 7},          {2, 5, 8},          {3, 6, 9},          {10, 13, 16},       {11, 14, 17},
    {12, 15, 18},       {19, 22, 25},       {28, 31, 34},       {29, 32, 35},       {30, 33, 36},
    {301, 304, 307},    {501, 503, 505},    {502, 504, 506},    {507, 509, 511},    {508, 510, 512},
    {513, 515, 517},    {519, 521, 523},    {520, 522, 524},    {801, 804, 807},    {802, 805, 808},
    {803, 806, 809},    {1001, 1002, 1003}, {1004, 1005, 1006}, {1007, 1008, 1009}, {828, 831, 834},
    {829, 832, 835},    {830, 833, 836},    {302, 305, 308},    {303, 306, 309},    {20, 23, 26},
    {21, 24, 27},
};

// Sums of fields (Diagnostics_Vorticity_Field.F90 Compute_Vorticity_Field): vort_theta (302)
// = (csc dv_r/dphi - v_phi) / r - dv_phi/dr, vort_phi (303) = dv_theta/dr + (v_theta -
// dv_r/dtheta) / r, from the buffer fields as the other codes form them (v_theta, v_phi and
// their r and theta derivatives divided by sin(theta)); dv_theta/dtheta (20) and
// dv_phi/dtheta (21) as the physical-space stage forms them (Compute_dvtheta_by_dtheta,
// Compute_dvphi_by_dtheta, Sphere_Physical_Space.F90:226-248): -v_r (r dlnrho + 2) - r
// dv_r/dr - v_theta cot - csc dv_phi/dphi and r omega_r + csc dv_theta/dphi - v_phi cot.
// DiagTerm: field, d/dphi, theta factor (1 csc, 2 cot, 3 csc cot, 4 csc^2), radial factor
// (1 1/r, 2 r, 3 r dlnrho + 2), coefficient.
struct LinearSource { int code, nt; DiagTerm t[4]; };
static const LinearSource kLinear[] = {
    {302, 3, {{A_VR, 1, 1, 1, 1.0}, {A_VP, 0, 1, 1, -1.0}, {A_DVPDR, 0, 1, 0, -1.0}}},
    {303, 3, {{A_DVTDR, 0, 1, 0, 1.0}, {A_VT, 0, 1, 1, 1.0}, {A_DVRDT, 0, 1, 1, -1.0}}},
    {20, 4, {{A_VR, 0, 0, 3, -1.0}, {A_DVRDR, 0, 0, 2, -1.0}, {A_VT, 0, 3, 0, -1.0}, {A_VP, 1, 4, 0, -1.0}}},
    {21, 3, {{A_OMR, 0, 0, 2, 1.0}, {A_VT, 1, 4, 0, 1.0}, {A_VP, 0, 3, 0, -1.0}}},
};

// The buffer-field sum of quantity `code` (a row of kQuantities or kLinear), of its part mpart.
static DiagCombo combo_of(const Ctx& c, int code, int mpart, int asked) {
    DiagCombo C{};
    C.mpart = mpart;
    for (const LinearSource& k : kLinear)
        if (k.code == code) {
            C.nt = k.nt;
            for (int i = 0; i < k.nt; ++i) C.t[i] = k.t[i];
            return C;
        }
    for (const QuantitySource& k : kQuantities)
        if (k.code == code) {
            if (k.field >= c.nfa)
                throw ArgError("diagnostics: quantity code " + std::to_string(asked) + " needs magnetism");
            C.nt = 1;
            C.t[0] = DiagTerm{k.field, k.dphi, k.csc, k.orad, 1.0};
            return C;
        }
    throw ArgError("diagnostics: quantity code " + std::to_string(asked) + " is not provided");
}

// Products of vector components (parts: 0 the field, 1 fluctuating, 2 mean), summed over the
// three components (comp 0) or of one (comp 1..3):
//   kinetic_energy_codes.F (keoffset = 400): 1/2 rho |v|^2 and its parts 401-404, of the mean
//     flow 405-408, of the fluctuations 409-412; v^2 likewise without rho 413-424
//     (Diagnostics_Energies.F90 Compute_Kinetic_Energy);
//   magnetic_energy_codes.F (meoffset = 1100): 1/2 Lorentz_Coeff |B|^2 in the same order,
//     1101-1112 (Compute_Magnetic_Energy);
//   current_density_codes.F: J.J 1010, J'.J' 1011, mean J.J 1012, mean J . J' 1013, J_r^2,
//     J_theta^2, J_phi^2 each with its fluctuating and mean forms 1014-1022;
//   vorticity_field_codes.F (vort_off = 300): enstrophy 310, omega'.mean omega 311, of the
//     mean 312, of the fluctuations 313; omega_r^2, omega_theta^2, omega_phi^2 314-316, of the
//     fluctuations 317-319, of the means 320-322; kinetic helicity v_i omega_i 324-326 and its
//     (v, omega) parts (fluct, fluct) 327-329, (mean, mean) 330-332, (mean, fluct) 333-335,
//     (fluct, mean) 336-338; v.omega 339 and the same four part pairs 340-343
//     (Diagnostics_Vorticity_Field.F90).
//   mass_flux_codes.F (rhovoffset = 200): rho v_r, rho v_theta, rho v_phi 201-203, of the
//     fluctuations 204-206, of the means 207-209 (Diagnostics_Velocity_Field.F90);
//   thermal_energy_codes.F (teoffset = 700): rho T S of the reference state and its
//     fluctuating and mean parts 701-703, their squares 707-709 (Diagnostics_Thermal_Energies.F90
//     Compute_Thermal_Energy); b = nullptr: the constant 1.
struct Product { const int* a; int apart; const int* b; int bpart; int comp, coef; bool square; };
static const int kVelocity[3] = {1, 2, 3}, kVorticity[3] = {301, 302, 303}, kBfield[3] = {801, 802, 803},
                 kCurrent[3] = {1001, 1004, 1007}, kEntropy[1] = {501};
static bool product_of(int code, Product& p) {
    static const int kGroupPart[3] = {0, 2, 1};   // field, mean, fluctuations
    if (code >= 201 && code <= 209) {
        static const int part[3] = {0, 1, 2};
        const int k = code - 201;
        p = Product{kVelocity, part[k / 3], nullptr, 0, k % 3 + 1, 5, false};
        return true;
    }
    if ((code >= 701 && code <= 703) || (code >= 707 && code <= 709)) {
        const bool sq = code >= 707;
        const int part = sq ? code - 707 : code - 701;   // 0 field, 1 fluctuations, 2 mean
        p = Product{kEntropy, part, sq ? kEntropy : nullptr, part, 1, sq ? 4 : 3, sq};
        return true;
    }
    if (code >= 401 && code <= 424) {
        const int k = code - 401, g = k / 4;
        p = Product{kVelocity, kGroupPart[g % 3], kVelocity, kGroupPart[g % 3], k % 4, g < 3 ? 1 : 0, true};
        return true;
    }
    if (code >= 1101 && code <= 1112) {
        const int k = code - 1101, g = k / 4;
        p = Product{kBfield, kGroupPart[g], kBfield, kGroupPart[g], k % 4, 2, true};
        return true;
    }
    if (code >= 1010 && code <= 1013) {
        static const int ap[4] = {0, 1, 2, 2}, bp[4] = {0, 1, 2, 1};
        const int k = code - 1010;
        p = Product{kCurrent, ap[k], kCurrent, bp[k], 0, 0, k < 3};
        return true;
    }
    if (code >= 1014 && code <= 1022) {
        const int k = code - 1014;
        p = Product{kCurrent, k % 3, kCurrent, k % 3, k / 3 + 1, 0, true};
        return true;
    }
    if (code >= 310 && code <= 313) {
        static const int ap[4] = {0, 1, 2, 1}, bp[4] = {0, 2, 2, 1};
        const int k = code - 310;
        p = Product{kVorticity, ap[k], kVorticity, bp[k], 0, 0, k != 1};
        return true;
    }
    if (code >= 314 && code <= 322) {
        static const int part[3] = {0, 1, 2};
        const int k = code - 314;
        p = Product{kVorticity, part[k / 3], kVorticity, part[k / 3], k % 3 + 1, 0, true};
        return true;
    }
    if (code >= 324 && code <= 343) {   // (velocity part, vorticity part) per group
        static const int vp[5] = {0, 1, 2, 2, 1}, wp[5] = {0, 1, 2, 1, 2};
        const int k = code - 324;
        const int g = k < 15 ? k / 3 : k - 15, comp = k < 15 ? k % 3 + 1 : 0;
        p = Product{kVelocity, vp[g], kVorticity, wp[g], comp, 0, false};
        return true;
    }
    return false;
}

static std::vector<SliceSpec> quantity_specs(const Ctx& c, const int* quantities, int nq) {
    std::vector<SliceSpec> spec(nq);
    for (int q = 0; q < nq; ++q) {
        const int asked = quantities[q];
        Product pr;
        if (product_of(asked, pr)) {
            SliceSpec S{};
            S.nprod = pr.comp ? 1 : 3;
            if (pr.coef >= 3 && c.custom_reference)   // ra_set_reference gives no temperature
                throw ArgError("diagnostics: the thermal energy codes need the library's own reference state");
            for (int i = 0; i < S.nprod; ++i) {
                const int j = pr.comp ? pr.comp - 1 : i;
                S.a[i] = combo_of(c, pr.a[j], pr.apart, asked);
                S.bsame[i] = pr.square ? 1 : 0;
                if (!pr.square && pr.b) S.b[i] = combo_of(c, pr.b[j], pr.bpart, asked);
            }
            S.field = S.a[0].t[0].field;
            S.coef = pr.coef;
            S.cval = 0.5 * c.rad.lorentz;   // magnetic_energy: 1/2 Lorentz_Coeff
            spec[q] = S;
            continue;
        }
        int code = asked, mpart = 0;
        for (const QuantityParts& p : kParts) {
            if (p.fluct == code) { code = p.full; mpart = 1; break; }
            if (p.mean == code) { code = p.full; mpart = 2; break; }
        }
        bool linear = false;
        for (const LinearSource& k : kLinear) linear |= k.code == code;
        if (linear) {   // nprod 1 with b the constant 1
            SliceSpec S{};
            S.nprod = 1;
            S.a[0] = combo_of(c, code, mpart, asked);
            S.field = S.a[0].t[0].field;
            spec[q] = S;
            continue;
        }
        const QuantitySource* src = nullptr;
        for (const QuantitySource& k : kQuantities)
            if (k.code == code) src = &k;
        if (!src) throw ArgError("diagnostics: quantity code " + std::to_string(asked) + " is not provided");
        if (src->field >= c.nfa)
            throw ArgError("diagnostics: quantity code " + std::to_string(asked) + " needs magnetism");
        if (src->pressure && (c.cfg.reference_type != 1 || c.custom_reference))   // the anelastic state holds P / rho
            throw ArgError("diagnostics: the pressure codes are provided for the Boussinesq reference only");
        spec[q] = SliceSpec{};
        spec[q].field = src->field;
        spec[q].dphi = src->dphi;
        spec[q].csc = src->csc;
        spec[q].pressure = src->pressure;
        spec[q].orad = src->orad;
        spec[q].mpart = mpart;
    }
    return spec;
}

int ra_shell_slices(ra_ctx* ctx, const int* quantities, int nq, const int* levels, int nlev, double* out) {
    if (!ctx || !ctx->c.have_state) return RA_ERR_STATE;
    if (!quantities || !levels || !out || nq < 1 || nlev < 1) return RA_ERR_ARG;
    return guarded(ctx, [&] {
        Ctx& c = ctx->c;
        const std::vector<SliceSpec> spec = quantity_specs(c, quantities, nq);
        for (int l = 0; l < nlev; ++l)
            if (levels[l] < 0 || levels[l] >= c.d.nr) throw ArgError("shell slice: radial index out of range");
        // the slices go through p2b, which the step rewrites before reading
        const long per = (long)c.d.nth * c.d.nphi;
        const long room = (long)c.d.L * c.d.nth * c.nfb * 2 * c.d.nr;
        if (room < per) throw ArgError("shell slice: no room for one slice");
        const int chunk = (int)std::min<long>(SliceSpec::MAXL, room / per);
        int phase = -1;   // which fields p2a holds: 0 velocity and T, 1 with P in T's place
        for (int q = 0; q < nq; ++q)
            for (int l0 = 0; l0 < nlev; l0 += chunk) {
                SliceSpec S = spec[q];
                S.nl = std::min(chunk, nlev - l0);
                for (int i = 0; i < S.nl; ++i) S.level[i] = levels[l0 + i];
                need_phase(c, phase, S);
                launch_shell_slice(c, S, c.d_p2b);
                RA_CUDA(cudaMemcpyAsync(out + ((long)q * nlev + l0) * per, c.d_p2b, (size_t)S.nl * per * sizeof(double),
                                        cudaMemcpyDeviceToHost, c.stream));
            }
        RA_CUDA(cudaStreamSynchronize(c.stream));
        check_status(c);
    });
}

int ra_shell_averages(ra_ctx* ctx, const int* quantities, int nq, double* out) {
    if (!ctx || !ctx->c.have_state) return RA_ERR_STATE;
    if (!quantities || !out || nq < 1) return RA_ERR_ARG;
    return guarded(ctx, [&] {
        Ctx& c = ctx->c;
        const std::vector<SliceSpec> spec = quantity_specs(c, quantities, nq);
        // row sums and the moments go through p2b, which the step rewrites before reading
        const long nrows = (long)c.d.nth * c.d.nr;
        double* rows = c.d_p2b;
        double* dev_out = c.d_p2b + 4 * nrows;
        int phase = -1;   // which fields p2a holds: 0 velocity and T, 1 with P in T's place
        for (int q = 0; q < nq; ++q) {
            need_phase(c, phase, spec[q]);
            launch_shell_moments(c, spec[q], rows, dev_out);
            RA_CUDA(cudaMemcpyAsync(out + (long)q * 4 * c.d.nr, dev_out, 4 * (size_t)c.d.nr * sizeof(double),
                                    cudaMemcpyDeviceToHost, c.stream));
            RA_CUDA(cudaStreamSynchronize(c.stream));   // dev_out is reused by the next quantity
        }
        check_status(c);
    });
}

int ra_azimuthal_averages(ra_ctx* ctx, const int* quantities, int nq, double* out) {
    if (!ctx || !ctx->c.have_state) return RA_ERR_STATE;
    if (!quantities || !out || nq < 1) return RA_ERR_ARG;
    return guarded(ctx, [&] {
        Ctx& c = ctx->c;
        const std::vector<SliceSpec> spec = quantity_specs(c, quantities, nq);
        const long nrows = (long)c.d.nth * c.d.nr;
        int phase = -1;   // which fields p2a holds: 0 velocity and T, 1 with P in T's place
        for (int q = 0; q < nq; ++q) {
            need_phase(c, phase, spec[q]);
            launch_azimuthal_average(c, spec[q], c.d_p2b);   // p2b: scratch between steps
            RA_CUDA(cudaMemcpyAsync(out + (long)q * nrows, c.d_p2b, (size_t)nrows * sizeof(double),
                                    cudaMemcpyDeviceToHost, c.stream));
            RA_CUDA(cudaStreamSynchronize(c.stream));
        }
        check_status(c);
    });
}

int ra_shell_spectra(ra_ctx* ctx, const int* quantities, int nq, const int* levels, int nlev, double* out) {
    if (!ctx || !ctx->c.have_state) return RA_ERR_STATE;
    if (!quantities || !levels || !out || nq < 1 || nlev < 1) return RA_ERR_ARG;
    return guarded(ctx, [&] {
        Ctx& c = ctx->c;
        const std::vector<SliceSpec> spec = quantity_specs(c, quantities, nq);
        for (int l = 0; l < nlev; ++l)
            if (levels[l] < 0 || levels[l] >= c.d.nr) throw ArgError("shell spectra: radial index out of range");
        int phase = -1;   // which fields p2a holds: 0 velocity and T, 1 with P in T's place
        // (quantity, level) pairs fill the 4 n_r column slots of the p2b / s2b layouts, which the
        // step rewrites before reading; each batch of slots goes through one forward transform
        const long total = (long)nq * nlev;
        const int cap = c.nfb * c.d.nr;
        const long per = 2L * c.d.L * c.d.L;
        for (long s0 = 0; s0 < total; s0 += cap) {
            const int ns = (int)std::min<long>(cap, total - s0);
            for (long s = s0; s < s0 + ns;) {   // runs of one quantity, at most 64 levels each
                const int q = (int)(s / nlev), l0 = (int)(s % nlev);
                SliceSpec S = spec[q];
                S.nl = (int)std::min<long>({(long)SliceSpec::MAXL, (long)(nlev - l0), s0 + ns - s});
                for (int i = 0; i < S.nl; ++i) S.level[i] = levels[l0 + i];
                need_phase(c, phase, S);   // the phases' preparations leave p2b alone
                launch_spectra_rows(c, S, (int)(s - s0), c.d_p2b);
                s += S.nl;
            }
            launch_lt_forward(c, c.d_p2b, c.d_s2b, c.nfb * c.d.nr * 2);
            launch_spectra_gather(c, c.d_s2b, ns, c.d_p2b);
            RA_CUDA(cudaMemcpyAsync(out + s0 * per, c.d_p2b, (size_t)ns * per * sizeof(double),
                                    cudaMemcpyDeviceToHost, c.stream));
            RA_CUDA(cudaStreamSynchronize(c.stream));
        }
        check_status(c);
    });
}

int ra_equatorial_slices(ra_ctx* ctx, const int* quantities, int nq, double* out) {
    if (!ctx || !ctx->c.have_state) return RA_ERR_STATE;
    if (!quantities || !out || nq < 1) return RA_ERR_ARG;
    return guarded(ctx, [&] {
        Ctx& c = ctx->c;
        const std::vector<SliceSpec> spec = quantity_specs(c, quantities, nq);
        const long per = (long)c.d.nr * c.d.nphi;
        int phase = -1;   // which fields p2a holds: 0 velocity and T, 1 with P in T's place
        for (int q = 0; q < nq; ++q) {
            need_phase(c, phase, spec[q]);
            launch_equatorial_slice(c, spec[q], c.d_p2b);   // p2b: scratch between steps
            RA_CUDA(cudaMemcpyAsync(out + (long)q * per, c.d_p2b, (size_t)per * sizeof(double),
                                    cudaMemcpyDeviceToHost, c.stream));
            RA_CUDA(cudaStreamSynchronize(c.stream));
        }
        check_status(c);
    });
}

int ra_meridional_slices(ra_ctx* ctx, const int* quantities, int nq, const int* phi_indices, int nphi_sel,
                         double* out) {
    if (!ctx || !ctx->c.have_state) return RA_ERR_STATE;
    if (!quantities || !phi_indices || !out || nq < 1 || nphi_sel < 1) return RA_ERR_ARG;
    return guarded(ctx, [&] {
        Ctx& c = ctx->c;
        const std::vector<SliceSpec> spec = quantity_specs(c, quantities, nq);
        for (int j = 0; j < nphi_sel; ++j)
            if (phi_indices[j] < 0 || phi_indices[j] >= c.d.nphi)
                throw ArgError("meridional slices: phi index out of range");
        const long per = (long)c.d.nth * c.d.nr;
        int phase = -1;   // which fields p2a holds: 0 velocity and T, 1 with P in T's place
        for (int q = 0; q < nq; ++q)
            for (int j0 = 0; j0 < nphi_sel; j0 += SliceSpec::MAXL) {
                SliceSpec S = spec[q];
                S.nl = std::min(SliceSpec::MAXL, nphi_sel - j0);
                for (int i = 0; i < S.nl; ++i) S.level[i] = phi_indices[j0 + i];
                need_phase(c, phase, S);
                launch_meridional_slice(c, S, c.d_p2b);   // p2b: scratch between steps
                RA_CUDA(cudaMemcpyAsync(out + ((long)q * nphi_sel + j0) * per, c.d_p2b,
                                        (size_t)S.nl * per * sizeof(double), cudaMemcpyDeviceToHost, c.stream));
                RA_CUDA(cudaStreamSynchronize(c.stream));
            }
        check_status(c);
    });
}

int ra_global_averages(ra_ctx* ctx, const int* quantities, int nq, double* out) {
    if (!ctx || !ctx->c.have_state) return RA_ERR_STATE;
    if (!quantities || !out || nq < 1) return RA_ERR_ARG;
    return guarded(ctx, [&] {
        Ctx& c = ctx->c;
        const std::vector<SliceSpec> spec = quantity_specs(c, quantities, nq);
        const long nrows = (long)c.d.nth * c.d.nr;
        double* rows = c.d_p2b;                       // scratch between steps
        double* mean = c.d_p2b + nrows;
        double* res = mean + c.d.nr;                  // nq results
        int phase = -1;   // which fields p2a holds: 0 velocity and T, 1 with P in T's place
        for (int q = 0; q < nq; ++q) {
            need_phase(c, phase, spec[q]);
            launch_global_average(c, spec[q], rows, mean, res + q);
        }
        RA_CUDA(cudaMemcpyAsync(out, res, (size_t)nq * sizeof(double), cudaMemcpyDeviceToHost, c.stream));
        RA_CUDA(cudaStreamSynchronize(c.stream));
        check_status(c);
    });
}

int ra_point_probes(ra_ctx* ctx, const int* quantities, int nq, const int* r_idx, int nr_p, const int* theta_idx,
                    int ntheta_p, const int* phi_idx, int nphi_p, double* out) {
    if (!ctx || !ctx->c.have_state) return RA_ERR_STATE;
    if (!quantities || !r_idx || !theta_idx || !phi_idx || !out || nq < 1) return RA_ERR_ARG;
    return guarded(ctx, [&] {
        Ctx& c = ctx->c;
        const std::vector<SliceSpec> spec = quantity_specs(c, quantities, nq);
        if (nr_p < 1 || nr_p > ProbeSet::MAXP || ntheta_p < 1 || ntheta_p > ProbeSet::MAXP || nphi_p < 1 ||
            nphi_p > ProbeSet::MAXP)
            throw ArgError("point probes: 1 .. 64 indices per direction");
        ProbeSet Q{};
        Q.nr = nr_p;
        Q.ntheta = ntheta_p;
        Q.nphi = nphi_p;
        for (int i = 0; i < nr_p; ++i) {
            if (r_idx[i] < 0 || r_idx[i] >= c.d.nr) throw ArgError("point probes: radial index out of range");
            Q.r[i] = r_idx[i];
        }
        for (int i = 0; i < ntheta_p; ++i) {
            if (theta_idx[i] < 0 || theta_idx[i] >= c.d.nth) throw ArgError("point probes: theta index out of range");
            Q.theta[i] = theta_idx[i];
        }
        for (int i = 0; i < nphi_p; ++i) {
            if (phi_idx[i] < 0 || phi_idx[i] >= c.d.nphi) throw ArgError("point probes: phi index out of range");
            Q.phi[i] = phi_idx[i];
        }
        const long per = (long)nr_p * ntheta_p * nphi_p;
        int phase = -1;   // which fields p2a holds: 0 velocity and T, 1 with P in T's place
        for (int q = 0; q < nq; ++q) {
            need_phase(c, phase, spec[q]);
            launch_point_probes(c, spec[q], Q, c.d_p2b + q * per);   // p2b: scratch
        }
        RA_CUDA(cudaMemcpyAsync(out, c.d_p2b, (size_t)nq * per * sizeof(double), cudaMemcpyDeviceToHost, c.stream));
        RA_CUDA(cudaStreamSynchronize(c.stream));
        check_status(c);
    });
}

int ra_rlm_b(ra_ctx* ctx) {
    if (!ctx || !ctx->c.have_state) return RA_ERR_STATE;
    return guarded(ctx, [&] {
        double n, o;
        ab_factors(ctx->c, n, o);
        run_stage(ctx->c, 5, n, o);
        run_stage(ctx->c, 6, n, o);
    });
}

int ra_advance(ra_ctx* ctx) {
    if (!ctx || !ctx->c.have_state) return RA_ERR_STATE;
    return guarded(ctx, [&] {
        run_stage(ctx->c, 7, 0.0, 0.0);
        ctx->c.old_dt = ctx->c.dt;
        ++ctx->c.iteration;
        check_status(ctx->c);
    });
}

static const char* kKernelNames[] = {"cheb_synthesis", "post_assemble", "rlm_a",  "lt_inverse",
                                     "physics",        "lt_forward",    "rlm_b",  "solve"};

int ra_kernels_per_step(void) { return kNK; }
const char* ra_kernel_name(int i) { return (i >= 0 && i < kNK) ? kKernelNames[i] : nullptr; }

int ra_time_steps(ra_ctx* ctx, int nsteps, double* total_ms, double* kernel_ms, int nk) {
    if (!ctx || !ctx->c.have_state) return RA_ERR_STATE;
    if (nsteps <= 0 || !total_ms) return RA_ERR_ARG;
    return guarded(ctx, [&] {
        Ctx& c = ctx->c;
        c.launches = 0;
        std::vector<cudaEvent_t> ev((size_t)nsteps * (kNK + 1));
        for (auto& e : ev) RA_CUDA(cudaEventCreate(&e));
        try {
            for (int s = 0; s < nsteps; ++s) {
                double new_ab, old_ab;
                ab_factors(c, new_ab, old_ab);
                cudaEvent_t* E = ev.data() + (size_t)s * (kNK + 1);
                for (int k = 0; k < kNK; ++k) {
                    RA_CUDA(cudaEventRecord(E[k], c.stream));
                    run_stage(c, k, new_ab, old_ab);
                }
                RA_CUDA(cudaEventRecord(E[kNK], c.stream));
                c.old_dt = c.dt;
                ++c.iteration;
            }
            RA_CUDA(cudaStreamSynchronize(c.stream));
            check_status(c);
            float ms = 0.f;
            RA_CUDA(cudaEventElapsedTime(&ms, ev.front(), ev.back()));
            *total_ms = ms;
            if (kernel_ms) {
                for (int k = 0; k < nk && k < kNK; ++k) kernel_ms[k] = 0.0;
                for (int s = 0; s < nsteps; ++s) {
                    cudaEvent_t* E = ev.data() + (size_t)s * (kNK + 1);
                    for (int k = 0; k < nk && k < kNK; ++k) {
                        RA_CUDA(cudaEventElapsedTime(&ms, E[k], E[k + 1]));
                        kernel_ms[k] += ms;
                    }
                }
            }
        } catch (...) {
            for (auto& e : ev) cudaEventDestroy(e);
            throw;
        }
        for (auto& e : ev) cudaEventDestroy(e);
    });
}

int ra_sync(ra_ctx* ctx) {
    if (!ctx || ctx->c.d.L == 0) return RA_ERR_STATE;
    return guarded(ctx, [&] { RA_CUDA(cudaStreamSynchronize(ctx->c.stream)); });
}

long ra_launch_count(const ra_ctx* ctx) { return ctx ? ctx->c.launches : -1; }

int ra_debug_buffer(ra_ctx* ctx, int which, double* out, long n, long* n_out) {
    if (!ctx || ctx->c.d.L == 0) return RA_ERR_STATE;
    return guarded(ctx, [&] {
        Ctx& c = ctx->c;
        const long nlm = c.d.nlm, nr = c.d.nr, L = c.d.L, nth = c.d.nth;
        const double* src = nullptr;
        long size = 0;
        switch (which) {
            case RA_BUF_GRID: src = c.d_g; size = c.ng * nlm * 2 * nr; break;
            case RA_BUF_S2A: src = c.d_s2a; size = nlm * NS2A * 2 * nr; break;
            case RA_BUF_S2A11: src = c.d_s2a11; size = nlm * c.nfa * 2 * nr; break;
            case RA_BUF_P2A: src = c.d_p2a; size = L * nth * c.nfa * 2 * nr; break;
            case RA_BUF_P2B: src = c.d_p2b; size = L * nth * c.nfb * 2 * nr; break;
            case RA_BUF_S2B: src = c.d_s2b; size = nlm * c.nfb * 2 * nr; break;
            case RA_BUF_AB: src = c.d_ab; size = (c.mag ? 6 : 4) * nlm * 2 * nr; break;
            case RA_BUF_RHS_WPT: src = c.d_rhs_wpt; size = nlm * 2 * 3 * nr; break;
            case RA_BUF_RHS_Z: src = c.d_rhs_z; size = nlm * 2 * nr; break;
            case RA_BUF_PTAB: src = c.d_Ptab; size = nlm * c.d.nth2; break;
            case RA_BUF_IPTAB: src = c.d_iPtab; size = nlm * c.d.nth2; break;
            case RA_BUF_S2AM: src = c.d_s2am; size = c.mag ? nlm * NS2AM * 2 * nr : 0; break;
            case RA_BUF_RHS_C: src = c.d_rhs_c; size = c.mag ? nlm * 2 * nr : 0; break;
            case RA_BUF_RHS_A: src = c.d_rhs_a; size = c.mag ? nlm * 2 * nr : 0; break;
            default: throw ArgError("unknown buffer id");
        }
        if (!src) throw ArgError("this buffer exists only with magnetism");
        if (n_out) *n_out = size;
        if (!out) return;
        if (n < size) throw ArgError("output capacity too small");
        RA_CUDA(cudaMemcpyAsync(out, src, size * sizeof(double), cudaMemcpyDeviceToHost, c.stream));
        RA_CUDA(cudaStreamSynchronize(c.stream));
    });
}

int ra_radius(const ra_ctx* ctx, double* radius) {
    if (!ctx || ctx->c.d.L == 0 || !radius) return RA_ERR_ARG;
    std::copy(ctx->c.rad.radius.begin(), ctx->c.rad.radius.end(), radius);
    return RA_OK;
}

int ra_costheta(const ra_ctx* ctx, double* ct) {
    if (!ctx || ctx->c.d.L == 0 || !ct) return RA_ERR_ARG;
    std::copy(ctx->c.costheta_h.begin(), ctx->c.costheta_h.end(), ct);
    return RA_OK;
}

// ---- math-layer operators ----
int ra_legendre_s2p(ra_ctx* ctx, const double* s, double* p, int nf, int nr) {
    if (!ctx || ctx->c.d.L == 0) return RA_ERR_STATE;
    if (!s || !p || nf <= 0 || nr <= 0) return RA_ERR_ARG;
    return guarded(ctx, [&] {
        Ctx& c = ctx->c;
        const int L = c.d.L, nth = c.d.nth;
        const int ncol = nf * nr * 2;
        std::vector<double> hs((size_t)c.d.nlm * ncol), hp((size_t)L * nth * ncol);
        // host s: per m, Fortran (l, r, ri, f) -> device s2[row(m,l)][f][r][ri]
        size_t off = 0;
        for (int m = 0; m < L; ++m) {
            const int nl = L - m;
            for (int f = 0; f < nf; ++f)
                for (int ri = 0; ri < 2; ++ri)
                    for (int r = 0; r < nr; ++r)
                        for (int j = 0; j < nl; ++j)
                            hs[(size_t)row_index(m, m + j, L) * ncol + ((size_t)f * nr + r) * 2 + ri] =
                                s[off + (((size_t)f * 2 + ri) * nr + r) * nl + j];
            off += (size_t)nl * nr * 2 * nf;
        }
        double *ds = nullptr, *dp = nullptr;
        dalloc(ds, hs.size());
        dalloc(dp, hp.size());
        RA_CUDA(cudaMemcpyAsync(ds, hs.data(), hs.size() * sizeof(double), cudaMemcpyHostToDevice, c.stream));
        launch_lt_inverse(c, ds, dp, ncol);
        RA_CUDA(cudaMemcpyAsync(hp.data(), dp, hp.size() * sizeof(double), cudaMemcpyDeviceToHost, c.stream));
        RA_CUDA(cudaStreamSynchronize(c.stream));
        cudaFree(ds);
        cudaFree(dp);
        // device p2[th_h][m][par][f][r][ri] (E, O) -> host p2a(th, (r, ri, f), m):
        // south th_h: E + O, north nth-1-th_h: E - O (Legendre_Transforms.F90:1030-1064)
        const int nth2 = nth / 2;
        for (int m = 0; m < L; ++m)
            for (int f = 0; f < nf; ++f)
                for (int ri = 0; ri < 2; ++ri)
                    for (int r = 0; r < nr; ++r)
                        for (int th = 0; th < nth2; ++th) {
                            const size_t cidx = ((size_t)f * nr + r) * 2 + ri;
                            const double e = hp[(((size_t)th * L + m) * 2 + 0) * ncol + cidx];
                            const double o = hp[(((size_t)th * L + m) * 2 + 1) * ncol + cidx];
                            double* dst = p + ((((size_t)m * nf + f) * 2 + ri) * nr + r) * nth;
                            dst[th] = e + o;
                            dst[nth - 1 - th] = e - o;
                        }
    });
}

int ra_legendre_p2s(ra_ctx* ctx, const double* p, double* s, int nf, int nr) {
    if (!ctx || ctx->c.d.L == 0) return RA_ERR_STATE;
    if (!s || !p || nf <= 0 || nr <= 0) return RA_ERR_ARG;
    return guarded(ctx, [&] {
        Ctx& c = ctx->c;
        const int L = c.d.L, nth = c.d.nth;
        const int ncol = nf * nr * 2;
        std::vector<double> hs((size_t)c.d.nlm * ncol), hp((size_t)L * nth * ncol);
        // equatorial fold of PtS_4d_dgpv3 (Legendre_Transforms.F90:1109-1122) into p2[m][par][th_h][col]
        const int nth2 = nth / 2;
        for (int m = 0; m < L; ++m)
            for (int f = 0; f < nf; ++f)
                for (int ri = 0; ri < 2; ++ri)
                    for (int r = 0; r < nr; ++r)
                        for (int th = 0; th < nth2; ++th) {
                            const size_t cidx = ((size_t)f * nr + r) * 2 + ri;
                            const double* src = p + ((((size_t)m * nf + f) * 2 + ri) * nr + r) * nth;
                            hp[(((size_t)m * 2 + 0) * nth2 + th) * ncol + cidx] = src[th] + src[nth - 1 - th];
                            hp[(((size_t)m * 2 + 1) * nth2 + th) * ncol + cidx] = src[th] - src[nth - 1 - th];
                        }
        double *ds = nullptr, *dp = nullptr;
        dalloc(ds, hs.size());
        dalloc(dp, hp.size());
        RA_CUDA(cudaMemcpyAsync(dp, hp.data(), hp.size() * sizeof(double), cudaMemcpyHostToDevice, c.stream));
        launch_lt_forward(c, dp, ds, ncol);
        RA_CUDA(cudaMemcpyAsync(hs.data(), ds, hs.size() * sizeof(double), cudaMemcpyDeviceToHost, c.stream));
        RA_CUDA(cudaStreamSynchronize(c.stream));
        cudaFree(ds);
        cudaFree(dp);
        size_t off = 0;
        for (int m = 0; m < L; ++m) {
            const int nl = L - m;
            for (int f = 0; f < nf; ++f)
                for (int ri = 0; ri < 2; ++ri)
                    for (int r = 0; r < nr; ++r)
                        for (int j = 0; j < nl; ++j)
                            s[off + (((size_t)f * 2 + ri) * nr + r) * nl + j] =
                                hs[(size_t)row_index(m, m + j, L) * ncol + ((size_t)f * nr + r) * 2 + ri];
            off += (size_t)nl * nr * 2 * nf;
        }
    });
}

static int fft_op(ra_ctx* ctx, double* x, long howmany, int inverse) {
    if (!ctx || ctx->c.d.L == 0) return RA_ERR_STATE;
    if (!x || howmany <= 0) return RA_ERR_ARG;
    return guarded(ctx, [&] {
        Ctx& c = ctx->c;
        const size_t n = (size_t)howmany * (c.d.nphi + 2);
        double* dx = nullptr;
        dalloc(dx, n);
        RA_CUDA(cudaMemcpyAsync(dx, x, n * sizeof(double), cudaMemcpyHostToDevice, c.stream));
        launch_fft_rows(c, dx, howmany, inverse);
        RA_CUDA(cudaMemcpyAsync(x, dx, n * sizeof(double), cudaMemcpyDeviceToHost, c.stream));
        RA_CUDA(cudaStreamSynchronize(c.stream));
        cudaFree(dx);
    });
}

int ra_fft_c2r(ra_ctx* ctx, double* x, long howmany) { return fft_op(ctx, x, howmany, 1); }

int ra_transform_dev(ra_ctx* ctx, int direction, int precision, double* d_spec, double* d_grid, double* d_work,
                     int nfr, double* stage_ms) {
    if (!ctx || ctx->c.d.L == 0) return RA_ERR_STATE;
    if (!d_spec || !d_grid || !d_work || nfr <= 0 || (direction != 0 && direction != 1)) return RA_ERR_ARG;
    if (precision != RA_PREC_FP64 && precision != RA_PREC_MIXED) return RA_ERR_ARG;
    return guarded(ctx, [&] {
        Ctx& c = ctx->c;
        // the operands may have been written by work queued on the legacy default stream (where
        // frameworks queue by default); the context's non-blocking stream waits for it
        cudaEvent_t ready;
        RA_CUDA(cudaEventCreateWithFlags(&ready, cudaEventDisableTiming));
        RA_CUDA(cudaEventRecord(ready, cudaStreamLegacy));
        RA_CUDA(cudaStreamWaitEvent(c.stream, ready, 0));
        cudaEventDestroy(ready);
        RA_CUDA(cudaMemsetAsync(c.d_status, 0, sizeof(int), c.stream));
        transform_dev(c, direction, precision, d_spec, d_grid, d_work, nfr, stage_ms);
        check_status(c);
    });
}
int ra_fft_r2c(ra_ctx* ctx, double* x, long howmany) { return fft_op(ctx, x, howmany, 0); }

static int cheb_op(ra_ctx* ctx, const double* in, double* out, long ncols, int mode, int order) {
    if (!ctx || ctx->c.d.L == 0) return RA_ERR_STATE;
    if (!in || !out || ncols <= 0) return RA_ERR_ARG;
    if (mode == 2 && (order < 1 || order > 3)) return RA_ERR_ARG;
    return guarded(ctx, [&] {
        Ctx& c = ctx->c;
        if (!c.cfg.chebyshev)
            throw StateError("the Chebyshev operators need a context with chebyshev = 1 (finite differences hold "
                             "grid values: to_spectral and from_spectral are the identity)");
        const size_t n = (size_t)ncols * c.d.nr;
        double *di = nullptr, *dout = nullptr;
        dalloc(di, n);
        dalloc(dout, n);
        RA_CUDA(cudaMemcpyAsync(di, in, n * sizeof(double), cudaMemcpyHostToDevice, c.stream));
        launch_cheb_columns(c, di, dout, ncols, mode, order);
        RA_CUDA(cudaMemcpyAsync(out, dout, n * sizeof(double), cudaMemcpyDeviceToHost, c.stream));
        RA_CUDA(cudaStreamSynchronize(c.stream));
        cudaFree(di);
        cudaFree(dout);
    });
}

int ra_mixed_gemm(ra_ctx* ctx, const double* a, const double* b, double* cc, int m, int n, int k) {
    if (!ctx || ctx->c.d.L == 0) return RA_ERR_STATE;
    if (!a || !b || !cc || m <= 0 || n <= 0 || k <= 0) return RA_ERR_ARG;
    return guarded(ctx, [&] {
        if (k > OZ_MAX_K) throw ArgError("ra_mixed_gemm: k exceeds the exact int32 accumulation limit");
        Ctx& c = ctx->c;
        const int ntm = oz_tiles_of(m, OZ_HA), ntn = oz_tiles_of(n, OZ_HB), nks = oz_ksteps(k);
        double *da = nullptr, *db = nullptr, *dc = nullptr;
        int8_t *sa = nullptr, *sb = nullptr;
        int *ea = nullptr, *eb = nullptr, *dst = nullptr, *dtiles = nullptr;
        OzProblem* dprob = nullptr;
        OzSplitJob* djobs = nullptr;
        dalloc(da, (size_t)m * k);
        dalloc(db, (size_t)k * n);
        dalloc(dc, (size_t)m * n);
        dalloc(sa, (size_t)ntm * nks * OZ_ABLK);
        dalloc(sb, (size_t)ntn * nks * OZ_BBLK);
        dalloc(ea, (size_t)m);
        dalloc(eb, (size_t)n);
        dalloc(dst, 1);
        RA_CUDA(cudaMemsetAsync(dst, 0, sizeof(int), c.stream));
        RA_CUDA(cudaMemcpyAsync(da, a, (size_t)m * k * sizeof(double), cudaMemcpyHostToDevice, c.stream));
        RA_CUDA(cudaMemcpyAsync(db, b, (size_t)k * n * sizeof(double), cudaMemcpyHostToDevice, c.stream));
        // rows of A (k contiguous) and columns of B (rows of B^T, n apart)
        OzSplitJob jobs[2] = {{da, (long)k, 1L, m, k, OZ_HA, ntm, nks, sa, ea},
                              {db, 1L, (long)n, n, k, OZ_HB, ntn, nks, sb, eb}};
        dalloc(djobs, 2);
        RA_CUDA(cudaMemcpyAsync(djobs, jobs, sizeof(jobs), cudaMemcpyHostToDevice, c.stream));
        ozaki_split(c, djobs, 2, std::max(ntm * OZ_HA, ntn * OZ_HB));
        OzProblem pr{sa, sb, (long)nks * OZ_ABLK, (long)nks * OZ_BBLK, ea, eb, m, n, nks, dc, (long)n, 1L};
        std::vector<OzProblem> probs{pr};
        std::vector<int> tiles = ozaki_tiles(probs);
        dalloc(dprob, 1);
        dalloc(dtiles, tiles.size());
        RA_CUDA(cudaMemcpyAsync(dprob, probs.data(), sizeof(OzProblem), cudaMemcpyHostToDevice, c.stream));
        RA_CUDA(cudaMemcpyAsync(dtiles, tiles.data(), tiles.size() * sizeof(int), cudaMemcpyHostToDevice, c.stream));
        ozaki_gemm(c, dprob, dtiles, (int)(tiles.size() / 4), dst);
        int status = 0;
        RA_CUDA(cudaMemcpyAsync(cc, dc, (size_t)m * n * sizeof(double), cudaMemcpyDeviceToHost, c.stream));
        RA_CUDA(cudaMemcpyAsync(&status, dst, sizeof(int), cudaMemcpyDeviceToHost, c.stream));
        RA_CUDA(cudaStreamSynchronize(c.stream));
        cudaFree(da); cudaFree(db); cudaFree(dc); cudaFree(sa); cudaFree(sb);
        cudaFree(ea); cudaFree(eb); cudaFree(dst); cudaFree(dprob); cudaFree(dtiles); cudaFree(djobs);
        if (status) throw ArgError("tensor-core product timed out waiting on its pipeline barrier");
    });
}

int ra_cheby_to_spectral(ra_ctx* ctx, const double* f, double* cc, long ncols) { return cheb_op(ctx, f, cc, ncols, 0, 0); }
int ra_cheby_from_spectral(ra_ctx* ctx, const double* cc, double* f, long ncols) { return cheb_op(ctx, cc, f, ncols, 1, 0); }
int ra_cheby_deriv(ra_ctx* ctx, const double* cc, double* dc, int order, long ncols) {
    return cheb_op(ctx, cc, dc, ncols, 2, order);
}

}  // extern "C"
