"""NumPy/SciPy restatement of Rayleigh's timestep hot path (test infrastructure).

Every function cites the reference file:line it restates (paths inside the
geodynamics/Rayleigh 1.2.0 source tree).  Layouts follow the reference's
Fortran buffers, written here in C order with the axes reversed:

* ``p1`` (solve configuration, ``Spherical_Buffer.F90`` p1a/p1b):
  ``[field][lm][re/im][r]`` with the (l, m) pairs l-major, m ascending
  (``Load_Balance.F90:357-368``).
* ``s2`` (spectral, one array per m, ``s2a(mp)%data(m:l_max, r, imi, f)``):
  ``s2[m]`` has shape ``(nf, 2, n_r, l_max - m + 1)``.
* ``p2`` (hybrid, ``p2a(theta, nrhs, m)`` with nrhs = (r, imi, f)):
  ``[m][f][ri][r][theta]``.
* ``p3`` (physical, ``p3a(1:n_phi+2, r, theta, f)``): ``[f][theta][r][n_phi+2]``.

The REAL*16 parts of the reference (Gauss-Legendre roots, P_l^m recurrence)
are carried in ``numpy.longdouble`` (x86 80-bit), as the reference's own
NumPy port ``post_processing/spectral_utils.py:577-620,1887-2005`` does.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field, replace

import numpy as np
import scipy.linalg as sla

LD = np.longdouble
PI_LD = LD("3.14159265358979323846264338327950288")

# Field indices of the forward-leg buffers, 0-based restatement of
# Fields.F90:232-335 (no scalars); C and A follow Z when magnetism is on (:240-243).
WVAR, PVAR, TVAR, ZVAR, CVAR, AVAR = 0, 1, 2, 3, 4, 5
# equation ids (Fields.F90:86-88), 0-based
WEQ, PEQ, TEQ, ZEQ, CEQ, AEQ = 0, 1, 2, 3, 4, 5


@dataclass
class Config:
    """Problem description (restates the namelist values the path reads)."""

    n_r: int = 48
    l_max: int = 63
    n_theta: int = 0                 # 3(l_max+1)/2 when 0 (ProblemSize.F90:431-452)
    aspect_ratio: float = 0.35
    shell_depth: float = 1.0
    rayleigh: float = 1.0e5          # Rayleigh_Number (Ra/Pr is the buoyancy coefficient)
    ekman: float = 1.0e-3
    prandtl: float = 1.0
    magnetic_prandtl: float = 1.0
    gravity_power: float = 1.0
    rotation: bool = True
    magnetism: bool = False
    lorentz_forces: bool = True      # Controls.F90:63 (on whenever magnetism is on)
    momentum_advection: bool = True
    no_slip_top: bool = True
    no_slip_bottom: bool = True
    fix_tvar_top: bool = True
    fix_tvar_bottom: bool = True
    t_top: float = 0.0
    t_bottom: float = 1.0
    dtdr_top: float = 0.0
    dtdr_bottom: float = 0.0
    dt: float = 1.0e-4
    alpha_implicit: float = 0.5
    chebyshev: bool = True           # Numerical_Controls (Controls.F90): False = finite differences, uniform grid
    # Reference_Namelist (PDE_Coefficients.F90:84-160): 1 Constant_Reference (Boussinesq),
    # 2 Polytropic_Reference (dimensional, cgs), 3 Polytropic_ReferenceND
    reference_type: int = 1
    poly_n: float = 0.0
    poly_nrho: float = 0.0
    poly_mass: float = 0.0
    poly_rho_i: float = 0.0
    pressure_specific_heat: float = 1.0
    angular_velocity: float = -1.0
    modified_rayleigh: float = -1.0
    # Transport_Namelist (PDE_Coefficients.F90:186-207): type 1 constant, type 2
    # x_top (rho / rho_top)^power; the tops are read for reference_type 2 only
    nu_type: int = 1
    kappa_type: int = 1
    eta_type: int = 1
    nu_power: float = 0.0
    kappa_power: float = 0.0
    eta_power: float = 0.0
    nu_top: float = -1.0
    kappa_top: float = -1.0
    eta_top: float = -1.0
    # Controls.F90:64-65 (Constant_Reference turns both off)
    viscous_heating: bool = True
    ohmic_heating: bool = True

    def __post_init__(self):
        if self.n_theta <= 0:
            self.n_theta = (3 * (self.l_max + 1)) // 2
        if self.n_theta % 2:
            raise ValueError("n_theta must be even")
        if self.n_r % 2 and self.chebyshev:
            raise ValueError("n_r must be even (single Chebyshev domain, parity split)")

    @property
    def n_phi(self):
        return 2 * self.n_theta

    @property
    def n_m(self):
        return self.l_max + 1


# ---------------------------------------------------------------------------
# Horizontal grid: Gauss-Legendre nodes and P_l^m tables
# ---------------------------------------------------------------------------

def _nth_legendre(x, n):
    """Legendre_Polynomials.F90:377-393 (nth_legendre)."""
    pn = LD(1)
    pm1 = LD(0)
    for j in range(1, n + 1):
        pm2 = pm1
        pm1 = pn
        pn = ((LD(2 * j) - 1) * x * pm1 - (LD(j) - 1) * pm2) / LD(j)
    dpn = n * (x * pn - pm1) / (x * x - 1)
    return pn, dpn


def gauss_legendre(n, eps="3e-14"):
    """Find_Colocation (Legendre_Polynomials.F90:332-373): nodes ascending in (-1, 1).

    ``eps`` is the Newton stopping tolerance (3e-14 in the Fortran; the
    reference's NumPy port uses 3e-15).  The weight of each pass uses the
    derivative at the pre-update root, as the reference does, so the weights
    carry an O(eps) relative difference between the two.
    """
    x = np.zeros(n, dtype=LD)
    w = np.zeros(n, dtype=LD)
    eps = LD(eps)
    for i in range(1, (n + 1) // 2 + 1):
        root = np.cos(PI_LD * (LD(i) - LD("0.25")) / (LD(n) + LD("0.5")))
        while True:
            pn, dpn = _nth_legendre(root, n)
            new = root - pn / dpn
            delta = abs(root - new)
            root = new
            x[i - 1] = -root
            x[n - i] = root
            w[i - 1] = 2 / ((1 - root * root) * dpn * dpn)
            w[n - i] = w[i - 1]
            if delta <= eps:
                break
    return x, w


class Horizontal:
    """Gauss-Legendre grid plus parity-split P_l^m tables for one (l_max, n_theta)."""

    def __init__(self, l_max, n_theta, eps="3e-14"):
        self.l_max = l_max
        self.n_theta = n_theta
        self.n_phi = 2 * n_theta
        self.n_m = l_max + 1
        xq, wq = gauss_legendre(n_theta, eps)
        self.xq, self.wq = xq, wq
        self.costheta = xq.astype(np.float64)           # ProblemSize.F90:490
        self.sintheta = np.sqrt(1.0 - self.costheta ** 2)
        self.csctheta = 1.0 / self.sintheta
        self.cottheta = self.costheta / self.sintheta
        nth2 = n_theta // 2
        self.p_even, self.p_odd, self.ip_even, self.ip_odd = [], [], [], []
        self.l_even, self.l_odd = [], []
        x = xq[:nth2]
        renorm = 2 * PI_LD * wq[:nth2]
        for m in range(self.n_m):
            nl = l_max - m + 1
            pq = np.zeros((nl, nth2), dtype=LD)
            # closed form for l = m (Legendre_Polynomials.F90:190-212)
            ratio = LD(1)
            for i in range(1, m + 1):
                ratio = ratio * np.sqrt((LD(i) - LD("0.5")) / LD(i))
            amp = np.sqrt((LD(m) + LD("0.5")) / (2 * PI_LD)) * ratio
            tmp = 1 - x * x
            if m % 2 == 1:
                pq[0] = -amp * tmp ** (LD(m // 2) + LD("0.5"))
            else:
                pq[0] = amp * tmp ** LD(m // 2)
            if m < l_max:
                pq[1] = pq[0] * x * np.sqrt(LD(2 * m + 3))
            # three-term recurrence (Legendre_Polynomials.F90:215-226)
            for l in range(m + 2, l_max + 1):
                a = (LD(l - 1) ** 2 - LD(m * m)) / (4 * LD(l - 1) ** 2 - 1)
                a = np.sqrt(a)
                t = pq[l - 1 - m] * x - a * pq[l - 2 - m]
                b = (4 * LD(l) * LD(l) - 1) / (LD(l * l) - LD(m * m))
                pq[l - m] = t * np.sqrt(b)
            # the normalisations are double-precision literals stored into REAL*16 (:270-276)
            if m == 0:
                pts = LD(np.float64(1.0) / (2.0 * n_theta))
                stp = LD(1)
            else:
                pts = LD(np.float64(1.0) / n_theta)
                stp = LD("0.5")
            ev = pq[0::2]
            od = pq[1::2]
            self.l_even.append(np.arange(m, l_max + 1, 2))
            self.l_odd.append(np.arange(m + 1, l_max + 1, 2))
            self.p_even.append((ev * stp).astype(np.float64))
            self.p_odd.append((od * stp).astype(np.float64))
            self.ip_even.append(((ev * renorm) * pts).T.astype(np.float64).copy())
            self.ip_odd.append(((od * renorm) * pts).T.astype(np.float64).copy())
        # angular derivative coefficients (Spectral_Derivatives.F90:49-83)
        self.dcoef, self.sdcoef = [], []
        for m in range(self.n_m):
            ls = np.arange(m, l_max + 1, dtype=np.float64)
            num = (ls + m) * (ls - m)
            den = (2 * ls + 1) * (2 * ls - 1)
            c1 = np.sqrt(num / den)
            num2 = (ls + 1 + m) * (ls + 1 - m)
            den2 = (2 * ls + 1) * (2 * ls + 3)
            c2 = np.sqrt(num2 / den2)
            self.dcoef.append(((ls - 1) * c1, -(ls + 2) * c2))
            self.sdcoef.append(((ls + 1) * c1, -ls * c2))

    # ----- Legendre transforms (Legendre_Transforms.F90:968-1175) -----
    def s2p(self, s2, ms=None):
        """StP_4d_dgp2: spectral s2[m] (nf,2,nr,nl) -> p2 [m][nf][2][nr][theta].

        ``ms`` restricts the work to a subset of m (returns that many arrays)."""
        nth, nth2 = self.n_theta, self.n_theta // 2
        out = []
        for m in (range(self.n_m) if ms is None else ms):
            a = s2[m]
            nf, _, nr, nl = a.shape
            a2 = a.reshape(-1, nl).T           # (nl, nrhs)
            o = np.zeros((nth, a2.shape[1]))
            if len(self.l_even[m]):
                te = self.p_even[m].T @ a2[0::2]       # (nth2, nrhs) :1028
                o[:nth2] = te
                o[nth - 1:nth2 - 1:-1] = te             # reflect about the equator :1030-1036
            if len(self.l_odd[m]):
                to = self.p_odd[m].T @ a2[1::2]         # :1058
                o[:nth2] += to
                o[nth - 1:nth2 - 1:-1] -= to            # :1059-1064
            out.append(o.T.reshape(nf, 2, nr, nth))
        return out

    def p2s(self, p2, ms=None):
        """PtS_4d_dgpv3: p2 [m](nf,2,nr,theta) -> s2[m] (nf,2,nr,nl); ``ms`` as in s2p."""
        nth, nth2 = self.n_theta, self.n_theta // 2
        out = []
        for m in (range(self.n_m) if ms is None else ms):
            d = p2[m]
            nf, _, nr, _ = d.shape
            d2 = d.reshape(-1, nth).T          # (nth, nrhs)
            south = d2[:nth2]
            north = d2[nth - 1:nth2 - 1:-1]
            fe = south + north                 # :1109-1122
            fo = south - north
            nl = self.l_max - m + 1
            o = np.zeros((nl, d2.shape[1]))
            if len(self.l_even[m]):
                o[0::2] = self.ip_even[m].T @ fe   # :1130
            if len(self.l_odd[m]):
                o[1::2] = self.ip_odd[m].T @ fo    # :1150
            out.append(o.T.reshape(nf, 2, nr, nl))
        return out

    # ----- angular derivatives in (l, m) space -----
    def d_by_dtheta(self, a, m):
        """sin(theta) d/dtheta (Spectral_Derivatives.F90:329-350); a[..., l-m]."""
        return self._ell_couple(a, m, self.dcoef[m])

    def d_by_sdtheta(self, a, m):
        """(1/sin) d(sin^2 .)/dtheta (Spectral_Derivatives.F90:381-401)."""
        return self._ell_couple(a, m, self.sdcoef[m])

    def _ell_couple(self, a, m, coef):
        c1, c2 = coef
        out = np.zeros_like(a)
        if m == self.l_max:
            return out
        # interior l = m+1 .. lmax-1
        out[..., 1:-1] = a[..., 0:-2] * c1[1:-1] + a[..., 2:] * c2[1:-1]
        out[..., 0] = a[..., 1] * c2[0]
        out[..., -1] = a[..., -2] * c1[-1]
        return out

    @staticmethod
    def d_by_dphi(a, m):
        """d/dphi on (re, im) pairs (Spectral_Derivatives.F90:495-509); a[..., ri, r, l]."""
        out = np.empty_like(a)
        out[..., 0, :, :] = -m * a[..., 1, :, :]
        out[..., 1, :, :] = m * a[..., 0, :, :]
        return out


# ---------------------------------------------------------------------------
# FFT in phi (Fourier_Transform.F90:100-183): unnormalised, packed n+2 layout
# ---------------------------------------------------------------------------

# Threads of the phi FFTs: 1 (NumPy's FFT) by default; the CPU baseline sets the
# host's core count (SciPy's FFT with that many workers, the same transform).
FFT_WORKERS = 1


def set_fft_workers(n):
    """Threads for the phi FFTs (1 = NumPy's single-threaded FFT)."""
    global FFT_WORKERS
    FFT_WORKERS = max(1, int(n))


def _irfft(c, n):
    if FFT_WORKERS > 1:
        import scipy.fft
        return scipy.fft.irfft(c, n=n, axis=-1, workers=FFT_WORKERS)
    return np.fft.irfft(c, n=n, axis=-1)


def _rfft(x):
    if FFT_WORKERS > 1:
        import scipy.fft
        return scipy.fft.rfft(x, axis=-1, workers=FFT_WORKERS)
    return np.fft.rfft(x, axis=-1)


def fft_c2r(p3, n_phi):
    """c2r_ip4D_fftw: last axis (n_phi+2 packed re/im) -> n_phi real values (unnormalised)."""
    c = p3[..., 0::2] + 1j * p3[..., 1::2]
    y = _irfft(c, n_phi) * n_phi
    out = np.zeros_like(p3)
    out[..., :n_phi] = y
    return out


def fft_r2c(p3, n_phi):
    """r2c_ip4D_fftw: first n_phi real values -> packed spectrum (unnormalised)."""
    c = _rfft(p3[..., :n_phi])
    out = np.empty(p3.shape[:-1] + (n_phi + 2,))
    out[..., 0::2] = c.real
    out[..., 1::2] = c.imag
    return out


# ---------------------------------------------------------------------------
# Finite-difference radial grid (chebyshev = .false.): the uniform grid of
# Initialize_Radial_Grid (ProblemSize.F90:607-618) and the stencils of
# Finite_Difference.F90 (Initialize_Derivatives :69-93, Initialize_dcoefs
# :464-521, Generate_Coefs :525-689, with the default 5-point stencils and
# boundary accuracy 2).  The state holds grid values, so to_spectral,
# from_spectral and dealias are identities and a derivative is the banded
# matrix D_d applied along the radius (d_by_dx3d3 :374-460; the same rows
# Load_Interior_RowsFD / Load_Single_RowFD put in the implicit matrices, :717-866).
# ---------------------------------------------------------------------------
def fd_generate_coefs(grid, n_stencil, deriv_order, boundary_accuracy):
    """Generate_Coefs (transition type 1): coefs[n_stencil, ngrid] (0-based rows of the
    Fortran coefs(1:n_stencil, i)).  Interior points use the centred stencil clipped at the
    ends; the two end points one-sided stencils of deriv_order + boundary_accuracy points.
    Each stencil's weights are a row of the inverse of the Vandermonde matrix of the
    point offsets (scaled by their mean, rescaled after), times j!."""
    ngrid = len(grid)
    sr = n_stencil // 2
    sc = sr + 1                                              # stencil centre, 1-based
    coefs = np.zeros((n_stencil, ngrid))

    def weights(dees, dmean, nxy):
        temp = np.zeros((nxy, nxy))
        temp[:, 0] = 1.0
        for k in range(1, nxy):
            temp[:, k] = dees ** k
        inv = np.linalg.inv(temp)                            # dgetrf + dgetri
        jfact = 1.0
        for j in range(2, nxy + 1):                          # Fortran rows j = 2 .. nxy
            jfact = jfact * float(j - 1)
            inv[j - 1, :] = inv[j - 1, :] * jfact * (1.0 / dmean) ** (j - 1)
        return inv[deriv_order, :]

    for i in range(2, ngrid):                                # Fortran i = 2 .. ngrid - 1
        jstart = max(1, sc - i + 1)
        jend = min(n_stencil, (ngrid - i) + sc)
        nxy = jend - jstart + 1
        dees = np.zeros(n_stencil + 1)                       # 1-based
        dsum = 0.0
        for j in range(jstart, jend + 1):
            dees[j] = grid[i + j - sc - 1] - grid[i - 1]
            dsum = dsum + abs(dees[j])
        dees[sc] = 0.0
        dmean = dsum / float(nxy - 1)
        d = dees[jstart:jend + 1] / dmean
        coefs[jstart - 1:jend, i - 1] = weights(d, dmean, nxy)
    nxy = deriv_order + boundary_accuracy
    for this_pt, diff_dir in ((1, 1), (ngrid, -1)):
        dees = np.zeros(nxy)
        dsum = 0.0
        if diff_dir == 1:
            for j in range(2, nxy + 1):
                dees[j - 1] = grid[this_pt + j - 2] - grid[this_pt - 1]
                dsum = dsum + dees[j - 1]
        else:
            for j in range(1, nxy):
                dees[j - 1] = grid[this_pt + (j - nxy) - 1] - grid[this_pt - 1]
                dsum = dsum + dees[j - 1]
        dmean = dsum / float(nxy - 1)
        w = weights(dees / dmean, dmean, nxy)
        if diff_dir == 1:
            coefs[0:nxy, this_pt - 1] = w
        else:
            coefs[n_stencil - nxy:n_stencil, this_pt - 1] = w
    return coefs


class FiniteDifference:
    N_STENCIL = (5, 5, 5)          # n_stencil_1..3 (Finite_Difference.F90:10-12)
    BOUNDARY_ACCURACY = (2, 2, 2)  # boundary_accuracy_1..3 (:14-16)

    def __init__(self, n, rmin, rmax, dmax=3):
        self.n = n
        r = np.zeros(n)
        r[n - 1] = rmin
        dr = 1.0 / (n - 1.0) * (rmax - rmin)
        for i in range(n - 2, -1, -1):
            r[i] = dr + r[i + 1]
        self.radius = r
        self.delta_r = np.full(n, dr)
        ns = max(self.N_STENCIL)
        kd = (ns + 1) // 2
        d = np.zeros((dmax + 1, n, n))
        d[0] = np.eye(n)
        for dd in range(1, dmax + 1):
            st, ba = self.N_STENCIL[dd - 1], self.BOUNDARY_ACCURACY[dd - 1]
            c = fd_generate_coefs(r, st, dd, ba)
            off = (ns - st) // 2
            full = np.zeros((ns, n))
            full[off:ns - off, 1:n - 1] = c[:, 1:n - 1]
            full[0:st, 0] = c[:, 0]
            full[ns - st:ns, n - 1] = c[:, n - 1]
            nb = dd + ba
            m = np.zeros((n, n))
            m[0, 0:nb] = full[0:nb, 0]
            m[n - 1, n - nb:n] = full[ns - nb:ns, n - 1]
            for i in range(1, n - 1):                        # Fortran r = i + 1
                rr = i + 1
                kstart = max(1, kd - rr + 1)
                kend = min(st, (n - rr) + kd)
                for kk in range(kstart, kend + 1):
                    m[i, rr + kk - kd - 1] = full[kk - 1, i]
            d[dd] = m
        self.dcheby = d
        self.rda = n + 1           # every column of a boundary row (no dealiasing)
        # Initialize_Derivatives' integration weights: (r_{i-1} - r_{i+1}) / 2 r_i^2, normalised
        w = np.zeros(n)
        for i in range(1, n - 1):
            w[i] = (r[i - 1] - r[i + 1]) / 2.0 * r[i] ** 2
        w[0] = (r[0] - r[1]) / 2.0 * r[0] ** 2
        w[n - 1] = (r[n - 2] - r[n - 1]) / 2.0 * r[n - 1] ** 2
        self.integration_weights = w / w.sum()

    def to_spectral(self, f):
        return np.array(f, copy=True)

    def from_spectral(self, c):
        return np.array(c, copy=True)

    def dealias(self, c):
        return np.array(c, copy=True)

    def deriv(self, c, d):
        return np.einsum("rk,...k->...r", self.dcheby[d], c)


# ---------------------------------------------------------------------------
# Chebyshev grid (Chebyshev_Polynomials.F90:65-644), single domain
# ---------------------------------------------------------------------------

class Chebyshev:
    def __init__(self, n, rmin, rmax, dmax=3):
        self.n = n
        # Gen_Colocation_Points: zeros of T_N, theta accumulated by repeated addition (:233-244)
        dth = math.pi / n
        arg = dth * 0.5
        theta = np.zeros(n)
        for i in range(n):
            theta[i] = arg
            arg = arg + dth
        self.theta = theta
        x = np.cos(theta)
        self.x = x
        # Gen_Tn (:251-297)
        k = np.arange(n)
        cheby = np.cos(k[None, :] * theta[:, None])      # cheby(r, i) = cos((i-1) theta_r)
        n_odd = n // 2
        n_even = n_odd + n % 2
        self.n_even, self.n_odd = n_even, n_odd
        self.cheby_even = cheby[:n_even, 0::2].copy()     # (n_x, n_even)
        self.cheby_odd = cheby[:n_even, 1::2].copy()
        # Gen_Tn_Deriv_Arrays (:299-351)
        alpha = np.zeros((n, n))
        alpha[n - 2, n - 1] = 2.0 * (n - 1)
        for kk in range(n - 3, -1, -1):                   # Fortran k = N-2 .. 1
            alpha[kk, kk + 1] = 2.0 * (kk + 1)
            alpha[kk, :] = alpha[kk, :] + alpha[kk + 2, :]
        d = np.zeros((dmax + 1, n, n))
        d[0] = cheby.copy()
        d[0][:, 0] -= 0.5                                  # -c_0/2 of from_spectral (:332-333)
        for dd in range(1, dmax + 1):
            d[dd] = d[dd - 1] @ alpha
        # grid and scalings (Initialize_Cheby_Grid :168-200); bounds reversed: r(1) = rmax
        xmin, xmax = x[n - 1], x[0]
        delta = rmax - rmin
        scaling = delta / (xmax - xmin)
        self.radius = (x - xmin) * scaling + rmin
        inv = 1.0 / scaling
        for dd in range(1, dmax + 1):
            d[dd] = d[dd] * inv ** dd
        self.dcheby = d                                    # dcheby[d][r, n]
        self.deriv_scaling = inv
        self.rda = (2 * n) // 3 + 1                        # 1-based dealias index (:128)

    def dealias(self, c):
        """dealias_buffer4d (:353-374): zero coefficients rda..N (1-based) along the last axis."""
        c = c.copy()
        c[..., self.rda - 1:] = 0.0
        return c

    def to_spectral(self, f):
        """To_Spectral4D (:375-448): grid values (last axis r) -> coefficients."""
        n, nx = self.n, self.n_even
        alpha = 2.0 / n
        fe = f[..., :nx] + f[..., n - 1:n - 1 - nx:-1]
        fo = f[..., :nx] - f[..., n - 1:n - 1 - nx:-1]
        c = np.empty_like(f)
        c[..., 0::2] = alpha * (fe @ self.cheby_even)
        c[..., 1::2] = alpha * (fo @ self.cheby_odd)
        return c

    def from_spectral(self, c):
        """From_Spectral4D (:450-558): coefficients -> grid values (even N)."""
        n, nx = self.n, self.n_even
        fe = c[..., 0::2] @ self.cheby_even.T
        fo = c[..., 1::2] @ self.cheby_odd.T
        f = np.empty_like(c)
        f[..., :nx] = fe
        f[..., n - 1:n - 1 - nx:-1] = fe
        f[..., :nx] += fo
        f[..., n - 1:n - 1 - nx:-1] -= fo
        return f - c[..., 0:1] / 2.0

    def deriv(self, c, order):
        """Cheby_Deriv_Buffer_4D (:560-644): coefficient recursion, then scaling**order."""
        n = self.n
        cur = c
        for _ in range(order):
            d = np.zeros_like(cur)
            d[..., n - 2] = 2.0 * (n - 1) * cur[..., n - 1]
            for i in range(n - 3, -1, -1):
                d[..., i] = d[..., i + 2] + 2.0 * (i + 1) * cur[..., i + 1]
            cur = d
        return cur * self.deriv_scaling ** order


# ---------------------------------------------------------------------------
# The time stepper
# ---------------------------------------------------------------------------

def lm_pairs(l_max):
    """(l, m) ordering of the solve configuration (Load_Balance.F90:357-368)."""
    ls, ms = [], []
    for l in range(l_max + 1):
        for m in range(l + 1):
            ls.append(l)
            ms.append(m)
    return np.array(ls), np.array(ms)


class Oracle:
    """Rotating convection in a spherical shell, single Chebyshev domain, on a
    Boussinesq (reference_type 1) or anelastic polytropic (2 dimensional, 3
    nondimensional) reference state; with ``cfg.magnetism`` the dynamo equation
    set (poloidal C and toroidal A potentials of B, Lorentz force, induction by
    the EMF)."""

    NF1A = 8     # W P T Z W' T' Z' W''  (Fields.F90:244-252, aliases :317-335); + C A C' A' C'' with magnetism
    NF2A = 12    # + Br, (curl B)_r, (curl B)_theta, (curl B)_phi, B_theta, B_phi with magnetism
    NFB = 4      # + EMF_theta (C slot), EMF_r (A slot), EMF_phi with magnetism (Fields.F90:365-368)

    def __init__(self, cfg: Config, horizontal: Horizontal | None = None):
        self.mag = bool(cfg.magnetism)
        if self.mag:
            self.NF1A, self.NF2A, self.NFB = 13, 18, 7
        self.cfg = cfg
        self.h = horizontal if horizontal is not None else Horizontal(cfg.l_max, cfg.n_theta)
        rmax = cfg.shell_depth / (1.0 - cfg.aspect_ratio)
        rmin = rmax * cfg.aspect_ratio
        self.rmin, self.rmax = rmin, rmax
        self.cg = Chebyshev(cfg.n_r, rmin, rmax) if cfg.chebyshev else FiniteDifference(cfg.n_r, rmin, rmax)
        r = self.cg.radius
        self.radius = r
        nr = cfg.n_r
        if cfg.chebyshev:
            # Delta_r (ProblemSize.F90:541-549)
            dr = np.empty(nr)
            dr[0] = r[0] - r[1]
            dr[1:] = r[:-1] - r[1:]
        else:
            dr = self.cg.delta_r                               # uniform_dr (:611-613)
        self.delta_r = dr
        self._reference_state()
        self.ls, self.ms = lm_pairs(cfg.l_max)
        self.n_lm = len(self.ls)
        self.l_start = np.searchsorted(self.ls, np.arange(cfg.l_max + 1))
        # index maps between l-major lm and per-m blocks
        self.old_dt = cfg.dt
        self.dt = cfg.dt
        self.iteration = 1
        self._build_linear()
        self.last_cfl = 0.0
        self.bc_values = None   # None: the built-in boundary values (only l = 0 T carries one)

    # ----- reference state and transport coefficients (PDE_Coefficients.F90) -----
    def _reference_state(self):
        cfg, r, nr = self.cfg, self.radius, self.cfg.n_r
        rmin, rmax = self.rmin, self.rmax
        one = np.ones(nr)
        self.dsdr = np.zeros(nr)
        if cfg.reference_type == 1:
            # Constant_Reference (:335-435)
            self.density, self.dlnrho, self.d2lnrho = one.copy(), np.zeros(nr), np.zeros(nr)
            self.temperature, self.dlnT = one.copy(), np.zeros(nr)
            self.buoy = (cfg.rayleigh / cfg.prandtl) * (r / r[0]) ** cfg.gravity_power
            pscaling = 1.0 / cfg.ekman if cfg.rotation else 1.0
            self.coriolis = 2.0 / cfg.ekman
            nu_top, kappa_top = 1.0, 1.0 / cfg.prandtl
            self.viscous_amp = np.full(nr, 2.0)
            self.lorentz = 1.0 / (cfg.magnetic_prandtl * cfg.ekman) if self.mag else 0.0
            eta_top = 1.0 / cfg.magnetic_prandtl if self.mag else 0.0
            self.ohmic_amp = np.full(nr, self.lorentz)
            self.viscous_heating = self.ohmic_heating = False
        elif cfg.reference_type == 2:
            # Polytropic_Reference (:925-1051), cgs
            if cfg.poly_n <= 0 or cfg.poly_nrho <= 0 or cfg.poly_mass <= 0 or cfg.poly_rho_i <= 0:
                raise ValueError("reference_type 2 needs poly_n, poly_nrho, poly_mass, poly_rho_i > 0")
            G = 6.67e-8
            n = cfg.poly_n
            ri, ro = r[-1], r[0]
            beta = ri / ro
            zeta0 = (beta + 1.0) / (beta * math.exp(cfg.poly_nrho / n) + 1.0)
            c0 = (2.0 * zeta0 - beta - 1.0) / (1.0 - beta)
            c1 = (1.0 + beta) * (1.0 - zeta0) / (1.0 - beta) ** 2
            d = ro - ri
            zeta = c0 + c1 * d / r
            dlnzeta = -c1 * d / r ** 2 / zeta
            rho_c = cfg.poly_rho_i / zeta[-1] ** n
            P_c = G * cfg.poly_mass * rho_c / ((n + 1.0) * d * c1)
            T_c = (n + 1.0) * P_c / (cfg.pressure_specific_heat * rho_c)
            gravity = G * cfg.poly_mass / r ** 2
            self.density = rho_c * zeta ** n
            self.dlnrho = -n * c1 * d / (zeta * r ** 2)
            self.d2lnrho = -self.dlnrho * (2.0 / r - c1 * d / zeta / r ** 2)
            self.temperature = T_c * zeta
            self.dlnT = dlnzeta
            self.buoy = gravity / cfg.pressure_specific_heat * self.density
            pscaling = 1.0
            self.coriolis = 2.0 * cfg.angular_velocity
            nu_top, kappa_top, eta_top = cfg.nu_top, cfg.kappa_top, cfg.eta_top
            self.viscous_amp = 2.0 / self.temperature
            self.lorentz = 1.0 / (4.0 * math.pi) if self.mag else 0.0
            self.ohmic_amp = self.lorentz / self.density / self.temperature
            self.viscous_heating, self.ohmic_heating = cfg.viscous_heating, cfg.ohmic_heating
        elif cfg.reference_type == 3:
            # Polytropic_ReferenceND (:437-537)
            if cfg.poly_n <= 0 or cfg.poly_nrho <= 0:
                raise ValueError("reference_type 3 needs poly_n, poly_nrho > 0")
            n = cfg.poly_n
            beta = cfg.aspect_ratio
            diss = beta * (math.exp(cfg.poly_nrho / n) - 1.0)
            dtmp = 1.0 / (1.0 - beta)
            self.temperature = dtmp * diss * (dtmp / r - 1.0) + 1.0
            self.density = self.temperature ** n
            gravity = rmax ** 2 / r ** 2
            self.buoy = gravity * cfg.modified_rayleigh * self.density
            self.dlnT = -diss * gravity / self.temperature
            self.dlnrho = n * self.dlnT
            self.d2lnrho = -n * self.dlnT ** 2 + (n / self.temperature) * (2.0 * diss * gravity / r)
            pscaling = 1.0
            self.coriolis = 2.0
            nu_top, kappa_top = cfg.ekman, cfg.ekman / cfg.prandtl
            self.viscous_amp = 2.0 / self.temperature * diss / cfg.modified_rayleigh
            if self.mag:
                self.lorentz = cfg.ekman / cfg.magnetic_prandtl
                eta_top = cfg.ekman / cfg.magnetic_prandtl
                otmp = diss * cfg.ekman ** 2 / (cfg.modified_rayleigh * cfg.magnetic_prandtl ** 2)
                self.ohmic_amp = otmp / self.density / self.temperature
            else:
                self.lorentz, eta_top, self.ohmic_amp = 0.0, 0.0, np.zeros(nr)
            self.viscous_heating, self.ohmic_heating = cfg.viscous_heating, cfg.ohmic_heating
        else:
            raise ValueError(f"reference_type {cfg.reference_type} is not restated (1, 2, 3)")
        if not self.mag:
            eta_top = 0.0
        self.dpdr_w_term = self.density * pscaling
        self.pressure_dwdr_term = -1.0 * self.density * pscaling

        # Initialize_Diffusivity / Vary_With_Density (:1906-1981)
        def diffusivity(top, kind, power):
            if kind == 1:
                return np.full(nr, top), np.zeros(nr)
            if kind == 2:
                return top * (self.density / self.density[0]) ** power, power * self.dlnrho
            raise ValueError(f"transport type {kind} is not restated (1, 2)")
        self.nu, self.dlnu = diffusivity(nu_top, cfg.nu_type, cfg.nu_power)
        self.kappa, self.dlnkappa = diffusivity(kappa_top, cfg.kappa_type, cfg.kappa_power)
        if self.mag:
            self.eta, self.dlneta = diffusivity(eta_top, cfg.eta_type, cfg.eta_power)
        else:
            self.eta, self.dlneta = np.zeros(nr), np.zeros(nr)
        # Initialize_Transport_Coefficients (:1822-1836)
        self.viscous_heating_coeff = self.viscous_amp * self.nu if self.viscous_heating else None
        self.ohmic_heating_coeff = (self.ohmic_amp * self.eta if (self.mag and self.ohmic_heating) else None)
        # Compute_Diffusion_Coefs (:2032-2098)
        nu, dlnu, dlnrho, d2lnrho = self.nu, self.dlnu, self.dlnrho, self.d2lnrho
        self.w_diff0 = -nu * (4.0 / 3.0) * (dlnu * dlnrho + d2lnrho + dlnrho / r + 3.0 * dlnu / r)
        self.w_diff1 = nu * (2.0 * dlnu - dlnrho / 3.0)
        self.dw_diff2 = (dlnu - dlnrho) * nu
        self.dw_diff1 = -(d2lnrho + 2.0 / r * dlnrho + 2.0 / r * dlnu + dlnu * dlnrho) * nu
        self.dw_diff0 = -(2.0 * dlnrho / 3.0 + dlnu) * nu
        self.s_diff1 = self.kappa * (self.dlnkappa + dlnrho + self.dlnT)
        self.z_diff0 = -nu * (2.0 * dlnu / r + dlnrho * dlnu + d2lnrho + 2.0 * dlnrho / r)
        self.z_diff1 = nu * (dlnu - dlnrho)
        self.a_diff1 = self.eta * self.dlneta
        r_out, r_in = r[0], r[-1]
        pref = r_out * r_in / (r_in - r_out)
        self.s_conductive = pref * (1.0 / r_out - 1.0 / r)

    # ----- linear system (Sphere_Linear_Terms.F90:79-537, Linear_Solve.F90:494-539) -----
    def _build_linear(self):
        cfg, nr, cg = self.cfg, self.cfg.n_r, self.cg
        r = self.radius
        dt, a = self.dt, cfg.alpha_implicit
        lf = -dt * a
        rf = dt * (1.0 - a)
        D = cg.dcheby
        rda = cg.rda
        self.coefs = []     # per l: dict (eq, var, d) -> vector(r)
        self.lu_wpt = []
        self.lu_z = []
        self.mat_wpt = []
        self.mat_z = []
        self.mat_c, self.mat_a, self.lu_c, self.lu_a = [], [], [], []
        over_r2 = 1.0 / r ** 2
        for l in range(cfg.l_max + 1):
            coefs = {}
            A = np.zeros((3 * nr, 3 * nr))
            Z = np.zeros((nr, nr))
            Cm = np.zeros((nr, nr))
            Am = np.zeros((nr, nr))
            blk = {WEQ: 0, PEQ: nr, TEQ: 2 * nr, WVAR: 0, PVAR: nr, TVAR: 2 * nr}

            def add(eq, var, d, amp, static=False, mat=None, rb=None, cb=None):
                key = (eq, var, d)
                coefs[key] = coefs.get(key, 0.0) + (amp if static else amp * rf)
                fac = amp if static else amp * lf
                mm = A if mat is None else mat
                r0 = blk[eq] if rb is None else rb
                c0 = blk[var] if cb is None else cb
                mm[r0:r0 + nr, c0:c0 + nr] += fac[:, None] * D[d]      # Load_Interior_Rows_Cheby

            ones = np.ones(nr)
            H = -l * (l + 1) * over_r2
            if l == 0:
                add(TEQ, TVAR, 0, ones, static=True)
                add(TEQ, TVAR, 1, 2.0 / r * self.kappa)
                add(TEQ, TVAR, 2, 1.0 * self.kappa)
                add(TEQ, TVAR, 1, self.s_diff1)            # S_Diffusion_Coefs_1
                add(PEQ, TVAR, 0, -self.buoy, static=True)
                add(PEQ, PVAR, 1, self.dpdr_w_term, static=True)
                add(WEQ, WVAR, 0, ones, static=True)
            else:
                add(WEQ, TVAR, 0, -self.buoy / H)
                add(WEQ, PVAR, 1, self.dpdr_w_term / H)
                add(WEQ, WVAR, 0, ones, static=True)
                add(WEQ, WVAR, 0, H * self.nu)
                add(WEQ, WVAR, 2, self.nu)
                add(WEQ, WVAR, 0, self.w_diff0)            # W_Diffusion_Coefs_0
                add(WEQ, WVAR, 1, self.w_diff1)            # W_Diffusion_Coefs_1
                add(PEQ, PVAR, 0, self.pressure_dwdr_term)
                add(PEQ, WVAR, 1, ones, static=True)
                add(PEQ, WVAR, 0, -self.nu * H * 2.0 / r)
                add(PEQ, WVAR, 1, H * self.nu)
                add(PEQ, WVAR, 3, self.nu)
                add(PEQ, WVAR, 0, self.dw_diff0 * H)       # dW_Diffusion_Coefs_0*H
                add(PEQ, WVAR, 1, self.dw_diff1)
                add(PEQ, WVAR, 2, self.dw_diff2)
                add(TEQ, TVAR, 0, ones, static=True)
                add(TEQ, TVAR, 0, H * self.kappa)
                add(TEQ, TVAR, 1, 2.0 / r * self.kappa)
                add(TEQ, TVAR, 2, self.kappa)
                add(TEQ, TVAR, 1, self.s_diff1)
                add(ZEQ, ZVAR, 0, ones, static=True, mat=Z, rb=0, cb=0)
                add(ZEQ, ZVAR, 0, H * self.nu, mat=Z, rb=0, cb=0)
                add(ZEQ, ZVAR, 2, self.nu, mat=Z, rb=0, cb=0)
                add(ZEQ, ZVAR, 0, self.z_diff0, mat=Z, rb=0, cb=0)
                add(ZEQ, ZVAR, 1, self.z_diff1, mat=Z, rb=0, cb=0)
                if self.mag:
                    # Btor (A) and Bpol (C) equations (Sphere_Linear_Terms.F90:473-499)
                    blk[AEQ] = blk[AVAR] = 0
                    blk[CEQ] = blk[CVAR] = 0
                    add(AEQ, AVAR, 0, ones, static=True, mat=Am)
                    add(AEQ, AVAR, 0, H * self.eta, mat=Am)
                    add(AEQ, AVAR, 2, self.eta, mat=Am)
                    add(AEQ, AVAR, 1, self.a_diff1, mat=Am)    # A_Diffusion_Coefs_1
                    add(CEQ, CVAR, 0, ones, static=True, mat=Cm)
                    add(CEQ, CVAR, 0, H * self.eta, mat=Cm)
                    add(CEQ, CVAR, 2, self.eta, mat=Cm)
            # Set_Boundary_Conditions (Sphere_Linear_Terms.F90:539-1100)
            def bc(mat, row, col0, d, amp):
                # Load_Single_Row_Cheby (Linear_Solve.F90:1483-1522): dealiased columns only
                mat[row, col0:col0 + rda - 1] += amp * D[d][row % nr, :rda - 1]

            top, bot = 0, nr - 1
            if l == 0:
                A[nr + top, :] = 0.0
                A[2 * nr + top, :] = 0.0
                A[2 * nr + bot, :] = 0.0
                if cfg.fix_tvar_top:
                    bc(A, 2 * nr + top, 2 * nr, 0, 1.0)
                else:
                    bc(A, 2 * nr + top, 2 * nr, 1, 1.0)
                if cfg.fix_tvar_bottom:
                    bc(A, 2 * nr + bot, 2 * nr, 0, 1.0)
                else:
                    bc(A, 2 * nr + bot, 2 * nr, 1, 1.0)
                bc(A, nr + top, nr, 0, 1.0)                  # pressure node at the top
            else:
                for rb in (0, nr, 2 * nr):
                    A[rb + top, :] = 0.0
                    A[rb + bot, :] = 0.0
                Z[top, :] = 0.0
                Z[bot, :] = 0.0
                if cfg.fix_tvar_top:
                    bc(A, 2 * nr + top, 2 * nr, 0, 1.0)
                else:
                    bc(A, 2 * nr + top, 2 * nr, 1, 1.0)
                if cfg.fix_tvar_bottom:
                    bc(A, 2 * nr + bot, 2 * nr, 0, 1.0)
                else:
                    bc(A, 2 * nr + bot, 2 * nr, 1, 1.0)
                bc(A, top, 0, 0, 1.0)                       # impenetrable
                bc(A, bot, 0, 0, 1.0)
                if cfg.no_slip_top:
                    bc(Z, top, 0, 0, 1.0)
                    bc(A, nr + top, 0, 1, 1.0)
                else:
                    samp = -(2.0 / r[top] + self.dlnrho[top])
                    bc(A, nr + top, 0, 2, 1.0)
                    bc(A, nr + top, 0, 1, samp)
                    bc(Z, top, 0, 1, 1.0)
                    bc(Z, top, 0, 0, samp)
                if cfg.no_slip_bottom:
                    bc(A, nr + bot, 0, 1, 1.0)
                    bc(Z, bot, 0, 0, 1.0)
                else:
                    samp = -(2.0 / r[bot] + self.dlnrho[bot])
                    bc(A, nr + bot, 0, 2, 1.0)
                    bc(A, nr + bot, 0, 1, samp)
                    bc(Z, bot, 0, 1, 1.0)
                    bc(Z, bot, 0, 0, samp)
                if self.mag:
                    # insulating boundaries (:1041-1077): A = 0; C matched to a potential field,
                    # dC/dr + l C / r = 0 at the top, dC/dr - (l + 1) C / r = 0 at the bottom
                    for mm in (Cm, Am):
                        mm[top, :] = 0.0
                        mm[bot, :] = 0.0
                    bc(Am, top, 0, 0, 1.0)
                    bc(Am, bot, 0, 0, 1.0)
                    bc(Cm, top, 0, 1, 1.0)
                    bc(Cm, top, 0, 0, l / r[top])
                    bc(Cm, bot, 0, 1, 1.0)
                    bc(Cm, bot, 0, 0, -(l + 1) / r[bot])
            self.coefs.append(coefs)
            self.mat_wpt.append(A)
            self.mat_z.append(Z)
            # LU_Decompose_full -> DGETRF (Linear_Solve.F90:1028-1036)
            self.lu_wpt.append(sla.lu_factor(A, check_finite=False))
            self.lu_z.append(sla.lu_factor(Z, check_finite=False) if l > 0 else None)
            if self.mag:
                self.mat_c.append(Cm)
                self.mat_a.append(Am)
                self.lu_c.append(sla.lu_factor(Cm, check_finite=False) if l > 0 else None)
                self.lu_a.append(sla.lu_factor(Am, check_finite=False) if l > 0 else None)
        # bc_values (BoundaryConditions.F90:364-402): only l=0 T rows carry values
        self.bc_t = (cfg.t_top * math.sqrt(4 * math.pi) if cfg.fix_tvar_top else cfg.dtdr_top * math.sqrt(4 * math.pi),
                     cfg.t_bottom * math.sqrt(4 * math.pi) if cfg.fix_tvar_bottom else cfg.dtdr_bottom * math.sqrt(4 * math.pi))

    def set_dt(self, dt):
        """Reset_Linear_Equations (Sphere_Linear_Terms.F90:67-76) for a new dt."""
        self.dt = dt
        self._build_linear()

    # ----- state -----
    def init_state(self, wpt_coeffs, z_coeffs, ab=None, c_coeffs=None, a_coeffs=None):
        """State in the equation-set RHS layout: wpt[lm, ri, 3nr], z[lm, ri, nr] (Chebyshev coefficients);
        with magnetism also c[lm, ri, nr], a[lm, ri, nr] (zero when None) and ab[6] (W P T Z C A)."""
        nr = self.cfg.n_r
        self.rhs_wpt = np.array(wpt_coeffs, dtype=np.float64).reshape(self.n_lm, 2, 3 * nr)
        self.rhs_z = np.array(z_coeffs, dtype=np.float64).reshape(self.n_lm, 2, nr)
        nab = 6 if self.mag else 4
        self.ab = np.zeros((nab, self.n_lm, 2, nr)) if ab is None else np.array(ab, dtype=np.float64)
        if self.mag:
            z0 = np.zeros((self.n_lm, 2, nr))
            self.rhs_c = z0.copy() if c_coeffs is None else np.array(c_coeffs, dtype=np.float64).reshape(z0.shape)
            self.rhs_a = z0.copy() if a_coeffs is None else np.array(a_coeffs, dtype=np.float64).reshape(z0.shape)

    def get_all_rhs(self):
        """Get_All_RHS (Linear_Solve.F90:691-711) -> p1 [f][lm][ri][r] for W P T Z (C A)."""
        nr = self.cfg.n_r
        p = np.empty((6 if self.mag else 4, self.n_lm, 2, nr))
        p[WVAR] = self.rhs_wpt[:, :, 0:nr]
        p[PVAR] = self.rhs_wpt[:, :, nr:2 * nr]
        p[TVAR] = self.rhs_wpt[:, :, 2 * nr:3 * nr]
        p[ZVAR] = self.rhs_z
        if self.mag:
            p[CVAR] = self.rhs_c
            p[AVAR] = self.rhs_a
        return p

    def _coef(self, l, eq, var, d):
        return self.coefs[l].get((eq, var, d))

    def _add_derivative(self, addto, eq, var, d, dfield):
        """Add_Derivative (Linear_Solve.F90:758-796): addto[eq] += coef(r) * dfield per l block."""
        for l in range(self.cfg.l_max + 1):
            c = self._coef(l, eq, var, d)
            if c is None:
                continue
            s, e = self.l_start[l], self.l_start[l] + l + 1
            addto[eq, s:e] += dfield[s:e] * c

    # ----- the five stages of one step (Sphere_Driver.F90:305-328) -----
    def post_solve(self):
        """Sphere_Spectral_Space.F90:178-413 (Chebyshev branch; the finite-difference branch
        Post_Solve_FD :37-176 is the same with identity transforms and the deriv_cluge),
        ending with Transpose_1a2a."""
        cg = self.cg
        if self.iteration == 1:
            self.new_ab, self.old_ab = self.dt, 0.0
        else:
            self.new_ab = 0.5 * self.dt * (2 + self.dt / self.old_dt)
            self.old_ab = -0.5 * self.dt ** 2 / self.old_dt
        p1b = self.ab * self.old_ab
        c = cg.dealias(self.get_all_rhs())                    # :217-221
        W, P, T, Z = c[WVAR], c[PVAR], c[TVAR], c[ZVAR]
        d3w = cg.deriv(W, 3)
        dw = cg.deriv(W, 1)
        d2w = cg.deriv(W, 2)
        dp = cg.deriv(P, 1)
        d2t = cg.deriv(T, 2)
        dt_ = cg.deriv(T, 1)
        d2z = cg.deriv(Z, 2)
        dz = cg.deriv(Z, 1)
        ct = [d3w, dp, d2t, d2z]
        gl = [W, P, T, Z, dw, dt_, dz, d2w]
        if self.mag:                                           # :268-274
            C, A = c[CVAR], c[AVAR]
            ct.append(cg.deriv(A, 2))
            gl += [C, A, cg.deriv(C, 1), cg.deriv(A, 1), cg.deriv(C, 2)]
        ctemp = cg.from_spectral(cg.dealias(np.stack(ct)))    # :277-283
        self._add_derivative(p1b, PEQ, WVAR, 3, ctemp[0])
        self._add_derivative(p1b, WEQ, PVAR, 1, ctemp[1])
        self._add_derivative(p1b, TEQ, TVAR, 2, ctemp[2])
        self._add_derivative(p1b, ZEQ, ZVAR, 2, ctemp[3])
        if self.mag:
            self._add_derivative(p1b, AEQ, AVAR, 2, ctemp[4])  # :295-297
        g = cg.from_spectral(cg.dealias(np.stack(gl)))         # :301-309
        Wg, Pg, Tg, Zg, dWg, dTg, dZg, d2Wg = g[:8]
        self.last_pressure_grids = np.stack([Pg, ctemp[1]])   # P and dP/dr, for pressure_fields
        self._add_derivative(p1b, PEQ, WVAR, 0, Wg)
        self._add_derivative(p1b, PEQ, WVAR, 1, dWg)
        self._add_derivative(p1b, PEQ, WVAR, 2, d2Wg)
        self._add_derivative(p1b, WEQ, WVAR, 0, Wg)
        self._add_derivative(p1b, WEQ, WVAR, 1, dWg)
        self._add_derivative(p1b, WEQ, WVAR, 2, d2Wg)
        self._add_derivative(p1b, PEQ, PVAR, 0, Pg)
        self._add_derivative(p1b, TEQ, TVAR, 1, dTg)
        self._add_derivative(p1b, TEQ, TVAR, 0, Tg)
        self._add_derivative(p1b, WEQ, TVAR, 0, Tg)
        self._add_derivative(p1b, ZEQ, ZVAR, 0, Zg)
        self._add_derivative(p1b, ZEQ, ZVAR, 1, dZg)
        if not self.cfg.chebyshev:
            # Post_Solve_FD's deriv_cluge (Sphere_Spectral_Space.F90:96-98, Controls.F90:44): the
            # d2W/dr2 that goes on to rlm_spacea is d/dr of dW/dr
            g = g.copy()
            g[7] = cg.deriv(dWg, 1)
        if self.mag:                                            # :370-384
            Cg, Ag, dCg, dAg, d2Cg = g[8:13]
            self._add_derivative(p1b, AEQ, AVAR, 0, Ag)
            self._add_derivative(p1b, AEQ, AVAR, 1, dAg)
            self._add_derivative(p1b, CEQ, CVAR, 2, d2Cg)
            self._add_derivative(p1b, CEQ, CVAR, 0, Cg)
        self._set_all_rhs(p1b)                                  # :391
        return g                                                # p1a grid fields (8; 13 with magnetism)

    def _set_all_rhs(self, p1b):
        nr = self.cfg.n_r
        self.rhs_wpt[:, :, 0:nr] = p1b[WEQ]
        self.rhs_wpt[:, :, nr:2 * nr] = p1b[PEQ]
        self.rhs_wpt[:, :, 2 * nr:3 * nr] = p1b[TEQ]
        self.rhs_z[:] = p1b[ZEQ]
        if self.mag:
            self.rhs_c[:] = p1b[CEQ]
            self.rhs_a[:] = p1b[AEQ]

    def transpose_1a2a(self, p1):
        """Transpose_1a2a (Spherical_Buffer.F90:849-949): p1[f][lm][ri][r] -> s2[m](f,2,r,l)."""
        nf = p1.shape[0]
        L = self.cfg.l_max
        s2 = []
        for m in range(L + 1):
            idx = self.l_start[m:] + m            # lm index of (l, m) for l = m..L
            s2.append(np.ascontiguousarray(p1[:, idx].transpose(0, 2, 3, 1)))
        return s2

    def transpose_2b1b(self, s2):
        """Transpose_2b1b (Spherical_Buffer.F90:705-847): s2[m](f,2,r,l) -> p1[f][lm][ri][r]."""
        nf = s2[0].shape[0]
        L = self.cfg.l_max
        p1 = np.empty((nf, self.n_lm, 2, self.cfg.n_r))
        for m in range(L + 1):
            idx = self.l_start[m:] + m
            p1[:, idx] = s2[m].transpose(0, 3, 1, 2)
        return p1

    def rlm_spacea(self, s2, ms=None):
        """Sphere_Hybrid_Space.F90:64-125 (hydro): 8 fields -> 12 fields, then StP."""
        h, L = self.h, self.cfg.l_max
        r = self.radius
        over_rhorsq = (1.0 / r ** 2 / self.density)[:, None]
        over_rhor = (1.0 / r / self.density)[:, None]
        drho = (self.dlnrho + 1.0 / r)[:, None]
        two_over_r = (2.0 / r)[:, None]
        out = []
        for m in (range(L + 1) if ms is None else ms):
            a = s2[m].copy()
            a[..., -1] = 0.0                                          # zero l_max (:73-75)
            ls = np.arange(m, L + 1, dtype=np.float64)
            llp1 = ls * (ls + 1)
            W, P, T, Z = a[0], a[1], a[2], a[3]
            dW, dT, dZ, d2W = a[4], a[5], a[6], a[7]
            b = np.zeros((self.NF2A,) + W.shape)
            vr = llp1 * W * over_rhorsq                               # Velocity_Components :246-248
            vt = (h.d_by_dtheta(dW, m) + h.d_by_dphi(Z[None], m)[0]) * over_rhor
            vp = (h.d_by_dphi(dW[None], m)[0] - h.d_by_dtheta(Z, m)) * over_rhor
            dvtdr = (h.d_by_dtheta(d2W, m) + h.d_by_dphi(dZ[None], m)[0]) * over_rhor
            dvtdr = dvtdr - vt * drho                                  # :295-297
            dvpdr = (h.d_by_dphi(d2W[None], m)[0] - h.d_by_dtheta(dZ, m)) * over_rhor
            dvpdr = dvpdr - vp * drho
            dvrdr = llp1 * dW * over_rhorsq
            dvrdr = dvrdr - vr * two_over_r
            dvrdr = dvrdr - vr * self.dlnrho[:, None]
            dvrdt = h.d_by_dtheta(vr, m)
            omr = llp1 * Z * over_rhorsq
            dtdt = h.d_by_dtheta(T, m)
            b[0] = vr            # vr   (wvar)
            b[1] = P             # pvar
            b[2] = T             # tvar
            b[3] = omr           # zvar -> omega_r
            b[4] = dvrdr         # dwdr slot
            b[5] = dT            # dtdr
            b[6] = dvrdt         # dzdr slot
            b[7] = dtdt          # d2wdr2 slot
            b[8] = vt
            b[9] = vp
            b[10] = dvtdr
            b[11] = dvpdr
            if self.mag:
                # Compute_BandCurlB (Sphere_Hybrid_Space.F90:357-435), each times r sin(theta)
                # except B_r and (curl B)_r
                C, A, dC, dA, d2C = a[8], a[9], a[10], a[11], a[12]
                over_rsq = (1.0 / r ** 2)[:, None]
                br = llp1 * C * over_rsq
                x = d2C - br
                b[12] = br
                b[13] = llp1 * A * over_rsq                           # (curl B)_r
                b[14] = h.d_by_dtheta(dA, m) - h.d_by_dphi(x[None], m)[0]   # (curl B)_theta
                b[15] = h.d_by_dphi(dA[None], m)[0] + h.d_by_dtheta(x, m)   # (curl B)_phi
                b[16] = h.d_by_dphi(A[None], m)[0] + h.d_by_dtheta(dC, m)   # B_theta
                b[17] = h.d_by_dphi(dC[None], m)[0] - h.d_by_dtheta(A, m)   # B_phi
            b[..., -1] = 0.0                                          # :100-102
            out.append(b)
        return out

    def physical_space(self, p3, thetas=None, diagnostics=True):
        """Sphere_Physical_Space.F90:98-224 (hydro): p3a (18 fields) -> p3b (4 fields) + CFL.

        ``thetas`` (index array) says which theta rows p3 holds (all when None).
        ``diagnostics=False`` skips what only the diagnostics read (the pressure
        and its phi derivative on the grid, the copy of every grid field)."""
        cfg, h = self.cfg, self.h
        th = slice(None) if thetas is None else np.asarray(thetas)
        nphi = cfg.n_phi
        L = cfg.l_max
        # Phi_Derivatives (:745-759) in packed m-space
        mvec = np.repeat(np.arange(nphi // 2 + 1), 2).astype(np.float64)
        def dphi(a):
            o = np.empty_like(a)
            o[..., 0::2] = -mvec[0::2] * a[..., 1::2]
            o[..., 1::2] = mvec[1::2] * a[..., 0::2]
            return o
        f = {}
        names = ["vr", "p", "t", "omr", "dvrdr", "dtdr", "dvrdt", "dtdt", "vt", "vp", "dvtdr", "dvpdr"]
        if self.mag:
            names += ["br", "curlbr", "curlbt", "curlbp", "bt", "bp"]
        for i, n in enumerate(names):
            f[n] = p3[i]
        f["dvrdp"] = dphi(f["vr"])
        f["dvtdp"] = dphi(f["vt"])
        f["dvpdp"] = dphi(f["vp"])
        f["dtdp"] = dphi(f["t"])
        if diagnostics:
            f["dpdp"] = dphi(f["p"])     # the diagnostics' pressure_dphi (only read by them)
        else:
            del f["p"]
        for k in list(f.keys()):
            f[k] = fft_c2r(f[k], nphi)[..., :nphi]
        csc = h.csctheta[th][:, None, None]
        cot = h.cottheta[th][:, None, None]
        sin = h.sintheta[th][:, None, None]
        cos = h.costheta[th][:, None, None]
        for k in ("vt", "vp", "dvtdr", "dvpdr", "dtdt", "dvrdt", "dvpdp", "dvtdp"):
            f[k] = f[k] * csc                                          # sintheta_div (:119-126)
        if self.mag:
            orad = (1.0 / self.radius)[None, :, None]
            for k in ("curlbt", "curlbp", "bt", "bp"):
                f[k] = f[k] * csc * orad                               # rsintheta_div (:142-147)
            self.last_magnetic = (f["br"], f["bt"], f["bp"], th)
        # the velocity and temperature Benchmark_Checkup reads at this point of the step (:158-159)
        self.last_velocity = (f["vr"], f["vt"], f["vp"], th)
        self.last_temperature = f["t"]
        if diagnostics:
            self.last_fields = dict(f)   # every physical-space field, [theta, r, phi]: the diagnostics' buffer
        r = self.radius[None, :, None]
        dlnrho = self.dlnrho[None, :, None]
        one_over_r = 1.0 / r
        r2 = r * r
        rho = self.density[None, :, None]
        # CFL (Find_MyMinDT :784-813)
        llp1max = L * (L + 1.0)
        ovht2 = (np.max(f["vt"] ** 2 + f["vp"] ** 2, axis=(0, 2)) / self.radius ** 2 * llp1max)
        ovrt2 = np.max(f["vr"] ** 2, axis=(0, 2)) / self.delta_r ** 2
        cfl = max(ovht2.max(), ovrt2.max(), 0.0)
        if self.mag:   # the Alfven speed (:798-806)
            ovht2 = (np.max(f["bt"] ** 2 + f["bp"] ** 2, axis=(0, 2)) / self.radius ** 2 * llp1max
                     / self.density * self.lorentz)
            ovrt2 = np.max(f["br"] ** 2, axis=(0, 2)) / self.delta_r ** 2 / self.density * self.lorentz
            cfl = max(cfl, ovht2.max(), ovrt2.max())
        self.last_cfl = float(cfl)
        vr, vt, vp = f["vr"], f["vt"], f["vp"]
        out = np.zeros((self.NFB,) + vr.shape)
        lorentz = self.mag and cfg.lorentz_forces
        # Temperature_Advection (:303-318)
        out[TVAR] = -vr * f["dtdr"] - one_over_r * (f["dtdt"] * vt + vp * f["dtdp"] * csc)
        if self.viscous_heating_coeff is not None:
            # Compute_Viscous_Heating (:337-443) with the colatitude derivatives of
            # Compute_dvtheta_by_dtheta / Compute_dvphi_by_dtheta (:226-248)
            dvpdp, dvtdp = f["dvpdp"], f["dvtdp"]
            dvtdt = -vr * (r * dlnrho + 2.0) - r * f["dvrdr"] - vt * cot - dvpdp * csc
            dvpdt = r * f["omr"] + dvtdp * csc - vp * cot
            tmp = (dvpdp * csc + vr + vt * cot) * one_over_r          # e_phi_phi
            tmp2 = (dvtdt + vr) * one_over_r                          # e_theta_theta
            ht = f["dvrdr"] * f["dvrdr"] + tmp * tmp + tmp2 * tmp2
            tmp = (f["dvrdp"] * csc - vp) * one_over_r + f["dvpdr"]   # 2 e_r_phi
            ht = ht + tmp * tmp * 0.5
            tmp = (f["dvrdt"] - vt) * one_over_r + f["dvtdr"]         # 2 e_r_theta
            ht = ht + tmp * tmp * 0.5
            tmp = (dvpdt + dvtdp * csc - vp * cot) * one_over_r       # 2 e_phi_theta
            ht = ht + tmp * tmp * 0.5
            tmp = -vr * dlnrho                                        # div u
            ht = ht - tmp * tmp * (1.0 / 3.0)
            out[TVAR] = out[TVAR] + self.viscous_heating_coeff[None, :, None] * ht
        # Momentum_Advection_Radial (:466-529)
        w = -vr * f["dvrdr"] * r2 - vt * (f["dvrdt"] - vt) * r - vp * (f["dvrdp"] * csc - vp) * r
        if cfg.rotation:
            w = w + self.coriolis * sin * vp * r2
        out[WVAR] = w * rho
        if lorentz:   # r^2 [J x B]_r (:512-519)
            out[WVAR] = out[WVAR] + r2 * self.lorentz * (f["curlbt"] * f["bp"] - f["curlbp"] * f["bt"])
        # Momentum_Advection_Theta (:583-645)
        pth = f["dvrdr"] + (f["dvpdp"] * csc + vt * cot + vr) * one_over_r + vr * dlnrho
        pth = -pth * vt + vr * f["dvtdr"] + vp * (f["dvtdp"] * csc - vp * cot) * one_over_r
        if cfg.rotation:
            pth = pth - self.coriolis * cos * vp
        pth = pth * rho
        if lorentz:   # -[J x B]_theta (:635-641)
            pth = pth - self.lorentz * (f["curlbp"] * f["br"] - f["curlbr"] * f["bp"])
        out[PVAR] = pth * r * csc
        # Momentum_Advection_Phi (:648-700)
        z = vt * (f["omr"] + f["dvtdp"] * csc * one_over_r) + vr * f["dvpdr"] + vp * (f["dvpdp"] * csc + vr) * one_over_r
        if cfg.rotation:
            z = z + self.coriolis * cos * vt + self.coriolis * sin * vr
        z = z * rho
        if lorentz:   # -[J x B]_phi (:712-718)
            z = z - self.lorentz * (f["curlbr"] * f["bt"] - f["curlbt"] * f["br"])
        out[ZVAR] = z * r * csc
        if self.ohmic_heating_coeff is not None:   # Compute_Ohmic_Heating (:446-466)
            out[TVAR] = out[TVAR] + (f["curlbr"] * f["curlbr"] + f["curlbt"] * f["curlbt"]
                                     + f["curlbp"] * f["curlbp"]) * self.ohmic_heating_coeff[None, :, None]
        if self.mag:
            # Compute_EMF (:534-581): u x B; the theta and phi parts times r / sin(theta)
            br, bt, bp = f["br"], f["bt"], f["bp"]
            out[4] = (-vr * bp + vp * br) * csc * r      # emftheta (C slot)
            out[5] = vt * bp - vp * bt                   # emfr (A slot)
            out[6] = (vr * bt - vt * br) * csc * r       # emfphi
        pad = np.zeros(out.shape[:-1] + (nphi + 2,))
        pad[..., :nphi] = out
        return fft_r2c(pad, nphi)

    def transpose_2a3a(self, p2):
        """Transpose_2a3a (Spherical_Buffer.F90:196-316): p2[m](f,2,r,theta) -> p3[f][theta][r][nphi+2]."""
        nf, _, nr, nth = p2[0].shape
        P = np.stack(p2, axis=0)                       # (m, f, 2, r, th)
        p3 = np.zeros((nf, nth, nr, self.cfg.n_phi + 2))
        M = P.shape[0]
        p3[..., 0:2 * M:2] = P[:, :, 0].transpose(1, 3, 2, 0)
        p3[..., 1:2 * M:2] = P[:, :, 1].transpose(1, 3, 2, 0)
        return p3

    def transpose_3b2b(self, p3):
        """Transpose_3b2b (Spherical_Buffer.F90:461-581): m > l_max discarded."""
        M = self.cfg.l_max + 1
        re = p3[..., 0:2 * M:2]          # (f, th, r, m)
        im = p3[..., 1:2 * M:2]
        P = np.stack([re, im], axis=0).transpose(4, 1, 0, 3, 2)   # (m, f, 2, r, th)
        return [np.ascontiguousarray(P[m]) for m in range(M)]

    def rlm_spaceb(self, s2, ms=None):
        """Sphere_Hybrid_Space.F90:127-222 (hydro): curl algebra on the NL terms."""
        h, L = self.h, self.cfg.l_max
        out = []
        for m in (range(L + 1) if ms is None else ms):
            a = s2[m].copy()
            ls = np.arange(m, L + 1, dtype=np.float64)
            ollp1 = np.zeros_like(ls)
            ollp1[ls > 0] = 1.0 / (ls[ls > 0] * (ls[ls > 0] + 1))
            ollp1[ls == 0] = 1.0                              # over_l_l_plus1(0) = 1 (ProblemSize.F90:506)
            a[WVAR] = a[WVAR] * ollp1
            ft1 = h.d_by_sdtheta(a[ZVAR], m)
            ft2 = h.d_by_dphi(a[PVAR][None], m)[0]
            ft1 = (ft2 - ft1) * ollp1
            ft2 = h.d_by_dphi(a[ZVAR][None], m)[0]
            zsd = h.d_by_sdtheta(a[PVAR], m)
            a[PVAR] = (zsd + ft2) * ollp1
            a[ZVAR] = ft1
            if m == 0:
                a[PVAR][..., 0] = 0.0
                a[WVAR][..., 0] = 0.0
                a[ZVAR][..., 0] = 0.0
            if self.mag:
                # Adjust_Emf (:557-602): C RHS from the radial curl of the EMF in the C slot;
                # the A slot keeps EMF_r; slot 7 the term Finalize_EMF differentiates in r
                ft1 = h.d_by_sdtheta(a[6], m)
                ft2 = h.d_by_dphi(a[4][None], m)[0]
                ft3 = a[4].copy()
                a[4] = (ft1 - ft2) * ollp1
                ft2 = h.d_by_dphi(a[6][None], m)[0]
                a[6] = ft3
                ft1 = h.d_by_sdtheta(a[6], m)
                a[6] = (ft2 + ft1) * ollp1
            a[..., -1] = 0.0
            out.append(a)
        return out

    def advance_time(self, p1b_new, ls=None):
        """AdvanceTime (Sphere_Spectral_Space.F90:415-435): add AB term, BCs, solve (``ls``: subset of l)."""
        nr = self.cfg.n_r
        if self.mag:
            # Finalize_EMF (:436-488), Chebyshev branch: A RHS += d/dr of slot 7 (grid ->
            # coefficients -> derivative -> dealias -> grid)
            cg = self.cg
            dx = cg.from_spectral(cg.dealias(cg.deriv(cg.to_spectral(p1b_new[6]), 1)))
            p1b_new = p1b_new[:6].copy()
            p1b_new[AEQ] = p1b_new[AEQ] + dx
        self.ab = p1b_new
        nab = self.new_ab
        self.rhs_wpt[:, :, 0:nr] += nab * p1b_new[WEQ]
        self.rhs_wpt[:, :, nr:2 * nr] += nab * p1b_new[PEQ]
        self.rhs_wpt[:, :, 2 * nr:3 * nr] += nab * p1b_new[TEQ]
        self.rhs_z += nab * p1b_new[ZEQ]
        if self.mag:
            self.rhs_c += nab * p1b_new[CEQ]
            self.rhs_a += nab * p1b_new[AEQ]
            for arr in (self.rhs_c, self.rhs_a):     # the magnetic boundary values are zero
                arr[:, :, 0] = 0.0
                arr[:, :, nr - 1] = 0.0
        # Apply_Boundary_Mask (Linear_Solve.F90:401-418)
        for b in (0, nr, 2 * nr):
            self.rhs_wpt[:, :, b] = 0.0
            self.rhs_wpt[:, :, b + nr - 1] = 0.0
        self.rhs_z[:, :, 0] = 0.0
        self.rhs_z[:, :, nr - 1] = 0.0
        if self.bc_values is None:
            self.rhs_wpt[0, 0, 2 * nr] = self.bc_t[0]          # l=0, m=0, real, top
            self.rhs_wpt[0, 0, 3 * nr - 1] = self.bc_t[1]
        else:
            # bc_values(top/bottom, re/im, lm, eq) (BoundaryConditions.F90:364-531), here [eq][lm][ri][tb]
            bv = self.bc_values
            for eq, (arr, b) in enumerate(((self.rhs_wpt, 0), (self.rhs_wpt, nr), (self.rhs_wpt, 2 * nr),
                                           (self.rhs_z, 0))):
                arr[:, :, b] = bv[eq, :, :, 0]
                arr[:, :, b + nr - 1] = bv[eq, :, :, 1]
        # Implicit_Solve -> DGETRS (Linear_Solve.F90:423-457,1088-1110)
        for l in (range(self.cfg.l_max + 1) if ls is None else ls):
            s, e = self.l_start[l], self.l_start[l] + l + 1
            b = self.rhs_wpt[s:e].reshape(-1, 3 * nr).T
            x = sla.lu_solve(self.lu_wpt[l], b, check_finite=False)
            self.rhs_wpt[s:e] = x.T.reshape(e - s, 2, 3 * nr)
            if l > 0:
                bz = self.rhs_z[s:e].reshape(-1, nr).T
                xz = sla.lu_solve(self.lu_z[l], bz, check_finite=False)
                self.rhs_z[s:e] = xz.T.reshape(e - s, 2, nr)
                if self.mag:
                    for arr, lu in ((self.rhs_c, self.lu_c[l]), (self.rhs_a, self.lu_a[l])):
                        x = sla.lu_solve(lu, arr[s:e].reshape(-1, nr).T, check_finite=False)
                        arr[s:e] = x.T.reshape(e - s, 2, nr)

    # ----- the reference's accuracy benchmark (Christensen et al. 2001, case 0) -----
    def benchmark_init_hydro(self):
        """Benchmark_Init_Hydro (Initial_Conditions.F90:731-787): W = P = Z = 0;
        T(l=0) = sqrt(4 pi) (r_o r_i / r - r_i) and the real part of T(l=4, m=4) =
        0.2 (1 - 3x^2 + 3x^4 - x^6), x = 2r - r_i - r_o, on the collocation grid,
        then To_Spectral.  Returns (wpt, z) in the init_state layout."""
        nr, L = self.cfg.n_r, self.cfg.l_max
        r = self.radius
        ri, ro = self.rmin, self.rmax
        x = 2.0 * r - ri - ro
        grid = np.zeros((self.n_lm, 2, nr))
        grid[0, 0, :] = (ro * ri / r - ri) * math.sqrt(4.0 * math.pi)
        if L >= 4:
            grid[4 * 5 // 2 + 4, 0, :] = 0.2 * (1.0 - 3.0 * x * x + 3.0 * x ** 4 - x ** 6)
        wpt = np.zeros((self.n_lm, 2, 3 * nr))
        wpt[:, :, 2 * nr:] = self.cg.to_spectral(grid)
        return wpt, np.zeros((self.n_lm, 2, nr))

    def abenchmark_init_hydro(self, temp_amp=1.0):
        """ABenchmark_Init_Hydro (Initial_Conditions.F90:789-879), init_type 6 of the Jones et al.
        (2011) anelastic benchmark: W = P = Z = 0; on the collocation grid the l = 0 entropy
        Delta_S (zeta_o^-n - zeta^-n) / (zeta_o^-n - zeta_i^-n) sqrt(4 pi) with Delta_S = t_bottom,
        zeta = c0 + c1 d / r of the n = 2, N_rho = 5 polytrope, and the real parts of
        S(19, 19) = temp_amp (1 - cos(2 pi (r - r_i) / d)) and S(1, 1) = 0.1 of that; then
        To_Spectral.  Returns (wpt, z) in the init_state layout."""
        nr = self.cfg.n_r
        r = self.radius
        d = r[0] - r[-1]
        beta = r[-1] / r[0]
        n_rho, bm_n = 5.0, 2.0
        zeta0 = (beta + 1.0) / (beta * math.exp(n_rho / bm_n) + 1.0)
        c0 = (2.0 * zeta0 - beta - 1.0) / (1.0 - beta)
        c1 = (1.0 + beta) * (1.0 - zeta0) / (1.0 - beta) ** 2
        zeta = c0 + c1 * d / r
        ee = -bm_n
        denom = zeta[0] ** ee - zeta[-1] ** ee
        rfunc2 = self.cfg.t_bottom * (zeta[0] ** ee - zeta ** ee) / denom
        rfunc1 = (1.0 - np.cos(2.0 * math.pi / d * (r - r[-1]))) * temp_amp
        grid = np.zeros((self.n_lm, 2, nr))
        grid[0, 0, :] = rfunc2 * math.sqrt(4.0 * math.pi)
        if self.cfg.l_max >= 19:
            grid[19 * 20 // 2 + 19, 0, :] = rfunc1
        grid[1 * 2 // 2 + 1, 0, :] = rfunc1 * 0.1
        wpt = np.zeros((self.n_lm, 2, 3 * nr))
        wpt[:, :, 2 * nr:] = self.cg.to_spectral(grid)
        return wpt, np.zeros((self.n_lm, 2, nr))

    def benchmark_mean_flow_energies(self, avr, avt, avp):
        """Benchmark_Checkup's zonal and meridional kinetic energies (Benchmarking.F90:658-687):
        0.5 rho <v_phi>^2 and 0.5 rho (<v_r>^2 + <v_theta>^2) of the phi means <.>, given as
        [theta, r] arrays, averaged over theta (Gauss-Legendre weights / 2) and radius (the
        radial integration weights) as the kinetic energy is."""
        tw = (self.h.wq / 2.0).astype(np.float64)
        w = self.radial_integration_weights()
        rho = self.density[None, :]
        zonal = 0.5 * rho * avp * avp
        merid = 0.5 * rho * (avr * avr + avt * avt)
        return (float(np.dot(w, np.einsum("t,tr->r", tw, zonal))),
                float(np.dot(w, np.einsum("t,tr->r", tw, merid))))

    def benchmark_insulating_init(self):
        """Benchmark_Insulating_Init (Initial_Conditions.F90:1011-1073): on the collocation grid
        C(l=1, m=0) = (8 r_o - 6 r - 2 r_i^4 / r^3) (5/8) sqrt(pi/3) r^2 and
        A(l=2, m=0) = sin(pi (r - r_i)) r sqrt(pi/5) (4/3) 5 (real parts), then To_Spectral.
        Returns (c, a) in the init_state layout."""
        nr = self.cfg.n_r
        r = self.radius
        ri, ro = self.rmin, self.rmax
        nrm2 = math.sqrt(math.pi / 5.0) * (4.0 / 3.0) * 5.0
        nrm1 = (5.0 / 8.0) * math.sqrt(math.pi / 3.0)
        rf1 = 8.0 * ro - 6.0 * r
        rf1 = rf1 - 2.0 * (ri ** 4) / (r ** 3)
        rf1 = rf1 * nrm1 * r ** 2
        rf2 = np.sin(math.pi * (r - ri)) * r * nrm2
        gc = np.zeros((self.n_lm, 2, nr))
        ga = np.zeros((self.n_lm, 2, nr))
        gc[1, 0, :] = rf1                  # lm(1, 0) = 1
        if self.cfg.l_max >= 2:
            ga[3, 0, :] = rf2              # lm(2, 0) = 3
        return self.cg.to_spectral(gc), self.cg.to_spectral(ga)

    def benchmark_magnetic_energy(self):
        """Benchmark_Checkup's magnetic energy (Benchmarking.F90:689-696, 846) of the field
        the last step's physical-space stage formed: |B|^2 averaged as the kinetic energy,
        times mag_factor = 1 / (2 Ek Pm)."""
        br, bt, bp, th = self.last_magnetic
        if not (isinstance(th, slice) and th == slice(None)):
            raise ValueError("the last physical-space stage did not cover every theta row")
        q = bp * bp + br * br + bt * bt
        tw = (self.h.wq / 2.0).astype(np.float64)
        ell0 = np.einsum("t,tr->r", tw, q.mean(axis=2))
        return float(np.dot(self.radial_integration_weights(), ell0)) / (2.0 * self.cfg.ekman *
                                                                           self.cfg.magnetic_prandtl)

    def radial_integration_weights(self):
        """Initialize_Cheby_Grid's integration_weights (Chebyshev_Polynomials.F90:165-194):
        3 pi scaling / ((r_o^3 - r_i^3) N) r^2 sqrt(1 - x^2), halved at the two end
        points; they sum to ~1 (a volume average over the shell)."""
        cg, n = self.cg, self.cfg.n_r
        if not self.cfg.chebyshev:   # finite differences: Initialize_Derivatives (Finite_Difference.F90:69-93)
            return cg.integration_weights.copy()
        scaling = (self.rmax - self.rmin) / (cg.x[0] - cg.x[n - 1])
        int_scale = 3.0 * math.pi * scaling / ((self.rmax ** 3 - self.rmin ** 3) * n)
        w = int_scale * self.radius ** 2 * np.sqrt(1.0 - cg.x * cg.x)
        w[0] *= 0.5
        w[n - 1] *= 0.5
        return w

    def benchmark_kinetic_energy(self):
        """Benchmark_Checkup's kinetic energy (Benchmarking.F90:645-656, 733-736) of the
        velocity the last step's physical-space stage formed: 0.5 rho |u|^2 averaged
        over phi, over theta with the Gauss-Legendre weights / 2 (ComputeEll0,
        Spherical_IO.F90:1350-1391) and over radius with the radial integration
        weights (Compute_Radial_Average, :1436-1470)."""
        vr, vt, vp, th = self.last_velocity
        if not (isinstance(th, slice) and th == slice(None)):
            raise ValueError("the last physical-space stage did not cover every theta row")
        q = 0.5 * self.density[None, :, None] * (vr * vr + vt * vt + vp * vp)   # [theta, r, phi]
        tw = (self.h.wq / 2.0).astype(np.float64)
        ell0 = np.einsum("t,tr->r", tw, q.mean(axis=2))
        return float(np.dot(self.radial_integration_weights(), ell0))

    def pressure_fields(self):
        """dP/dr and dP/dtheta on the physical grid for the state the last step started from
        (the diagnostics' pressure_dr and pressure_dtheta,
        Diagnostics_Thermodynamic_Gradients.F90:197-223): Post_Solve's P and dP/dr grids
        through Transpose_1a2a, l_max zeroed as rlm_spacea does (Sphere_Hybrid_Space.F90:73-75),
        d/dtheta as for dT/dtheta (sin(theta) d/dtheta in (l, m), then 1/sin(theta)), StP and
        the c2r.  Returns {"dpdr", "dpdt"} as [theta, r, phi]."""
        h = self.h
        b = []
        for m, a in enumerate(self.transpose_1a2a(self.last_pressure_grids)):   # [m](2, 2, r, l)
            a = a.copy()
            a[..., -1] = 0.0
            b.append(np.stack([a[1], h.d_by_dtheta(a[0], m)]))
        p3 = self.transpose_2a3a(h.s2p(b))
        nphi = self.cfg.n_phi
        return {"dpdr": fft_c2r(p3[0], nphi)[..., :nphi],
                "dpdt": fft_c2r(p3[1], nphi)[..., :nphi] * h.csctheta[:, None, None]}

    def shell_averages(self, names):
        """Shell_Averages (Spherical_IO.F90 Add_Quantity :548-575 with ComputeEll0
        :1350-1391) of the last physical-space stage's fields (keys of last_fields): per
        radius the mean over phi and over theta with the Gauss-Legendre weights / 2, and
        the same average of (q - mean)^m for m = 2, 3, 4.  Returns [len(names), 4, n_r]."""
        th = self.last_velocity[3]
        if not (isinstance(th, slice) and th == slice(None)):
            raise ValueError("the last physical-space stage did not cover every theta row")
        tw = (self.h.wq / 2.0).astype(np.float64)
        out = np.zeros((len(names), 4, self.cfg.n_r))
        for i, name in enumerate(names):
            q = self.last_fields[name]                      # [theta, r, phi]
            mean = np.einsum("t,tr->r", tw, q.mean(axis=2))
            out[i, 0] = mean
            d = q - mean[None, :, None]
            for m in (2, 3, 4):
                out[i, m - 1] = np.einsum("t,tr->r", tw, (d ** m).mean(axis=2))
        return out

    def shell_spectra(self, names, levels):
        """Shell_Spectra (Parallel_IO.F90 Spectral_Prep :973-1047) of the last physical-space
        stage's fields at the radial indices ``levels``: the unnormalised r2c along phi
        (FFT_To_Spectral) and PtS_4d_dgpv3.  Returns [len(names), len(levels), 2, L, L] as
        [re/im][m][l], zero for l < m."""
        th = self.last_velocity[3]
        if not (isinstance(th, slice) and th == slice(None)):
            raise ValueError("the last physical-space stage did not cover every theta row")
        L = self.cfg.l_max + 1
        lv = list(levels)
        out = np.zeros((len(names), len(lv), 2, L, L))
        for i, name in enumerate(names):
            q = self.last_fields[name][:, lv, :]              # [theta, level, phi]
            X = np.fft.rfft(q, axis=2)                         # unnormalised, like FFTW's r2c
            p2 = [np.stack([X[:, :, m].real.T, X[:, :, m].imag.T])[None] for m in range(L)]   # (1, 2, nlev, theta)
            s2 = self.h.p2s(p2)
            for m in range(L):
                out[i, :, :, m, m:] = s2[m][0].transpose(1, 0, 2)   # (2, nlev, nl) -> (nlev, 2, nl)
        return out

    def benchmark_point_observations(self, msymm=4, fields=None, btheta=None):
        """Assemble_Strips and Point_Observations (Benchmarking.F90:934-1063) on the last
        physical-space stage, or on ``fields`` = (v_r, v_phi, T) given as [theta, r, phi]
        arrays: the phi strips of v_r, v_phi and T at the two radii that straddle
        mid-depth (n_r/2, n_r/2 + 1) and the two colatitudes that straddle the equator,
        averaged; at the first msymm points (in phi order, starting across the wrap)
        where v_r changes sign upwards, v_phi and T are interpolated linearly and
        averaged.  Returns (v_phi, T); with ``btheta`` (True: the last stage's B_theta, or a
        [theta, r, phi] array) the fourth observation of the magnetic case (Benchmarking.F90:
        1017-1063, nobs = 4) as well: (v_phi, T, B_theta)."""
        if fields is None:
            vr, vt, vp, th = self.last_velocity
            if not (isinstance(th, slice) and th == slice(None)):
                raise ValueError("the last physical-space stage did not cover every theta row")
            temperature = self.last_temperature
        else:
            vr, vp, temperature = fields
        nth, nr, nphi = self.cfg.n_theta, self.cfg.n_r, self.cfg.n_phi
        t1, t2 = nth // 2 - 1, nth // 2
        r1, r2 = nr // 2 - 1, nr // 2

        def strip(a):   # strips 1..4 = (r_one, th_one), (r_one, th_two), (r_two, th_one), (r_two, th_two)
            s = np.zeros(nphi)
            for rr, tt in ((r1, t1), (r1, t2), (r2, t1), (r2, t2)):
                s = s + a[tt, rr, :]
            return s * (1.0 / 4)

        strips = [strip(vr), strip(vp), strip(temperature)]
        if btheta is not None:
            strips.append(strip(self.last_magnetic[1] if btheta is True else btheta))
        nobs = len(strips)
        vsave = np.zeros((msymm, nobs))
        xind = 0
        im1 = nphi - 1
        for i in range(nphi):
            vrnext, vrlast = strips[0][i], strips[0][im1]
            dvr = vrnext - vrlast
            if vrnext * vrlast < 0 and xind < msymm and dvr > 0:
                x = -vrlast / dvr
                for j in range(nobs):
                    y1, y2 = strips[j][im1], strips[j][i]
                    vsave[xind, j] = (y2 - y1) * x + y1
                xind += 1
            im1 = i
        obs = vsave.sum(axis=0) / msymm
        if btheta is not None:
            return float(obs[1]), float(obs[2]), float(obs[3])
        return float(obs[1]), float(obs[2])

    def step(self):
        """One pass of Main_Loop_Sphere (Sphere_Driver.F90:305-328) at fixed dt."""
        g = self.post_solve()
        s2a = self.transpose_1a2a(g)
        s2a12 = self.rlm_spacea(s2a)
        p2a = self.h.s2p(s2a12)
        p3a = self.transpose_2a3a(p2a)
        p3b = self.physical_space(p3a)
        p2b = self.transpose_3b2b(p3b)
        s2b = self.h.p2s(p2b)
        s2b = self.rlm_spaceb(s2b)
        p1b = self.transpose_2b1b(s2b)
        self.advance_time(p1b)
        self.old_dt = self.dt
        self.iteration += 1
        return self.last_cfl


def c2001_case0_config(n_r=48, n_theta=64, chebyshev=True):
    """The settings benchmark_mode = 1 imposes (Benchmarking.F90:107-149: Christensen
    et al. 2001, hydrodynamic case 0) on an n_r x n_theta grid; l_max from n_theta as
    ProblemSize.F90:431-436 derives it (2 n_theta / 3 - 1).  chebyshev=False: the
    finite-difference radial mode on its uniform grid."""
    return Config(n_r=n_r, l_max=(2 * n_theta) // 3 - 1, n_theta=n_theta, aspect_ratio=0.35, shell_depth=1.0,
                  rayleigh=1.0e5, ekman=1.0e-3, prandtl=1.0, gravity_power=1.0, rotation=True,
                  no_slip_top=True, no_slip_bottom=True, fix_tvar_top=True, fix_tvar_bottom=True,
                  t_top=0.0, t_bottom=1.0, dt=1.0e-4, alpha_implicit=0.50001, chebyshev=chebyshev)


def c2001_case1_config(n_r=64, n_theta=96):
    """The settings benchmark_mode = 2 imposes (Benchmarking.F90:150-199: Christensen et al.
    2001, MHD case 1: case 0's settings with magnetism, Pm = 5 and insulating boundaries)."""
    return replace(c2001_case0_config(n_r, n_theta), magnetism=True, magnetic_prandtl=5.0)


def j2011_hydro_config(n_r=128, n_theta=192):
    """The settings benchmark_mode = 3 imposes (Benchmarking.F90:202-247: Jones et al. 2011,
    anelastic hydrodynamic case): the cgs polytrope (reference_type 2) with n = 2, N_rho = 5,
    M = 1.9e30 g, rho_i = 1.1 g/cm^3, c_P = 1.0509e8, Omega = 1.76e-4 rad/s between
    r_i = 2.45e9 and r_o = 7e9 cm; nu = kappa = 3.64364e12; stress-free; entropy 0 at the
    top and 851225.7 at the bottom; viscous heating on (Controls.F90:64); dt <= 30 s."""
    return Config(n_r=n_r, l_max=(2 * n_theta) // 3 - 1, n_theta=n_theta, aspect_ratio=0.35, shell_depth=4.55e9,
                  reference_type=2, poly_n=2.0, poly_nrho=5.0, poly_mass=1.9e30, poly_rho_i=1.1,
                  pressure_specific_heat=1.0509e8, angular_velocity=1.76e-4, nu_top=3.64364e12,
                  kappa_top=3.64364e12, rotation=True, no_slip_top=False, no_slip_bottom=False,
                  fix_tvar_top=True, fix_tvar_bottom=True, t_top=0.0, t_bottom=851225.7, dt=30.0,
                  alpha_implicit=0.50001)


def anelastic_mhd_config(n_r=128, l_max=255, **kw):
    """The anelastic MHD step workload: the nondimensional polytrope (reference_type 3,
    Polytropic_ReferenceND) with 5 density scale heights and polytropic index 2 in a
    shell of radius ratio 0.35; fields W, Z, P, S (entropy in T's place), C, A;
    stress-free, fixed-entropy, insulating boundaries; viscous and ohmic heating on
    (Controls.F90:64-65).  Ek = 1e-3, Pr = 1, Pm = 2, Ra* = 0.5, dt = 1e-4 rotation times."""
    base = dict(n_r=n_r, l_max=l_max, aspect_ratio=0.35, shell_depth=1.0, reference_type=3, poly_n=2.0,
                poly_nrho=5.0, modified_rayleigh=0.5, ekman=1.0e-3, prandtl=1.0, magnetic_prandtl=2.0,
                magnetism=True, rotation=True, no_slip_top=False, no_slip_bottom=False, t_top=0.0,
                t_bottom=1.0, dt=1.0e-4)
    base.update(kw)
    return Config(**base)


def seeded_state(cfg: Config, seed=0x5241594C, amp=1.0e-3, lmin=1, lmax_pert=20, cheby=None):
    """Seeded initial state: conductive T plus a Gaussian perturbation on l in [lmin, lmax_pert].

    Returns (wpt[lm,2,3nr], z[lm,2,nr]) in Chebyshev-coefficient form.  The
    perturbation is a random set of Chebyshev coefficients on the dealiased
    modes with amplitude amp*(l+1)^-2 that vanishes at both boundaries
    (multiplied by the grid function (r-rmin)(rmax-r) before the transform).
    """
    rng = np.random.Generator(np.random.PCG64(seed))
    nr = cfg.n_r
    rmax = cfg.shell_depth / (1.0 - cfg.aspect_ratio)
    rmin = rmax * cfg.aspect_ratio
    cg = cheby if cheby is not None else Chebyshev(nr, rmin, rmax)
    r = cg.radius
    ls, ms = lm_pairs(cfg.l_max)
    n_lm = len(ls)
    wpt = np.zeros((n_lm, 2, 3 * nr))
    z = np.zeros((n_lm, 2, nr))
    r_out, r_in = r[0], r[-1]
    pref = r_out * r_in / (r_in - r_out)
    tcond = pref * (1.0 / r_out - 1.0 / r) * math.sqrt(4 * math.pi)
    tgrid = np.zeros((n_lm, 2, nr))
    tgrid[0, 0] = tcond
    shape = (r - rmin) * (rmax - r)
    shape = shape / shape.max()
    radial = np.sin(np.pi * (r - rmin) / (rmax - rmin))
    for i in range(n_lm):
        l, m = ls[i], ms[i]
        if lmin <= l <= lmax_pert:
            a = amp * (l + 1.0) ** -2
            re, im = rng.standard_normal(2) * a
            if m == 0:
                im = 0.0
            tgrid[i, 0] += re * radial * shape
            tgrid[i, 1] += im * radial * shape
    wpt[:, :, 2 * nr:] = cg.to_spectral(tgrid)
    return wpt, z


def seeded_magnetic_state(cfg: Config, seed=0x5241594D, amp=1.0e-3, lmin=1, lmax_pert=20, cheby=None):
    """Seeded magnetic perturbation: (c[lm,2,nr], a[lm,2,nr]) Chebyshev coefficients of the
    poloidal (C) and toroidal (A) potentials, complex Gaussian of amplitude amp*(l+1)^-2 on
    l in [lmin, lmax_pert] (m = 0 imaginary parts zero) times the grid function
    sin(pi (r - rmin) / (rmax - rmin)), which vanishes at both boundaries."""
    rng = np.random.Generator(np.random.PCG64(seed))
    nr = cfg.n_r
    rmax = cfg.shell_depth / (1.0 - cfg.aspect_ratio)
    rmin = rmax * cfg.aspect_ratio
    cg = cheby if cheby is not None else Chebyshev(nr, rmin, rmax)
    r = cg.radius
    ls, ms = lm_pairs(cfg.l_max)
    radial = np.sin(np.pi * (r - rmin) / (rmax - rmin))
    grids = np.zeros((2, len(ls), 2, nr))
    for i in range(len(ls)):
        l, m = ls[i], ms[i]
        if lmin <= l <= lmax_pert:
            for k in range(2):
                re, im = rng.standard_normal(2) * amp * (l + 1.0) ** -2
                if m == 0:
                    im = 0.0
                grids[k, i, 0] = re * radial
                grids[k, i, 1] = im * radial
    return cg.to_spectral(grids[0]), cg.to_spectral(grids[1])
