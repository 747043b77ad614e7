"""Layout helpers shared by the GPU parity tests: convert the oracle's
reference-layout arrays into the device buffer layouts that
``Rayleigh.debug_buffer`` returns (see include/rayleigh_b200.h, RA_BUF_*)."""
import numpy as np


def m_off(m, L):
    return m * L - m * (m - 1) // 2


def row_index(m, l, L):
    d = l - m
    ne = (L - m + 1) // 2
    return m_off(m, L) + ((ne + (d - 1) // 2) if (d & 1) else d // 2)


def s2_to_rows(s2, fields, r_major=False):
    """list over m of (nf, 2, nr, nl) -> [row][F][nr][2], or [row][nr][F][2] when r_major."""
    L = len(s2)
    nr = s2[0].shape[2]
    nlm = L * (L + 1) // 2
    F = len(fields)
    out = np.zeros((nlm, nr, F, 2) if r_major else (nlm, F, nr, 2))
    for m in range(L):
        a = s2[m][list(fields)]                      # (F, 2, nr, nl)
        rows = [row_index(m, m + j, L) for j in range(L - m)]
        out[rows] = a.transpose(3, 2, 0, 1) if r_major else a.transpose(3, 0, 2, 1)
    return out


def p2_to_dev(p2, fields):
    """list over m of (nf, 2, nr, nth) -> [m][nth][nr][F][2]."""
    P = np.stack([p[list(fields)] for p in p2])     # (m, F, 2, nr, nth)
    return P.transpose(0, 4, 3, 1, 2).copy()


def rel_err(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    den = np.linalg.norm(b.ravel())
    if den == 0:
        return float(np.linalg.norm(a.ravel()))
    return float(np.linalg.norm((a - b).ravel()) / den)


def p2_eo_to_full(dev, L, nth, F, nr):
    """device [nth/2][m][par][nr][F][2] (E, O) -> [m][nth][nr][F][2] with south E+O, north E-O."""
    d = dev.reshape(nth // 2, L, 2, nr, F, 2).transpose(1, 2, 0, 3, 4, 5)
    e, o = d[:, 0], d[:, 1]
    full = np.empty((L, nth, nr, F, 2))
    full[:, :nth // 2] = e + o
    full[:, nth - 1:nth // 2 - 1:-1] = e - o
    return full


def p2_fold(full):
    """[m][nth][nr][F][2] -> [m][2][nth/2][nr][F][2] folded (s + n, s - n)."""
    nth = full.shape[1]
    s = full[:, :nth // 2]
    n = full[:, nth - 1:nth // 2 - 1:-1]
    return np.stack([s + n, s - n], axis=1)
