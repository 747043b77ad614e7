"""Generate the golden fixtures that pin the oracle's Legendre path.

The fixtures come from the reference's own NumPy port of Rayleigh's
spherical-harmonic machinery, ``post_processing/spectral_utils.py`` (class
``SHT``, ``_compute_Plm`` at :1887-2005, ``_LT_to_spectral`` at :2106-2240,
``_LT_to_physical`` just below it).  That port restates
``src/Math_Layer/Legendre_Polynomials.F90`` and ``Legendre_Transforms.F90``
with the same REAL*16 -> longdouble recurrence, parity split and FFT
normalisation folding.

Run from the repository root in a container that has the reference tree:

    python tests/golden/make_golden.py /path/to/reference

The output ``tests/golden/sht_golden.npz`` is committed; nothing at test
time reads the reference tree.
"""
import os
import sys
import warnings

import numpy as np

if len(sys.argv) != 2:
    sys.exit("usage: python %s /path/to/reference" % os.path.relpath(__file__))
REF = sys.argv[1]
sys.path.insert(0, os.path.join(REF, "post_processing"))
warnings.simplefilter("ignore")
if not hasattr(np, "ComplexWarning"):          # removed from the numpy namespace in 2.x
    np.ComplexWarning = np.exceptions.ComplexWarning

import spectral_utils as su  # noqa: E402

SEED = 0x5241594C
CASES = [(15, 24, None), (41, 64, None), (63, 96, (0, 1, 2, 17, 31, 62, 63))]


def main():
    out = {}
    rng = np.random.Generator(np.random.PCG64(SEED))
    for lmax, nth, keep in CASES:
        sht = su.SHT(lmax, spectral=True, dealias=(nth + 0.5) / (lmax + 1))
        assert sht.nth == nth, (sht.nth, nth)
        assert sht.lmax == lmax, (sht.lmax, lmax)
        tag = f"l{lmax}"
        out[f"{tag}_x"] = sht.x
        out[f"{tag}_w"] = sht.w
        ms = range(sht.nm) if keep is None else keep
        out[f"{tag}_ms"] = np.array(list(ms))
        for m in ms:
            for name in ("p_lm_even", "p_lm_odd", "ip_lm_even", "ip_lm_odd"):
                arr = getattr(sht, name)[m]
                if isinstance(arr, np.ndarray):
                    out[f"{tag}_{name}_{m}"] = arr
        # Legendre transforms of seeded data: spectral (l, m, k) -> hybrid (theta, m, k) and back
        nk = 3
        spec = rng.standard_normal((sht.nl, sht.nm, nk)) + 1j * rng.standard_normal((sht.nl, sht.nm, nk))
        for l in range(sht.nl):
            spec[l, l + 1:] = 0.0
        spec[:, 0].imag = 0.0
        hyb = sht._LT_to_physical(spec, axis=0, m_axis=1)
        out[f"{tag}_spec_in"] = spec
        out[f"{tag}_hyb_out"] = hyb
        hyb_in = rng.standard_normal((sht.nth, sht.nm, nk)) + 1j * rng.standard_normal((sht.nth, sht.nm, nk))
        out[f"{tag}_hyb_in"] = hyb_in
        out[f"{tag}_spec_out"] = sht._LT_to_spectral(hyb_in, axis=0, m_axis=1)
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "sht_golden.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main()
