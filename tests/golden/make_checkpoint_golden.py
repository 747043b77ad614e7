"""Decode the reference's sample checkpoint field with the reference's own reader.

``post_processing/sample_checkpoint_T`` of the reference is one field file of a
Rayleigh checkpoint (N_r = 48, N_theta = 48, so l_max = 31).  This script reads
it with ``post_processing/rayleigh_diagnostics.py``'s ``checkpoint_read`` and
stores the decoded (l, m, radial index) coefficients together with the SHA-256
of the file's bytes in ``tests/golden/checkpoint_sample_T.npz``.  The tests
re-encode the decoded values with this library's checkpoint writer and compare
the SHA-256: equal digests mean the library writes the reference's byte layout.

    python tests/golden/make_checkpoint_golden.py /path/to/reference
"""
import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def main(ref):
    sys.path.insert(0, os.path.join(ref, "post_processing"))
    import rayleigh_diagnostics as rd
    path = os.path.join(ref, "post_processing", "sample_checkpoint_T")
    n_r, n_theta = 48, 48
    a = rd.checkpoint_read(path, n_r, n_theta)          # [m][l][radial index], zero for l < m
    nell = a.shape[0]
    m_idx, l_idx = np.nonzero(np.triu(np.ones((nell, nell), dtype=bool)))
    np.savez_compressed(os.path.join(HERE, "checkpoint_sample_T.npz"),
                        re=a.real[m_idx, l_idx, :], im=a.imag[m_idx, l_idx, :], m=m_idx, l=l_idx,
                        n_r=n_r, n_theta=n_theta,
                        sha256=hashlib.sha256(open(path, "rb").read()).hexdigest())
    print("pairs", len(m_idx), "n_r", n_r)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_checkpoint_golden.py /path/to/reference")
    main(sys.argv[1])
