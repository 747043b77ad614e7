"""Checkpoint field files in the reference's byte layout (host only, no GPU).

tests/golden/checkpoint_sample_T.npz holds the reference's sample checkpoint
field (post_processing/sample_checkpoint_T, N_r = 48, l_max = 31) as decoded by
the reference's own reader, and the SHA-256 of its bytes
(tests/golden/make_checkpoint_golden.py).  Re-encoding the decoded values with
this library's writer gives the same bytes; reading them back gives the values."""
import hashlib
import os

import numpy as np

GOLD = os.path.join(os.path.dirname(__file__), "golden", "checkpoint_sample_T.npz")


def _state_layout(g):
    n_r = int(g["n_r"])
    l_max = int(g["l"].max())
    n_lm = (l_max + 1) * (l_max + 2) // 2
    field = np.zeros((n_lm, 2, n_r))
    lm = g["l"] * (g["l"] + 1) // 2 + g["m"]
    field[lm, 0, :] = g["re"]
    field[lm, 1, :] = g["im"]
    return field, n_r, l_max


def test_writer_reproduces_the_reference_sample_bytes(tmp_path):
    import rayleigh_b200 as rb
    g = np.load(GOLD)
    field, n_r, l_max = _state_layout(g)
    path = os.path.join(tmp_path, "T")
    rb.checkpoint_write_field(path, field, n_r, l_max)
    data = open(path, "rb").read()
    assert len(data) == n_r * (l_max + 1) * (l_max + 2) * 8       # the size Read_Checkpoint checks
    assert hashlib.sha256(data).hexdigest() == str(g["sha256"])
    back = rb.checkpoint_read_field(path, n_r, l_max)
    assert np.array_equal(back, field)


def test_reader_refuses_another_grid(tmp_path):
    import pytest
    import rayleigh_b200 as rb
    g = np.load(GOLD)
    field, n_r, l_max = _state_layout(g)
    path = os.path.join(tmp_path, "T")
    rb.checkpoint_write_field(path, field, n_r, l_max)
    with pytest.raises(rb.RayleighError):
        rb.checkpoint_read_field(path, n_r, l_max + 1)
    with pytest.raises(rb.RayleighError):
        rb.checkpoint_read_field(os.path.join(tmp_path, "missing"), n_r, l_max)
