"""The allocation-free split-precision product (ra_mixed_gemm_noalloc) against
the allocating entry point (ra_mixed_gemm), through the C ABI.

Collected last on purpose: it must pass both in a fresh process and after
every other test has run in the same process."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _call_noalloc(lib, da, db, dc, m, n, k, stream):
    msg = ctypes.create_string_buffer(512)
    rc = lib.ra_mixed_gemm_noalloc(ctypes.c_void_p(da.data_ptr()), ctypes.c_void_p(db.data_ptr()),
                                   ctypes.c_void_p(dc.data_ptr()), m, n, k, ctypes.c_void_p(stream), msg, 512)
    return rc, msg.value.decode()


def test_noalloc_matches_allocating_entry_point():
    import torch
    import rayleigh_b200 as rb
    from rayleigh_b200 import build as rbuild
    rbuild.build()
    lib = rb.load_library()
    ctx = rb.Rayleigh(rb.Config(n_r=16, l_max=15, n_theta=24))
    rng = np.random.Generator(np.random.PCG64(17))
    m, n, k = 300, 200, 130
    a = rng.standard_normal((m, k))
    b = rng.standard_normal((k, n))
    ref = ctx.mixed_gemm(a, b)
    exact = (a.astype(np.longdouble) @ b.astype(np.longdouble)).astype(np.float64)
    dev = torch.device("cuda", 0)
    da = torch.from_numpy(a).to(dev)
    db = torch.from_numpy(b).to(dev)
    stream = torch.cuda.current_stream(dev).cuda_stream
    tol = 1e-10 * np.abs(exact).max()
    for _ in range(2):
        dc = torch.full((m, n), float("nan"), dtype=torch.float64, device=dev)
        torch.cuda.synchronize()
        rc, msg = _call_noalloc(lib, da, db, dc, m, n, k, stream)
        assert rc == 0, msg
        got = dc.cpu().numpy()
        assert np.abs(got - ref).max() <= tol
        assert np.abs(got - exact).max() <= tol


def test_noalloc_rejects_oversize():
    import torch
    import rayleigh_b200 as rb
    lib = rb.load_library()
    dev = torch.device("cuda", 0)
    d = torch.zeros(4, dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev).cuda_stream
    # 4096 x 4096 x 4096 needs ~200 MB of digits: refused before any launch
    rc, msg = _call_noalloc(lib, d, d, d, 4096, 4096, 4096, stream)
    assert rc == rb.RA_ERR_ARG and "static limit" in msg, (rc, msg)
