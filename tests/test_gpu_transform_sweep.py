"""The standalone Legendre + FFT transform sweep: l_max in {255, 511, 1023}
(N_theta = 3 (l_max + 1) / 2, N_phi = 2 N_theta), 16 complex FP64 fields x N_r = 128 radial
levels, coefficients seeded complex Gaussian with amplitude (l + 1)^-1.5 and the m = 0
imaginary parts zero; forward and inverse transforms (StP_4d_dgp2 + FFT_To_Physical,
FFT_To_Spectral + PtS_4d_dgpv3; Legendre_Transforms.F90:968-1175, Fourier_Transform.F90:100-183)
through ra_transform_dev on device buffers, all-FP64 (FP64 tensor-core products) against the
split int8 form, timed on the device per stage.  Errors per l_max: the FP64 round trip
(spectral -> physical -> spectral, exact for the band-limited input on the Gauss-Legendre
grid), the mixed form against the FP64 form in each direction, and at l_max = 255 the FP64
physical values against the oracle's StP + c2r on sampled columns.  The 128 levels run as four
chunks of 32 (16 x 32 = 512 complex columns per call)."""
import numpy as np
import pytest

import oracle as O
from layouts import row_index

pytestmark = pytest.mark.gpu
NF, NR, CHUNK = 16, 128, 32


def _row_map(L):
    """row index of every (l, m) in l-major order and the (l+1)^-1.5 amplitude and m of each row."""
    nlm = L * (L + 1) // 2
    amp = np.zeros(nlm)
    mrow = np.zeros(nlm, dtype=np.int64)
    lrow = np.zeros(nlm, dtype=np.int64)
    for m in range(L):
        for l in range(m, L):
            r = row_index(m, l, L)
            amp[r] = (l + 1.0) ** -1.5
            mrow[r] = m
            lrow[r] = l
    return amp, mrow, lrow


@pytest.mark.parametrize("lmax", [255, 511, 1023])
def test_transform_sweep(lmax):
    import torch
    import rayleigh_b200 as rb
    from rayleigh_b200 import build as rbuild
    rbuild.build()
    L = lmax + 1
    ctx = rb.Rayleigh(rb.Config(n_r=8, l_max=lmax, use_graph=False))
    nth, nphi = ctx.n_theta, ctx.n_phi
    assert nth == 3 * L // 2 and nphi == 2 * nth
    nlm = L * (L + 1) // 2
    nfr = NF * CHUNK
    amp, mrow, lrow = _row_map(L)
    dev = torch.device("cuda")
    amp_d = torch.tensor(amp, device=dev)[:, None, None]
    m0 = torch.tensor(mrow == 0, device=dev)
    gen = torch.Generator(device=dev).manual_seed(0x5241594C + lmax)
    spec = torch.empty((nlm, nfr, 2), dtype=torch.float64, device=dev)
    back = torch.empty_like(spec)
    grid = torch.empty((nth, nfr, nphi + 2), dtype=torch.float64, device=dev)
    work = torch.empty((L * nth * nfr * 2,), dtype=torch.float64, device=dev)
    times = {p: np.zeros((2, 3)) for p in (rb.PREC_FP64, rb.PREC_MIXED)}
    worst = {"fp64_round_trip": 0.0, "mixed_vs_fp64_inverse": 0.0, "mixed_vs_fp64_forward": 0.0}

    def rel(a, b):
        return float(torch.linalg.norm(a - b) / torch.linalg.norm(b))

    ref_grid = None
    spec.zero_()
    for prec in (rb.PREC_FP64, rb.PREC_MIXED):   # untimed: builds the split-product plans
        ctx.transform_dev(0, prec, spec.data_ptr(), grid.data_ptr(), work.data_ptr(), nfr)
        ctx.transform_dev(1, prec, back.data_ptr(), grid.data_ptr(), work.data_ptr(), nfr)
    for chunk in range(NR // CHUNK):
        spec.normal_(generator=gen)
        spec.mul_(amp_d)
        spec[m0, :, 1] = 0.0
        # FP64: inverse into grid (kept), forward from it in place (r2c overwrites the grid)
        times[rb.PREC_FP64][0] += ctx.transform_dev(0, rb.PREC_FP64, spec.data_ptr(), grid.data_ptr(),
                                                    work.data_ptr(), nfr)
        phys64 = grid[..., :nphi].clone()
        if chunk == 0 and lmax == 255:
            ref_grid = (spec.cpu().numpy(), phys64.cpu().numpy())
        times[rb.PREC_FP64][1] += ctx.transform_dev(1, rb.PREC_FP64, back.data_ptr(), grid.data_ptr(),
                                                    work.data_ptr(), nfr)
        worst["fp64_round_trip"] = max(worst["fp64_round_trip"], rel(back, spec))
        back64 = back.clone()
        # mixed, from the same coefficients; each direction compared with the FP64 one
        times[rb.PREC_MIXED][0] += ctx.transform_dev(0, rb.PREC_MIXED, spec.data_ptr(), grid.data_ptr(),
                                                     work.data_ptr(), nfr)
        worst["mixed_vs_fp64_inverse"] = max(worst["mixed_vs_fp64_inverse"], rel(grid[..., :nphi], phys64))
        grid[..., :nphi] = phys64          # the forward direction from the FP64 physical values
        times[rb.PREC_MIXED][1] += ctx.transform_dev(1, rb.PREC_MIXED, back.data_ptr(), grid.data_ptr(),
                                                     work.data_ptr(), nfr)
        worst["mixed_vs_fp64_forward"] = max(worst["mixed_vs_fp64_forward"], rel(back, back64))
        del phys64, back64
    if ref_grid is not None:   # the oracle's StP and c2r on 6 sampled complex columns
        s_h, g_h = ref_grid
        cols = [0, 1, 77, 200, 311, nfr - 1]
        h = O.Horizontal(lmax, nth)
        s2 = []
        for m in range(L):
            rows = [row_index(m, l, L) for l in range(m, L)]
            a = s_h[rows][:, cols, :]                               # (nl, k, 2)
            s2.append(a.transpose(2, 1, 0)[None].copy())            # (1, 2, k, nl)
        p2 = h.s2p(s2)                                              # [m](1, 2, k, nth)
        p3 = np.zeros((nth, len(cols), nphi + 2))
        for m in range(L):
            p3[:, :, 2 * m] = p2[m][0, 0].T
            p3[:, :, 2 * m + 1] = p2[m][0, 1].T
        ref = O.fft_c2r(p3, nphi)[..., :nphi]
        got = g_h[:, cols, :]
        worst["fp64_vs_oracle"] = float(np.linalg.norm(got - ref) / np.linalg.norm(ref))
    f, x = times[rb.PREC_FP64], times[rb.PREC_MIXED]
    print(f"l_max {lmax} (N_theta {nth}, N_phi {nphi}), 16 fields x 128 levels, device ms per sweep "
          f"[Legendre, relayout, FFT]: inverse FP64 {np.round(f[0], 2).tolist()} mixed {np.round(x[0], 2).tolist()}; "
          f"forward FP64 {np.round(f[1], 2).tolist()} mixed {np.round(x[1], 2).tolist()}; "
          f"errors { {k: f'{v:.2e}' for k, v in worst.items()} }")
    ctx.close()
    # the round trip goes through the P_lm and the weighted P_lm tables (each within ~5e-12 of
    # its largest entry at l_max 255, the table test's bound): measured 3.2e-13, 4.3e-12 and
    # 2.2e-12 at l_max 255, 511, 1023
    assert worst["fp64_round_trip"] < 1e-11
    assert worst["mixed_vs_fp64_inverse"] < 1e-9 and worst["mixed_vs_fp64_forward"] < 1e-9
    if "fp64_vs_oracle" in worst:
        assert worst["fp64_vs_oracle"] < 1e-12
