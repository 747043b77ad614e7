"""The radial split of the spherical-harmonic transforms on the device.

A batch of nf = 4 complex fields on N_r = 17 levels at l_max = 63 (N_theta = 96, N_phi = 192),
coefficients seeded with (l + 1)^-1.5 amplitude, is owned per mode by three ranks (contiguous
pair blocks of 694 / 693 / 693 pairs, LM_Load_Balance) and transformed by radius (blocks of
6 / 6 / 5 levels, Standard_Balance): Transpose_1a2a, the inverse transform of each rank's
levels (ra_transform_dev), then the forward transform and Transpose_2b1b back to the
per-mode owners.  The ranks are emulated in one process, the all-to-all by in-process
copies (no rank waits on another).  Every rank's physical values and returned coefficients
must equal the transform of the whole batch on one rank bit for bit, in both forms (the
products see the same columns with the same operands, whatever the batch), and the round
trip the input (relative L2; measured 9.6e-13 FP64, 2.3e-10 mixed).  The same path through
a one-rank NCCL process group (all_to_all_single on device buffers) must reproduce the
group-less path bit for bit."""
import os
import socket

import numpy as np
import pytest
import torch

from rayleigh_b200 import radial_split as RS

pytestmark = pytest.mark.gpu
LMAX, NR, NF, WORLD = 63, 17, 4, 3


def _ctx():
    import rayleigh_b200 as rb
    from rayleigh_b200 import build as rbuild
    rbuild.build()
    return rb.Rayleigh(rb.Config(n_r=8, l_max=LMAX, use_graph=False))


def _modes(dev, seed=5):
    L = LMAX + 1
    ls = np.concatenate([np.full(l + 1, l) for l in range(L)])
    ms = np.concatenate([np.arange(l + 1) for l in range(L)])
    g = torch.Generator(device=dev).manual_seed(seed)
    x = torch.randn((len(ls), NF, NR, 2), generator=g, dtype=torch.float64, device=dev)
    x *= torch.tensor((ls + 1.0) ** -1.5, device=dev)[:, None, None, None]
    x[torch.tensor(ms == 0, device=dev), :, :, 1] = 0.0
    return x


def _rel(a, b):
    return float(torch.linalg.norm(a - b) / torch.linalg.norm(b))


def _whole(ctx, x, precision):
    sp = RS.RadialSplit(LMAX, NR, 1, 0, NF, device=x.device)
    ws = RS.TransformWorkspace(ctx, sp)
    grid = RS.to_physical(ctx, sp, x, precision, ws).clone()
    back = RS.to_spectral(ctx, sp, grid.clone(), precision, ws)
    return grid, back


@pytest.mark.parametrize("precision", [0, 1])
def test_radial_split_transforms(precision):
    ctx = _ctx()
    dev = torch.device("cuda")
    x = _modes(dev)
    nth, nphi = ctx.n_theta, ctx.n_phi
    grid_all, back_all = _whole(ctx, x, precision)
    ga = grid_all.view(nth, NF, NR, nphi + 2)
    splits = [RS.RadialSplit(LMAX, NR, WORLD, k, NF, device=dev) for k in range(WORLD)]
    assert [sp.nlm_local for sp in splits] == [694, 693, 693] and [sp.nr_local for sp in splits] == [6, 6, 5]
    wss = [RS.TransformWorkspace(ctx, sp) for sp in splits]
    # Transpose_1a2a, then each rank's inverse transform
    sends = [sp.pack_1a2a(x[sp.lm_lo:sp.lm_hi].contiguous()) for sp in splits]
    recvs = RS.all_to_all_in_process(sends, [sp.send_splits_1a2a() for sp in splits],
                                     [sp.recv_splits_1a2a() for sp in splits])
    errs = {"inverse": 0.0, "forward": 0.0, "round_trip": 0.0}
    exact = True
    for sp, ws, r in zip(splits, wss, recvs):
        sp.unpack_1a2a(r, out=ws.spec)
        ctx.transform_dev(0, precision, ws.spec.data_ptr(), ws.grid.data_ptr(), ws.work.data_ptr(), ws.nfr)
        got = ws.grid.view(nth, NF, sp.nr_local, nphi + 2)[..., :nphi]
        want = ga[:, :, sp.r_lo:sp.r_hi, :nphi]
        errs["inverse"] = max(errs["inverse"], _rel(got, want))
        exact &= bool(torch.equal(got, want))
    # each rank's forward transform of its own levels (in place), then Transpose_2b1b
    sends = []
    for sp, ws in zip(splits, wss):
        ctx.transform_dev(1, precision, ws.spec.data_ptr(), ws.grid.data_ptr(), ws.work.data_ptr(), ws.nfr)
        sends.append(sp.pack_2b1b(ws.spec))
    recvs = RS.all_to_all_in_process(sends, [sp.send_splits_2b1b() for sp in splits],
                                     [sp.recv_splits_2b1b() for sp in splits])
    for sp, r in zip(splits, recvs):
        out = sp.unpack_2b1b(r)
        errs["forward"] = max(errs["forward"], _rel(out, back_all[sp.lm_lo:sp.lm_hi]))
        exact &= bool(torch.equal(out, back_all[sp.lm_lo:sp.lm_hi]))
        errs["round_trip"] = max(errs["round_trip"], _rel(out, x[sp.lm_lo:sp.lm_hi]))
    print(precision, {k: f"{v:.2e}" for k, v in errs.items()})
    assert exact, errs
    assert errs["round_trip"] < (1e-11 if precision == 0 else 1e-9), errs
    ctx.close()


def test_radial_split_through_nccl():
    import torch.distributed as dist
    ctx = _ctx()
    dev = torch.device("cuda:0")
    x = _modes(dev, seed=9)
    grid_ref, back_ref = _whole(ctx, x, 0)
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("nccl", rank=0, world_size=1, device_id=dev)
    try:
        sp = RS.RadialSplit(LMAX, NR, 1, 0, NF, device=dev)
        ws = RS.TransformWorkspace(ctx, sp)
        grid = RS.to_physical(ctx, sp, x, 0, ws).clone()
        back = RS.to_spectral(ctx, sp, grid.clone(), 0, ws)
        torch.cuda.synchronize()
        assert torch.equal(grid[..., :ctx.n_phi], grid_ref[..., :ctx.n_phi])
        assert torch.equal(back, back_ref)
    finally:
        dist.destroy_process_group()
        ctx.close()
