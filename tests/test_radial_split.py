"""The radial split and its r <-> (l, m) all-to-all on CPU.

The balances against the reference's own loops (Standard_Balance, Load_Balance.F90:80-105;
the pair dealing of LM_Load_Balance, :400-418), the device row order against the layout
helpers, and Transpose_1a2a / Transpose_2b1b (Spherical_Buffer.F90:705-949) against the
single-rank arrays: bit for bit, for ranks emulated in one process and for 2 and 3 gloo
ranks, with ragged radial and pair blocks and the round trip."""
import json
import os
import socket
import tempfile

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from layouts import row_index
from rayleigh_b200 import radial_split as RS


def _standard_balance(nx, np_):
    """Standard_Balance's loop (1-based min, delta, max per rank) -> [(lo, hi)] 0-based."""
    nx_local = nx // np_
    mcheck = nx % np_ - 1
    out, mn = [], 1
    for p in range(np_):
        if p > 0:
            mn = out[-1][1] + 1
        delta = nx_local + 1 if p <= mcheck else nx_local
        out.append((mn, mn + delta - 1))
    return [(a - 1, b) for a, b in out]


def _lm_owner_blocks(count, n):
    """LM_Load_Balance's owner loop -> [(lo, hi)] per rank."""
    per, rem = divmod(count, n)
    owner = []
    for i in range(1, n + 1):
        owner += [i - 1] * per
        if i <= rem:
            owner.append(i - 1)
    owner = np.array(owner)
    return [(int(np.argmax(owner == k)), int(np.argmax(owner == k)) + int((owner == k).sum())) for k in range(n)]


@pytest.mark.parametrize("n,world", [(10, 4), (10, 3), (192, 8), (128, 3), (7, 7), (528, 5), (131328, 6)])
def test_balances_are_the_references(n, world):
    assert RS.balance(n, world) == _standard_balance(n, world)
    assert RS.balance(n, world) == _lm_owner_blocks(n, world)


@pytest.mark.parametrize("l_max", [0, 1, 7, 8, 31])
def test_device_rows(l_max):
    L = l_max + 1
    rows = RS.device_rows(l_max)
    want = [row_index(m, l, L) for l in range(L) for m in range(l + 1)]
    assert rows.tolist() == want
    assert sorted(rows.tolist()) == list(range(L * (L + 1) // 2))


def _globals(l_max, n_r, nf, seed=11):
    nlm = (l_max + 1) * (l_max + 2) // 2
    g = torch.Generator().manual_seed(seed)
    x = torch.randn((nlm, nf, n_r, 2), generator=g, dtype=torch.float64)        # pair order, all levels
    s = torch.randn((nlm, nf, n_r, 2), generator=g, dtype=torch.float64)        # device row order
    return x, s


def _expected(split, x, s):
    rows = torch.from_numpy(RS.device_rows(split.l_max))
    spec = torch.empty_like(x)
    spec[rows] = x
    spec = spec[:, :, split.r_lo:split.r_hi, :].contiguous()
    modes = s[rows][split.lm_lo:split.lm_hi].contiguous()
    return spec, modes


@pytest.mark.parametrize("l_max,n_r,world", [(7, 11, 1), (7, 11, 2), (7, 11, 3), (8, 13, 5), (3, 6, 6)])
def test_transposes_in_process(l_max, n_r, world):
    nf = 3
    x, s = _globals(l_max, n_r, nf)
    splits = [RS.RadialSplit(l_max, n_r, world, k, nf) for k in range(world)]
    # Transpose_1a2a
    sends = [sp.pack_1a2a(x[sp.lm_lo:sp.lm_hi].contiguous()) for sp in splits]
    recvs = RS.all_to_all_in_process(sends, [sp.send_splits_1a2a() for sp in splits],
                                     [sp.recv_splits_1a2a() for sp in splits])
    specs = [sp.unpack_1a2a(r) for sp, r in zip(splits, recvs)]
    # Transpose_2b1b, of the radial blocks of s and of what 1a2a produced
    for src, want_x in ((s, None), (None, x)):
        blocks = [(src[:, :, sp.r_lo:sp.r_hi, :].contiguous() if src is not None else specs[k])
                  for k, sp in enumerate(splits)]
        sends = [sp.pack_2b1b(b) for sp, b in zip(splits, blocks)]
        recvs = RS.all_to_all_in_process(sends, [sp.send_splits_2b1b() for sp in splits],
                                         [sp.recv_splits_2b1b() for sp in splits])
        modes = [sp.unpack_2b1b(r) for sp, r in zip(splits, recvs)]
        for k, sp in enumerate(splits):
            want_spec, want_modes = _expected(sp, x, s)
            assert torch.equal(specs[k], want_spec)
            if want_x is None:
                assert torch.equal(modes[k], want_modes)
            else:                                   # the round trip
                assert torch.equal(modes[k], x[sp.lm_lo:sp.lm_hi])
    if world > 1:
        with pytest.raises(ValueError):
            splits[0].pack_1a2a(x)                  # the whole array is not a rank's share
        with pytest.raises(RuntimeError):           # several ranks and no process group
            splits[0].transpose_1a2a(x[splits[0].lm_lo:splits[0].lm_hi].contiguous())


def _free_port():
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        return sk.getsockname()[1]


def _rank_main(rank, world, port, out_dir, l_max, n_r, nf):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        x, s = _globals(l_max, n_r, nf)
        sp = RS.RadialSplit(l_max, n_r, world, rank, nf)
        want_spec, want_modes = _expected(sp, x, s)
        spec = sp.transpose_1a2a(x[sp.lm_lo:sp.lm_hi].contiguous())
        modes = sp.transpose_2b1b(s[:, :, sp.r_lo:sp.r_hi, :].contiguous())
        back = sp.transpose_2b1b(spec)
        res = {"spec": bool(torch.equal(spec, want_spec)), "modes": bool(torch.equal(modes, want_modes)),
               "round_trip": bool(torch.equal(back, x[sp.lm_lo:sp.lm_hi])),
               "blocks": [sp.nlm_local, sp.nr_local]}
        other = RS.RadialSplit(l_max, n_r, world + 1, rank, nf)    # a split for another group size
        try:
            other.transpose_1a2a(x[other.lm_lo:other.lm_hi].contiguous())
            res["mismatch_refused"] = False
        except ValueError as e:
            res["mismatch_refused"] = "process group" in str(e)
        dist.barrier()
        with open(os.path.join(out_dir, f"rank{rank}.json"), "w") as f:
            json.dump(res, f)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,l_max,n_r", [(2, 15, 17), (3, 10, 16)])
def test_transposes_gloo(world, l_max, n_r):
    nf = 2
    with tempfile.TemporaryDirectory() as d:
        mp.start_processes(_rank_main, args=(world, _free_port(), d, l_max, n_r, nf), nprocs=world,
                           start_method="spawn")
        res = [json.load(open(os.path.join(d, f"rank{r}.json"))) for r in range(world)]
    nlm = (l_max + 1) * (l_max + 2) // 2
    assert sum(r["blocks"][0] for r in res) == nlm and sum(r["blocks"][1] for r in res) == n_r
    for r in res:
        assert r["spec"] and r["modes"] and r["round_trip"] and r["mismatch_refused"], r
