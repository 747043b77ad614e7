"""The radial split of the transform stages over ranks (one process per GPU) and the
r <-> (l, m) all-to-all that joins it to the per-mode layout of the solve stages.

Rayleigh's decomposition with nprow = 1 and npcol = G ranks:

* the radial levels in contiguous blocks, the first mod(n_r, G) ranks one level more
  (Standard_Balance, Load_Balance.F90:80-105); level 0 is the outer boundary, as on the
  Chebyshev grid;
* the (l, m) pairs ordered l slowest, m fastest (the order of the C ABI's state arrays,
  lm = l (l + 1) / 2 + m) and dealt in contiguous chunks, the first mod(n_lm, G) ranks one
  pair more (LM_Load_Balance, Load_Balance.F90:311-470): every rank owns whole radial
  columns of its modes, which is what the per-l implicit solves and the radial synthesis
  need;
* Transpose_1a2a (Spherical_Buffer.F90:849-949): each rank sends every other rank that
  rank's radial block of its own modes and receives its own radial block of every rank's
  modes, which then covers all (l, m) of its levels, as the Legendre transforms and the
  physical-space stage need;
* Transpose_2b1b (Spherical_Buffer.F90:705-847): the reverse.

Each exchange is one all-to-all with ragged splits (torch.distributed.all_to_all_single:
NCCL's grouped send/recv over NVLink between GPUs, gloo between CPU processes) plus one
pack and one row permutation on the sending or receiving side.  Layouts:

* per-mode side: x[mode][field][r][re, im], the rank's n_lm_local modes in pair order, all
  n_r levels;
* radial side: spec[row][field][r_local][re, im], all n_lm rows in the device row order of
  ra_transform_dev (m-major, even l - m first), which reads it as [row][nfr][re, im] with
  nfr = fields x local levels.

``to_physical`` and ``to_spectral`` join the exchange to the library's device-resident
transforms (ra_transform_dev: Legendre products, (theta, pi - theta) relayout, phi FFT):
the transform batch of the spectral-transform sweep, split by radius over the ranks."""
import numpy as np
import torch


def balance(n, world):
    """[(lo, hi)] per rank: contiguous blocks of n indices, the first mod(n, world) ranks one more."""
    base, extra = divmod(n, world)
    out, lo = [], 0
    for k in range(world):
        hi = lo + base + (1 if k < extra else 0)
        out.append((lo, hi))
        lo = hi
    return out


def device_rows(l_max):
    """Device row of every (l, m) pair in pair order (l slowest): row(m, l) = off(m) +
    (l - m even ? (l - m)/2 : ne(m) + (l - m - 1)/2), off(m) = m L - m (m - 1)/2,
    ne(m) = (L - m + 1)/2, L = l_max + 1."""
    L = l_max + 1
    rows = np.empty(L * (L + 1) // 2, dtype=np.int64)
    p = 0
    for l in range(L):
        for m in range(l + 1):
            d = l - m
            off = m * L - m * (m - 1) // 2
            ne = (L - m + 1) // 2
            rows[p] = off + (ne + (d - 1) // 2 if d & 1 else d // 2)
            p += 1
    return rows


class RadialSplit:
    """Rank ``rank``'s share of an l_max, n_r problem over ``world`` ranks, for batches of
    ``nf`` complex fields."""

    def __init__(self, l_max, n_r, world, rank, nf, device="cpu"):
        if not (0 <= rank < world):
            raise ValueError("rank out of range")
        if n_r < world:
            raise ValueError("fewer radial levels than ranks")
        self.l_max, self.n_r, self.world, self.rank, self.nf = l_max, n_r, world, rank, nf
        self.n_lm = (l_max + 1) * (l_max + 2) // 2
        self.r_blocks = balance(n_r, world)
        self.lm_blocks = balance(self.n_lm, world)
        self.r_lo, self.r_hi = self.r_blocks[rank]
        self.lm_lo, self.lm_hi = self.lm_blocks[rank]
        self.nr_local = self.r_hi - self.r_lo
        self.nlm_local = self.lm_hi - self.lm_lo
        self.device = torch.device(device)
        self.rows = torch.from_numpy(device_rows(l_max)).to(self.device)

    # ---- Transpose_1a2a: per-mode -> radial ----
    def send_splits_1a2a(self):
        return [self.nlm_local * self.nf * (hi - lo) * 2 for lo, hi in self.r_blocks]

    def recv_splits_1a2a(self):
        return [(hi - lo) * self.nf * self.nr_local * 2 for lo, hi in self.lm_blocks]

    def pack_1a2a(self, x):
        """x[n_lm_local][nf][n_r][2] -> the send buffer, ordered by destination rank."""
        self._check(x, (self.nlm_local, self.nf, self.n_r, 2))
        return torch.cat([x[:, :, lo:hi, :].reshape(-1) for lo, hi in self.r_blocks])

    def unpack_1a2a(self, recv, out=None):
        """The received blocks (every rank's modes, in rank order = pair order) -> spec in
        device row order [n_lm][nf][nr_local][2]."""
        src = recv.view(self.n_lm, self.nf, self.nr_local, 2)
        if out is None:
            out = torch.empty_like(src)
        out.index_copy_(0, self.rows, src)
        return out

    def transpose_1a2a(self, x, group=None, out=None):
        send = self.pack_1a2a(x)
        recv = torch.empty(sum(self.recv_splits_1a2a()), dtype=x.dtype, device=x.device)
        self._exchange(recv, send, self.recv_splits_1a2a(), self.send_splits_1a2a(), group)
        return self.unpack_1a2a(recv, out)

    # ---- Transpose_2b1b: radial -> per-mode ----
    def send_splits_2b1b(self):
        return [(hi - lo) * self.nf * self.nr_local * 2 for lo, hi in self.lm_blocks]

    def recv_splits_2b1b(self):
        return [self.nlm_local * self.nf * (hi - lo) * 2 for lo, hi in self.r_blocks]

    def pack_2b1b(self, spec):
        """spec[n_lm][nf][nr_local][2] in device row order -> pair order, which is the send
        buffer (rank j's modes are a contiguous block of pairs)."""
        self._check(spec, (self.n_lm, self.nf, self.nr_local, 2))
        return spec.index_select(0, self.rows).reshape(-1)

    def unpack_2b1b(self, recv, out=None):
        """Every rank's radial block of this rank's modes -> x[n_lm_local][nf][n_r][2]."""
        if out is None:
            out = torch.empty((self.nlm_local, self.nf, self.n_r, 2), dtype=recv.dtype, device=recv.device)
        for (lo, hi), part in zip(self.r_blocks, torch.split(recv, self.recv_splits_2b1b())):
            out[:, :, lo:hi, :] = part.view(self.nlm_local, self.nf, hi - lo, 2)
        return out

    def transpose_2b1b(self, spec, group=None, out=None):
        send = self.pack_2b1b(spec)
        recv = torch.empty(sum(self.recv_splits_2b1b()), dtype=spec.dtype, device=spec.device)
        self._exchange(recv, send, self.recv_splits_2b1b(), self.send_splits_2b1b(), group)
        return self.unpack_2b1b(recv, out)

    def _exchange(self, recv, send, recv_splits, send_splits, group):
        import torch.distributed as dist
        if dist.is_available() and dist.is_initialized():
            if dist.get_world_size(group) != self.world or dist.get_rank(group) != self.rank:
                raise ValueError("the process group does not match the split's world size and rank")
            dist.all_to_all_single(recv, send, recv_splits, send_splits, group=group)
        elif self.world == 1:
            recv.copy_(send)
        else:
            raise RuntimeError("a split over several ranks needs an initialised process group")

    @staticmethod
    def _check(t, shape):
        if tuple(t.shape) != tuple(shape) or t.dtype != torch.float64 or not t.is_contiguous():
            raise ValueError(f"expected a contiguous float64 tensor of shape {tuple(shape)}, got "
                             f"{tuple(t.shape)} {t.dtype}")


def all_to_all_in_process(sends, send_splits, recv_splits):
    """The same exchange for ranks that live in one process (each rank's send buffer in
    ``sends``): rank k receives block k of every rank's send buffer, in rank order."""
    world = len(sends)
    parts = [torch.split(sends[j], send_splits[j]) for j in range(world)]
    out = []
    for k in range(world):
        recv = torch.cat([parts[j][k] for j in range(world)])
        if recv.numel() != sum(recv_splits[k]):
            raise ValueError("send and receive splits disagree")
        out.append(recv)
    return out


class TransformWorkspace:
    """Device buffers of one rank's radial batch for ra_transform_dev: spec[n_lm][nfr][2],
    grid[n_theta][nfr][n_phi + 2], work (l_max + 1) n_theta nfr complex."""

    def __init__(self, ctx, split):
        dev = split.device
        nfr = split.nf * split.nr_local
        self.nfr = nfr
        self.spec = torch.empty((split.n_lm, split.nf, split.nr_local, 2), dtype=torch.float64, device=dev)
        self.grid = torch.empty((ctx.n_theta, nfr, ctx.n_phi + 2), dtype=torch.float64, device=dev)
        self.work = torch.empty(((split.l_max + 1) * ctx.n_theta * nfr * 2,), dtype=torch.float64, device=dev)


def to_physical(ctx, split, x, precision, ws=None, group=None):
    """Fields x[n_lm_local][nf][n_r][2] of this rank's modes -> physical values of this rank's
    levels, grid[n_theta][nf * nr_local][n_phi + 2] (Transpose_1a2a, StP, c2r)."""
    ws = ws or TransformWorkspace(ctx, split)
    split.transpose_1a2a(x, group=group, out=ws.spec)
    ctx.transform_dev(0, precision, ws.spec.data_ptr(), ws.grid.data_ptr(), ws.work.data_ptr(), ws.nfr)
    return ws.grid


def to_spectral(ctx, split, grid, precision, ws=None, group=None):
    """Physical values of this rank's levels grid[n_theta][nf * nr_local][n_phi + 2] (consumed:
    the r2c runs in place) -> x[n_lm_local][nf][n_r][2] of this rank's modes (r2c, PtS,
    Transpose_2b1b)."""
    ws = ws or TransformWorkspace(ctx, split)
    if grid.data_ptr() != ws.grid.data_ptr():
        ws.grid.copy_(grid)
    ctx.transform_dev(1, precision, ws.spec.data_ptr(), ws.grid.data_ptr(), ws.work.data_ptr(), ws.nfr)
    return split.transpose_2b1b(ws.spec, group=group)
