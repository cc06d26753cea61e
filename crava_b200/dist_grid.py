"""One posterior unit whose grids are split over several GPUs.

The reference transforms a whole grid on one host (FFTGrid::fftInPlace,
src/fftgrid.cpp:1803-1829) and solves every bin in one loop
(src/crava.cpp:1042-1151).  For a grid too large for one GPU the unit is
split the way the transform factorises:

* z slabs: rank r holds planes [z0_r, z1_r) of every real grid and runs the
  x and y passes on them (crava_gpu_fft_xy, scaled as the full grid);
* one all-to-all moves the spectra to (kx, ky) column shards: rank r then
  holds rows [y0_r, y1_r) of every kz plane, runs the z pass
  (crava_gpu_fft_z) and the per-bin solve (crava_gpu_posterior), which
  needs nothing outside its own bins, and the inverse z pass;
* one all-to-all back to z slabs and the inverse y and x passes.

Per posterior the exchange moves (10 + nt) grids out and (9 + nt) back,
each rank sending (P - 1) / P of its share; received blocks land in local
memory before use.  The transforms and the solve are passed in as
functions, so the same exchange code runs with the device kernels on GPUs
(``device_ops``) and with numpy stand-ins in the two-rank gloo tests.
"""
from __future__ import annotations

import math
from dataclasses import dataclass


def split_range(n: int, parts: int, r: int):
    """[lo, hi) of the r-th of `parts` nearly equal pieces of range(n)."""
    base, extra = divmod(n, parts)
    lo = r * base + min(r, extra)
    return lo, lo + base + (1 if r < extra else 0)


@dataclass
class Layout:
    """z-slab and ky-column partition of an (nxp, nyp, nzp) grid over P ranks."""
    nxp: int
    nyp: int
    nzp: int
    world: int

    @property
    def cnxp(self):
        return self.nxp // 2 + 1

    def z(self, r):
        return split_range(self.nzp, self.world, r)

    def y(self, r):
        return split_range(self.nyp, self.world, r)


def _smooth(n: int) -> bool:
    for f in (2, 3, 5, 7):
        while n % f == 0:
            n //= f
    return n == 1


def check_layout(lay: Layout):
    """Every rank's slab (z planes) and column shard (ky rows) must be a
    transform length the contexts plan (2, 3, 5, 7-smooth); raises
    ValueError naming the first that is not."""
    for r in range(lay.world):
        nz = lay.z(r)[1] - lay.z(r)[0]
        ny = lay.y(r)[1] - lay.y(r)[0]
        if nz < 1 or ny < 1 or not _smooth(nz) or not _smooth(ny):
            raise ValueError(f"rank {r}: slab of {nz} planes / shard of {ny} rows is not 2,3,5,7-smooth; "
                             f"choose a rank count that splits nyp={lay.nyp} and nzp={lay.nzp} so")


def exchange_plan(lay: Layout, rank: int, direction: str):
    """The point-to-point operations of one exchange on this rank, in the
    order they are posted: a list of (kind, peer, z range, y range) with
    kind "send" or "recv".

    direction "to_columns": this rank sends rows [py0, py1) of its z slab to
    each peer and receives the peer's planes [pz0, pz1) of its own rows;
    "to_slabs" is the reverse.  The list depends on the layout and the rank
    only (never on the backend), so NCCL and gloo post the same operations;
    every send of rank r to p has the shape of p's receive from r."""
    z0, z1 = lay.z(rank)
    y0, y1 = lay.y(rank)
    ops = []
    for peer in range(lay.world):
        if peer == rank:
            continue
        pz0, pz1 = lay.z(peer)
        py0, py1 = lay.y(peer)
        if direction == "to_columns":
            ops.append(("send", peer, (z0, z1), (py0, py1)))
            ops.append(("recv", peer, (pz0, pz1), (y0, y1)))
        elif direction == "to_slabs":
            ops.append(("send", peer, (pz0, pz1), (y0, y1)))
            ops.append(("recv", peer, (z0, z1), (py0, py1)))
        else:
            raise ValueError(direction)
    return ops


def _post(dist, p2p):
    """Posts one exchange as a single group (dist.batch_isend_irecv) and
    waits for it.  Grouping lets NCCL match every rank's sends and receives
    together: posting them one by one in the same order on every rank
    deadlocks once a send is larger than NCCL's eager buffer (each rank's
    send waits for a receive queued behind the peer's own send)."""
    if not p2p:
        return
    ops = [dist.P2POp(dist.isend if kind == "send" else dist.irecv, t, peer) for kind, peer, t in p2p]
    for w in dist.batch_isend_irecv(ops):
        w.wait()


def to_columns(slab, lay: Layout, rank: int, dist):
    """z slab [nz_r, nyp, 2 cnxp] (float32, complex pairs after the xy
    passes) -> column shard [nzp, ny_r, 2 cnxp] of this rank.  Each source's
    block lands directly in its z slice of the shard."""
    import torch

    z0, z1 = lay.z(rank)
    y0, y1 = lay.y(rank)
    assert tuple(slab.shape) == (z1 - z0, lay.nyp, 2 * lay.cnxp)
    out = torch.empty((lay.nzp, y1 - y0, 2 * lay.cnxp), dtype=slab.dtype, device=slab.device)
    out[z0:z1].copy_(slab[:, y0:y1, :])
    if dist is not None and lay.world > 1:
        p2p = []
        for kind, peer, (a, b), (c, d) in exchange_plan(lay, rank, "to_columns"):
            if kind == "send":
                p2p.append((kind, peer, slab[:, c:d, :].contiguous()))
            else:
                p2p.append((kind, peer, out[a:b]))  # a contiguous z slice
        _post(dist, p2p)
    return out


def to_slabs(cols, lay: Layout, rank: int, dist, out):
    """Column shard [nzp, ny_r, 2 cnxp] -> this rank's z slab `out`
    [nz_r, nyp, 2 cnxp]: each source's block is written into its ky rows."""
    import torch

    z0, z1 = lay.z(rank)
    y0, y1 = lay.y(rank)
    assert tuple(cols.shape) == (lay.nzp, y1 - y0, 2 * lay.cnxp)
    assert tuple(out.shape) == (z1 - z0, lay.nyp, 2 * lay.cnxp)
    out[:, y0:y1, :].copy_(cols[z0:z1])
    if dist is not None and lay.world > 1:
        p2p, blocks = [], []
        for kind, peer, (a, b), (c, d) in exchange_plan(lay, rank, "to_slabs"):
            if kind == "send":
                p2p.append((kind, peer, cols[a:b]))  # a contiguous z slice
            else:
                blk = torch.empty((b - a, d - c, 2 * lay.cnxp), dtype=cols.dtype, device=cols.device)
                p2p.append((kind, peer, blk))
                blocks.append((c, d, blk))
        _post(dist, p2p)
        for c, d, blk in blocks:
            out[:, c:d, :].copy_(blk)
    return out


# grid types (FFTGrid::gridTypes, src/fftgrid.h:172)
DATA, PARAMETER, COVARIANCE = 1, 2, 3


def scales(n: int, gtype: int):
    """Forward and inverse scale of a whole grid of n cells (fftInPlace /
    invFFTInPlace, src/fftgrid.cpp:1817, 1848-1859): the device computes
    its own; host stand-ins of the passes use these."""
    if gtype == COVARIANCE:
        return 1.0, 1.0 / n
    return 1.0 / math.sqrt(n), 1.0 / math.sqrt(n)


def posterior_unit_split(ops, lay: Layout, rank: int, dist, mu, data, cov, err):
    """The posterior unit on this rank's z slabs (real padded layout,
    [nz_r, nyp, rnxp] float32), in place: means, stacks and covariances
    come back as posterior means, residuals and posterior covariances.
    ops: fft_xy(grid, dir, grid_type) on slabs (scaled as the whole grid
    of that type), fft_z(grid, dir) and solve(mu, data, cov, err) on
    column shards."""
    types = [PARAMETER] * len(mu) + [DATA] * len(data) + [COVARIANCE] * (len(cov) + 1)
    grids = list(mu) + list(data) + list(cov) + [err]
    cols = []
    for g, t in zip(grids, types):
        ops.fft_xy(g, -1, t)
        c = to_columns(g, lay, rank, dist)
        ops.fft_z(c, -1)
        cols.append(c)
    nm, nd, nc = len(mu), len(data), len(cov)
    cm, cd, cc, ce = cols[:nm], cols[nm:nm + nd], cols[nm + nd:nm + nd + nc], cols[-1]
    ops.solve(cm, cd, cc, ce)
    for g, c, t in zip(grids[:-1], cols[:-1], types[:-1]):
        ops.fft_z(c, 1)
        to_slabs(c, lay, rank, dist, g)
        ops.fft_xy(g, 1, t)


def spectra_to_columns(ops, lay: Layout, rank: int, dist, mu, data, cov, err):
    """The forward half of the split unit: the slabs' spectra on this
    rank's column shards (mu, data, cov, err), the slabs left as they were
    after their x and y passes."""
    types = [PARAMETER] * len(mu) + [DATA] * len(data) + [COVARIANCE] * (len(cov) + 1)
    cols = []
    for g, t in zip(list(mu) + list(data) + list(cov) + [err], types):
        ops.fft_xy(g, -1, t)
        c = to_columns(g, lay, rank, dist)
        ops.fft_z(c, -1)
        cols.append(c)
    nm, nd, nc = len(mu), len(data), len(cov)
    return cols[:nm], cols[nm:nm + nd], cols[nm + nd:nm + nd + nc], cols[-1]


def loglik_grad_split(loglik, dist, mu_c, data_c, cov_c, err_c, *args):
    """The log marginal likelihood and its gradients over a grid split
    into column shards: every rank evaluates its own bins (`loglik`, e.g.
    a column-shard context's loglik_grad) and one all-reduce sums the value,
    the gradients and the failed-bin count (5 + 5 + 2 (nzp/2 + 1) 5 + 2
    doubles for five angles)."""
    import numpy as np

    L, gs, gv, gw, nf = loglik(mu_c, data_c, cov_c, err_c, *args)
    if dist is None:
        return L, gs, gv, gw, nf
    import torch

    gw = np.asarray(gw)
    flat = np.concatenate([[L], gs, gv, gw.real.reshape(-1), gw.imag.reshape(-1), [nf]]).astype(np.float64)
    t = torch.from_numpy(flat)
    if dist.get_backend() == "nccl":
        t = t.cuda()
    dist.all_reduce(t)
    f = t.cpu().numpy()
    nt, nw = len(gs), gw.size
    gwr = f[1 + 2 * nt:1 + 2 * nt + nw].reshape(gw.shape)
    gwi = f[1 + 2 * nt + nw:1 + 2 * nt + 2 * nw].reshape(gw.shape)
    return float(f[0]), f[1:1 + nt], f[1 + nt:1 + 2 * nt], gwr + 1j * gwi, int(round(f[-1]))


class device_ops:
    """The device kernels for posterior_unit_split: x/y passes on a z-slab
    context, z pass and solve on a column-shard context (crava_b200.api)."""

    def __init__(self, ctx_slab, ctx_cols, precision, nzp_full):
        self.s, self.c, self.p, self.nzp = ctx_slab, ctx_cols, precision, nzp_full

    def fft_xy(self, g, d, gtype):
        self.s.fft_xy(g, d, gtype, self.nzp)

    def fft_z(self, g, d):
        self.c.fft_z(g, d)

    def solve(self, mu, data, cov, err):
        self.c.posterior(mu, data, cov, err, self.p)


def shard_case(case, nyp=None, nzp=None):
    """The case seen by a slab (nzp planes) or column-shard (nyp rows)
    context: same model constants, local geometry.  A slab context only
    transforms along x and y, so its wavelets are the first nzp samples."""
    from types import SimpleNamespace

    c = SimpleNamespace(**{k: getattr(case, k) for k in
                           ("nxp", "nyp", "nzp", "ntheta", "nz", "lz", "min_rel_thick", "low_cut",
                            "high_cut", "wnc", "wavelet", "A", "theta_cov", "var0")})
    c.thickness_mode = int(getattr(case, "thickness_mode", 0))
    if nyp is not None:
        c.nyp = nyp
    if nzp is not None:
        c.nzp = nzp
        c.wavelet = case.wavelet[:, :nzp].copy()
        c.nz = min(case.nz, nzp)
    return c
