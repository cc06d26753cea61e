"""The multi-rank plumbing on CPU with two gloo ranks (no GPU)."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    from crava_b200 import dist as D

    dist = D.init("gloo", timeout_s=60)
    r, w, _ = D.rank_env()
    m = D.max_over_ranks(dist, 10.0 * (r + 1))
    D.barrier(dist)
    items = list(range(11))
    mine = D.shard(items, r, w)
    out.put((r, m, mine))
    dist.destroy_process_group()


def test_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[1] for r in res] == [20.0, 20.0]
    shares = res[0][2] + res[1][2]
    assert sorted(shares) == list(range(11)) and not set(res[0][2]) & set(res[1][2])


def test_single_process_identity():
    from crava_b200 import dist as D
    assert D.max_over_ranks(None, 3.5) == 3.5
    assert D.shard([1, 2, 3], 0, 1) == [1, 2, 3]


# ------------------------------------------- one grid split over ranks
SPLIT_SHAPE = (8, 6, 10)  # nxp, nyp, nzp: uneven slabs and column shards over 3 ranks


class _NumpyOps:
    """Stand-ins of the device passes with the same conventions (unscaled
    complex passes, the x pass real <-> half-complex and scaled), and a
    per-bin stand-in of the solve."""

    def __init__(self, nxp, n):
        self.nxp, self.n = nxp, n

    def fft_xy(self, g, d, gtype):
        import numpy as np
        import torch
        from crava_b200 import dist_grid as G
        scale = G.scales(self.n, gtype)[0 if d < 0 else 1]
        a = g.numpy()
        nx, c = self.nxp, self.nxp // 2 + 1
        if d < 0:
            z = np.fft.rfft(a[..., :nx].astype(np.float64), axis=-1) * scale
            z = np.fft.fft(z, axis=1)
            a[...] = z.astype(np.complex64).view(np.float32)
        else:
            z = a.view(np.complex64).astype(np.complex128)
            z = np.fft.ifft(z, axis=1) * a.shape[1]
            out = np.zeros_like(a)
            out[..., :nx] = np.fft.irfft(z, n=nx, axis=-1) * nx * scale
            a[...] = out
        g.copy_(torch.from_numpy(a))

    def fft_z(self, g, d):
        import numpy as np
        import torch
        z = g.numpy().view(np.complex64).astype(np.complex128)
        z = np.fft.fft(z, axis=0) if d < 0 else np.fft.ifft(z, axis=0) * z.shape[0]
        g.copy_(torch.from_numpy(z.astype(np.complex64).view(np.float32)))

    def solve(self, mu, data, cov, err):
        # a per-bin map of the spectra (what the real solve is: bins do not mix)
        e = err.clone()
        for q in range(3):
            mu[q].mul_(0.5).add_(data[q % len(data)] * 0.25)
        for l in range(len(data)):
            data[l].sub_(mu[0] * 0.1).add_(e * 0.01)
        for t in range(6):
            cov[t].mul_(0.8)


def _split_inputs():
    import numpy as np
    nxp, nyp, nzp = SPLIT_SHAPE
    rng = np.random.default_rng(17)
    mk = lambda: rng.standard_normal((nzp, nyp, 2 * (nxp // 2 + 1))).astype(np.float32)
    return [mk() for _ in range(3)], [mk() for _ in range(2)], [mk() for _ in range(6)], mk()


def _split_worker(rank, world, port, out):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import torch
    from crava_b200 import dist as D
    from crava_b200 import dist_grid as G

    dist = D.init("gloo", timeout_s=60)
    lay = G.Layout(*SPLIT_SHAPE, world)
    z0, z1 = lay.z(rank)
    mu, data, cov, err = _split_inputs()
    t = lambda gs: [torch.from_numpy(g[z0:z1].copy()) for g in gs]
    mu_t, data_t, cov_t, err_t = t(mu), t(data), t(cov), t([err])[0]
    G.posterior_unit_split(_NumpyOps(lay.nxp, lay.nxp * lay.nyp * lay.nzp), lay, rank, dist, mu_t, data_t, cov_t, err_t)
    out.put((rank, [g.numpy() for g in mu_t + data_t + cov_t]))
    dist.destroy_process_group()


def test_grid_split_over_three_gloo_ranks():
    """The split unit (z slabs -> column shards -> z slabs) on 3 gloo ranks
    equals the same passes on the whole grid in one process."""
    import numpy as np
    import torch
    from crava_b200 import dist_grid as G

    world = 3
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_split_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=180) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    lay = G.Layout(*SPLIT_SHAPE, 1)
    mu, data, cov, err = _split_inputs()
    t = lambda gs: [torch.from_numpy(g.copy()) for g in gs]
    mu_t, data_t, cov_t, err_t = t(mu), t(data), t(cov), t([err])[0]
    G.posterior_unit_split(_NumpyOps(lay.nxp, lay.nxp * lay.nyp * lay.nzp), lay, 0, None, mu_t, data_t, cov_t, err_t)
    whole = [g.numpy() for g in mu_t + data_t + cov_t]
    split = [np.concatenate([res[r][i] for r in range(world)], axis=0) for i in range(len(whole))]
    for a, b in zip(split, whole):
        nx = SPLIT_SHAPE[0]
        assert np.allclose(a[..., :nx], b[..., :nx], rtol=1e-5, atol=1e-6)
    # and the split passes are the 3-D transforms: with no solve the
    # round trip returns the inputs
    assert not np.allclose(whole[0][..., :nx], mu[0][..., :nx])


def test_split_layout_ranges():
    from crava_b200 import dist_grid as G
    lay = G.Layout(16, 10, 7, 3)
    assert [lay.z(r) for r in range(3)] == [(0, 3), (3, 5), (5, 7)]
    assert [lay.y(r) for r in range(3)] == [(0, 4), (4, 7), (7, 10)]


def test_split_round_trip_is_identity():
    """With a solve that changes nothing, the split passes (forward with the
    full grid's scale, inverse with its inverse scale) return every grid."""
    import numpy as np
    import torch
    from crava_b200 import dist_grid as G

    class Ops(_NumpyOps):
        def solve(self, mu, data, cov, err):
            pass

    lay = G.Layout(*SPLIT_SHAPE, 1)
    mu, data, cov, err = _split_inputs()
    t = lambda gs: [torch.from_numpy(g.copy()) for g in gs]
    mu_t, data_t, cov_t, err_t = t(mu), t(data), t(cov), t([err])[0]
    G.posterior_unit_split(Ops(lay.nxp, lay.nxp * lay.nyp * lay.nzp), lay, 0, None, mu_t, data_t, cov_t, err_t)
    nx = SPLIT_SHAPE[0]
    for a, b in zip(mu_t + data_t + cov_t, mu + data + cov):
        assert np.allclose(a.numpy()[..., :nx], b[..., :nx], rtol=1e-5, atol=1e-5)


def _loglik_worker(rank, world, port, out):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import torch
    from crava_b200 import dist as D
    from crava_b200 import dist_grid as G

    dist = D.init("gloo", timeout_s=60)
    lay = G.Layout(*SPLIT_SHAPE, world)
    z0, z1 = lay.z(rank)
    mu, data, cov, err = _split_inputs()
    t = lambda gs: [torch.from_numpy(g[z0:z1].copy()) for g in gs]
    cols = G.spectra_to_columns(_NumpyOps(lay.nxp, lay.nxp * lay.nyp * lay.nzp), lay, rank, dist,
                                t(mu), t(data), t(cov), t([err])[0])
    out.put((rank, G.loglik_grad_split(_toy_loglik, dist, *cols)))
    dist.destroy_process_group()


def _toy_loglik(mu, data, cov, err):
    """A per-bin sum with the shape of the real functional's outputs."""
    import numpy as np
    c = lambda g: g.numpy().view(np.complex64).astype(np.complex128)
    L = float(sum((np.abs(c(d)) ** 2).sum() for d in data))
    gs = np.array([float(np.abs(c(d)).sum()) for d in data])
    gv = np.array([float(c(m).real.sum()) for m in mu[:len(data)]])
    gw = np.stack([c(d).sum(axis=(1, 2)) for d in data], -1)[: SPLIT_SHAPE[2] // 2 + 1]
    return L, gs, gv, gw, int((np.abs(c(err)) > 1.0).sum())


def test_loglik_over_split_grid_sums_the_shards():
    """The all-reduced per-shard functional over 3 gloo ranks equals the
    whole grid's."""
    import numpy as np
    import torch
    from crava_b200 import dist_grid as G

    world = 3
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_loglik_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=180) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    lay = G.Layout(*SPLIT_SHAPE, 1)
    mu, data, cov, err = _split_inputs()
    t = lambda gs: [torch.from_numpy(g.copy()) for g in gs]
    cols = G.spectra_to_columns(_NumpyOps(lay.nxp, lay.nxp * lay.nyp * lay.nzp), lay, 0, None,
                                t(mu), t(data), t(cov), t([err])[0])
    L, gs, gv, gw, nf = G.loglik_grad_split(_toy_loglik, None, *cols)
    for r in range(world):
        L2, gs2, gv2, gw2, nf2 = res[r]
        assert np.isclose(L2, L, rtol=1e-6) and nf2 == nf
        assert np.allclose(gs2, gs, rtol=1e-6) and np.allclose(gv2, gv, rtol=1e-5, atol=1e-6)
        assert np.allclose(gw2, gw, rtol=1e-5, atol=1e-5)


def test_split_layout_check():
    from crava_b200 import dist_grid as G
    G.check_layout(G.Layout(256, 256, 512, 2))
    G.check_layout(G.Layout(256, 256, 512, 4))
    with pytest.raises(ValueError):
        G.check_layout(G.Layout(256, 256, 512, 3))  # 86 / 85 rows


def test_exchange_plan_pairs_match():
    """Every send of rank r to p has the shape of p's receive from r, in
    both directions, for even and uneven splits."""
    from crava_b200 import dist_grid as G

    for shape, world in ((SPLIT_SHAPE, 3), ((256, 256, 512), 4), ((16, 10, 7), 3)):
        lay = G.Layout(*shape, world)
        for direction in ("to_columns", "to_slabs"):
            plans = {r: G.exchange_plan(lay, r, direction) for r in range(world)}
            for r in range(world):
                sends = {peer: (z, y) for kind, peer, z, y in plans[r] if kind == "send"}
                for p in range(world):
                    if p == r:
                        continue
                    recv = [(z, y) for kind, peer, z, y in plans[p] if kind == "recv" and peer == r]
                    assert len(recv) == 1
                    (sz, sy), (rz, ry) = sends[p], recv[0]
                    assert (sz[1] - sz[0], sy[1] - sy[0]) == (rz[1] - rz[0], ry[1] - ry[0])


class _RecordingDist:
    """Stands in for torch.distributed: records the grouped point-to-point
    operations instead of sending them (receive buffers stay as they are)."""

    def __init__(self, backend):
        self.backend, self.posted = backend, []

    def get_backend(self):
        return self.backend

    isend, irecv = "isend", "irecv"

    class P2POp:
        def __init__(self, op, tensor, peer):
            self.op, self.tensor, self.peer = op, tensor, peer

    def batch_isend_irecv(self, ops):
        self.posted.append([(o.op, o.peer, tuple(o.tensor.shape)) for o in ops])
        return []


def test_exchange_posts_one_group_and_same_ops_on_both_backends():
    """Each exchange is one batch_isend_irecv group, and NCCL and gloo are
    given the same operations in the same order."""
    import torch
    from crava_b200 import dist_grid as G

    lay = G.Layout(*SPLIT_SHAPE, 3)
    rank = 1
    z0, z1 = lay.z(rank)
    y0, y1 = lay.y(rank)
    posted = {}
    for backend in ("nccl", "gloo"):
        d = _RecordingDist(backend)
        slab = torch.zeros((z1 - z0, lay.nyp, 2 * lay.cnxp))
        cols = G.to_columns(slab, lay, rank, d)
        G.to_slabs(cols, lay, rank, d, slab)
        posted[backend] = d.posted
    assert len(posted["nccl"]) == 2  # one group per direction
    assert posted["nccl"] == posted["gloo"]
    assert [op for op, _, _ in posted["nccl"][0]] == ["isend", "irecv"] * 2
