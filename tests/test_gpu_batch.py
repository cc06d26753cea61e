"""Launch-shape choices, the autotuner and the vintage batch (CUDA graph):
every tile choice gives the same transform, and a batch run gives exactly
what the separate entry points give."""
import numpy as np
import pytest
import torch

from crava_b200 import api, synth

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(np.asarray(b)), 1e-30))


# every column length with compiled kernels, as y and as z; z planes of 30
# lines (a ragged last TMA tile) and of 35 (odd: no TMA box, the choice
# falls back to the register-resident pass)
TILE_SHAPES = [(8, 64, 128), (8, 256, 512), (8, 96, 160), (8, 192, 200), (8, 300, 384),
               (8, 128, 64), (8, 384, 300), (8, 96, 256), (8, 6, 512), (8, 7, 64)]


@pytest.mark.parametrize("shape", TILE_SHAPES)
def test_column_tiles_match_numpy(shape):
    nx, ny, nz = shape
    case = synth.make_case(nx, ny, nz, (10.0,), 0.1, seed=4)
    ctx = api.Context(case)
    g = case.data[0]
    ref = np.fft.rfftn(g[..., :nx].astype(np.float64), axes=(0, 1, 2)) / np.sqrt(nx * ny * nz)
    res = {}
    for ty in (1, 16, 8, 0):
        for tz in (1, 16, 8, 0, 2):
            ctx.set_tuning(ty, tz, 0)
            t = api.to_device(g)
            ctx.fft_r2c(t, api.DATA)
            out = api.complex_view(t.cpu().numpy(), nx).copy()
            assert rel(out, ref) < 2e-6, (ty, tz)
            ctx.fft_c2r(t, api.DATA)
            back = t.cpu().numpy()[..., :nx]
            assert rel(back, g[..., :nx]) < 2e-6, (ty, tz)
            res[(ty, tz)] = (out, back)
    # the in-place pass does the same arithmetic per line whatever the
    # tile, and so do the register-resident pass (1) where it exists and its
    # TMA-fed z pass (2)
    same = lambda a, b: all(np.array_equal(x, y) for x, y in zip(res[a], res[b]))
    assert same((16, 16), (8, 8)) and same((16, 8), (8, 16))
    assert same((1, 1), (16, 16)) and same((1, 16), (16, 16)) and same((16, 1), (16, 16))
    assert same((1, 2), (1, 1)) and same((16, 2), (16, 1))
    assert ctx.stats().tile_wait_timeouts == 0


# even nxp whose half length has register-resident row kernels, and one without
@pytest.mark.parametrize("shape", [(128, 24, 32), (256, 8, 16), (512, 6, 8), (1024, 4, 8), (96, 12, 16)])
def test_row_pass_choices_match(shape):
    """The register-resident x pass (rows_x 1) and the in-place x pass
    (rows_x 0) give the same transform bit for bit, forward and inverse,
    with and without an addend; both match numpy."""
    nx, ny, nz = shape
    case = synth.make_case(nx, ny, nz, (10.0,), 0.1, seed=6)
    ctx = api.Context(case)
    g = case.data[0]
    ref = np.fft.rfftn(g[..., :nx].astype(np.float64), axes=(0, 1, 2)) / np.sqrt(nx * ny * nz)
    res = {}
    for rx in (1, 0):
        ctx.set_tuning(-1, -1, 0, 2, rx)
        t = api.to_device(g)
        ctx.fft_r2c(t, api.DATA)
        out = t.cpu().numpy().copy()
        assert rel(api.complex_view(out, nx), ref) < 2e-6, rx
        ctx.fft_c2r(t, api.DATA)
        back = t.cpu().numpy().copy()
        assert rel(back[..., :nx], g[..., :nx]) < 2e-6, rx
        res[rx] = (out, back)
    assert np.array_equal(res[0][0], res[1][0]) and np.array_equal(res[0][1], res[1][1])


# planes of 21 x 36 bins (fewer than one CTA's bins in every shape) and of
# 33 x 40; five and two angles
@pytest.mark.parametrize("shape,angles", [((40, 36, 96), (0.0, 10.0, 20.0, 30.0, 40.0)),
                                          ((64, 40, 64), (10.0, 30.0))])
@pytest.mark.parametrize("prec,kappa", [(api.FP64, None), (api.MIXED, None), (api.MIXED, 0.0)])
def test_solve_shapes_match(shape, angles, prec, kappa):
    """Every launch shape of the square-root solves (solve_shape 0-5) gives
    the same outputs and counters bit for bit; kappa_refine 0 sends every
    inverted bin of the mixed form through the FP64 refinement step.  Shape
    6, the Woodbury form of the FP64 solve (the built-in FP64 choice),
    computes the same posterior by other operations: within 1e-9 relative
    L2 of shape 0 per output, same counters (for the mixed form shape 6
    falls back to shape 3)."""
    nx, ny, nz = shape
    case = synth.make_case(nx, ny, nz, angles, 0.1, seed=12)
    ctx = api.Context(case)
    spec = _dev(case)
    mu, data, cov, err = spec
    for g in mu:
        ctx.fft_r2c(g, api.PARAMETER)
    for g in data:
        ctx.fft_r2c(g, api.DATA)
    for g in cov + [err]:
        ctx.fft_r2c(g, api.COVARIANCE)
    res = {}
    for sh in (-1, 0, 1, 2, 3, 4, 5, 6, 7, 8):
        ctx.set_tuning(-1, -1, 0, 2, -1, kappa, None, sh)
        assert ctx.tuning().solve_shape == sh
        m, d, c = [g.clone() for g in mu], [g.clone() for g in data], [g.clone() for g in cov]
        ctx.posterior(m, d, c, err, prec)
        st = ctx.stats()
        res[sh] = ([g.cpu().numpy() for g in m + d + c], st.chol_fail_bins, st.nonfinite_bins, st.refined_bins)
    if kappa == 0.0:
        assert res[0][3] > 0
    woodbury = (-1, 6, 7, 8) if prec == api.FP64 else ()
    for sh in res:
        assert res[sh][1:] == res[0][1:], sh
        if sh in woodbury:
            for a, b in zip(res[sh][0], res[0][0]):
                assert rel(a, b) < 1e-9, (sh, rel(a, b))
        else:
            assert all(np.array_equal(a, b) for a, b in zip(res[sh][0], res[0][0])), sh
    assert all(np.array_equal(a, b) for a, b in zip(res[-1][0], res[6][0]))
    if prec == api.FP64:  # the Woodbury kernel ran (its roundings differ somewhere)
        assert not all(np.array_equal(a, b) for a, b in zip(res[6][0], res[0][0]))
    with pytest.raises(api.CravaGpuError):
        ctx.set_tuning(-1, -1, 0, 2, -1, None, None, 9)


def test_tma_z_pass_unit_matches():
    """The whole out-of-place unit at 128x128x512, 5 angles, with the
    TMA-fed z pass equals the unit with the register-resident z pass bit
    for bit, FP64 and mixed."""
    case = synth.make_case(128, 128, 512, (0.0, 10.0, 20.0, 30.0, 40.0), 0.1, seed=21)
    ctx = api.Context(case)
    src = _dev(case)
    for prec in (api.FP64, api.MIXED):
        outs = {}
        for tz in (1, 2):
            ctx.set_tuning(-1, tz, 0)
            dst = _dev(case)
            ctx.posterior_unit_oop(src, dst, prec)
            outs[tz] = [g.cpu().numpy() for g in dst[0] + dst[1] + dst[2]]
        assert all(np.array_equal(a, b) for a, b in zip(outs[1], outs[2])), prec
    assert ctx.stats().tile_wait_timeouts == 0


def _dev(case):
    d = lambda gs: [api.to_device(g) for g in gs]
    return d(case.mu), d(case.data), d(case.cov), d([case.err_corr])[0]


def test_autotune_keeps_the_fastest_and_the_results():
    case = synth.make_case(64, 64, 128, (10.0, 20.0, 30.0), 0.1, seed=8)
    ctx = api.Context(case, precision=api.FP64)
    src, dst = _dev(case), _dev(case)
    ref = _dev(case)
    ctx.posterior_unit_oop(src, ref, api.FP64)
    best = ctx.autotune(src, dst, api.FP64, reps=2)
    assert best.ms > 0.0
    t = ctx.tuning()
    assert (t.cols_y_tile, t.cols_z_tile, t.fused) == (best.cols_y_tile, best.cols_z_tile, best.fused)
    ctx.posterior_unit_oop(src, dst, api.FP64)
    for a, b in zip(dst[0] + dst[1] + dst[2], ref[0] + ref[1] + ref[2]):
        assert rel(a.cpu().numpy(), b.cpu().numpy()) < 1e-5
    with pytest.raises(api.CravaGpuError):
        ctx.autotune(src, src, api.FP64)  # inputs would be overwritten


def _separate(ctx, case, nsim, seed, first, precision):
    """The batch's work through the separate entry points (reference order:
    transforms, solve, inverse means/residuals, realisations, inverse
    covariances)."""
    mu, data, cov, err = _dev(case)
    for g in mu:
        ctx.fft_r2c(g, api.PARAMETER)
    for g in data:
        ctx.fft_r2c(g, api.DATA)
    for g in cov + [err]:
        ctx.fft_r2c(g, api.COVARIANCE)
    ctx.posterior(mu, data, cov, err, precision)
    for g in mu:
        ctx.fft_c2r(g, api.PARAMETER)
    for g in data:
        ctx.fft_c2r(g, api.DATA)
    sims = [torch.zeros_like(mu[0]) for _ in range(3 * nsim)]
    if nsim:
        ctx.simulate(cov, mu, seed, first, sims)
    for g in cov:
        ctx.fft_c2r(g, api.COVARIANCE)
    return mu, data, cov, sims


@pytest.mark.parametrize("flags", [0, api.BATCH_NO_GRAPH])
def test_batch_matches_separate_calls(flags):
    cases = [synth.make_case(32, 24, 64, (10.0, 20.0, 30.0), 0.1, seed=31),
             synth.make_case(20, 18, 30, (0.0, 10.0, 20.0, 30.0, 40.0), 0.1, seed=32),
             synth.make_case(64, 48, 40, (5.0, 25.0), 0.1, seed=33)]
    nsims, seeds, firsts = [3, 2, 0], [5, 6, 7], [0, 10, 0]
    precs = [api.MIXED, api.FP64, api.FP64]
    ctxs = [api.Context(c, precision=p) for c, p in zip(cases, precs)]
    ctxs[2].set_fused(True)  # the fused unit inside the graph too
    vint, dsts, simss = [], [], []
    for c, ctx, n, s, f, p in zip(cases, ctxs, nsims, seeds, firsts, precs):
        src, dst = _dev(c), _dev(c)
        sims = [torch.zeros_like(src[0][0]) for _ in range(3 * n)]
        vint.append(dict(ctx=ctx, src=src, dst=dst, precision=p, nsim=n, seed=s, first_index=f,
                         sims=sims))
        dsts.append(dst)
        simss.append(sims)
    b = api.Batch(vint, flags)
    n0 = api.launch_count()
    for run in range(2):
        b.run()
        b.sync()
        for k, (c, ctx) in enumerate(zip(cases, ctxs)):
            if k == 2:
                ref = _dev(c)
                ctx.posterior_unit_oop(_dev(c), ref, precs[k])
                mu, data, cov = ref[0], ref[1], ref[2]
                sims = []
            else:
                mu, data, cov, sims = _separate(ctx, c, nsims[k], seeds[k],
                                                firsts[k] + run * nsims[k], precs[k])
            mine = dsts[k]
            for a, r in zip(mine[0] + mine[1] + mine[2], mu + data + cov):
                assert torch.equal(a, r), (run, k)
            for a, r in zip(simss[k], sims):
                assert torch.equal(a, r), (run, k)
    assert api.launch_count() - n0 > 0
    b.close()


def test_batch_rejects_in_place_vintages():
    case = synth.make_case(16, 12, 32, (10.0,), 0.1, seed=1)
    ctx = api.Context(case)
    g = _dev(case)
    with pytest.raises(api.CravaGpuError):
        api.Batch([dict(ctx=ctx, src=g, dst=g, precision=api.FP64)])


@pytest.mark.parametrize("shape", [(256, 256, 16), (128, 128, 24), (256, 256, 512)])
def test_fused_xy_pass_matches_numpy_and_separate_passes(shape):
    """The x and y passes as one cluster kernel (xy_fused) against numpy
    and against the separate passes (float rounding: the y transform is
    factorised differently), forward and inverse, in place."""
    nx, ny, nz = shape
    case = synth.make_case(nx, ny, nz, (10.0,), 0.1, seed=12)
    ctx = api.Context(case)
    g = case.data[0]
    ref = np.fft.rfftn(g[..., :nx].astype(np.float64), axes=(0, 1, 2)) / np.sqrt(nx * ny * nz)
    res = {}
    for xy in (1, 0):
        ctx.set_tuning(-1, -1, 0, 2, -1, None, xy)
        t = api.to_device(g)
        ctx.fft_r2c(t, api.DATA)
        out = api.complex_view(t.cpu().numpy(), nx).copy()
        assert rel(out, ref) < 2e-6, xy
        ctx.fft_c2r(t, api.DATA)
        back = t.cpu().numpy()
        assert rel(back[..., :nx], g[..., :nx]) < 2e-6, xy
        assert np.all(back[..., nx:] == 0.0)  # the padding floats
        res[xy] = (out, back)
    assert rel(res[1][0], res[0][0]) < 1e-6 and rel(res[1][1][..., :nx], res[0][1][..., :nx]) < 1e-6


def test_fused_xy_unit_out_of_place_matches_separate_passes():
    """The whole out-of-place unit (forward transforms read the inputs and
    write the work grids) with and without the fused x + y pass."""
    case = synth.make_case(128, 128, 64, (0.0, 15.0, 30.0), 0.1, seed=13)
    ctx = api.Context(case, precision=api.FP64)
    src = _dev(case)
    outs = {}
    for xy in (1, 0):
        ctx.set_tuning(-1, -1, 0, 2, -1, None, xy)
        dst = _dev(case)
        ctx.posterior_unit_oop(src, dst, api.FP64)
        outs[xy] = [t.cpu().numpy() for t in dst[0] + dst[1] + dst[2]]
    for a, b in zip(outs[1], outs[0]):
        assert rel(a[..., :128], b[..., :128]) < 1e-5
    for t, h in zip(src[0] + src[1] + src[2] + [src[3]], case.mu + case.data + case.cov + [case.err_corr]):
        assert np.array_equal(t.cpu().numpy(), h)  # inputs untouched
