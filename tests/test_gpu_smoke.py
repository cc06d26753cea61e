"""First end-to-end GPU checks against the CPU oracle (small grids)."""
import numpy as np
import pytest

from crava_b200 import api, synth
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(np.asarray(b)), 1e-30))


@pytest.mark.parametrize("shape", [(16, 12, 32), (20, 18, 30), (15, 16, 20), (64, 64, 128),
                                   (96, 200, 30), (192, 160, 24), (75, 21, 35), (128, 128, 256),
                                   (16, 1, 32), (15, 1, 20)])
@pytest.mark.parametrize("gtype", [api.DATA, api.COVARIANCE])
def test_fft_roundtrip_and_oracle(shape, gtype):
    nx, ny, nz = shape
    case = synth.make_case(nx, ny, nz, (10.0, 20.0), 0.1, seed=5)
    ctx = api.Context(case)
    g = case.data[0] if gtype == api.DATA else case.cov[0]
    t = api.to_device(g)
    ctx.fft_r2c(t, gtype)
    out = t.cpu().numpy()
    ref = O.fft_r2c(g, nx, ny, nz, gtype, "orc")
    assert rel(api.complex_view(out, nx), O.complex_view(ref, nx)) < 1e-6
    ctx.fft_c2r(t, gtype)
    back = t.cpu().numpy()
    assert rel(back[..., :nx], g[..., :nx]) < 1e-6


def _spectra_dev(case, sp):
    mu = [api.to_device(g) for g in sp["mu"]]
    data = [api.to_device(g) for g in sp["data"]]
    cov = [api.to_device(g) for g in sp["cov"]]
    err = api.to_device(sp["err"])
    return mu, data, cov, err


@pytest.mark.parametrize("shape,angles", [((16, 12, 32), (10.0, 20.0, 30.0)),
                                          ((20, 18, 30), (0.0, 10.0, 20.0, 30.0, 40.0)),
                                          ((15, 16, 20), (5.0, 25.0))])
def test_solve_fp32_bitexact_vs_reference_order(shape, angles):
    case = synth.make_case(*shape, angles, 0.1, seed=7)
    sp = O.forward_spectra(case, "orc")
    tables = O.kz_tables(case, "orc")
    ctx = api.Context(case)
    ctx.set_kz_tables(tables)
    mu, data, cov, err = _spectra_dev(case, sp)
    ctx.posterior(mu, data, cov, err, api.FP32)
    st = ctx.stats()
    omu, ores, ocov, ofail = O.posterior_fp32_tables(case, sp, tables, "orc")
    nx = case.nxp
    for g, o in zip(mu + data + cov, omu + ores + ocov):
        a = api.complex_view(g.cpu().numpy(), nx)
        b = O.complex_view(o, nx)
        assert np.array_equal(a.view(np.uint64), b.view(np.uint64)), rel(a, b)
    assert st.chol_fail_bins == ofail


@pytest.mark.parametrize("prec,tol", [(api.FP64, 1e-7), (api.MIXED, 1e-5)])
@pytest.mark.parametrize("noise", [0.1, 0.01])
def test_solve_vs_fp64_oracle(prec, tol, noise):
    case = synth.make_case(16, 12, 64, (0.0, 10.0, 20.0, 30.0, 40.0), noise, seed=11)
    sp = O.forward_spectra(case, "orc")
    tables = O.kz_tables(case, "orc")
    ctx = api.Context(case)
    ctx.set_kz_tables(tables)
    mu, data, cov, err = _spectra_dev(case, sp)
    ctx.posterior(mu, data, cov, err, prec)
    dmu, dres, dcov, dfail = O.posterior_fp64(case, sp)
    nx = case.nxp
    errs = []
    for g, o in zip(mu + data + cov, dmu + dres + dcov):
        errs.append(rel(api.complex_view(g.cpu().numpy(), nx), o))
    assert max(errs) < tol, errs


@pytest.mark.parametrize("angles", [(20.0,), (0.0, 5.0, 10.0, 15.0, 20.0, 25.0, 30.0, 35.0)])
def test_solve_one_and_eight_angles(angles):
    """The smallest and largest angle counts: FP32 form bit for bit with the
    reference order, FP64 and mixed forms against the FP64 oracle."""
    case = synth.make_case(12, 10, 32, angles, 0.1, seed=17)
    sp = O.forward_spectra(case, "orc")
    tables = O.kz_tables(case, "orc")
    nx = case.nxp
    ctx = api.Context(case)
    ctx.set_kz_tables(tables)
    mu, data, cov, err = _spectra_dev(case, sp)
    ctx.posterior(mu, data, cov, err, api.FP32)
    omu, ores, ocov, _ = O.posterior_fp32_tables(case, sp, tables, "orc")
    for g, o in zip(mu + data + cov, omu + ores + ocov):
        a = api.complex_view(g.cpu().numpy(), nx)
        assert np.array_equal(a.view(np.uint64), O.complex_view(o, nx).view(np.uint64))
    dmu, dres, dcov, _ = O.posterior_fp64(case, sp)
    for prec, tol in [(api.FP64, 1e-7), (api.MIXED, 1e-5)]:
        mu, data, cov, err = _spectra_dev(case, sp)
        ctx.posterior(mu, data, cov, err, prec)
        errs = [rel(api.complex_view(g.cpu().numpy(), nx), o) for g, o in zip(mu + data + cov, dmu + dres + dcov)]
        assert max(errs) < tol, (prec, errs)


def test_unit_vs_reference_unit():
    case = synth.config_small()
    ctx = api.Context(case)
    mu = [api.to_device(g) for g in case.mu]
    data = [api.to_device(g) for g in case.data]
    cov = [api.to_device(g) for g in case.cov]
    err = api.to_device(case.err_corr)
    ctx.posterior_unit(mu, data, cov, err, api.FP32)
    which = "ref" if O.have_ref() else "orc"
    omu, ores, ocov, ofail = O.unit_fp32(case, which)
    nx = case.nxp
    for g, o in zip(mu + data + cov, omu + ores + ocov):
        assert rel(g.cpu().numpy()[..., :nx], o[..., :nx]) < 2e-5


@pytest.mark.parametrize("shape", [(16, 1, 32), (15, 1, 20)])
def test_unit_single_line(shape):
    """A 2-D section (nyp = 1: length-1 y lines, every bin its own y
    partner) through the whole unit, against the reference's numerics."""
    case = synth.make_case(*shape, (10.0, 20.0, 30.0), 0.1, seed=5)
    ctx = api.Context(case)
    d = lambda gs: [api.to_device(g) for g in gs]
    mu, data, cov, err = d(case.mu), d(case.data), d(case.cov), d([case.err_corr])[0]
    ctx.posterior_unit(mu, data, cov, err, api.FP32)
    which = "ref" if O.have_ref() else "orc"
    omu, ores, ocov, ofail = O.unit_fp32(case, which)
    nx = case.nxp
    for g, o in zip(mu + data + cov, omu + ores + ocov):
        assert rel(g.cpu().numpy()[..., :nx], o[..., :nx]) < 2e-5


@pytest.mark.parametrize("shape", [(32, 24, 64), (15, 16, 20)])
def test_nonconstant_thickness_unit(shape):
    """The non-constant-thickness branch (K = diag(D) A and its error
    multipliers, src/crava.cpp:1059-1083): device tables vs the restatement
    and the whole unit vs the reference's numerics."""
    case = synth.make_case(*shape, (0.0, 15.0, 30.0), 0.1, seed=13)
    case.thickness_mode = 1
    case.min_rel_thick = 0.8
    ctx = api.Context(case)
    wd, e1, e2, e3, inv = ctx.kz_tables()
    owd, oe1, oe2, oe3, oinv = O.kz_tables(case, "orc")
    assert np.array_equal(inv, oinv)
    for a, b in [(wd, owd), (e1, oe1), (e2, oe2)]:
        assert np.abs(a - b).max() <= 1e-6 * np.abs(b).max()
    m = inv.astype(bool)
    assert np.abs(e3[m] - oe3[m]).max() <= 1e-6 * np.abs(oe3[m]).max()
    ctx.set_kz_tables(O.kz_tables(case, "ref" if O.have_ref() else "orc"))
    d = lambda gs: [api.to_device(g) for g in gs]
    mu, data, cov, err = d(case.mu), d(case.data), d(case.cov), d([case.err_corr])[0]
    ctx.posterior_unit(mu, data, cov, err, api.FP32)
    which = "ref" if O.have_ref() else "orc"
    omu, ores, ocov, ofail = O.unit_fp32(case, which)
    nx = case.nxp
    for g, o in zip(mu + data + cov, omu + ores + ocov):
        assert rel(g.cpu().numpy()[..., :nx], o[..., :nx]) < 2e-5


def test_host_entry_matches_device_unit():
    case = synth.make_case(32, 24, 64, (0.0, 15.0, 30.0), 0.1, seed=9)
    ctx = api.Context(case)
    d = lambda gs: [api.to_device(g) for g in gs]
    mu, data, cov, err = d(case.mu), d(case.data), d(case.cov), d([case.err_corr])[0]
    ctx.posterior_unit(mu, data, cov, err, api.MIXED)
    import torch
    h = [torch.from_numpy(g.copy()).pin_memory() for g in case.grids()]
    nt = case.ntheta
    ctx.posterior_unit_host(h[:3], h[3:3 + nt], h[3 + nt:9 + nt], h[9 + nt], api.MIXED)
    for a, b in zip(mu + data + cov, h[:9 + nt]):
        assert np.array_equal(a.cpu().numpy()[..., :32], b.numpy()[..., :32])
