"""The fused posterior unit (cluster xy-plane kernels + fused z/solve kernel)
against the CPU oracle and the three-pass path."""
import numpy as np
import pytest

from crava_b200 import api, synth
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(np.asarray(b)), 1e-30))


SHAPES = [
    ((16, 12, 32), (10.0, 20.0, 30.0)),
    ((64, 64, 128), (10.0, 20.0, 30.0)),
    ((20, 18, 30), (0.0, 10.0, 20.0, 30.0, 40.0)),
    ((15, 16, 20), (5.0, 25.0)),                      # odd nxp
    ((36, 40, 48), (0.0, 10.0, 20.0, 30.0, 40.0)),
    ((128, 96, 64), (10.0, 30.0)),                    # cluster of several CTAs
    ((96, 200, 60), (0.0, 15.0, 30.0)),
]


@pytest.mark.parametrize("shape,angles", SHAPES)
@pytest.mark.parametrize("prec", [api.FP64, api.MIXED])
def test_fused_unit_vs_oracle(shape, angles, prec):
    case = synth.make_case(*shape, angles, 0.1, seed=21)
    ctx = api.Context(case)
    ctx.set_fused(True)
    assert ctx.fused_available(prec)
    d = lambda gs: [api.to_device(g) for g in gs]
    src = (d(case.mu), d(case.data), d(case.cov), d([case.err_corr])[0])
    dst = (d(case.mu), d(case.data), d(case.cov), d([case.err_corr])[0])
    ctx.posterior_unit_oop(src, dst, prec)
    st = ctx.stats()
    assert st.nonfinite_bins == 0
    which = "ref" if O.have_ref() else "orc"
    omu, ores, ocov, ofail = O.unit_fp32(case, which)
    nx = case.nxp
    outs = dst[0] + dst[1] + dst[2]
    # tolerance: the reference's own FP32 solve and FFTs carry up to ~4e-5
    # relative error on the residuals (d - K mu cancels); 1e-4 bounds both.
    for g, o in zip(outs, omu + ores + ocov):
        assert rel(g.cpu().numpy()[..., :nx], o[..., :nx]) < 1e-4
    # inputs untouched
    for g, o in zip(src[0] + src[1] + src[2], case.mu + case.data + case.cov):
        assert np.array_equal(g.cpu().numpy(), o)


@pytest.mark.parametrize("shape,angles", SHAPES[:4])
def test_fused_matches_three_pass(shape, angles):
    case = synth.make_case(*shape, angles, 0.1, seed=22)
    ctx = api.Context(case)
    d = lambda gs: [api.to_device(g) for g in gs]
    src = (d(case.mu), d(case.data), d(case.cov), d([case.err_corr])[0])
    a = (d(case.mu), d(case.data), d(case.cov), d([case.err_corr])[0])
    b = (d(case.mu), d(case.data), d(case.cov), d([case.err_corr])[0])
    ctx.set_fused(True)
    ctx.posterior_unit_oop(src, a, api.FP64)
    ctx.set_fused(False)
    ctx.posterior_unit_oop(src, b, api.FP64)
    nx = case.nxp
    for x, y in zip(a[0] + a[1] + a[2], b[0] + b[1] + b[2]):
        assert rel(x.cpu().numpy()[..., :nx], y.cpu().numpy()[..., :nx]) < 2e-6
