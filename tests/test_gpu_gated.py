"""The band-gated covariance bins written by the forward z passes.

Outside the inversion band the per-bin loop of the reference only rewrites
the prior covariance (src/crava.cpp:1098-1147 with
getNextParameterCovariance, src/seismicparametersholder.cpp:355-427).  In
the unit the forward z pass of each covariance grid applies that rule as it
stores the spectrum, and the solve visits the inverted planes alone.  The
in-place z pass (column tile 16) has no such epilogue, so with it the solve
does those bins as before; its transform values equal the register-resident
and TMA-fed passes bit for bit, so the two runs must agree bit for bit, the
failure and non-finite counts included (a bin counts once however many of
its six covariance outputs are not finite).
"""
import numpy as np
import pytest

from crava_b200 import api, synth

pytestmark = pytest.mark.gpu

A5 = (0.0, 10.0, 20.0, 30.0, 40.0)
CASES = [
    ((64, 64, 128), A5),          # separate x and y passes, register-resident z pass
    ((128, 128, 256), A5),        # fused x + y pass, TMA-fed z pass
    ((48, 40, 64), (10.0, 20.0, 30.0)),
]


def _dev(case):
    d = lambda gs: [api.to_device(g) for g in gs]
    return d(case.mu), d(case.data), d(case.cov), d([case.err_corr])[0]


def _run(ctx, case, src, prec, tile_z):
    ctx.set_tuning(-1, tile_z, 0, 3, -1)
    dst = _dev(case)
    ctx.posterior_unit_oop(src, dst, prec)
    st = ctx.stats()
    return [g.cpu().numpy() for g in dst[0] + dst[1] + dst[2]], st.nonfinite_bins, st.chol_fail_bins


@pytest.mark.parametrize("shape,angles", CASES)
@pytest.mark.parametrize("prec", [api.FP64, api.MIXED])
def test_gated_rule_in_z_pass_equals_solve(shape, angles, prec):
    case = synth.make_case(*shape, angles, 0.1, seed=31)
    ctx = api.Context(case)
    src = _dev(case)
    got, nf_a, cf_a = _run(ctx, case, src, prec, -1)
    ref, nf_b, cf_b = _run(ctx, case, src, prec, 16)
    assert nf_a == nf_b == 0 and cf_a == cf_b
    for a, b in zip(got, ref):
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32))


@pytest.mark.parametrize("prec", [api.FP64, api.MIXED])
def test_gated_rule_nonfinite_bins_counted_once(prec):
    """A NaN planted in two of the six prior covariance grids makes every
    bin of both non-finite after the transform: each bin counts once, in
    both paths."""
    case = synth.make_case(64, 64, 128, A5, 0.1, seed=32)
    case.cov[1][5, 7, 9] = np.nan
    case.cov[4][60, 3, 2] = np.nan
    ctx = api.Context(case)
    src = _dev(case)
    got, nf_a, cf_a = _run(ctx, case, src, prec, -1)
    ref, nf_b, cf_b = _run(ctx, case, src, prec, 16)
    csize = (case.nxp // 2 + 1) * case.nyp * case.nzp
    assert nf_a == nf_b == csize
    assert cf_a == cf_b
    for a, b in zip(got, ref):
        assert np.array_equal(np.isnan(a), np.isnan(b))
        assert np.array_equal(a, b, equal_nan=True)
