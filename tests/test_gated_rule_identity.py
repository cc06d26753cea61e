"""The identity the forward z pass relies on for the FP64 form's band-gated
covariance rule (crava_b200/csrc/fft.cuh, zprior_apply): for a finite
float c and a double S0 with 1e-200 <= |S0| <= 1e200, the FP64 form's
prior |c / S0| S0 evaluated in double and rounded to float equals
sign(S0) |c| exactly, so the pass writes sign(S0) |c| without the double
division; outside that range (where c / S0 can overflow or lose bits) the
host makes the pass evaluate the double expression.  Checked here on the
CPU over random and edge-case values with IEEE double arithmetic (numpy),
which is what the solve's rule (solve_bin.cuh prior_d) computes."""
import numpy as np


def _fp64_rule(c, v):
    x = c.astype(np.float64)
    with np.errstate(over="ignore", under="ignore"):
        r = np.where(v != 0.0, np.abs(x / v) * v, np.abs(x))
    return r.astype(np.float32)


def _shortcut(c, v):
    a = np.abs(c)
    return np.where(v != 0.0, np.where(v < 0.0, -a, a), a).astype(np.float32)


def test_fp64_rule_equals_sign_times_abs():
    rng = np.random.default_rng(12)
    n = 1_000_000
    # spectra spanning the float range the transforms produce, both signs
    c = (rng.standard_normal(n) * 10.0 ** rng.uniform(-30, 30, n)).astype(np.float32)
    c[:8] = np.array([0.0, -0.0, 1e-45, -1e-45, 3.4e38, -3.4e38, 1.0, -1.0], np.float32)
    # the six Sigma0 entries: variances and covariances of either sign
    vs = [6.4e-3, 1.44e-2, 2.5e-3, 6.72e-3, -2.0e-3, 2.4e-3, 1.0, -7.3e-5, 1e-200, -1e-200, 1e200, -1e200]
    vs += list(rng.choice([-1.0, 1.0], 40) * 10.0 ** rng.uniform(-200, 200, 40))
    for v in vs:
        got, want = _shortcut(c, np.float64(v)), _fp64_rule(c, np.float64(v))
        assert np.array_equal(got.view(np.uint32), want.view(np.uint32)), v


def test_identity_fails_outside_the_guarded_range():
    """Why the range guard exists: with |S0| = 1e-300 the double quotient
    of a large float overflows."""
    c = np.array([3.0e38], np.float32)
    with np.errstate(over="ignore"):
        assert not np.array_equal(_shortcut(c, np.float64(1e-300)), _fp64_rule(c, np.float64(1e-300)))


def test_zero_variance_keeps_abs():
    c = np.array([-2.5, 0.0, 7.0], np.float32)
    assert np.array_equal(_shortcut(c, np.float64(0.0)), np.abs(c))
    assert np.array_equal(_fp64_rule(c, np.float64(0.0)), np.abs(c))
