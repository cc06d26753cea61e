"""Seeded time-lapse states for the State4D tests (src/state4d.cpp).

Per complex bin: a random Hermitian positive-definite 6x6 prior over
(static, dynamic) x (vp, vs, rho) with a random prior mean, and an inverted
current state (mean and covariance) derived from it.  Bins 0, fail_every,
2 fail_every, ... (none when fail_every is 0) have their prior negated, so
that the reference's 3x3 Cholesky of the current prior fails there and
split keeps the prior.  real_post_cov keeps only the real part of the
current covariance (as for symmetric correlation functions), so that the
reference's unconjugated copy of its lower triangle (src/state4d.cpp:370-372)
leaves it Hermitian.  Grids are float32
arrays in the padded real layout [nzp][nyp][2 (nxp/2 + 1)] holding
interleaved complex spectra, as the device grids hold them.
"""
import numpy as np

P = (0, 0, 0, 1, 1, 2)
Q = (0, 1, 2, 1, 2, 2)
UNIT = (0, 3, 4, 1, 5, 2)  # slot of State4D's (P[r], Q[r]) in the posterior order
KEYS = ("ms", "md", "ss", "dd", "sd")


def grid_shape(nxp, nyp, nzp):
    return (nzp, nyp, 2 * (nxp // 2 + 1))


def _grid(vals, shape):
    return np.ascontiguousarray(vals.astype(np.complex64)).view(np.float32).reshape(shape).copy()


def to_complex(g):
    return np.ascontiguousarray(g).view(np.complex64).reshape(-1)


def random_state(nxp, nyp, nzp, seed, fail_every=37, real_post_cov=False):
    shape = grid_shape(nxp, nyp, nzp)
    n = shape[0] * shape[1] * shape[2] // 2
    rng = np.random.default_rng(seed)
    Z = rng.standard_normal((n, 6, 6)) + 1j * rng.standard_normal((n, 6, 6))
    S = Z @ np.conj(np.transpose(Z, (0, 2, 1))) / 6.0 + 0.3 * np.eye(6)
    if fail_every:
        S[::fail_every] *= -1.0  # bins 0, fail_every, 2 fail_every, ...
    m = rng.standard_normal((n, 6)) + 1j * rng.standard_normal((n, 6))
    state = {
        "ms": [_grid(m[:, l], shape) for l in range(3)],
        "md": [_grid(m[:, l + 3], shape) for l in range(3)],
        "ss": [_grid(S[:, P[r], Q[r]], shape) for r in range(6)],
        "dd": [_grid(S[:, P[r] + 3, Q[r] + 3], shape) for r in range(6)],
        "sd": [_grid(S[:, l, k + 3], shape) for l in range(3) for k in range(3)],
    }
    C = S[:, :3, :3] + S[:, 3:, 3:] + S[:, 3:, :3] + S[:, :3, 3:]
    mc = m[:, :3] + m[:, 3:]
    cpost = 0.6 * (C.real if real_post_cov else C)
    mpost = 0.8 * mc + 0.1 * (rng.standard_normal((n, 3)) + 1j * rng.standard_normal((n, 3)))
    mu = [_grid(mpost[:, l], shape) for l in range(3)]
    cov = [None] * 6
    for r in range(6):
        cov[UNIT[r]] = _grid(cpost[:, P[r], Q[r]], shape)
    return state, mu, cov


def evolution(seed):
    """A transition of the (static, dynamic) state: E near the identity,
    a mean correction and a symmetric positive covariance correction."""
    rng = np.random.default_rng(seed)
    E = np.eye(6) + 0.1 * rng.standard_normal((6, 6))
    cm = rng.standard_normal(6)
    G = rng.standard_normal((6, 6))
    cc = G @ G.T / 6.0 + 0.1 * np.eye(6)
    return E, cm, cc


def copy_state(state):
    return {k: [g.copy() for g in state[k]] for k in KEYS}
