"""Synthetic seismic on the device (crava_gpu_synt_seismic) against the
reference's trace loop (committed golden outputs of FFTW 2.1.2) and the CPU
restatement at the lengths with compiled column kernels."""
import os

import numpy as np
import pytest
import torch

from crava_b200 import api, synth
from oracle import oracle as O
from tests import golden_cases as GC

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(np.asarray(b)), 1e-30))


def _run(case, m, nx, ny):
    ctx = api.Context(case)
    dm = [api.to_device(g) for g in m]
    outs = [torch.full_like(dm[0], float("nan")) for _ in range(case.ntheta)]
    ctx.synt_seismic(*dm, outs, nx, ny)
    torch.cuda.synchronize()
    for g, h in zip(dm, m):  # inputs untouched
        assert np.array_equal(g.cpu().numpy(), h)
    return [o.cpu().numpy() for o in outs]


@pytest.mark.parametrize("name", ["c3_12x10x16", "c2_9x8x20_odd", "c5_10x8x24"])
def test_synt_vs_reference_golden(name):
    z = np.load(os.path.join(GC.HERE, "synt_seismic.npz"))
    case, _ = GC.load(name)
    m = list(z[f"{name}_m"])
    k = 0
    while f"{name}_{k}_size" in z:
        nx, ny, nz = (int(v) for v in z[f"{name}_{k}_size"])
        case.nz = nz
        out = _run(case, m, nx, ny)
        for a, b in zip(out, z[f"{name}_{k}_out"]):
            assert rel(a, b) < 1e-5, (name, k, rel(a, b))
        k += 1


# compiled z lengths (fused kernels) and generic lengths
@pytest.mark.parametrize("shape,nz,nx,ny", [((16, 12, 64), 50, 13, 10), ((8, 6, 128), 128, 8, 6),
                                             ((10, 4, 96), 90, 10, 4), ((6, 4, 300), 260, 5, 4),
                                             ((12, 6, 384), 384, 12, 6), ((9, 5, 40), 33, 9, 5),
                                             # all angles in one pass (z lengths 128, 256, 512)
                                             ((12, 10, 128), 100, 10, 9), ((12, 8, 256), 200, 11, 7),
                                             ((10, 6, 512), 480, 9, 5)])
def test_synt_vs_restatement(shape, nz, nx, ny):
    case = synth.make_case(*shape, (0.0, 20.0, 40.0), 0.1, seed=9)
    case.nz = nz
    rng = np.random.default_rng(3)
    m = [rng.standard_normal(case.mu[0].shape).astype(np.float32) for _ in range(3)]
    out = _run(case, m, nx, ny)
    ref = O.synt_seismic(case, m, nx, ny, nz, "orc")
    for a, b in zip(out, ref):
        assert rel(a, b) < 1e-5, rel(a, b)
        # untouched traces are the impedance itself, bit for bit
        assert np.array_equal(a[:, ny:, :], b[:, ny:, :])
        assert np.array_equal(a[..., nx:], b[..., nx:])


def _run_local(case, m, nx, ny, rt, dz, shift, gain):
    ctx = api.Context(case)
    dm = [api.to_device(g) for g in m]
    outs = [torch.full_like(dm[0], float("nan")) for _ in range(case.ntheta)]
    ctx.synt_seismic_local(*dm, outs, rt, dz, shift, gain, nx, ny)
    torch.cuda.synchronize()
    for g, h in zip(dm, m):  # inputs untouched
        assert np.array_equal(g.cpu().numpy(), h)
    return [o.cpu().numpy() for o in outs]


@pytest.mark.parametrize("name", ["c3_12x10x16", "c2_9x8x20_odd"])
def test_synt_local_vs_reference_golden(name):
    """Every simbox trace filtered with its own local wavelet (relative
    thickness stretch, local shift and gain) against the reference's trace
    loop on FFTW 2.1.2 (golden fixture): < 1e-5; the other traces are the
    impedance bit for bit."""
    z = np.load(os.path.join(GC.HERE, "synt_local.npz"))
    case, _ = GC.load(name)
    nx, ny, nz = (int(v) for v in z[f"{name}_size"])
    case.nz = nz
    sh = z[f"{name}_shift"] if f"{name}_shift" in z else None
    ga = z[f"{name}_gain"] if f"{name}_gain" in z else None
    out = _run_local(case, list(z[f"{name}_m"]), nx, ny, z[f"{name}_rel_thick"], float(z[f"{name}_dz"]), sh, ga)
    for a, b in zip(out, z[f"{name}_out"]):
        assert rel(a, b) < 1e-5, rel(a, b)
        assert np.array_equal(a[:, ny:, :], b[:, ny:, :])
        assert np.array_equal(a[..., nx:], b[..., nx:])


@pytest.mark.skipif(not O.have_ref(), reason="oracle/_ref (the reference's FFTW build) is not built")
@pytest.mark.parametrize("shape,nz,nx,ny,local", [((12, 10, 128), 100, 10, 9, True),
                                                   ((12, 8, 256), 200, 11, 7, False),
                                                   ((10, 6, 512), 480, 9, 5, True),
                                                   ((9, 7, 96), 80, 8, 6, True)])
def test_synt_local_vs_reference_live(shape, nz, nx, ny, local):
    """At the z lengths of the one-pass filter kernel (128/256/512) and a
    multi-pass length: the device against the reference's trace loop run
    here (oracle/_ref), < 1e-5."""
    case = synth.make_case(*shape, (0.0, 20.0, 40.0), 0.1, seed=19)
    case.nz = nz
    rng = np.random.default_rng(5)
    m = [rng.standard_normal(case.mu[0].shape).astype(np.float32) for _ in range(3)]
    rt = rng.uniform(0.7, 1.3, (case.nyp, case.nxp))
    dz = float(np.float32(case.lz / nz))
    shift = gain = None
    if local:
        shift = rng.uniform(-6.0, 6.0, (case.ntheta, ny, nx)).astype(np.float32)
        gain = rng.uniform(0.6, 1.4, (case.ntheta, ny, nx)).astype(np.float32)
        gain[1, 0, 0] = -999.0  # WELLMISSING: no gain there
    out = _run_local(case, m, nx, ny, rt, dz, shift, gain)
    ref = O.synt_seismic_local(case, m, rt, dz, shift, gain, nx, ny, nz)
    for a, b in zip(out, ref):
        assert rel(a, b) < 1e-5, rel(a, b)
        assert np.array_equal(a[:, ny:, :], b[:, ny:, :])
