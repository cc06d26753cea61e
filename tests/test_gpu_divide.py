"""The data divided by the local scale wavelet (Crava::divideDataByScaleWavelet,
src/crava.cpp:591-722, without interpolateSeismic) on the device: against the
reference's FFTW sequence (committed fixture) and the restatement, with and
without local shift and gain grids, even and odd sizes; padding kept."""
import os

import numpy as np
import pytest

from crava_b200 import api, synth
from oracle import oracle as O
from tests import golden_cases as GC

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


@pytest.mark.parametrize("name", ["c3_12x10x16", "c2_9x8x20_odd"])
def test_divide_vs_reference_fixture(name):
    z = np.load(os.path.join(os.path.dirname(__file__), "golden", "divide.npz"))
    case, _ = GC.load(name)
    nx, ny, nz = (int(v) for v in z[f"{name}_size"])
    case.nz = nz
    shift = z[f"{name}_shift"] if f"{name}_shift" in z else None
    gain = z[f"{name}_gain"] if f"{name}_gain" in z else None
    ctx = api.Context(case)
    data = [api.to_device(g) for g in case.data]
    cov = api.to_device(case.cov[0])
    ctx.divide_data_by_scale_wavelet(data, cov, z[f"{name}_rel_thick"], nx, ny, float(z[f"{name}_dz"]),
                                     shift, gain)
    for g, ref, orig in zip(data, z[f"{name}_out"], case.data):
        out = g.cpu().numpy()
        assert rel(out[..., :case.nxp], ref[..., :case.nxp]) < 1e-5
        assert np.array_equal(out[..., case.nxp:], orig[..., case.nxp:])  # row padding kept


@pytest.mark.parametrize("shape,nxy,local", [((64, 48, 96), (56, 40), True), ((75, 21, 35), (70, 20), False),
                                             ((16, 1, 32), (14, 1), True),
                                             ((40, 30, 128), (36, 28), True),   # fused one-pass kernel
                                             ((35, 12, 256), (30, 12), False)])
def test_divide_vs_restatement(shape, nxy, local):
    nxp, nyp, nzp = shape
    nx, ny = nxy
    case = synth.make_case(nxp, nyp, nzp, (0.0, 15.0, 30.0), 0.1, seed=41)
    case.nz = nzp - 8
    rng = np.random.default_rng(5)
    rt = rng.uniform(0.75, 1.25, (nyp, nxp))
    shift = rng.uniform(-5, 5, (3, ny, nx)).astype(np.float32) if local else None
    gain = rng.uniform(0.7, 1.3, (3, ny, nx)).astype(np.float32) if local else None
    dz = float(np.float32(case.lz / case.nz))
    ctx = api.Context(case)
    data = [api.to_device(g) for g in case.data]
    ctx.divide_data_by_scale_wavelet(data, api.to_device(case.cov[0]), rt, nx, ny, dz, shift, gain)
    ref = O.divide_data(case, case.data, case.cov[0][:, 0, 0].copy(), rt, nx, ny, dz, shift, gain, "orc")
    for g, r in zip(data, ref):
        assert rel(g.cpu().numpy()[..., :nxp], r[..., :nxp]) < 1e-5


def test_divide_rejects_bad_arguments():
    case = synth.make_case(16, 12, 32, (10.0,), 0.1, seed=1)
    ctx = api.Context(case)
    data = [api.to_device(g) for g in case.data]
    cov = api.to_device(case.cov[0])
    rt = np.ones((12, 16))
    with pytest.raises(api.CravaGpuError):
        ctx.divide_data_by_scale_wavelet(data, cov, rt, 17, 12, 4.0)  # nx above nxp
    with pytest.raises(api.CravaGpuError):
        ctx.divide_data_by_scale_wavelet(data, cov, rt, 16, 12, 0.0)  # dz not positive


def _planted_grid(nxp, nyp, nzp, nx, ny, bad, seed=0):
    rng = np.random.default_rng(seed)
    g = rng.standard_normal((nzp, nyp, 2 * (nxp // 2 + 1))).astype(np.float32)
    for n, (i, j) in enumerate(bad):
        g[:, j, i] = 0.0 if n % 2 == 0 else 1e-3  # zero and low-energy traces
    return g


@pytest.mark.parametrize("shape,nxy,bad", [
    ((16, 12, 24), (12, 10), [(3, 4), (4, 4), (5, 4), (0, 0), (11, 9), (5, 0), (6, 6), (7, 7), (6, 7)]),
    ((20, 16, 30), (18, 14), [(0, j) for j in range(14)] + [(17, 3), (9, 9), (9, 10), (10, 9), (10, 10)]),
    ((15, 1, 20), (13, 1), [(2, 0), (3, 0), (12, 0)]),
])
def test_interpolate_seismic_vs_restatement(shape, nxy, bad):
    """interpolateSeismic: energies, the flag walk and the interpolations bit
    for bit; the extrapolated padding to 1 float ulp (pow of CUDA and of
    the C library)."""
    nxp, nyp, nzp = shape
    nx, ny = nxy
    case = synth.make_case(nxp, nyp, nzp, (10.0,), 0.1, seed=3)
    case.nz = nzp - 4
    ctx = api.Context(case)
    g = _planted_grid(nxp, nyp, nzp, nx, ny, bad)
    ref, ni, n0 = O.interpolate_seismic(g, nxp, nyp, nzp, nx, ny, case.nz, 0.05)
    t = api.to_device(g)
    gi, g0 = ctx.interpolate_seismic(t, nx, ny, 0.05)
    assert (gi, g0) == (ni, n0) and ni == len(bad)
    out = t.cpu().numpy()
    ob, rb = out.view(np.int32).astype(np.int64), ref.view(np.int32).astype(np.int64)
    assert np.array_equal(out[:, :ny, :nx], ref[:, :ny, :nx])  # simbox traces
    assert np.abs(ob - rb).max() <= 1


@pytest.mark.parametrize("shape,nxy,local", [((16, 12, 32), (12, 10), True), ((15, 10, 21), (13, 9), False),
                                             ((16, 1, 32), (14, 1), False),
                                             ((24, 20, 128), (20, 18), True),   # fused one-pass kernel
                                             ((15, 9, 256), (13, 9), False)])
def test_multiply_back_vs_restatement(shape, nxy, local):
    """multiplyDataByScaleWaveletAndWriteToFile (before the write): the
    inverse transform of the residual spectra, then each simbox trace times
    its local wavelet's conjugate spectrum; other traces unchanged."""
    nxp, nyp, nzp = shape
    nx, ny = nxy
    case = synth.make_case(nxp, nyp, nzp, (0.0, 15.0, 30.0), 0.1, seed=44)
    rng = np.random.default_rng(8)
    rt = rng.uniform(0.75, 1.25, (nyp, nxp))
    shift = rng.uniform(-5, 5, (3, ny, nx)).astype(np.float32) if local else None
    gain = rng.uniform(0.7, 1.3, (3, ny, nx)).astype(np.float32) if local else None
    dz = float(np.float32(case.lz / case.nz))
    ctx = api.Context(case)
    spec = [api.to_device(g) for g in case.data]
    for g in spec:
        ctx.fft_r2c(g, api.DATA)
    timed = [g.clone() for g in spec]
    for g in timed:
        ctx.fft_c2r(g, api.DATA)
    ctx.multiply_data_by_scale_wavelet(spec, rt, nx, ny, dz, shift, gain)
    ref = O.multiply_data(case, [g.cpu().numpy() for g in timed], rt, nx, ny, dz, shift, gain)
    for g, r, t0 in zip(spec, ref, timed):
        out = g.cpu().numpy()
        assert rel(out[:, :ny, :nx], r[:, :ny, :nx]) < 1e-5
        assert np.array_equal(out[:, :, nx:nxp], t0.cpu().numpy()[:, :, nx:nxp])  # traces left alone
        assert np.array_equal(out[:, ny:, :nxp], t0.cpu().numpy()[:, ny:, :nxp])
