"""The C++ host classes (crava_b200/host/crava_device.hpp) driven like the
reference's Crava drives FFTGrid, compared with the reference fixtures."""
import os
import subprocess

import numpy as np
import pytest

from tests import golden_cases as GC

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "host_mirror_test.cpp")
CUDA = "/usr/local/cuda"


def build(tmp):
    exe = os.path.join(tmp, "host_mirror_test")
    cmd = ["g++", "-O2", "-std=c++17", SRC, "-o", exe, f"-I{ROOT}/include", f"-I{ROOT}/crava_b200/host",
           f"-I{CUDA}/include", f"-L{ROOT}/crava_b200/lib", "-lcrava_gpu", f"-L{CUDA}/lib64", "-lcudart",
           f"-Wl,-rpath,{ROOT}/crava_b200/lib", f"-Wl,-rpath,{CUDA}/lib64"]
    subprocess.run(cmd, check=True)
    return exe


def test_host_mirror_compiles(tmp_path):
    build(str(tmp_path))


@pytest.mark.gpu
@pytest.mark.parametrize("mode", ["bulk", "cursor"])
@pytest.mark.parametrize("name", GC.NAMES)
def test_host_mirror_matches_reference(tmp_path, name, mode):
    """mode "cursor": inputs filled and outputs read through the element
    cursors (setNextReal / getNextReal / getNextComplex / setNextComplex),
    which must equal the bulk copies bit for bit."""
    exe = build(str(tmp_path))
    case, z = GC.load(name)
    d = str(tmp_path)
    np.array([case.nxp, case.nyp, case.nzp, case.ntheta, 2], np.int32).tofile(d + "/dims.bin")
    np.array([case.nz, case.lz, case.min_rel_thick, case.low_cut, case.high_cut, case.wnc],
             np.float64).tofile(d + "/scalars.bin")
    case.wavelet.astype(np.float32).tofile(d + "/wavelet.bin")
    case.A.astype(np.float32).tofile(d + "/A.bin")
    case.theta_cov.astype(np.float64).tofile(d + "/theta.bin")
    case.var0.astype(np.float64).tofile(d + "/var0.bin")
    for q in range(3):
        case.mu[q].tofile(d + f"/mu{q}.bin")
    for l in range(case.ntheta):
        case.data[l].tofile(d + f"/data{l}.bin")
    for t in range(6):
        case.cov[t].tofile(d + f"/cov{t}.bin")
    case.err_corr.tofile(d + "/err.bin")
    r = subprocess.run([exe, d] + (["cursor"] if mode == "cursor" else []), capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    if mode == "cursor":
        assert "cursor_mismatch 0" in r.stdout, r.stdout
    nx = case.nxp
    shape = case.mu[0].shape
    names = [f"mu{q}" for q in range(3)] + [f"data{l}" for l in range(case.ntheta)] + [f"cov{t}" for t in range(6)]
    refs = list(z["unit_mu"]) + list(z["unit_res"]) + list(z["unit_cov"])
    for n, ref in zip(names, refs):
        out = np.fromfile(d + f"/out_{n}.bin", np.float32).reshape(shape)
        err = np.linalg.norm(out[..., :nx] - ref[..., :nx]) / np.linalg.norm(ref[..., :nx])
        assert err < 2e-5, (n, err)
