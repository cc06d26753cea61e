"""The .crava grid file (FFTGrid::writeCravaFile / readCravaFile,
src/fftgrid.cpp:2399-2487 of the reference) through the device path,
against a restatement of the format: a type line, the simbox geometry and
the padded dimensions, then the rsize floats, all big-endian IEEE."""
import struct

import numpy as np
import pytest
import torch

from crava_b200 import api, synth

pytestmark = pytest.mark.gpu

GEOM = dict(x0=456000.5, y0=6780000.25, dx=25.0, dy=12.5, nx=15, ny=16, il0=1000.0, xl0=2000.0,
            il_step_x=0.5, il_step_y=-0.25, xl_step_x=0.125, xl_step_y=1.0, angle=0.3)


def write_ref(path, g, rnxp, nyp, nzp, grid):
    with open(path, "wb") as f:
        f.write(b"crava_fftgrid_binary\n")
        f.write(struct.pack(">4d2i7d3i", g["x0"], g["y0"], g["dx"], g["dy"], g["nx"], g["ny"],
                            g["il0"], g["xl0"], g["il_step_x"], g["il_step_y"], g["xl_step_x"],
                            g["xl_step_y"], g["angle"], rnxp, nyp, nzp))
        f.write(np.ascontiguousarray(grid, dtype=">f4").tobytes())


def read_ref(path):
    with open(path, "rb") as f:
        line = f.readline()
        assert line == b"crava_fftgrid_binary\n"
        vals = struct.unpack(">4d2i7d3i", f.read(4 * 8 + 2 * 4 + 7 * 8 + 3 * 4))
        data = np.frombuffer(f.read(), dtype=">f4").astype(np.float32)
    return vals, data


def test_write_then_read(tmp_path):
    case = synth.make_case(15, 16, 20, (10.0,), 0.1, seed=2)
    ctx = api.Context(case)
    g = api.to_device(case.data[0])
    hdr = api.GridHeader(**GEOM)
    p = str(tmp_path / "a.crava")
    ctx.write_crava_file(p, g, hdr)
    vals, data = read_ref(p)
    assert vals[:4] == (GEOM["x0"], GEOM["y0"], GEOM["dx"], GEOM["dy"])
    assert vals[4:6] == (GEOM["nx"], GEOM["ny"])
    assert vals[-3:] == (case.rnxp, case.nyp, case.nzp)
    assert np.array_equal(data.view(np.uint32), case.data[0].reshape(-1).view(np.uint32))
    # and back through the reader, into another grid
    out = torch.zeros_like(g)
    h2 = ctx.read_crava_file(p, out)
    assert torch.equal(out, g)
    assert (h2.x0, h2.angle, h2.ny) == (GEOM["x0"], GEOM["angle"], GEOM["ny"])


def test_read_reference_layout_and_reject_other_dims(tmp_path):
    case = synth.make_case(16, 12, 32, (10.0,), 0.1, seed=3)
    ctx = api.Context(case)
    grid = case.cov[2]
    p = str(tmp_path / "b.crava")
    write_ref(p, GEOM, case.rnxp, case.nyp, case.nzp, grid)
    out = torch.zeros_like(api.to_device(grid))
    ctx.read_crava_file(p, out)
    assert np.array_equal(out.cpu().numpy().view(np.uint32), grid.view(np.uint32))
    q = str(tmp_path / "c.crava")
    write_ref(q, GEOM, case.rnxp, case.nyp, case.nzp + 2, np.zeros(case.rnxp * case.nyp * (case.nzp + 2)))
    with pytest.raises(api.CravaGpuError):
        ctx.read_crava_file(q, out)
