"""Generates the golden fixtures of tests/golden/ from the reference's own
numerics (oracle/_ref: FFTW 2.1.2, lib_matr.c and random.cpp compiled from
the reference sources, driven as src/crava.cpp drives them).

Run in a checkout where the reference tree is present:
    python tests/golden/make_golden.py
The fixtures hold the seeded inputs and the reference outputs, so the tests
need neither the reference tree nor the generator's numpy version.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from crava_b200 import synth  # noqa: E402
from oracle import oracle as O  # noqa: E402

CASES = {
    "c3_12x10x16": dict(shape=(12, 10, 16), angles=(10.0, 20.0, 30.0), noise=0.10, seed=101, scale=None),
    "c5_10x8x24": dict(shape=(10, 8, 24), angles=(0.0, 10.0, 20.0, 30.0, 40.0), noise=0.30, seed=102,
                       scale=(0.8, 1.2)),
    "c2_9x8x20_odd": dict(shape=(9, 8, 20), angles=(5.0, 25.0), noise=0.01, seed=103, scale=None),
}


def make_case(spec):
    return synth.make_case(*spec["shape"], spec["angles"], spec["noise"], spec["seed"],
                           wavelet_scale_range=spec["scale"])


# Synthetic seismic: golden case geometry and wavelets, seeded N(0,1)
# parameter grids, unpadded sizes (nx, ny, nz) exercising the taper and
# the untouched traces.
SYNT = {
    "c3_12x10x16": [(12, 10, 16), (11, 9, 13)],
    "c2_9x8x20_odd": [(9, 8, 20), (7, 8, 17)],
    "c5_10x8x24": [(10, 8, 21)],
}


def make_synt():
    from tests import golden_cases as GC

    out = {}
    for name, sizes in SYNT.items():
        case, _ = GC.load(name)
        rng = np.random.default_rng(7)
        m = [rng.standard_normal(case.mu[0].shape).astype(np.float32) for _ in range(3)]
        out[f"{name}_m"] = np.stack(m)
        for k, (nx, ny, nz) in enumerate(sizes):
            out[f"{name}_{k}_size"] = np.array([nx, ny, nz])
            out[f"{name}_{k}_out"] = np.stack(O.synt_seismic(case, m, nx, ny, nz, "ref"))
    np.savez_compressed(os.path.join(HERE, "synt_seismic.npz"), **out)
    print("synt_seismic written")


# Synthetic seismic with local wavelets: golden case -> unpadded sizes and
# whether local shift / gain grids are given (relative thickness always).
SYNT_LOCAL = {
    "c3_12x10x16": (11, 9, 13, False),
    "c2_9x8x20_odd": (7, 8, 17, True),
}


def make_synt_local():
    """Crava::computeSyntSeismic with each trace's local wavelet (stretch,
    shift, gain) through the reference's FFTW (oracle/_ref)."""
    from tests import golden_cases as GC

    out = {}
    for name, (nx, ny, nz, local) in SYNT_LOCAL.items():
        case, _ = GC.load(name)
        rng = np.random.default_rng(8)
        m = [rng.standard_normal(case.mu[0].shape).astype(np.float32) for _ in range(3)]
        rt, shift, gain, dz = divide_inputs(case, nx, ny, local, seed=23)
        out[f"{name}_m"] = np.stack(m)
        out[f"{name}_size"] = np.array([nx, ny, nz])
        out[f"{name}_rel_thick"] = rt
        out[f"{name}_dz"] = np.float32(dz)
        if local:
            out[f"{name}_shift"], out[f"{name}_gain"] = shift, gain
        out[f"{name}_out"] = np.stack(O.synt_seismic_local(case, m, rt, dz, shift, gain, nx, ny, nz))
    np.savez_compressed(os.path.join(HERE, "synt_local.npz"), **out)
    print("synt_local written")


def make_state4d():
    """State4D merge and split of a seeded state through the reference's
    lib_matr (oracle/_ref)."""
    from tests import state4d_cases as SC

    nxp, nyp, nzp = 10, 6, 8
    state, mu, cov = SC.random_state(nxp, nyp, nzp, seed=404, fail_every=23)
    out = dict(shape=np.array([nxp, nyp, nzp]), mu_post=np.stack(mu), cov_post=np.stack(cov))
    for k in SC.KEYS:
        out[f"in_{k}"] = np.stack(state[k])
    mmu = [np.zeros_like(mu[0]) for _ in range(3)]
    mcov = [np.zeros_like(mu[0]) for _ in range(6)]
    O.state4d_merge(state, mmu, mcov, "ref")
    out["merge_mu"], out["merge_cov"] = np.stack(mmu), np.stack(mcov)
    st = SC.copy_state(state)
    out["split_fail"] = O.state4d_split(st, mu, cov, "ref")
    for k in SC.KEYS:
        out[f"split_{k}"] = np.stack(st[k])
    np.savez_compressed(os.path.join(HERE, "state4d.npz"), **out)
    print("state4d written, split shortcuts", out["split_fail"])


DIVIDE = {  # golden case -> (nx, ny, nz, with local shift and gain grids)
    "c3_12x10x16": (10, 8, 12, False),
    "c2_9x8x20_odd": (7, 6, 16, True),
}


def divide_inputs(case, nx, ny, local, seed=21):
    """Seeded relative thickness, local shift / gain grids, and dz."""
    rng = np.random.default_rng(seed)
    rt = rng.uniform(0.7, 1.3, (case.nyp, case.nxp))
    shift = gain = None
    if local:
        shift = rng.uniform(-6.0, 6.0, (case.ntheta, ny, nx)).astype(np.float32)
        gain = rng.uniform(0.6, 1.4, (case.ntheta, ny, nx)).astype(np.float32)
        shift[0, 0, 0] = -999.0  # WELLMISSING: no shift there
    dz = float(np.float32(case.lz / case.nz))
    return rt, shift, gain, dz


def make_divide():
    """Crava::divideDataByScaleWavelet through the reference's FFTW
    (oracle/_ref) on two golden cases."""
    from tests import golden_cases as GC

    out = {}
    for name, (nx, ny, nz, local) in DIVIDE.items():
        case, _ = GC.load(name)
        case.nz = nz
        rt, shift, gain, dz = divide_inputs(case, nx, ny, local)
        col = case.cov[0][:, 0, 0].copy()
        res = O.divide_data(case, case.data, col, rt, nx, ny, dz, shift, gain, "ref")
        out[f"{name}_out"] = np.stack(res)
        out[f"{name}_rel_thick"] = rt
        out[f"{name}_dz"] = np.float32(dz)
        out[f"{name}_size"] = np.array([nx, ny, nz])
        if local:
            out[f"{name}_shift"], out[f"{name}_gain"] = shift, gain
    np.savez_compressed(os.path.join(HERE, "divide.npz"), **out)
    print("divide written")


def main():
    if not O.have_ref():
        O.build(ref=True)
    if "--synt-only" in sys.argv:
        make_synt()
        return
    if "--synt-local-only" in sys.argv:
        make_synt_local()
        return
    if "--state4d-only" in sys.argv:
        make_state4d()
        return
    if "--divide-only" in sys.argv:
        make_divide()
        return
    for name, spec in CASES.items():
        case = make_case(spec)
        nx, ny, nz = case.nxp, case.nyp, case.nzp
        wd, e1, e2, e3, inv = O.kz_tables(case, "ref")
        sp = O.forward_spectra(case, "ref")
        pmu, pres, pcov, pfail = O.posterior_fp32_tables(case, sp, (wd, e1, e2, e3, inv), "ref")
        umu, ures, ucov, ufail = O.unit_fp32(case, "ref")
        seeds = [O.noise_fill(nx, ny, nz, 1000 + s, "ref")[0] for s in range(3)]
        sim, sfail = O.sim_filter(nx, ny, nz, pcov, seeds, "ref")
        out = dict(
            nxp=nx, nyp=ny, nzp=nz, angles=np.array(spec["angles"]), noise_frac=spec["noise"],
            seed=spec["seed"], wavelet=case.wavelet, A=case.A, theta_cov=case.theta_cov,
            var0=case.var0, low_cut=case.low_cut, high_cut=case.high_cut, wnc=case.wnc,
            nz=case.nz, lz=case.lz, min_rel_thick=case.min_rel_thick, dt=case.dt,
            mu=np.stack(case.mu), data=np.stack(case.data), cov=np.stack(case.cov),
            err_corr=case.err_corr,
            tab_wd=wd, tab_e1=e1, tab_e2=e2, tab_e3=e3, tab_inv=inv,
            spec_mu=np.stack(sp["mu"]), spec_data=np.stack(sp["data"]), spec_cov=np.stack(sp["cov"]),
            spec_err=sp["err"],
            post_mu=np.stack(pmu), post_res=np.stack(pres), post_cov=np.stack(pcov), post_fail=pfail,
            unit_mu=np.stack(umu), unit_res=np.stack(ures), unit_cov=np.stack(ucov), unit_fail=ufail,
            sim_noise=np.stack(seeds), sim=np.stack(sim), sim_fail=sfail,
        )
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)
        print(name, "written")
    normals, state = O.rng_normal(23665, 256, "ref")
    np.savez_compressed(os.path.join(HERE, "rng_23665.npz"), normals=normals, state=state)
    print("rng written")
    make_synt()
    make_synt_local()
    make_state4d()
    make_divide()


if __name__ == "__main__":
    main()
