"""Loads the committed golden fixtures (tests/golden/*.npz) as synth.Case
objects plus the reference outputs stored with them."""
import os

import numpy as np

from crava_b200.synth import Case

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
NAMES = ["c3_12x10x16", "c5_10x8x24", "c2_9x8x20_odd"]


def load(name):
    z = np.load(os.path.join(HERE, f"{name}.npz"))
    case = Case(nxp=int(z["nxp"]), nyp=int(z["nyp"]), nzp=int(z["nzp"]),
                angles_deg=[float(a) for a in z["angles"]], dt=float(z["dt"]),
                low_cut=float(z["low_cut"]), high_cut=float(z["high_cut"]), wnc=float(z["wnc"]),
                nz=int(z["nz"]), lz=float(z["lz"]), min_rel_thick=float(z["min_rel_thick"]),
                wavelet=z["wavelet"], A=z["A"], theta_cov=z["theta_cov"], var0=z["var0"],
                mu=list(z["mu"]), data=list(z["data"]), cov=list(z["cov"]), err_corr=z["err_corr"])
    return case, z


def spectra(z):
    return {"mu": list(z["spec_mu"]), "data": list(z["spec_data"]), "cov": list(z["spec_cov"]),
            "err": z["spec_err"]}


def tables(z):
    return (z["tab_wd"], z["tab_e1"], z["tab_e2"], z["tab_e3"], z["tab_inv"])
