"""Runs the posterior unit on a seeded synthetic case and prints the
per-kernel device times (CUDA events around every launch).

  python -m crava_b200.profile_unit NX,NY,NZ [precision 0|1|2] [fused 0|1] [repeats] [ntheta]

precision: 0 FP64, 1 mixed, 2 reference FP32.  Used for ncu captures of a
single kernel family on small cases.
"""
import sys

from crava_b200 import api, synth


def main(argv):
    nx, ny, nz = (int(v) for v in argv[1].split(","))
    prec = int(argv[2]) if len(argv) > 2 else 0
    fused = int(argv[3]) if len(argv) > 3 else 0
    reps = int(argv[4]) if len(argv) > 4 else 3
    nt = int(argv[5]) if len(argv) > 5 else 5
    angles = tuple(10.0 * i for i in range(nt))
    case = synth.make_case(nx, ny, nz, angles, 0.1, seed=2)
    ctx = api.Context(case)
    ctx.set_fused(bool(fused))
    d = lambda gs: [api.to_device(g) for g in gs]
    src = (d(case.mu), d(case.data), d(case.cov), d([case.err_corr])[0])
    dst = (d(case.mu), d(case.data), d(case.cov), d([case.err_corr])[0])
    ctx.set_profiling(True)
    for _ in range(reps):
        ctx.posterior_unit_oop(src, dst, prec)
        st = ctx.stats()
        print("forward %.3f solve %.3f inverse %.3f total %.3f ms" % (
            st.ms_forward, st.ms_solve, st.ms_inverse, st.ms_total))
    for k, v in ctx.profile().items():
        per = v[1] / v[0]
        print(f"{k:18s} launches {v[0]:4d}  {per:.4f} ms/launch  {v[2] / (per * 1e-3) / 1e9:8.1f} GB/s")


if __name__ == "__main__":
    main(sys.argv)
