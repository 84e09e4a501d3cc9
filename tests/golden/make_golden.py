#!/usr/bin/env python3
"""Generate the golden fixtures in tests/golden/ from the reference itself.

Builds the reference (oracle/build_ref.py: the reference's own C sources plus
the FM-torus config overlay, compiled with gcc) for small grids, runs it
through oracle/ref_harness.c, and stores the reference's geometry, initial
state and the states after the listed steps, cropped to NG ghost zones, as
compressed .npz files.  Needs the reference tree (HARM_REFERENCE_DIR or
/root/reference); the fixtures themselves are committed so that tests run
without it.

usage: python tests/golden/make_golden.py [case ...]
"""
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import build_ref  # noqa: E402
from oracle.pyoracle import RefDump  # noqa: E402

# ghost zones kept in the fixture: MC reads 2, PARA 3, WENO5 (with the
# reference's MAXBND=11 line lengths) 6 per side
NG = {"MC": 3, "PARA": 3, "WENO5": 6}

# name: (n1, n2, n3, lim, flux, cour, nsteps, dump steps[, TIMEORDER])
CASES = {
    "torus2d_16x16_mc_hll": (16, 16, 1, "MC", "HLL", 0.8, 5, [1, 5]),
    "torus3d_12x12x6_mc_laxf": (12, 12, 6, "MC", "LAXF", 0.8, 10, [1, 10]),
    "torus2d_16x16_weno5_hll": (16, 16, 1, "WENO5", "HLL", 0.8, 5, [1, 5]),
    "torus3d_12x12x6_weno5_laxf": (12, 12, 6, "WENO5", "LAXF", 0.8, 5, [1, 5]),
    "torus2d_16x16_para_hll": (16, 16, 1, "PARA", "HLL", 0.8, 5, [1, 5]),
    "torus3d_12x12x6_para_laxf": (12, 12, 6, "PARA", "LAXF", 0.8, 5, [1, 5]),
    "torus2d_16x16_mc_hll_rk4": (16, 16, 1, "MC", "HLL", 0.8, 5, [1, 5], 4),
    "torus2d_16x16_mc_hll_rk1": (16, 16, 1, "MC", "HLL", 0.8, 5, [1, 5], 1),
    "torus3d_12x12x6_weno5_laxf_rk3": (12, 12, 6, "WENO5", "LAXF", 0.8, 3, [1, 3], 3),
}


def make(name, spec, ref):
    n1, n2, n3, lim, flux, cour, nsteps, dumps = spec[:8]
    timeorder = spec[8] if len(spec) > 8 else 2
    ng = NG[lim]
    exe = build_ref.build(ref, n1, n2, n3, lim, flux, cour, 11, timeorder=timeorder)
    with tempfile.TemporaryDirectory() as tmp:
        out = os.path.join(tmp, "out")
        subprocess.run([exe, out, str(nsteps)] + [str(s) for s in dumps], cwd=tmp, check=True,
                       stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
        rd = RefDump(out)
        pr = rd.to_problem(ng, "init")
        data = dict(n=np.array(pr.n), ng=np.array(ng), dx=np.array(pr.dx), gam=pr.gam, cour=pr.cour,
                    lim=np.array(lim), flux=np.array(flux), bc=np.array(pr.bc), safe=pr.safe, defcon=pr.defcon,
                    tf=pr.tf, rhominlimit=pr.rhominlimit, uuminlimit=pr.uuminlimit, gammamax=pr.gammamax,
                    gammafail=pr.gammafail, gcov=pr.gcov, gcon=pr.gcon, gcovpert=pr.gcovpert, gdet=pr.gdet,
                    conn=pr.conn, floors=pr.floors, p_init=pr.p, pflag_init=pr.pflag, t_init=pr.t, dt_init=pr.dt,
                    steps=np.array(dumps), timeorder=np.array(timeorder))
        for s in dumps:
            m = rd.meta_of(f"s{s}")
            data[f"p_s{s}"] = rd.crop(rd.p(f"s{s}"), ng)
            data[f"pflag_s{s}"] = rd.crop(rd.pflag(f"s{s}"), ng)[..., 0]
            data[f"t_s{s}"] = m["t"]
            data[f"dt_s{s}"] = m["dt"]
            data[f"nstroke_s{s}"] = m["nstroke"]
    path = os.path.join(HERE, name + ".npz")
    np.savez_compressed(path, **data)
    print(f"wrote {path} ({os.path.getsize(path) / 1e6:.2f} MB)")


def main():
    ref = os.environ.get("HARM_REFERENCE_DIR", "/root/reference")
    if not os.path.isdir(ref):
        raise SystemExit(f"reference tree not found: {ref}")
    names = sys.argv[1:] or list(CASES)
    for name in names:
        make(name, CASES[name], ref)


if __name__ == "__main__":
    main()
