"""Load the committed golden fixtures (tests/golden/*.npz) into oracle Problems,
and summarise states into the compact records kept for the configurations
too large to store whole (tests/golden/records/*.npz)."""
import hashlib
import os

import numpy as np

from oracle.pyoracle import Problem

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
CASES = ["torus2d_16x16_mc_hll", "torus3d_12x12x6_mc_laxf", "torus2d_16x16_weno5_hll", "torus3d_12x12x6_weno5_laxf",
         "torus2d_16x16_para_hll", "torus3d_12x12x6_para_laxf", "torus2d_16x16_mc_hll_rk4",
         "torus2d_16x16_mc_hll_rk1", "torus3d_12x12x6_weno5_laxf_rk3", "torus2d_16x16_mc_hll_jon",
         "torus2d_16x16_para_hll_rk4_jon", "torus3d_12x12x6_weno5_laxf_jon", "torus2d_16x16_para_hll_rk4_jon_fv",
         "torus2d_16x16_mc_hll_fv", "torus3d_12x12x6_para_laxf_rk4_jon_fv", "torus3d_12x12x6_weno5_hll",
         "torus3d_12x12x6_mc_hll", "torus2d_16x16_mc_hll_beta1e-4"]


def load(name):
    d = np.load(os.path.join(GOLDEN, name + ".npz"))
    n = tuple(int(x) for x in d["n"])
    pr = Problem(n[0], n[1], n[2], int(d["ng"]), tuple(float(x) for x in d["dx"]), gam=float(d["gam"]),
                 cour=float(d["cour"]), lim=str(d["lim"]), flux=str(d["flux"]), bc=tuple(int(x) for x in d["bc"]),
                 safe=float(d["safe"]), defcon=float(d["defcon"]), tf=float(d["tf"]),
                 rhominlimit=float(d["rhominlimit"]), uuminlimit=float(d["uuminlimit"]),
                 gammamax=float(d["gammamax"]), gammafail=float(d["gammafail"]),
                 timeorder=int(d["timeorder"]) if "timeorder" in d else 2,
                 utoprim=str(d["utoprim"]) if "utoprim" in d else "2DFINAL",
                 doenoflux=str(d["doenoflux"]) if "doenoflux" in d else "NOENOFLUX")
    for k in ("gcov", "gcon", "gcovpert", "gdet", "conn", "floors"):
        getattr(pr, k)[...] = d[k]
    pr.p[...] = d["p_init"]
    pr.pflag[...] = d["pflag_init"]
    if "u_init" in d:
        pr.u = np.ascontiguousarray(d["u_init"])
    pr.t = float(d["t_init"])
    pr.dt = float(d["dt_init"])
    steps = [int(s) for s in d["steps"]]
    ref = {s: dict(p=d[f"p_s{s}"], pflag=d[f"pflag_s{s}"], t=float(d[f"t_s{s}"]), dt=float(d[f"dt_s{s}"]),
                   nstroke=float(d[f"nstroke_s{s}"]), u=d[f"u_s{s}"] if f"u_s{s}" in d else None,
                   unew=d[f"u_s{s}"] if f"u_s{s}" in d else (d[f"unew_s{s}"] if f"unew_s{s}" in d else None),
                   bsq=d[f"bsq_s{s}"] if f"bsq_s{s}" in d else None,
                   ffc=d[f"ffc_s{s}"] if f"ffc_s{s}" in d else None,
                   ener=d[f"ener_s{s}"] if f"ener_s{s}" in d else None) for s in steps}
    # the reference's ener.out line at init (dump_ener.c:287-295)
    pr.ener_init = d["ener_init"] if "ener_init" in d else None
    # the reference's failure and floor counters per zone at init
    pr.ffc_init = d["ffc_init"] if "ffc_init" in d else None
    # Bondi-integral boundaries: the x1 edge/ghost coordinate table and the
    # per-zone coordinate data (r, dx/dx', inverse, Kerr-Schild metric)
    pr.bondi_bc = np.ascontiguousarray(d["bondi_bc"]) if "bondi_bc" in d else None
    pr.bcgeom = d["bcgeom"] if "bcgeom" in d else None
    # the reference's bondigrid<N1>.dat the Bondi flow's init reads
    pr.bondigrid_dat = d["bondigrid_dat"].tobytes() if "bondigrid_dat" in d else None
    # the reference's restart dump after the last step (restart_write), bytes
    pr.rdump = d["rdump"].tobytes() if "rdump" in d else None
    return pr, ref


def same(a, b):
    """Bit-level equality up to the sign of zero (NaN equal to NaN)."""
    a = np.asarray(a)
    b = np.asarray(b)
    return a.shape == b.shape and bool(np.all((a == b) | (np.isnan(a) & np.isnan(b))))


def load_zones():
    """Zone-level inversion fixture (tests/golden/utoprim_zones.npz): inputs
    and the reference's Utoprimgen outputs for both inverters."""
    d = np.load(os.path.join(GOLDEN, "utoprim_zones.npz"))
    z = {k: d[k] for k in d.files}
    z["gam"] = float(d["gam"])
    z["gammafail"] = float(d["gammafail"])
    return z


RECORDS = os.path.join(GOLDEN, "records")


def sha(a):
    """SHA-256 of an array's bytes in C order (little-endian)."""
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def lattice(n, stride):
    """Sample indices of the active zones: every stride-th zone per axis,
    offset to the middle of the first stride."""
    return tuple(np.arange(min(st // 2, nn - 1), nn, st) for nn, st in zip(n, stride))


def summarise(p_active, pflag_active, stride):
    """Compact record of a state: hashes of the primitives and of the
    failure-flag map, per-primitive sums of |p|, and the primitives on a
    sparse lattice (for a relative-L1 estimate when the hashes differ)."""
    idx = lattice(p_active.shape[:3], stride)
    sample = p_active[np.ix_(*idx)]
    return dict(sha_p=sha(p_active), sha_pflag=sha(pflag_active.astype(np.int32)),
                l1=np.abs(p_active).reshape(-1, p_active.shape[-1]).sum(axis=0), sample=sample,
                nfail=int((pflag_active > 0).sum()))


def load_record(name):
    d = np.load(os.path.join(RECORDS, name + ".npz"))
    return {k: d[k] for k in d.files}


def reference_on_state(exe, tmp, mode, pr, args=(), with_flags=False):
    """Run the reference build `exe` (oracle/ref_harness.c --postfixup /
    --boundprim) on the state of `pr` and return its arrays cropped to pr's
    layout: p, or (p, FLAGUTOPRIMFAIL flags) with `with_flags`.  The init
    dump of `exe` in tmp/init gives the reference's
    own array shape (reference_problem writes it); its outer ghosts beyond
    pr's keep init's values."""
    import subprocess

    from oracle.pyoracle import RefDump
    rd = RefDump(os.path.join(tmp, "init"))
    off = tuple(b - g for b, g in zip(rd.bnd, pr.g))
    sl = tuple(slice(o, o + nt) for o, nt in zip(off, pr.nt))
    p_ref = rd.p("init").copy()
    p_ref[sl] = pr.p
    fin, fout = os.path.join(tmp, "in.bin"), os.path.join(tmp, "out.bin")
    with open(fin, "wb") as f:
        f.write(np.ascontiguousarray(p_ref).tobytes())
        if with_flags:
            f_ref = np.zeros(rd.NM, dtype=np.int32)
            f_ref[sl] = pr.pflag
            f.write(f_ref.tobytes())
    if os.path.exists(fout):
        os.remove(fout)
    r = subprocess.run([exe, mode, fin, fout] + [str(a) for a in args], cwd=tmp, capture_output=True, text=True)
    assert r.returncode == 0 and os.path.exists(fout), r.stderr[-400:]
    raw = np.fromfile(fout, dtype=np.uint8)
    nb = p_ref.nbytes
    p_out = raw[:nb].view(np.float64).reshape(p_ref.shape)[sl]
    if not with_flags:
        return p_out
    return p_out, raw[nb:].view(np.int32).reshape(rd.NM)[sl]


def reference_problem(exe, tmp, ng=3):
    """The initial state of the reference build `exe` as a Problem with ng
    ghosts (runs its init into tmp/init)."""
    import subprocess

    from oracle.pyoracle import RefDump
    out = os.path.join(tmp, "init")
    subprocess.run([exe, out, "0"], cwd=tmp, check=True, stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
    return RefDump(out).to_problem(ng, "init")
