#!/usr/bin/env python3
"""Generate the golden fixtures in tests/golden/ from the reference itself.

Builds the reference (oracle/build_ref.py: the reference's own C sources plus
the FM-torus config overlay, compiled with gcc) for small grids, runs it
through oracle/ref_harness.c, and stores the reference's geometry, initial
state and the states after the listed steps, cropped to NG ghost zones, as
compressed .npz files.

The benchmark configurations at their own sizes and step counts are too
large to store whole; for them (RECORDS) the reference's run is summarised
into tests/golden/records/<name>.npz: SHA-256 of the active primitives and
failure flags at init and after the listed steps, per-primitive sums of |p|,
the primitives on a sparse lattice, t and dt (tests/fixtures.summarise).
The GPU tests regenerate the initial state with the same reference binary
(built by __graft_entry__.build) and compare their run with the record.

Needs the reference tree (HARM_REFERENCE_DIR, else "reference" beside this
repository); the fixtures and records themselves are committed so that tests
run without it.

usage: python tests/golden/make_golden.py [case ...]
"""
import os
import shutil
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import build_ref  # noqa: E402
from oracle.pyoracle import RefDump  # noqa: E402
from tests.fixtures import RECORDS as RECORD_DIR  # noqa: E402
from tests.fixtures import summarise  # noqa: E402

# ghost zones kept in the fixture: MC reads 2, PARA 3, WENO5 (with the
# reference's MAXBND=11 line lengths) 6 per side.  The finite-volume cases
# keep all MAXBND ghosts: their fluxes and dt minimum run over every
# transverse ghost zone.
NG = {"MC": 3, "PARA": 3, "WENO5": 6}

# name: (n1, n2, n3, lim, flux, cour, nsteps, dump steps[, TIMEORDER[, inverter[, finite volume, MAXBND]]])
# [, {"phimodes": seed}] (the harness's azimuthal density modes)
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
    "torus2d_16x16_mc_hll_jon": (16, 16, 1, "MC", "HLL", 0.8, 5, [1, 5], 2, "JON"),
    "torus2d_16x16_para_hll_rk4_jon": (16, 16, 1, "PARA", "HLL", 0.8, 5, [1, 5], 4, "JON"),
    "torus3d_12x12x6_weno5_laxf_jon": (12, 12, 6, "WENO5", "LAXF", 0.8, 3, [1, 3], 2, "JON"),
    # the FM torus problem file's own scheme: PARA, HLL, RK4, Jon inverter,
    # ENOFINITEVOLUME with avgscheme=DONOR, MAXBND 11
    "torus2d_16x16_para_hll_rk4_jon_fv": (16, 16, 1, "PARA", "HLL", 0.8, 10, [1, 10], 4, "JON", True, 11),
    "torus2d_16x16_mc_hll_fv": (16, 16, 1, "MC", "HLL", 0.8, 5, [1, 5], 2, "2DFINAL", True, 11),
    "torus3d_12x12x6_para_laxf_rk4_jon_fv": (12, 12, 6, "PARA", "LAXF", 0.8, 3, [1, 3], 4, "JON", True, 3),
    # 3D with the HLL flux in all three directions, on a torus with azimuthal
    # density modes (x3 gradients in every primitive)
    "torus3d_12x12x6_weno5_hll": (12, 12, 6, "WENO5", "HLL", 0.8, 5, [1, 5], 2, "2DFINAL", False, 11,
                                  {"phimodes": 1}),
    "torus3d_12x12x6_mc_hll": (12, 12, 6, "MC", "HLL", 0.8, 10, [1, 10], 2, "2DFINAL", False, 11, {"phimodes": 1}),
    # a strongly magnetised torus (plasma beta 1e-4): b^2/rho and b^2/u above
    # the reference's flag limits in part of the grid, high-sigma inversions
    "torus2d_16x16_mc_hll_beta1e-4": (16, 16, 1, "MC", "HLL", 0.8, 5, [1, 5], 2, "2DFINAL", False, 11,
                                       {"beta": 1e-4}),
}

# The Bondi flow of the generic init.c (TESTNUMBER 153: the reference's
# bondigrid16.dat table on 16x16 zones, a = 0, its Bondi-integral x1
# boundaries, polar x2) with the MC + HLL point scheme and RK2 (its own
# inverter, Jon's); checked with a tolerance, not by the bit (pow).
BONDI_CASES = {
    "bondi2d_16x16_mc_hll": (16, 16, 1, "MC", "HLL", 0.5, 100, [1, 10, 100], 2, "JON", False, 11,
                             {"problem": "bondi"}),
    # the RAM paper's first relativistic shock tube (TESTNUMBER 101: 400 zones
    # on [0, 1], rho 10 | 1, p 13.33 | 1e-8, Gamma 5/3, CFL 0.5, to t = 0.4)
    # on the Minkowski line with the generic bounds.c's OUTFLOW copies
    "ram101_400_mc_hll": (400, 1, 1, "MC", "HLL", 0.5, 200, [1, 50, 200], 2, "JON", False, 11,
                          {"problem": "ram101"}),
    # its problems 2 (p 1000 | 0.01, a blast wave), 3 (a flow at v = 0.9 into
    # a denser, hotter state, Gamma 4/3) and 6.1 (the hard test), 400 zones
    "ram102_400_mc_hll": (400, 1, 1, "MC", "HLL", 0.5, 150, [1, 150], 2, "JON", False, 11, {"problem": "ram102"}),
    "ram103_400_mc_hll": (400, 1, 1, "MC", "HLL", 0.5, 150, [1, 150], 2, "JON", False, 11, {"problem": "ram103"}),
    "ram106_400_mc_hll": (400, 1, 1, "MC", "HLL", 0.5, 150, [1, 150], 2, "JON", False, 11, {"problem": "ram106"}),
}

# cases whose fixture also holds the reference's restart dump after the last
# step (restart_write(0) through the harness's --rdump: header line, then p
# and unew of every active zone as text), from a run without dump_ener
RDUMP = {"torus2d_16x16_mc_hll", "torus2d_16x16_mc_hll_beta1e-4", "torus2d_16x16_para_hll_rk4_jon_fv",
         "torus3d_12x12x6_weno5_hll"}

# Benchmark configurations run by the reference at their own sizes and step
# counts: name -> (n1, n2, n3, lim, flux, cour, nsteps, dump steps, harness
# options, lattice stride of the sample, keep the whole active state)
RECORDS = {
    # the 2D FM torus 64x64, MC + HLL + flux-CT, RK2, CFL 0.8, 200 steps
    "torus2d_64x64_mc_hll_200": (64, 64, 1, "MC", "HLL", 0.8, 200, [1, 200], [], (1, 1, 1), True),
    # the 3D torus 128x64x32 with azimuthal density modes, WENO5 + HLL, 500 steps
    "torus3d_128x64x32_weno5_hll_500": (128, 64, 32, "WENO5", "HLL", 0.8, 500, [1, 500],
                                        ["--phimodes", "1"], (8, 8, 4), False),
    # the precision-at-scale torus 256x128x128, WENO5 + HLL, first 5 steps
    "torus3d_256x128x128_weno5_hll_5": (256, 128, 128, "WENO5", "HLL", 0.8, 5, [1, 5],
                                        ["--phimodes", "1", "--geomplane"], (8, 8, 8), False),
    # the FM torus problem file's own scheme (PARA + HLL, RK4, Jon's inverter,
    # finite volume with avgscheme=DONOR, MAXBND 11) on the 3D torus 64x32x32
    # with azimuthal density modes, 20 steps
    "torus3d_64x32x32_para_hll_rk4_jon_fv_20": (64, 32, 32, "PARA", "HLL", 0.8, 20, [1, 20], ["--phimodes", "1"],
                                                (4, 4, 4), False, {"timeorder": 4, "utoprim": "JON", "fv": True}),
}


def make(name, spec, ref):
    n1, n2, n3, lim, flux, cour, nsteps, dumps = spec[:8]
    timeorder = spec[8] if len(spec) > 8 else 2
    utoprim = spec[9] if len(spec) > 9 else "2DFINAL"
    fv = spec[10] if len(spec) > 10 else False
    maxbnd = spec[11] if len(spec) > 11 else 11
    opts = spec[12] if len(spec) > 12 else {}
    hargs = ["--phimodes", str(opts["phimodes"])] if "phimodes" in opts else []
    problem = opts.get("problem", "fmtorus")
    if problem == "bondi":
        hargs = hargs + ["--bcgeom"]
    ng = maxbnd if fv else NG[lim]
    exe = build_ref.build(ref, n1, n2, n3, lim, flux, cour, maxbnd, timeorder=timeorder, utoprim=utoprim, fv=fv,
                          beta=opts.get("beta"), problem=problem)
    with tempfile.TemporaryDirectory() as tmp:
        out = os.path.join(tmp, "out")
        if problem == "bondi":
            # the analytic solution the reference's init reads (init.c:350-460)
            shutil.copy(os.path.join(ref, f"bondigrid{n1}.dat"), tmp)
        subprocess.run([exe, "--ener", "--ffc"] + hargs + [out, str(nsteps)] + [str(s) for s in dumps], cwd=tmp,
                       check=True, stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
        rd = RefDump(out)
        pr = rd.to_problem(ng, "init")
        if problem != "fmtorus":
            # the generic bounds.c's POLARAXIS (u~2, B2 negated) and OUTFLOW
            # (a plain copy) have their own ids here
            pr.bc = tuple({4: 1001, 0: 1000}.get(b, b) for b in pr.bc)
        # the reference's own ener.out (dump_ener.c:287-295), one line at init
        # and one after every dumped step: t, realnstep, the conserved
        # integrals U_tot[8], ..., divbmax, divbavg
        with open(os.path.join(tmp, "ener.out")) as f:
            ener = [np.array([float(v) for v in line.split()]) for line in f if line.strip()]
        data = dict(n=np.array(pr.n), ng=np.array(ng), dx=np.array(pr.dx), gam=pr.gam, cour=pr.cour,
                    lim=np.array(lim), flux=np.array(flux), bc=np.array(pr.bc), safe=pr.safe, defcon=pr.defcon,
                    tf=pr.tf, rhominlimit=pr.rhominlimit, uuminlimit=pr.uuminlimit, gammamax=pr.gammamax,
                    gammafail=pr.gammafail, gcov=pr.gcov, gcon=pr.gcon, gcovpert=pr.gcovpert, gdet=pr.gdet,
                    conn=pr.conn, floors=pr.floors, p_init=pr.p, pflag_init=pr.pflag, t_init=pr.t, dt_init=pr.dt,
                    steps=np.array(dumps), timeorder=np.array(timeorder), utoprim=np.array(utoprim),
                    doenoflux=np.array("ENOFINITEVOLUME" if fv else "NOENOFLUX"))
        if fv:
            data["u_init"] = pr.u
        data["ener_init"] = ener[0]
        # the reference's failure and floor counters per zone (failfloorcount,
        # fixup.c:206): at init (fixup at init counts too) and after each dump
        data["ffc_init"] = rd.crop(rd.ffc("init"), ng).astype(np.int32)
        for n_, s in enumerate(sorted(set(dumps) | {nsteps})):
            data[f"ener_s{s}"] = ener[1 + n_]
        for s in dumps:
            m = rd.meta_of(f"s{s}")
            data[f"p_s{s}"] = rd.crop(rd.p(f"s{s}"), ng)
            data[f"pflag_s{s}"] = rd.crop(rd.pflag(f"s{s}"), ng)[..., 0]
            # the b^2/rho and b^2/u flags of pre_fixup (FLAGBSQORHO, FLAGBSQOU)
            data[f"bsq_s{s}"] = rd.crop(rd.pflag(f"s{s}"), ng)[..., 2:4]
            data[f"ffc_s{s}"] = rd.crop(rd.ffc(f"s{s}"), ng).astype(np.int32)
            data[f"t_s{s}"] = m["t"]
            data[f"dt_s{s}"] = m["dt"]
            data[f"nstroke_s{s}"] = m["nstroke"]
            if fv:
                data[f"u_s{s}"] = rd.crop(rd.unew(f"s{s}"), ng)
            else:
                # unew of the other schemes: the last stage's conserved
                # update (what the restart dump holds beside p)
                data[f"unew_s{s}"] = rd.crop(rd.unew(f"s{s}"), ng)
        if problem == "bondi":
            # coordinate data of the x1 edge and ghost zones (hgpu_set_bondi_boundaries'
            # table: [side][q][j][49], q = 0 the edge zone, q >= 1 the ghosts)
            g = np.fromfile(os.path.join(out, "init_bcgeom.bin")).reshape(rd.NM[0], rd.NM[1], 49)
            b1, b2 = rd.bnd[0], rd.bnd[1]
            tab = np.zeros((2, ng + 1, n2, 49))
            for q in range(ng + 1):
                tab[0, q] = g[b1 - q, b2:b2 + n2]
                tab[1, q] = g[b1 + n1 - 1 + q, b2:b2 + n2]
            data["bondi_bc"] = tab
            data["bcgeom"] = rd.crop(g[:, :, None, :], ng)[:, :, 0, :]
            # the table file itself, for runs of the reference program
            with open(os.path.join(ref, f"bondigrid{n1}.dat"), "rb") as f:
                data["bondigrid_dat"] = np.frombuffer(f.read(), dtype=np.uint8)
        if name in RDUMP:
            # a run of its own without dump_ener, whose integrals would fill
            # the header's cumulative diagnostics (dump_ener.c:160-230)
            with tempfile.TemporaryDirectory() as tmp2:
                subprocess.run([exe, "--rdump"] + hargs + ["-", str(nsteps)], cwd=tmp2, check=True,
                               stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
                with open(os.path.join(tmp2, "dumps", "rdump-0"), "rb") as f:
                    data["rdump"] = np.frombuffer(f.read(), dtype=np.uint8)
    path = os.path.join(HERE, name + ".npz")
    np.savez_compressed(path, **data)
    print(f"wrote {path} ({os.path.getsize(path) / 1e6:.2f} MB)")


CENT = 7


def zone_inputs(nz=4096, seed=11):
    """Seeded zone-level inversion inputs on the MKS torus metric of the 16x16
    fixture: random primitives (rho log-uniform over 7 decades, u/rho over 6,
    Lorentz factors up to 2000, b^2/rho up to 1e3), their evolved conserved
    vector U (REMOVERESTMASSFROMUU 2: U[UU] = gdet (T^t_t + rho u^t)), a
    perturbed guess, and for a quarter of the zones an energy perturbed
    towards no physical solution."""
    g = np.load(os.path.join(HERE, "torus2d_16x16_mc_hll.npz"))
    gam = float(g["gam"])
    gcov_all = g["gcov"][:, :, CENT].reshape(-1, 4, 4)
    gcon_all = g["gcon"][:, :, CENT].reshape(-1, 4, 4)
    gdet_all = g["gdet"][:, :, CENT].reshape(-1)
    ok = np.abs(gdet_all) > 1e-8
    gcov_all, gcon_all, gdet_all = gcov_all[ok], gcon_all[ok], gdet_all[ok]
    rng = np.random.default_rng(seed)
    pick = rng.integers(0, len(gdet_all), nz)
    gcov, gcon, gdet = gcov_all[pick], gcon_all[pick], gdet_all[pick]
    rho = 10.0 ** rng.uniform(-6, 1, nz)
    uu = rho * 10.0 ** rng.uniform(-4, 2, nz)
    lor = 10.0 ** (rng.uniform(0, 1, nz) ** 2 * np.log10(2000.0))
    v = rng.normal(size=(nz, 3))
    norm = np.einsum("zi,zij,zj->z", v, gcov[:, 1:, 1:], v)
    ut = v * np.sqrt((lor * lor - 1.0) / norm)[:, None]
    alpha = 1.0 / np.sqrt(-gcon[:, 0, 0])
    ucon = np.zeros((nz, 4))
    ucon[:, 0] = lor / alpha
    ucon[:, 1:] = ut - ucon[:, :1] * gcon[:, 0, 1:] * (alpha * alpha)[:, None]
    ucov = np.einsum("zij,zj->zi", gcov, ucon)
    Bv = rng.normal(size=(nz, 3))
    bt = np.einsum("zi,zi->z", Bv, ucov[:, 1:])
    bcon = np.zeros((nz, 4))
    bcon[:, 0] = bt
    bcon[:, 1:] = (Bv + bt[:, None] * ucon[:, 1:]) / ucon[:, :1]
    bsq = np.einsum("zi,zij,zj->z", bcon, gcov, bcon)
    scale = np.sqrt(rho * 10.0 ** rng.uniform(-4, 3, nz) / bsq)
    Bv *= scale[:, None]
    bcon *= scale[:, None]
    bsq *= scale * scale
    bcov = np.einsum("zij,zj->zi", gcov, bcon)
    p = (gam - 1.0) * uu
    w = rho + uu + p
    Tt = (w + bsq)[:, None] * ucon[:, :1] * ucov - bcon[:, :1] * bcov
    Tt[:, 0] += p + 0.5 * bsq
    U = np.zeros((nz, 8))
    U[:, 0] = rho * ucon[:, 0]
    U[:, 1] = Tt[:, 0] + U[:, 0]
    U[:, 2:5] = Tt[:, 1:]
    U[:, 5:8] = Bv
    U *= gdet[:, None]
    bad = rng.random(nz) < 0.25
    U[bad, 1] *= 1.0 + rng.choice([-1.0, 1.0], bad.sum()) * 10.0 ** rng.uniform(-4, -0.3, bad.sum())
    prim = np.concatenate([rho[:, None], uu[:, None], ut, Bv], axis=1)
    guess = prim.copy()
    guess[:, 0:2] *= np.exp(rng.normal(scale=0.2, size=(nz, 2)))
    guess[:, 2:5] *= np.exp(rng.normal(scale=0.1, size=(nz, 1)))
    return dict(U=U, gcov=gcov, gcon=gcon, gdet=gdet, guess=guess, gam=gam, gammafail=float(g["gammafail"]),
                prim_true=prim)


def make_zones(ref):
    """Reference Utoprimgen outputs, both inverters, on zone_inputs()."""
    z = zone_inputs()
    n = len(z["gdet"])
    rec = np.concatenate([z["U"], z["gcov"].reshape(n, 16), z["gcon"].reshape(n, 16), z["gdet"][:, None],
                          z["guess"]], axis=1)
    data = dict(z)
    for inv in ("2DFINAL", "JON"):
        exe = build_ref.build(ref, 16, 16, 1, "MC", "HLL", 0.8, 11, utoprim=inv)
        with tempfile.TemporaryDirectory() as tmp:
            fin, fout = os.path.join(tmp, "in.bin"), os.path.join(tmp, "out.bin")
            with open(fin, "wb") as f:
                f.write(np.int64(n).tobytes())
                f.write(np.ascontiguousarray(rec).tobytes())
            subprocess.run([exe, "--invert", fin, fout], cwd=tmp, check=True, stdout=subprocess.DEVNULL,
                           stderr=subprocess.DEVNULL)
            raw = open(fout, "rb").read()
        data[f"pr_{inv}"] = np.frombuffer(raw[:n * 64], dtype=np.float64).reshape(n, 8).copy()
        data[f"pflag_{inv}"] = np.frombuffer(raw[n * 64:n * 68], dtype=np.int32).copy()
        data[f"iters_{inv}"] = np.frombuffer(raw[n * 68:n * 72], dtype=np.int32).copy()
    path = os.path.join(HERE, "utoprim_zones.npz")
    np.savez_compressed(path, **data)
    print(f"wrote {path} ({os.path.getsize(path) / 1e6:.2f} MB)")


def record_binary(ref, name):
    """Reference binary of a record (the one __graft_entry__.build also builds)."""
    n1, n2, n3, lim, flux, cour = RECORDS[name][:6]
    kw = RECORDS[name][11] if len(RECORDS[name]) > 11 else {}
    return build_ref.build(ref, n1, n2, n3, lim, flux, cour, 11, **kw)


def make_record(name, ref, workdir=None):
    n1, n2, n3, lim, flux, cour, nsteps, dumps, hargs, stride, whole = RECORDS[name][:11]
    exe = record_binary(ref, name)
    os.makedirs(RECORD_DIR, exist_ok=True)
    with tempfile.TemporaryDirectory(dir=workdir) as tmp:
        out = os.path.join(tmp, "out")
        subprocess.run([exe] + hargs + [out, str(nsteps)] + [str(s) for s in dumps], cwd=tmp, check=True,
                       stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
        rd = RefDump(out)
        data = dict(n=np.array((n1, n2, n3)), steps=np.array(dumps), stride=np.array(stride),
                    harness_args=np.array(" ".join(hargs)))
        for tag in ["init"] + [f"s{s}" for s in dumps]:
            p = rd.crop(rd.p(tag), 0)
            f = rd.crop(rd.pflag(tag), 0)[..., 0]
            m = rd.meta_of(tag)
            rec = summarise(p, f, stride)
            for k, v in rec.items():
                data[f"{tag}_{k}"] = np.array(v)
            data[f"{tag}_t"] = m["t"]
            data[f"{tag}_dt"] = m["dt"]
            data[f"{tag}_nstroke"] = m["nstroke"]
            if whole and tag != "init":
                data[f"{tag}_p"] = p
                data[f"{tag}_pflag"] = f
    path = os.path.join(RECORD_DIR, name + ".npz")
    np.savez_compressed(path, **data)
    print(f"wrote {path} ({os.path.getsize(path) / 1e6:.2f} MB)")


def make_bondigrid(ref):
    """The reference's tabulated Bondi solutions (bondigrid{N}.dat, read by
    readin_bondi_solution init.c:350-460): per table its header constants
    and the rows i, x, r, rho, u^r, u (the ghost rows included)."""
    data = {}
    for n in (32, 64, 128, 256):
        with open(os.path.join(ref, f"bondigrid{n}.dat")) as f:
            lines = f.read().splitlines()
        head = " ".join(lines[:2]).replace("#", " ").replace("=", " ").split()
        kv = {head[i]: float(head[i + 1]) for i in range(0, len(head) - 1, 2)}
        rows = np.array([[float(v) for v in ln.split()] for ln in lines[3:] if ln.strip()])
        data[f"n{n}_rows"] = rows
        data[f"n{n}_head"] = np.array([kv[k] for k in ("Gamma", "Rcr", "uu1cr", "rhocr", "Nx", "Rin", "Rout")])
    path = os.path.join(HERE, "bondigrid.npz")
    np.savez_compressed(path, **data)
    print(f"wrote {path} ({os.path.getsize(path) / 1e6:.2f} MB)")


def main():
    ref = build_ref.DEFAULT_REF
    if not os.path.isdir(ref):
        raise SystemExit(f"reference tree not found at {ref}: set HARM_REFERENCE_DIR")
    names = sys.argv[1:] or list(CASES) + list(BONDI_CASES) + ["utoprim_zones", "bondigrid"] + list(RECORDS)
    for name in names:
        if name == "utoprim_zones":
            make_zones(ref)
        elif name == "bondigrid":
            make_bondigrid(ref)
        elif name in RECORDS:
            make_record(name, ref)
        elif name in BONDI_CASES:
            make(name, BONDI_CASES[name], ref)
        else:
            make(name, CASES[name], ref)


if __name__ == "__main__":
    main()
