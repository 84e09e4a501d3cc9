#!/usr/bin/env python3
"""Build recipe for the reference HARM binary used as the pinning oracle.

Test infrastructure only.  It copies the reference C sources from the
read-only reference tree into a scratch directory OUTSIDE this repository,
applies two mechanical compatibility patches and a problem/config overlay,
swaps the reference main.c for oracle/ref_harness.c, and compiles with gcc.
Only the resulting executable is written, into oracle/_ref/ (git-ignored).

Mechanical patches (the reference targets icc):
  (a) block-scope ``static`` function prototypes are hoisted to file scope
      (gcc rejects them: "invalid storage class"); files: utoprim_jon.c,
      utoprim_jon_eos.c, u2p_util.c, utoprim_2d_final.c, utoprim_1d_final.c,
      utoprim_5d2_final.c, dudp_calc.c.
  (b) mpi_fileio.c:1978-2035 reuse one va_list across several vfprintf calls
      (undefined behaviour on x86-64); each call gets its own va_copy.
  (c) initbase.c:95-99 dumps the never-filled panalytic array at init; its
      wave-speed diagnostic hits myexit(10001) on the zeros (vchar.c:279).
      The dump is diagnostic output only, so the harness build skips it.

Config overlay (settings only, no algorithm change): the FM torus problem
file init.fishmon.c / init.fishmon.h / bounds.fishmon.c with
  EOMTYPE EOMGRMHD (init.fishmon.h:170 has EOMFFDE), defcoord=LOGRSINTH
  (init.fishmon.c:73 has 9), UTOPRIMVERSION=UTOPRIM2DFINAL unless the Jon
  inverter (UTOPRIMJONNONRELCOMPAT, init.fishmon.c:46) is asked for,
  lim/fluxmethod/cour as requested, TIMEORDER (2 unless asked),
  DOENOFLUX=NOENOFLUX unless the problem file's own ENOFINITEVOLUME
  (init.fishmon.c:112, with its avgscheme=DONOR) is asked for,
  rescaletype=0 (r^-1.5 / r^-2.5 floors), N1/N2/N3.

usage: python oracle/build_ref.py --n1 64 --n2 64 --n3 1 --lim MC --flux HLL
"""
import argparse
import os
import re
import shutil
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")
# the reference source tree: HARM_REFERENCE_DIR, else a checkout named
# "reference" beside this repository
DEFAULT_REF = os.environ.get("HARM_REFERENCE_DIR",
                             os.path.normpath(os.path.join(HERE, os.pardir, os.pardir, "reference")))

HOIST_FILES = ["utoprim_jon.c", "utoprim_jon_eos.c", "u2p_util.c", "utoprim_2d_final.c",
               "utoprim_1d_final.c", "utoprim_5d2_final.c", "dudp_calc.c"]

# maketail.harm.inc:185-232 (SRCSMANYPOINTS + SRCSONEPOINT); main.c replaced by the harness
SOURCES = """init.c initbase.c restart.c set_arrays.c set_grid.c
advance.c reconstructeno.c flux.c wavespeeds.c boundsflux.c fluxct.c fluxcompute.c
bounds.c boundsint.c diag.c dump.c dumpgen.c dump_ener.c image.c fail.c fixup.c
mpi_init.c mpi_fileio.c boundmpi.c boundmpiint.c
interppoint.c interpline.c monointerp.c jmonointerp.c smonointerp.c
metric.c coord.c phys.c step_ch.c phys.ffde.c phys.coldgrmhd.c eos.c
vchar.c transforms.c sources.c gaussj.c lubksb.c ludcmp.c mnewt.c nrutil.c ranc.c tensor.c
utoprimgen.c dudp_calc_3vel.c dudp_calc.c utoprim.c utoprim_2d.c utoprim_1d.c
utoprim_1d_opt.c utoprim_ldz.c utoprim_jon.c utoprim_1d_final.c utoprim_2d_final.c
utoprim_5d2_final.c freespace.c""".split()

LIMS = {"DONOR": "DONOR", "MC": "MC", "PARA": "PARA", "WENO5": "WENO5", "MINM": "MINM", "VANL": "VANL"}
FLUXES = {"HLL": "HLLFLUX", "LAXF": "LAXFFLUX"}


def hoist_block_statics(text):
    """Move block-scope `static <type> name(...);` prototypes to file scope."""
    lines = text.split("\n")
    depth = 0
    out = []
    hoisted = []
    seen = set()
    i = 0
    in_comment = False
    while i < len(lines):
        line = lines[i]
        stripped = line.strip()
        if depth > 0 and not in_comment and re.match(r"static\s+[A-Za-z_]", stripped) and "(" in stripped \
                and "=" not in stripped.split("(")[0]:
            # gather a possibly multi-line prototype up to ';' (must not open a body)
            j = i
            buf = [lines[j]]
            while ";" not in lines[j] and "{" not in lines[j] and j + 1 < len(lines):
                j += 1
                buf.append(lines[j])
            joined = " ".join(b.strip() for b in buf)
            if ";" in joined and "{" not in joined:
                key = re.sub(r"\s+", " ", joined)
                if key not in seen:
                    seen.add(key)
                    hoisted.append(joined)
                out.extend([""] * len(buf))
                i = j + 1
                continue
        # brace depth tracking (ignores braces inside // and /* */ comments and strings)
        k = 0
        s = line
        in_str = False
        while k < len(s):
            c = s[k]
            if in_comment:
                if s.startswith("*/", k):
                    in_comment = False
                    k += 2
                    continue
                k += 1
                continue
            if in_str:
                if c == "\\":
                    k += 2
                    continue
                if c == '"':
                    in_str = False
                k += 1
                continue
            if s.startswith("//", k):
                break
            if s.startswith("/*", k):
                in_comment = True
                k += 2
                continue
            if c == '"':
                in_str = True
            elif c == "'":
                k += 3 if k + 2 < len(s) and s[k + 2] == "'" else 1
                continue
            elif c == "{":
                depth += 1
            elif c == "}":
                depth -= 1
            k += 1
        out.append(line)
        i += 1
    if not hoisted:
        return text, 0
    # insert after the last #include/#define that precedes the first '{' of the file
    first_brace = next((n for n, l in enumerate(out) if "{" in l and not l.strip().startswith("//")), len(out))
    ins = 0
    for n in range(first_brace):
        if out[n].strip().startswith("#include") or out[n].strip().startswith("#define"):
            ins = n + 1
    block = ["/* prototypes hoisted to file scope by oracle/build_ref.py */"] + hoisted
    out = out[:ins] + block + out[ins:]
    return "\n".join(out), len(hoisted)


def patch_va_copy(text):
    pat = re.compile(r"vfprintf\s*\(\s*([A-Za-z_]+)\s*,\s*format\s*,\s*arglist\s*\)\s*;")
    new, n = pat.subn(r"{ va_list ac__; va_copy(ac__, arglist); vfprintf(\1, format, ac__); va_end(ac__); }", text)
    return new, n


def sub_once(text, old, new, count=1, where=""):
    n = text.count(old)
    if n != count:
        raise SystemExit(f"overlay: expected {count} occurrence(s) of {old!r} in {where}, found {n}")
    return text.replace(old, new)


def overlay_init_h(text, n1, n2, n3, maxbnd):
    text = sub_once(text, "#define EOMTYPE EOMFFDE", "#define EOMTYPE EOMGRMHD", where="init.fishmon.h")
    text = sub_once(text, "#define N1 64", f"#define N1 {n1}", where="init.fishmon.h")
    text = sub_once(text, "#define N2 64", f"#define N2 {n2}", where="init.fishmon.h")
    text = sub_once(text, "#define N3 1", f"#define N3 {n3}", where="init.fishmon.h")
    text = sub_once(text, "#define MAXBND 11", f"#define MAXBND {maxbnd}", where="init.fishmon.h")
    return text


UTOPRIMS = {"2DFINAL": "UTOPRIM2DFINAL", "JON": "UTOPRIMJONNONRELCOMPAT"}


def overlay_init_c(text, lim, flux, cour, timeorder=2, utoprim="2DFINAL", fv=False, beta=None):
    w = "init.fishmon.c"
    if beta is not None:
        # plasma beta of the field normalisation (init.fishmon.c:384)
        text = sub_once(text, "  beta = 1.e2 ;", f"  beta = {float(beta)!r} ;", where=w)
    text = sub_once(text, "  defcoord = 9;", "  defcoord = LOGRSINTH;", where=w)
    text = sub_once(text, "  UTOPRIMVERSION = UTOPRIMJONNONRELCOMPAT;", f"  UTOPRIMVERSION = {UTOPRIMS[utoprim]};", where=w)
    text = sub_once(text, "  lim = PARA;", f"  lim = {LIMS[lim]};", where=w)
    text = sub_once(text, "  TIMEORDER=4;", f"  TIMEORDER={int(timeorder)};", where=w)
    if not fv:
        text = sub_once(text, "  DOENOFLUX = ENOFINITEVOLUME;", "  DOENOFLUX = NOENOFLUX;", count=2, where=w)
    text = sub_once(text, "  fluxmethod=HLLFLUX;", f"  fluxmethod={FLUXES[flux]};", where=w)
    text = sub_once(text, "  rescaletype=1;", "  rescaletype=0;", where=w)
    text = sub_once(text, "  cour=0.8;", f"  cour={cour!r};", where=w)
    return text


# generic test problems (init.c / init.h / bounds.c) this recipe builds:
# problem name -> (TESTNUMBER, the marker line of its grid block in init.h)
GENERIC_PROBLEMS = {
    "bondi": (153, "#elif( TESTNUMBER == 153 )  // 1D Bondi problem"),
    "ram101": (101, "#elif( TESTNUMBER == 101 )  // 1D Riemann problem #1 from RAM paper"),
    "ram102": (102, "#elif( TESTNUMBER == 102 )  // 1D Riemann problem #2 from RAM paper"),
    "ram103": (103, "#elif( TESTNUMBER == 103 )  // 1D Riemann problem #3 from RAM paper"),
    "ram106": (106, "#elif( TESTNUMBER == 106 )  // 1D Riemann problem #6.1 from RAM paper (Hard test)"),
}


def overlay_bondi_h(text, n1, n2, problem="bondi"):
    """Generic init.h (the 1D/2D test-problem header) set to one of its test
    problems: the Bondi flow, TESTNUMBER 153 (init.h:578-582: 16x16 by
    default; the resolution must be one of the reference's bondigrid<N1>.dat
    tables), or the RAM paper's first relativistic shock tube, TESTNUMBER 101
    (init.h:515-520, 400 zones; init.c:2396-2411)."""
    w = "init.h"
    num, marker = GENERIC_PROBLEMS[problem]
    text = sub_once(text, "#define TESTNUMBER 49", f"#define TESTNUMBER {num}", where=w)
    i = text.index(marker)
    j = text.index("#elif", i + 5)
    block = re.sub(r"#define NXTEST \d+", f"#define NXTEST {n1}", text[i:j], count=1)
    block = re.sub(r"#define NYTEST \d+", f"#define NYTEST {n2}", block, count=1)
    text = text[:i] + block + text[j:]
    # the step's scheme settings of the FM torus problem file (init.fishmon.h),
    # which the test problems' header sets otherwise for non-FFDE tests
    # (init.h:209-220, 274, 283-293): primitives reconstructed as they are
    # (no rescaling, no extra interpolated quantities), checksolution on with
    # its limits, fixup1zone on
    k = text.rindex("#endif")
    return text[:k] + BONDI_SCHEME_SETTINGS + text[k:]


BONDI_SCHEME_SETTINGS = """
/* settings overlay (oracle/build_ref.py): the FM torus file's scheme */
#undef VARTOINTERP
#define VARTOINTERP PRIMTOINTERP
#undef RESCALEINTERP
#define RESCALEINTERP 0
#undef DOEXTRAINTERP
#define DOEXTRAINTERP 0
#undef CHECKSOLUTION
#define CHECKSOLUTION 1
#undef GAMMAPERCDIFFMAX
#define GAMMAPERCDIFFMAX 2.0
#undef UPERCDIFFMAX
#define UPERCDIFFMAX 10.0
#undef FIXUPZONES
#define FIXUPZONES FIXUP1ZONE
"""


def overlay_bondi_c(text, lim, flux, cour, timeorder=2, utoprim="2DFINAL"):
    """Generic init.c's GRMHD scheme block (init.c:915-934: WENO5BND finite
    volume, RK4, Jon's inverter) set to a point scheme, as the FM torus
    overlay does; everything else (grid from the bondigrid table, a = 0,
    LOGRSINTH with hslope 1, the Bondi-integral x1 boundaries, polar x2,
    periodic x3) is the reference's own TESTNUMBER 153 set-up."""
    w = "init.c"
    text = sub_once(text, "  avgscheme=WENO5BND;\n  //avgscheme=DONOR;", "  avgscheme=DONOR;\n  //avgscheme=DONOR;", where=w)
    text = sub_once(text, "  lim = WENO5BND;\n  //lim = WENO3;", f"  lim = {LIMS[lim]};\n  //lim = WENO3;", where=w)
    text = sub_once(text, "  TIMEORDER=4;\n  DOENOFLUX = ENOFINITEVOLUME;\n  //DOENOFLUX = NOENOFLUX;\n  fluxmethod= HLLFLUX; //LAXFFLUX;",
                    f"  TIMEORDER={int(timeorder)};\n  DOENOFLUX = NOENOFLUX;\n  //DOENOFLUX = NOENOFLUX;\n"
                    f"  fluxmethod= {FLUXES[flux]}; //LAXFFLUX;", where=w)
    text = sub_once(text, "  //UTOPRIMVERSION=UTOPRIM5D1;\n \tUTOPRIMVERSION = UTOPRIMJONNONRELCOMPAT;",
                    f"  //UTOPRIMVERSION=UTOPRIM5D1;\n \tUTOPRIMVERSION = {UTOPRIMS[utoprim]};", where=w)
    text = sub_once(text, "  SAFE=1.3;\n  cour = 0.5;", f"  SAFE=1.3;\n  cour = {cour!r};", where=w)
    return text


AFTER_MPI_STUB = """

/* bounds.fishmon.c has no bound_prim_user_after_mpi(); step_ch.c:bound_prim()
   calls one after bound_mpi().  With USEMPI=0 it has nothing to do. */
int bound_prim_user_after_mpi(int boundstage, FTYPE prim[][N2M][N3M][NPR])
{
  return(0);
}
"""


REPO = os.path.dirname(HERE)
SHIM = os.path.join(REPO, "harm_finalwham_b200", "dropin", "step_ch_gpu.c")
GPULIB = os.path.join(REPO, "harm_finalwham_b200", "lib")


def build(ref, n1, n2, n3, lim, flux, cour, maxbnd, name=None, keep=False, verbose=False, timeorder=2,
          utoprim="2DFINAL", fv=False, gpu_shim=False, beta=None, problem="fmtorus"):
    """gpu_shim: link the drop-in GPU step_ch (harm_finalwham_b200/dropin/step_ch_gpu.c
    against lib/libharmgpu.so) in place of the reference's own, which is kept
    as harm_cpu_step_ch (the only change to step_ch.c: the name at :16); the
    shim's restart_write, diag and dump_ener wrap the reference's, kept as
    harm_cpu_restart_write, harm_cpu_diag and harm_cpu_dump_ener (the names
    at restart.c:206, diag.c:9, dump_ener.c:3).

    problem: "fmtorus" (init.fishmon.c / init.fishmon.h / bounds.fishmon.c),
    or one of the generic init.c / init.h / bounds.c's test problems
    (GENERIC_PROBLEMS) with the FM torus file's scheme settings: "bondi"
    (TESTNUMBER 153, the Bondi flow with the Bondi-integral x1 boundaries,
    bounds.c:140-156, 295-308; n3 must be 1 and n1 x n2 a bondigrid table's
    size; the binary reads bondigrid<n1>.dat from its working directory) or
    "ram101" (TESTNUMBER 101, the first relativistic shock tube of the RAM
    paper on the Minkowski line, OUTFLOW copies at both ends)."""
    os.makedirs(OUT, exist_ok=True)
    name = name or ((f"harm_{problem}_" if problem in GENERIC_PROBLEMS else "harm_ref_")
                    + f"{n1}x{n2}x{n3}_{lim}_{flux}" + (f"_rk{timeorder}" if timeorder != 2 else "")
                    + ("_jon" if utoprim == "JON" else "") + ("_fv" if fv else "")
                    + (f"_beta{beta:g}" if beta is not None else "") + ("_gpushim" if gpu_shim else ""))
    scratch = tempfile.mkdtemp(prefix="harmref_")
    try:
        for fn in os.listdir(ref):
            if fn.endswith(".c") or fn.endswith(".h"):
                shutil.copy(os.path.join(ref, fn), os.path.join(scratch, fn))
        for fn in HOIST_FILES:
            p = os.path.join(scratch, fn)
            with open(p) as f:
                t = f.read()
            t, n = hoist_block_statics(t)
            with open(p, "w") as f:
                f.write(t)
            if verbose:
                print(f"hoisted {n} prototypes in {fn}")
        p = os.path.join(scratch, "mpi_fileio.c")
        with open(p) as f:
            t = f.read()
        t, n = patch_va_copy(t)
        if n < 6:
            raise SystemExit(f"va_copy patch matched {n} calls, expected >= 6")
        with open(p, "w") as f:
            f.write(t)
        p = os.path.join(scratch, "initbase.c")
        with open(p) as f:
            t = f.read()
        t = sub_once(t, "    if (dump(9999) >= 1){", "    if (0 && dump(9999) >= 1){", where="initbase.c")
        with open(p, "w") as f:
            f.write(t)
        # problem overlay
        if problem in GENERIC_PROBLEMS:
            if n3 != 1 or fv or beta is not None:
                raise SystemExit("the generic test problems here are 1D/2D, point scheme, as the reference sets them")
            with open(os.path.join(ref, "init.h")) as f:
                ih = overlay_bondi_h(f.read(), n1, n2, problem)
            with open(os.path.join(scratch, "init.h"), "w") as f:
                f.write(ih)
            with open(os.path.join(ref, "init.c")) as f:
                ic = overlay_bondi_c(f.read(), lim, flux, cour, timeorder, utoprim)
            with open(os.path.join(scratch, "init.c"), "w") as f:
                f.write(ic)
        else:
            with open(os.path.join(ref, "init.fishmon.h")) as f:
                ih = overlay_init_h(f.read(), n1, n2, n3, maxbnd)
            with open(os.path.join(scratch, "init.h"), "w") as f:
                f.write(ih)
            with open(os.path.join(ref, "init.fishmon.c")) as f:
                ic = overlay_init_c(f.read(), lim, flux, cour, timeorder, utoprim, fv, beta)
            with open(os.path.join(scratch, "init.c"), "w") as f:
                f.write(ic)
            with open(os.path.join(ref, "bounds.fishmon.c")) as f:
                bc = f.read() + AFTER_MPI_STUB
            with open(os.path.join(scratch, "bounds.c"), "w") as f:
                f.write(bc)
        shutil.copy(os.path.join(HERE, "ref_harness.c"), os.path.join(scratch, "ref_harness.c"))
        srcs = SOURCES + ["ref_harness.c"]
        extra = []
        if gpu_shim:
            p = os.path.join(scratch, "step_ch.c")
            with open(p) as f:
                t = f.read()
            t = sub_once(t, "int step_ch(void)\n{", "int harm_cpu_step_ch(void)\n{", where="step_ch.c")
            with open(p, "w") as f:
                f.write(t)
            # restart_write (restart.c:206), diag (diag.c:9) and dump_ener
            # (dump_ener.c:3) too: the shim's versions bring unew and the
            # failure/floor counters from the device first, then call them
            for fname, old, new in (
                    ("restart.c", "int restart_write(long dump_cnt)\n{", "int harm_cpu_restart_write(long dump_cnt)\n{"),
                    ("diag.c", "int diag(int call_code)\n{", "int harm_cpu_diag(int call_code)\n{"),
                    ("dump_ener.c", "int dump_ener(int doener, int dordump, int call_code)\n{",
                     "int harm_cpu_dump_ener(int doener, int dordump, int call_code)\n{")):
                p = os.path.join(scratch, fname)
                with open(p) as f:
                    t = f.read()
                t = sub_once(t, old, new, where=fname)
                with open(p, "w") as f:
                    f.write(t)
            shutil.copy(SHIM, os.path.join(scratch, "step_ch_gpu.c"))
            srcs = srcs + ["step_ch_gpu.c"]
            extra = ["-I" + os.path.join(REPO, "include"), "-L" + GPULIB, "-lharmgpu",
                     "-Wl,-rpath,$ORIGIN/../../harm_finalwham_b200/lib"]
            if problem in GENERIC_PROBLEMS:
                # the shim maps the generic bounds.c's boundary meanings
                extra.append("-DHARMGPU_GENERIC_BOUNDS")
        exe = os.path.join(OUT, name)
        cmd = ["gcc", "-O2", "-ffp-contract=off", "-fno-fast-math", "-fcommon", "-w",
               "-mcmodel=medium", "-o", exe] + srcs + extra + ["-lm"]
        r = subprocess.run(cmd, cwd=scratch, capture_output=True, text=True)
        if r.returncode != 0:
            sys.stderr.write(r.stderr[-6000:])
            raise SystemExit(f"reference build failed (scratch kept at {scratch})")
        if verbose:
            print("built", exe)
        return exe
    finally:
        if not keep:
            shutil.rmtree(scratch, ignore_errors=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=DEFAULT_REF)
    ap.add_argument("--n1", type=int, default=64)
    ap.add_argument("--n2", type=int, default=64)
    ap.add_argument("--n3", type=int, default=1)
    ap.add_argument("--lim", default="MC", choices=sorted(LIMS))
    ap.add_argument("--flux", default="HLL", choices=sorted(FLUXES))
    ap.add_argument("--cour", type=float, default=0.8)
    ap.add_argument("--maxbnd", type=int, default=11)
    ap.add_argument("--name", default=None)
    ap.add_argument("--keep", action="store_true")
    ap.add_argument("--timeorder", type=int, default=2, choices=[1, 2, 3, 4])
    ap.add_argument("--utoprim", default="2DFINAL", choices=sorted(UTOPRIMS))
    ap.add_argument("--fv", action="store_true", help="DOENOFLUX = ENOFINITEVOLUME (the problem file's own)")
    ap.add_argument("--gpu-shim", action="store_true",
                    help="link the drop-in GPU step_ch (harm_finalwham_b200/dropin) in place of the CPU one")
    a = ap.parse_args()
    if not os.path.isdir(a.ref):
        raise SystemExit(f"reference tree not found: {a.ref}")
    build(a.ref, a.n1, a.n2, a.n3, a.lim, a.flux, a.cour, a.maxbnd, a.name, a.keep, verbose=True,
          timeorder=a.timeorder, utoprim=a.utoprim, fv=a.fv, gpu_shim=a.gpu_shim)


if __name__ == "__main__":
    main()
