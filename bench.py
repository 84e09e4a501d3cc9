#!/usr/bin/env python3
"""Benchmark of the B200 per-zone conservative update (zone-updates/s).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload: 3D Fishbone-Moncrief torus around a Kerr hole (a=0.9375, beta=100,
MKS hslope=0.3, Rout=40) on 256x128x128 zones, FP64, WENO5 + HLL + flux-CT +
2D Noble inversion + fixups + boundaries, midpoint RK2 (the MC variants and
smaller grids are selectable with --workload).  One step = one full
time step (both RK substeps) of the whole domain; one zone-update = one
active zone advanced by one full step.

Our arm:
  value       zone-updates/s with the state resident in HBM, timed with CUDA
              events on the library's stream (max over ranks); the state
              arrays (300 MB each) exceed L2, so no flush is needed.
  e2e         the same metric through the C ABI with host-owned arrays
              (wall clock incl. copies from/to pinned host memory): every
              step uploads the active zones' primitives
              (hgpu_upload_active; the device rebuilds the ghosts with
              bound_prim), steps, and downloads primitives and flags
              (hgpu_download_active); e2e.full_arrays is the same with the
              arrays including ghost zones, as the drop-in step_ch() moves
              them (the finite-volume scheme, whose unew must travel too,
              reports that path).
  roofline    dominant kernel: algorithmic bytes per launch / its average
              CUDA-event duration vs the measured HBM peak, plus its FP64
              operation rate vs the FP64 peak measured in this run.
  cpu_baseline  the reference CPU build (oracle/_ref) on a bounded 3D torus
              sample on the host cores, one process per core.
Reference arm (--impl reference): the reference CPU build, one process per
host core on the bounded sample, aggregate zone-updates/s.

Multi-GPU (N > 1): one torus of n3 x N planes split along x3 (each rank
owns n3 planes, the reference's MPI decomposition with ncpux3 = N; ghost
planes exchanged over NCCL twice per stage, the ndt minima all-reduced once
per step), weak scaling; value = all ranks' zone-updates / max time.
--replicas instead runs N independent tori (no data-path collective).
"""
import argparse
import datetime
import json
import os
import re
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOADS = {
    # name: (n1, n2, n3, lim, flux)
    "torus3d_256x128x128": (256, 128, 128, "WENO5", "HLL"),
    "torus3d_256x128x64": (256, 128, 64, "WENO5", "HLL"),
    "torus3d_128x64x32": (128, 64, 32, "WENO5", "HLL"),
    "torus3d_256x128x128_mc": (256, 128, 128, "MC", "HLL"),
    "torus3d_256x128x64_mc": (256, 128, 64, "MC", "HLL"),
    "torus2d_64x64": (64, 64, 1, "MC", "HLL"),
    # the FM torus problem file's own scheme (init.fishmon.c:46, 97-127):
    # PARA + HLL, RK4, Jon's inverter, finite volume with avgscheme=DONOR,
    # all MAXBND=11 ghosts (its flux and dt loops cover them)
    "torus3d_256x128x128_fishmon": (256, 128, 128, "PARA", "HLL"),
    "torus3d_128x64x32_fishmon": (128, 64, 32, "PARA", "HLL"),
    "torus3d_256x128x64_fishmon": (256, 128, 64, "PARA", "HLL"),
}
# scheme settings beyond the 2D Noble / midpoint / standard-update default
SCHEMES = {
    "torus3d_256x128x128_fishmon": {"timeorder": 4, "utoprim": "JON", "doenoflux": "ENOFINITEVOLUME", "ng": 11},
    "torus3d_128x64x32_fishmon": {"timeorder": 4, "utoprim": "JON", "doenoflux": "ENOFINITEVOLUME", "ng": 11},
    "torus3d_256x128x64_fishmon": {"timeorder": 4, "utoprim": "JON", "doenoflux": "ENOFINITEVOLUME", "ng": 11},
}
DEFAULT_WORKLOAD = "torus3d_256x128x128"
# ghost zones kept on the device: MC reads 2 per side, PARA 3, WENO5 6 (the
# reference's MAXBND=11 lines never truncate a WENO5 stencil, and 6 is what
# its stencils read)
GHOSTS = {"MC": 3, "PARA": 3, "WENO5": 6}


def scheme_of(workload):
    sc = {"timeorder": 2, "utoprim": "2DFINAL", "doenoflux": "NOENOFLUX", "ng": None}
    sc.update(SCHEMES.get(workload, {}))
    return sc


def scheme_text(lim, flux, sc):
    inv = "2D Noble" if sc["utoprim"] == "2DFINAL" else "Jon 1D E'(W')"
    ti = {1: "Euler", 2: "midpoint RK2", 3: "TVD RK3", 4: "RK4"}[sc["timeorder"]]
    fv = ", finite volume (avgscheme DONOR)" if sc["doenoflux"] == "ENOFINITEVOLUME" else ""
    return f"{lim}+{flux}+flux-CT, {inv} inversion, {ti}{fv}"


def cpu_sample(workload):
    """CPU sample for the reference build: same problem and scheme, 3D 64x32x32."""
    lim = WORKLOADS[workload][3]
    return (64, 32, 32, lim, "HLL") + (scheme_of(workload),)

METRIC = "zone-updates/s FP64 vs mixed on 3D Kerr torus at stated L1; batch p50/p99 latency"


def rank_info():
    r = int(os.environ.get("RANK", "0"))
    w = int(os.environ.get("WORLD_SIZE", "1"))
    lr = int(os.environ.get("LOCAL_RANK", "0"))
    return r, w, lr


# the physical index of this process's GPU (for nvidia-smi)
PHYS_GPU = "0"


def select_device(local_rank, world):
    """One process per GPU: this rank's GPU (its local rank) for torch and
    for the library, whose statically linked CUDA runtime keeps its own
    current device.  Every GPU stays visible, so NCCL can reach its peers
    over NVLink."""
    global PHYS_GPU
    vis = os.environ.get("CUDA_VISIBLE_DEVICES")
    devs = vis.split(",") if vis else None
    PHYS_GPU = devs[local_rank % len(devs)].strip() if devs else str(local_rank)
    if world <= 1:
        return
    import torch

    from harm_finalwham_b200.gpu import set_device
    torch.cuda.set_device(local_rank)
    set_device(local_rank)


class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self):
        self.proc = None
        self.out = tempfile.NamedTemporaryFile(mode="w+", suffix=".csv", delete=False)

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                          "-lms", "200"], stdout=self.out, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.out.flush()
        self.out.seek(0)
        rows = [r.split(",") for r in self.out.read().strip().splitlines() if r.strip()]
        os.unlink(self.out.name)
        rows = [r for r in rows if len(r) >= 9 and r[0].strip() == PHYS_GPU] or [r for r in rows if len(r) >= 9]
        if not rows:
            return None
        sm = [float(r[1]) for r in rows]
        smax = max(float(r[2]) for r in rows)
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            for nm, v in zip(names, r[5:9]):
                if v.strip().lower() == "active":
                    reasons.add(nm)
        loaded = [s for s in sm if s > 0.5 * smax] or sm
        return {"sm_mhz": statistics.median(loaded), "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(rows), "power_w_max": max(float(r[3]) for r in rows if r[3].strip()
                                                           .replace('.', '', 1).isdigit()) if rows else None}


def bench_decomp(args, rank, world):
    """--decomp x3: one torus of n3 x world planes split along x3, rank r
    owning planes r*n3 .. (r+1)*n3-1 (weak scaling).  Each step runs the
    phase entry points with the x3 ghost planes sent to the neighbours over
    NCCL after each half-stage and the per-direction ndt minima all-reduced;
    with one rank the planes wrap onto the same context, which measures the
    cost of the phase-driven step against the one-call step."""
    import torch

    from harm_finalwham_b200 import torus
    from harm_finalwham_b200.decomp import CollectiveTransport, SplitRun, SlabContext, split_x3
    from harm_finalwham_b200.gpu import HarmGPU, load_library

    n1, n2, n3, lim, flux = WORKLOADS[args.workload]
    sc = scheme_of(args.workload)
    if args.utoprim:
        sc["utoprim"] = args.utoprim
    dist = None
    if world > 1:
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    dom = torus.fm_torus(n1, n2, n3 * world, ng=sc["ng"] or GHOSTS[lim], lim=lim, flux=flux, seed=7)
    dom.timeorder, dom.utoprim, dom.doenoflux = sc["timeorder"], sc["utoprim"], sc["doenoflux"]
    slab = split_x3(dom, world, rank)
    del dom
    L = load_library()
    g = HarmGPU.from_problem(slab, precision=args.precision)
    if args.tuning:
        g.set_tuning(dict(zip(("flux", "weno", "update", "invert"), (int(v) for v in args.tuning.split(",")))))
    else:
        g.autotune()
    sub = SlabContext(g)
    run = SplitRun([g], CollectiveTransport(sub))
    run.start(init_dt=True)
    run.step(args.warmup, stats=False)
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    launches0 = L.hgpu_launch_count(g.h)
    clocks = ClockSampler()
    clocks.start()
    e0.record(sub.stream)
    run.step(args.steps, stats=False)
    e1.record(sub.stream)
    e1.synchronize()
    clk = clocks.stop()
    launches = L.hgpu_launch_count(g.h) - launches0
    st = run.stats()
    ms = e0.elapsed_time(e1)
    if dist is not None:
        dist.barrier()
    ms_max = replica_max(ms, dist, "cuda")
    zones = n1 * n2 * n3
    norders = sc["timeorder"] or 2
    out = {"metric": METRIC, "value": replica_value(zones, args.steps, world, ms_max), "unit": "zone-updates/s",
           "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps,
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
           "dtype": "f64" if args.precision == "fp64" else "f64+f32", "data": "synthetic",
           "config": {"workload": f"{args.workload} per rank, x3 split of {n1}x{n2}x{n3 * world}",
                      "scheme": scheme_text(lim, flux, sc), "precision": args.precision,
                      "parallelism": f"x3 split over {world} ranks" + (" (NCCL halos)" if world > 1 else
                                                                         " (planes wrap onto the one rank)"),
                      "l2": "state larger than L2"},
           "halo": {"bytes_per_face_exchange": sub.nbytes, "exchanges_per_step": 2 * norders,
                    "bytes_sent_per_step": 2 * 2 * norders * sub.nbytes},
           "gpu_launches": launches, "clocks": clk, "newton_fail_err": st.err}
    if world == 1:
        # the same slab through the one-call step, for the phase-driven overhead
        ms1, _ = g.step_ch_timed(args.steps)
        out["one_call_ms_per_step"] = ms1 / args.steps
    run.close()
    if dist is not None:
        dist.destroy_process_group()
    return out


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f), "measured"
    except OSError:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


def _traffic_row(workload, kernel):
    """(DRAM bytes, FP64 instructions) per launch of `kernel` on `workload`
    from the committed ncu summary profiles/traffic.md, or None.  FP64
    instructions = DADD + DMUL + DFMA executed (thread-level), the unit of the
    FP64 issue-rate peak."""
    path = os.path.join(ROOT, "profiles", "traffic.md")
    try:
        txt = open(path).read()
    except OSError:
        return None
    m = re.search(rf"^\|\s*{re.escape(workload)}\s*\|\s*{re.escape(kernel)}\s*\|\s*([0-9.eE+]+)\s*\|\s*([0-9.eE+]+)\s*\|",
                  txt, re.M)
    return (float(m.group(1)), float(m.group(2))) if m else None


def step_dram_bytes(workload):
    """ncu DRAM bytes (read + write) of one whole time step of `workload`, from
    profiles/traffic.md, or None."""
    path = os.path.join(ROOT, "profiles", "traffic.md")
    try:
        txt = open(path).read()
    except OSError:
        return None
    m = re.search(rf"^\|\s*{re.escape(workload)}\s*\|\s*step\s*\|\s*([0-9.eE+]+)\s*\|", txt, re.M)
    return float(m.group(1)) if m else None


def profile_traffic(workload, kernel):
    """DRAM bytes per launch of `kernel` from the committed ncu summary, if any."""
    r = _traffic_row(workload, kernel)
    return r[0] if r else None


# ---------------------------------------------------------------------------
# reference CPU build
# ---------------------------------------------------------------------------
def ref_binary(sample):
    n1, n2, n3, lim, flux, sc = sample
    suffix = ((f"_rk{sc['timeorder']}" if sc["timeorder"] != 2 else "") + ("_jon" if sc["utoprim"] == "JON" else "")
              + ("_fv" if sc["doenoflux"] == "ENOFINITEVOLUME" else ""))
    return os.path.join(ROOT, "oracle", "_ref", f"harm_ref_{n1}x{n2}x{n3}_{lim}_{flux}{suffix}")


def run_reference(sample, steps, warmup, procs):
    """Run `procs` independent reference processes; return aggregate zone-updates/s."""
    exe = ref_binary(sample)
    if not os.path.exists(exe):
        return None, f"reference binary {os.path.basename(exe)} not built"
    n1, n2, n3 = sample[:3]
    total = warmup + steps
    with tempfile.TemporaryDirectory() as tmp:
        ps = []
        for i in range(procs):
            wd = os.path.join(tmp, f"r{i}")
            os.makedirs(wd)
            ps.append(subprocess.Popen([exe, "-", str(total)], cwd=wd, stdout=subprocess.DEVNULL,
                                       stderr=subprocess.PIPE, text=True))
        spans = []
        for p in ps:
            _, err = p.communicate()
            if p.returncode != 0:
                return None, f"reference run failed rc={p.returncode}"
            st = {int(a): float(b) for a, b in re.findall(r"harness: step (\d+) start ([0-9.]+)", err)}
            en = {int(a): float(b) for a, b in re.findall(r"harness: step (\d+) end ([0-9.]+)", err)}
            spans.append((st[warmup + 1], en[total]))
    # aggregate throughput of the concurrent processes: sum of per-process rates
    zu = float(n1 * n2 * n3) * steps
    return sum(zu / (e - s) for s, e in spans), None


def replica_max(v, dist=None, device="cuda"):
    """Max over ranks of a per-rank value (the timed region's device ms):
    replicas advance independent tori, so the job's time is the slowest."""
    if dist is None:
        return v
    import torch
    t = torch.tensor([v], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_value(zones, steps, world, ms_max):
    """Whole-job zone-updates/s: every rank's zones over the slowest rank's time."""
    return zones * steps * world / (ms_max / 1e3)


def host_cores():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------
def bench_ours(args, rank, world):
    import numpy as np

    from harm_finalwham_b200 import torus
    from harm_finalwham_b200.gpu import HarmGPU, load_library

    n1, n2, n3, lim, flux = WORKLOADS[args.workload]
    sc = scheme_of(args.workload)
    if args.utoprim:
        sc["utoprim"] = args.utoprim
    t_gen = time.time()
    dom = torus.fm_torus(n1, n2, n3, ng=sc["ng"] or GHOSTS[lim], lim=lim, flux=flux, seed=7 + rank)
    t_gen = time.time() - t_gen
    L = load_library()
    g = HarmGPU(n1, n2, n3, dom.ng, dom.dx, lim=lim, flux=flux, precision=args.precision, gam=dom.gam,
                cour=dom.cour, utoprim=sc["utoprim"], timeorder=sc["timeorder"], doenoflux=sc["doenoflux"])
    g.upload_geometry(dom.gcov, dom.gcon, dom.gcovpert, dom.gdet, dom.conn, dom.floors)
    g.upload_state(dom.p, dom.pflag, 0.0, 0.0)
    dt0 = g.init_dt()
    diag0 = g.diagnostics()
    if args.tuning:
        # a known choice (e.g. for profiler runs that should not see the trials)
        tuning = dict(zip(("flux", "weno", "update", "invert"), (int(v) for v in args.tuning.split(","))))
        g.set_tuning(tuning)
    else:
        tuning = g.autotune()

    dist = None
    if world > 1:
        import torch
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    def barrier():
        if dist is not None:
            dist.barrier()

    def allmax(v):
        return replica_max(v, dist, "cuda")

    # warm-up
    g.step_ch(args.warmup)
    barrier()
    launches0 = L.hgpu_launch_count(g.h)
    clocks = ClockSampler()
    clocks.start()
    ms, st = g.step_ch_timed(args.steps)
    clk = clocks.stop()
    launches = L.hgpu_launch_count(g.h) - launches0
    barrier()
    ms_max = allmax(ms)
    zones = n1 * n2 * n3
    value = replica_value(zones, args.steps, world, ms_max)
    if args.kernels_only:
        g.close()
        return {"metric": METRIC, "value": value, "unit": "zone-updates/s", "note": "kernels-only run",
                "ms_per_step": ms_max / args.steps, "gpu_launches": launches}

    # the other precision mode on the same initial state: its rate and its
    # error against this run after the same number of steps
    other = None
    if not args.no_compare:
        other_prec = "mixed" if args.precision == "fp64" else "fp64"
        # a longer comparison continues both runs untimed to --compare-steps
        extra = max(0, args.compare_steps - (args.warmup + args.steps))
        if extra:
            g.step_ch(extra, stats=False)
        p_this, _, _, _ = g.download_state()
        g2 = HarmGPU(n1, n2, n3, dom.ng, dom.dx, lim=lim, flux=flux, precision=other_prec, gam=dom.gam, cour=dom.cour,
                     utoprim=sc["utoprim"], timeorder=sc["timeorder"], doenoflux=sc["doenoflux"])
        g2.upload_geometry(dom.gcov, dom.gcon, dom.gcovpert, dom.gdet, dom.conn, dom.floors)
        g2.upload_state(dom.p, dom.pflag, 0.0, 0.0)
        g2.init_dt()
        if not args.tuning:
            g2.autotune()
        g2.step_ch(args.warmup)
        barrier()
        ms2, st2 = g2.step_ch_timed(args.steps)
        barrier()
        ms2 = allmax(ms2)
        if extra:
            g2.step_ch(extra, stats=False)
        p_other, _, _, _ = g2.download_state()
        diag_other = g2.diagnostics()
        g2.close()
        diag_this = g.diagnostics()
        p64, p32 = (p_this, p_other) if args.precision == "fp64" else (p_other, p_this)
        a32, a64 = g.active(p32), g.active(p64)
        names = ["rho", "u", "u1", "u2", "u3", "B1", "B2", "B3"]
        err = {nm: float(np.abs(a32[..., q] - a64[..., q]).sum() / np.abs(a64[..., q]).sum())
               for q, nm in enumerate(names)}
        d64, d32 = (diag_this, diag_other) if args.precision == "fp64" else (diag_other, diag_this)

        def drift(dg, q):
            a0 = diag0["integral"][q]
            return (dg["integral"][q] - a0) / abs(a0) if a0 else None

        # the torus's single field loop has zero net magnetic flux: its
        # drift is reported as the absolute change of the integral
        cons = {prec: {"mass_drift": drift(dg, 0), "energy_drift": drift(dg, 1),
                       "magnetic_flux_change": [dg["integral"][q] - diag0["integral"][q] for q in (5, 6, 7)],
                       "divb_max_interior": dg["divb_max_interior"], "failures_last_step": dg["nfail"]}
                for prec, dg in (("fp64", d64), ("mixed", d32))}
        other = {"precision": other_prec, "value": zones * args.steps * world / (ms2 / 1e3),
                 "ms_per_step": ms2 / args.steps, "steps_compared": args.warmup + args.steps + extra,
                 "rel_l1_mixed_vs_fp64": err, "conservation": cons,
                 "note": "mixed = FP32 WENO5 reconstruction (on differences from each cell's value, FP64 "
                         "epsilons; MC/PARA: FP32 Riemann kernel); WENO5's Riemann fluxes FP64 with FP32 wave speeds; "
                         "flux-CT, conserved update, con-to-prim and fixups FP64; both runs from the same "
                         "initial state"}

    # per-kernel device times for the roofline (a separate profiled pass)
    g.set_profiling(True)
    prof_steps = max(2, min(args.steps, 5))
    g.step_ch(prof_steps)
    ktimes = g.kernel_times()
    g.set_profiling(False)

    # e2e through the C ABI with host-owned arrays
    e2e = None
    if not args.no_e2e:
        e2e_steps = max(1, min(args.steps, args.e2e_steps))
        fv = sc["doenoflux"] == "ENOFINITEVOLUME"
        # (a) arrays with ghosts, as the drop-in step_ch moves them: p + pflag
        # up and down every step (the finite-volume scheme's unew too)
        p_host, pf_host = g.pinned_state_buffers()
        u_host = g.download_conserved() if fv else None
        _, _, t_now, dt_now = g.download_state(out=(p_host, pf_host))
        barrier()
        t0 = time.perf_counter()
        for _ in range(e2e_steps):
            g.upload_state(p_host, pf_host, t_now, dt_now)
            if fv:
                g.upload_conserved(u_host)
            g.step_ch(1)
            _, _, t_now, dt_now = g.download_state(out=(p_host, pf_host))
            if fv:
                u_host = g.download_conserved()
        el_full = allmax(time.perf_counter() - t0)
        nb_full = p_host.nbytes + pf_host.nbytes + (2 * u_host.nbytes if fv else 0)
        full = {"value": zones * e2e_steps * world / el_full, "h2d_bytes_per_step": nb_full,
                "d2h_bytes_per_step": nb_full,
                "mode": "arrays with ghosts: upload p+pflag, step_ch(1), download p+pflag every step"}
        if fv:
            e2e = dict(full, unit="zone-updates/s", steps=e2e_steps)
        else:
            # (b) active zones only (hgpu_upload_active / hgpu_download_active:
            # the ghosts rebuilt by bound_prim on the device)
            pa_host, fa_host = g.pinned_active_buffers()
            _, _, t_now, dt_now = g.download_active(out=(pa_host, fa_host))
            barrier()
            t0 = time.perf_counter()
            for _ in range(e2e_steps):
                g.upload_active(pa_host, t_now, dt_now)
                g.step_ch(1)
                _, _, t_now, dt_now = g.download_active(out=(pa_host, fa_host))
            el = allmax(time.perf_counter() - t0)
            e2e = {"value": zones * e2e_steps * world / el, "unit": "zone-updates/s",
                   "h2d_bytes_per_step": pa_host.nbytes, "d2h_bytes_per_step": pa_host.nbytes + fa_host.nbytes,
                   "steps": e2e_steps,
                   "mode": "host-owned active-zone arrays: upload p, step_ch(1), download p+pflag every step",
                   "full_arrays": full}

    # roofline on the dominant kernel
    dom_k = max(ktimes, key=lambda k: ktimes[k]["ms"])
    kt = ktimes[dom_k]
    avg_s = kt["ms"] / kt["launches"] / 1e3
    alg = algorithmic_bytes(dom_k, n1, n2, n3, lim, tx=dom.ng if sc["doenoflux"] == "ENOFINITEVOLUME" else 1)
    peaks, peaks_kind = measured_peaks()
    achieved = alg / avg_s / 1e9
    roof = {"kernel": dom_k, "bound": "hbm", "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
            "frac": achieved / peaks["hbm_gbs"], "traffic": profile_traffic(args.workload, dom_k),
            "peak_source": f"hbm_gbs ({peaks_kind})", "algorithmic_bytes_per_launch": alg,
            "avg_launch_ms": avg_s * 1e3,
            "share": kt["ms"] / sum(v["ms"] for v in ktimes.values())}
    fp64 = fp64_roof(kt, dom_k, args)
    if fp64:
        roof["fp64"] = fp64
    # the whole step against the path's compulsory bytes: 392 B per
    # zone-update (2 substeps x [read p_b 64 + read p^n 64 + write p_f 64 +
    # pflag 4], state resident, metric per (i,j) amortised over x3), beside
    # the DRAM bytes ncu counted for one step
    step_s = ms_max / args.steps / 1e3
    step_alg = 392.0 * zones
    sdb = step_dram_bytes(args.workload)
    roof["step"] = {"algorithmic_bytes": step_alg, "achieved_gbs": step_alg / step_s / 1e9,
                    "frac": step_alg / step_s / 1e9 / peaks["hbm_gbs"], "dram_bytes_ncu": sdb,
                    "dram_over_algorithmic": (sdb / step_alg) if sdb else None,
                    "dram_gbs": (sdb / step_s / 1e9) if sdb else None}

    result = {
        "metric": METRIC, "value": value, "unit": "zone-updates/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64" if args.precision == "fp64" else "f64+f32", "data": "synthetic",
        "config": {"workload": f"{args.workload}: 3D Fishbone-Moncrief torus a=0.9375 beta=100 MKS, "
                               f"{scheme_text(lim, flux, sc)}, {args.precision}",
                   "zones": zones, "ghosts": dom.ng, "parallelism": f"replicas x{world}" if world > 1 else "single",
                   "l2": "inputs larger than L2 (300 MB per state array)", "init_dt": dt0,
                   "newton_iters_per_zone_step": st.newton_iters / (zones * args.steps * float(sc["timeorder"])),
                   "autotune": tuning},
        "gpu_launches": launches,
        "roofline": roof,
        "kernels": {k: {"ms": round(v["ms"], 4), "launches": v["launches"]} for k, v in ktimes.items() if v["launches"]},
        "e2e": e2e,
        "clocks": clk,
    }
    if other is not None:
        result["other_precision"] = other
    if not args.no_batch:
        result["batch_riemann1d"] = bench_riemann_batch()
        result["serving"] = bench_serving()
        # a longer stream of the same mix through the server alone: its
        # time-to-solution percentiles over 200 requests
        long = bench_serving(count=200, one_at_a_time=False)
        result["serving"]["stream_200"] = {k: long[k] for k in ("requests", "kinds", "value", "makespan_s",
                                                                "time_to_solution_ms")}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        procs = min(host_cores(), args.cpu_procs) if args.cpu_procs > 0 else host_cores()
        cs = cpu_sample(args.workload)
        v, why = run_reference(cs, args.cpu_steps, 2, procs)
        result["cpu_baseline"] = ({"value": v, "unit": "zone-updates/s", "cores": procs, "kind": "reference",
                                   "sample": f"reference CPU build (gcc -O2 -ffp-contract=off), 3D torus "
                                             f"{cs[0]}x{cs[1]}x{cs[2]} {cs[3]}+{cs[4]}, {args.cpu_steps} steps "
                                             f"after 2 warm-up, one process per core"}
                                  if v else {"value": None, "unavailable": why})
    result["gen_seconds"] = t_gen
    if dist is not None:
        dist.destroy_process_group()
    g.close()
    return result


def bench_riemann_batch(ninst=256, seed=2024, sample_single=12, check_every=25):
    """Batched uneven 1D relativistic-MHD Riemann problems (MC + HLL, CFL 0.5,
    x in [-0.5, 0.5], t = 0.4): all instances advanced together by shared
    launches (hgpu_create_batch, CUDA-graph steps) until each reaches t = 0.4,
    against the same solves run one at a time."""
    import numpy as np

    from harm_finalwham_b200 import riemann
    from harm_finalwham_b200.gpu import HarmBatch, HarmGPU

    ng, tf = 3, 0.4
    probs = riemann.draw(ninst, seed=seed)

    def batch_of(ps):
        b = HarmBatch([p.n for p in ps], [p.dx for p in ps], [p.gam for p in ps], [tf] * len(ps), ng=ng, lim="MC",
                      flux="HLL", cour=0.5)
        b.upload_geometry(*riemann.minkowski_geometry(b.nt[0]))
        b.upload_state(b.join([riemann.primitives(p, ng) for p in ps]), None, 0.0, 0.0)
        b.init_dt()
        return b

    # warm-up: graph capture and instantiation on a small batch
    w = batch_of(probs[:4])
    w.run(check_every)
    w.close()
    b = batch_of(probs)
    tuning = b.autotune()
    steps, ms, per, fin = b.run(check_every)
    b.close()
    zu = float(np.sum(np.array([p.n for p in probs]) * per))
    fin = fin[fin >= 0]
    out = {"instances": ninst, "zones": int(sum(p.n for p in probs)), "zone_updates": zu, "batch_steps": steps,
           "ms": ms, "value": zu / (ms / 1e3), "unit": "zone-updates/s",
           "time_to_solution_ms": {"p50": float(np.percentile(fin, 50)), "p99": float(np.percentile(fin, 99)),
                                   "resolution_steps": check_every},
           "scheme": "MC + HLL + flux-CT, CFL 0.5, t = 0.4, N ~ U{200..2000}, seeded states",
           "autotune": tuning,
           "timing": "device time (CUDA events) of the whole run incl. the done-flag polls"}
    # one solve at a time: (a) the plain host loop, one step_ch(1) and a time read per step;
    # (b) the same graph machinery on a batch of one
    sub = probs[:sample_single]
    t_plain = 0.0
    zu_sub = 0.0
    for pb in sub:
        g = HarmGPU(pb.n, 1, 1, ng, (pb.dx, 1.0, 1.0), lim="MC", flux="HLL",
                    bc=("OUTFLOW_COPY", "OUTFLOW_COPY", "OUTFLOW", "OUTFLOW", "OUTFLOW", "OUTFLOW"), gam=pb.gam,
                    cour=0.5, tf=tf)
        g.upload_geometry(*riemann.minkowski_geometry(pb.n + 2 * ng))
        g.upload_state(riemann.primitives(pb, ng), None, 0.0, 0.0)
        g.init_dt()
        g.sync()
        t0 = time.perf_counter()
        n = 0
        while n < 100000:
            g.step_ch(1, stats=False)
            n += 1
            if g.time()[0] >= tf:
                break
        t_plain += time.perf_counter() - t0
        zu_sub += pb.n * n
        g.close()
    ms_graph = 0.0
    zu_graph = 0.0
    for pb in sub:
        one = batch_of([pb])
        st, m1, per1, _ = one.run(check_every)
        one.close()
        ms_graph += m1
        zu_graph += pb.n * float(per1[0])
    out["one_at_a_time"] = {"instances": len(sub), "plain_launches": zu_sub / t_plain,
                            "graph_batch_of_one": zu_graph / (ms_graph / 1e3), "unit": "zone-updates/s",
                            "timing": "wall clock per solve (plain), device time (graph)"}
    out["speedup_vs_one_at_a_time"] = {"plain_launches": out["value"] / (zu_sub / t_plain),
                                       "graph_batch_of_one": out["value"] / (zu_graph / (ms_graph / 1e3))}
    return out


def serving_requests(count, seed, shock_tubes=0.0):
    """A seeded request stream of (kind, domain, end time): 60% Kerr torus,
    40% Bondi (Schwarzschild, r_s = 8M, monopole field), both to t = 50 on
    grids from {32x32, 64x64, 128x128, 256x128} (2D) or {64x32x16, 96x48x32}
    (3D tori), spin a ~ U(0, 0.99), beta ~ logU[10, 1000], 4% internal-energy
    noise; arrival gaps exponential.  With shock_tubes > 0 that fraction of
    the requests are 1D relativistic-MHD shock tubes instead (MC + HLL, CFL
    0.5, N ~ U{200..2000}, seeded states, to t = 0.4)."""
    import numpy as np

    from harm_finalwham_b200 import bondi, riemann, torus

    rng = np.random.default_rng(seed)
    grids2 = [(32, 32), (64, 64), (128, 128), (256, 128)]
    grids3 = [(64, 32, 16), (96, 48, 32)]
    out = []
    for q in range(count):
        beta = 10.0 ** rng.uniform(1.0, 3.0)
        if shock_tubes and rng.random() < shock_tubes:
            prob = riemann.draw(1, seed=int(rng.integers(1 << 30)))[0]
            out.append(("shock tube", riemann.domain(prob), 0.4))
            continue
        if rng.random() < 0.6:
            a = rng.uniform(0.0, 0.99)
            if rng.random() < 0.2:
                n = grids3[rng.integers(len(grids3))]
            else:
                n = grids2[rng.integers(len(grids2))] + (1,)
            dom = torus.fm_torus(*n, ng=3, a=a, beta=beta, seed=int(rng.integers(1 << 30)))
            kind = "torus"
        else:
            n = grids2[rng.integers(len(grids2))]
            dom = bondi.bondi(*n, ng=3, beta=beta, seed=int(rng.integers(1 << 30)))
            kind = "bondi"
        out.append((kind, dom, 50.0))
    return out


def bench_serving(count=64, mean_gap_ms=2.0, seed=11, budget_bytes=32e9, max_active=32, steps_per_chunk=8,
                  one_at_a_time=True, shock_tubes=0.0):
    """Continuous batching: requests arrive on a seeded Poisson clock fast
    enough to keep the GPU saturated and go through hgpu_server (admission by
    device footprint, overlapped solves, each solve's step replayed from its
    captured graph), against the same requests solved one at a time."""
    import numpy as np

    from harm_finalwham_b200.gpu import HarmGPU, HarmServer

    reqs = serving_requests(count, seed, shock_tubes)
    rng = np.random.default_rng(seed + 1)
    arrivals = np.cumsum(rng.exponential(mean_gap_ms / 1e3, count))
    srv = HarmServer(max_device_bytes=int(budget_bytes), max_active=max_active, steps_per_chunk=steps_per_chunk)
    ids = {}
    t0 = time.perf_counter()
    done_at = {}
    nsub = 0
    while len(done_at) < count:
        now = time.perf_counter() - t0
        while nsub < count and arrivals[nsub] <= now:
            ids[srv.submit(reqs[nsub][1], reqs[nsub][2])] = nsub
            nsub += 1
        srv.poll()
        for rid, q in ids.items():
            if q not in done_at and srv.result(rid) is not None:
                done_at[q] = time.perf_counter() - t0
        if now > 600:
            break
    makespan = max(done_at.values())
    zu = 0.0
    lat = []
    for rid, q in ids.items():
        res = srv.result(rid)
        if res is None:
            continue
        zu += float(np.prod(reqs[q][1].n)) * res[3]
        lat.append((done_at[q] - arrivals[q]) * 1e3)
    srv.close()
    # the same requests one at a time (each alone, in arrival order): plain
    # launches (the one-solve-at-a-time baseline) and graph replays.  As the
    # server does, one context per allocation shape is kept and reused
    # (geometry and state uploaded per request), so neither arm pays
    # cudaMalloc/cudaFree per request.
    inv = {0: "OUTFLOW", 4: "POLARAXIS", 7: "PERIODIC", 1000: "OUTFLOW_COPY"}
    alone = {}
    for mode in (("plain_launches", "graph") if one_at_a_time else ()):
        pool = {}
        t1 = time.perf_counter()
        zu1 = 0.0
        for kind, dom, tf in reqs:
            key = (dom.n, dom.ng, dom.lim, dom.flux, tuple(dom.bc))
            g = pool.get(key)
            if g is None:
                g = pool[key] = HarmGPU(*dom.n, dom.ng, dom.dx, lim=dom.lim, flux=dom.flux,
                                        bc=tuple(inv[b] for b in dom.bc), gam=dom.gam, cour=dom.cour, tf=tf)
            else:
                g.reconfigure(dx=dom.dx, gam=dom.gam, cour=dom.cour, tf=tf)
            g.upload_geometry(dom.gcov, dom.gcon, dom.gcovpert, dom.gdet, dom.conn, dom.floors)
            g.upload_state(dom.p, None, 0.0, 0.0)
            g.init_dt()
            n = 0
            while n < 1000000:
                if mode == "graph":
                    g.step_graph(8, stats=False)
                else:
                    g.step_ch(8, stats=False)
                n += 8
                if g.time()[0] >= tf:
                    break
            n = g.diagnostics()["nsteps"]      # steps taken before the end time froze the state
            zu1 += float(np.prod(dom.n)) * n
        t_seq = time.perf_counter() - t1
        for g in pool.values():
            g.close()
        alone[mode] = {"value": zu1 / t_seq, "seconds": t_seq, "contexts": len(pool)}
    return {"requests": count, "kinds": {k: sum(1 for r in reqs if r[0] == k) for k in ("torus", "bondi", "shock tube")},
            "tf": {"torus": 50.0, "bondi": 50.0, "shock tube": 0.4}, "value": zu / makespan, "unit": "zone-updates/s", "makespan_s": makespan,
            "time_to_solution_ms": {"p50": float(np.percentile(lat, 50)), "p90": float(np.percentile(lat, 90)),
                                    "p99": float(np.percentile(lat, 99))},
            "one_at_a_time": alone,
            "speedup_vs_one_at_a_time": {m: (zu / makespan) / v["value"] for m, v in alone.items()},
            "slots": max_active, "steps_per_chunk": steps_per_chunk,
            "note": "wall clock; arrivals Poisson (mean gap %.0f ms, saturating); time-to-solution = finish - "
                    "arrival; one at a time = each solve alone in arrival order on a context reused per "
                    "allocation shape, 8 steps per host check, with plain launches or with its captured step "
                    "graph" % mean_gap_ms}


def algorithmic_bytes(kernel, n1, n2, n3, lim="MC", tx=1):
    """Compulsory HBM bytes per launch (FP64, state resident; per-(i,j) metric
    amortised over x3).  Units: faces for the flux kernels, zones otherwise.
    tx: transverse zones beyond the grid that the flux loops cover (1; all
    ghosts for the finite-volume scheme)."""
    zones = n1 * n2 * n3
    t = 2 * tx
    faces = {"flux_x1": (n1 + 1) * (n2 + t) * (n3 + t), "flux_x2": (n1 + t) * (n2 + 1) * (n3 + t),
             "flux_x3": (n1 + t) * (n2 + t) * (n3 + 1)}
    if kernel in faces:
        if lim == "WENO5":
            return faces[kernel] * (128 + 64)     # read the two face states (16 doubles), write 8 fluxes
        return faces[kernel] * (64 + 64)          # read one zone's 8 primitives, write 8 face fluxes
    # the WENO5 passes run once per direction under one name: mean cells per launch
    nd = [n for n in (n1, n2, n3) if n > 1]
    if kernel == "weno5":
        # output cells -1..n along the direction (mean over the directions):
        # read 8 primitives and the 2 dP/P state pieces, write 16 face values
        cells = sum(zones / n * (n + 2) for n in nd) / len(nd)
        return cells * (64 + 16 + 128)
    if kernel == "w5_state":
        # zones -2..n+1: read 8 primitives, write 2 state pieces
        ext = 1.0
        for n in (n1, n2, n3):
            ext *= (n + 4) / n if n > 1 else 1.0
        return zones * ext * (64 + 16)
    if kernel == "update":
        # mean of the two substeps: p(64) [+pk 64] + 5 F comps x3 dirs (120) + 3 EMFs (24)
        # + uf/ucum write (128) [+read 128] + pf (64) + pflag (4)
        return zones * (468 + 596) / 2.0
    if kernel == "emf":
        return zones * (6 * 8 + 3 * 8)
    if kernel == "bound_ghost":
        return zones * 0.0 + (2 * 3 * 8 * 8) * ((n2 + 6) * (n3 + 6) + (n1 + 6) * (n3 + 6) + (n1 + 6) * (n2 + 6))
    return zones * 8.0


def fp64_roof(kt, kernel, args):
    """FP64 issue rate of the dominant kernel: FP64 instructions per launch
    (DADD + DMUL + DFMA, ncu, profiles/traffic.md) over its CUDA-event time,
    against the FP64 instruction issue rate measured here (hgpu_fp64_peak:
    independent DADD/DMUL streams; a DFMA issues at the same rate).  Both
    numbers count instructions, one per FP64 operation issued."""
    r = _traffic_row(args.workload, kernel)
    if not r or r[1] <= 0:
        return None
    inst_per_launch = r[1]
    avg_s = kt["ms"] / kt["launches"] / 1e3
    achieved = inst_per_launch / avg_s / 1e12
    peak = measure_fp64_peak()
    return {"achieved_tinst_s": achieved, "peak_tinst_s": peak, "frac": achieved / peak if peak else None,
            "unit": "T FP64 instructions/s",
            "note": "DADD+DMUL+DFMA instructions per launch from ncu over the CUDA-event launch time; peak = "
                    "measured FP64 issue rate of this GPU (the FP64 path is built with -fmad=false for "
                    "bit-identity, so its FMAs are those inside the IEEE division/sqrt sequences)"}


_FP64_PEAK = None


def measure_fp64_peak():
    global _FP64_PEAK
    if _FP64_PEAK is None:
        from harm_finalwham_b200.gpu import fp64_peak_tflops
        _FP64_PEAK = fp64_peak_tflops()
    return _FP64_PEAK


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default=DEFAULT_WORKLOAD, choices=sorted(WORKLOADS))
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"])
    ap.add_argument("--utoprim", default=None, choices=["2DFINAL", "JON"],
                    help="con-to-prim inverter (default: the workload's): utoprim_2d_final.c or utoprim_jon.c")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-batch", action="store_true",
                    help="skip the batched 1D Riemann-problem measurement")
    ap.add_argument("--no-compare", action="store_true",
                    help="skip the run of the other precision mode (rate and error vs FP64)")
    ap.add_argument("--e2e-steps", type=int, default=5)
    ap.add_argument("--compare-steps", type=int, default=1000,
                    help="steps of the FP64-vs-mixed comparison (the precision-at-scale configuration runs 1000; "
                         "0: warm-up + timed steps)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-steps", type=int, default=3)
    ap.add_argument("--cpu-procs", type=int, default=0,
                    help="processes of the reference CPU build (default: every host core this process may use)")
    ap.add_argument("--tuning", default=None,
                    help="blocks per SM for flux,weno,update,invert instead of running the autotuner")
    ap.add_argument("--kernels-only", action="store_true",
                    help="set-up, warm-up and the timed steps only (for profiler runs)")
    ap.add_argument("--decomp", default=None, choices=["x3"],
                    help="split one torus along x3 over the ranks (NCCL halo exchange); the default for N > 1")
    ap.add_argument("--replicas", action="store_true",
                    help="N > 1: independent tori per rank instead of the x3 split")
    args = ap.parse_args()
    rank, world, local = rank_info()
    if args.warmup < 3:
        args.warmup = 3

    if args.impl == "reference":
        if rank != 0:
            return 0
        procs = min(host_cores(), args.cpu_procs) if args.cpu_procs > 0 else host_cores()
        cs = cpu_sample(args.workload)
        # each step: one step of every process's bounded sample
        v, why = run_reference(cs, args.steps, args.warmup, procs)
        if v is None:
            print(json.dumps({"impl": "reference", "unavailable": why}))
            return 0
        n1, n2, n3 = cs[:3]
        sample = (f"reference CPU build (its own C sources, gcc -O2 -ffp-contract=off): 3D torus {n1}x{n2}x{n3} "
                  f"{cs[3]}+{cs[4]} per process, {procs} processes (the code is single-threaded "
                  f"and non-reentrant), {args.steps} timed steps after {args.warmup}")
        out = {"impl": "reference", "metric": METRIC, "value": v, "unit": "zone-updates/s", "n_gpus": args.gpus,
               "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
               "vs_baseline": None, "dtype": "f64", "data": "synthetic",
               "config": {"workload": f"{args.workload} (CPU sample {n1}x{n2}x{n3} per core)"},
               "cpu_baseline": {"value": v, "unit": "zone-updates/s", "cores": procs, "kind": "reference",
                                "sample": sample},
               "e2e": {"value": v, "unit": "zone-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(out))
        return 0

    select_device(local, world)
    if world > 1 and not args.replicas and not args.decomp:
        args.decomp = "x3"
    res = bench_decomp(args, rank, world) if args.decomp else bench_ours(args, rank, world)
    if rank == 0:
        print(json.dumps(res))
    return 0


if __name__ == "__main__":
    sys.exit(main())
