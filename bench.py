#!/usr/bin/env python
"""Benchmark: cell-updates/s of the self-gravitating hydro step on one B200.

Headline workload (the configuration the target is quoted on): the 5-level
ZTWD binary of the reference's BINARY build -- two zero-temperature white
dwarfs (the reference's two-polytrope initial data, binary/initialize.cpp),
mass ratio q = 0.7, separation 0.5, donor near its Roche lobe, co-rotating
frame, Helmholtz EOS (synthetic table in the reference's format), PPM with
BW 3 on 8^3-cell bricks, CFL 0.3; one step = BinaryDriver::step: three RK3
substeps, each hydro followed by a multigrid Poisson solve to L1 error
1e-7 (ELL_TOLER), regrid every 8 steps.  `value` is the mixed-precision
persistent form (FP32 multigrid correction inside FP64 defect correction,
each solve one persistent kernel); the plain FP64 form, the FP64 persistent
form and the mixed form's errors after 100 steps are reported beside it,
with the reference's own BINARY build timed on the host cores.  A step's
work is the leaf cells it advances (GridNode::get_zone_cnt).

Secondary sections: the single star (n=1.5 polytrope, 4 levels, Euler
state, minmod, the graph and persistent forms), the batched uneven-brick
substep on a random-field octree, the Helmholtz EOS at 2^24 points.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

N > 1 runs independent replicas (the path is not sharded in this build):
value = all ranks' cell updates / max over ranks of the timed region.
"""

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "3d-eulerian-amr_b200")

LEVELS = 4
TOL = 1.0e-6
ZT_LEVELS = 5
ZT_NX = 12  # interior cells per brick edge of the BINARY build (binary/binary_defs.h:31-35)
ZT_TOL = 1.0e-7  # ELL_TOLER of the BINARY build (binary/binary_defs.h:64)
ZT_STEPS_TOTAL = 100
DYNAMIC_RANGE = 1.0e6
REF_CXXFLAGS = "g++ -O3 -fopenmp -ffp-contract=off"  # oracle/build_ref.py CXXFLAGS
METRIC = "cell-updates/s (hydro+gravity step), 1 B200: mixed+batched vs FP64 at set error"
# The headline's precision: the FP32 multigrid correction inside FP64 defect
# correction, the hydro (PPM, KT flux, EOS) in FP64.  The FP32 flux as well
# (AMR_PREC_MIXED) runs at the same speed within 1% on this workload (the
# flux kernel is 3% of the step) and moves the density 1000 times further
# from the FP64 form over 100 steps, so it is measured beside the headline.
def ZT_PREC(amr):
    return amr.PREC_MIXED_SOLVE


ZT_FORM = "mixed persistent: FP32 multigrid correction in FP64 defect correction, FP64 hydro"
UNIT = "cell-updates/s"
WORKLOAD = "single star: n=1.5 polytrope, 4 levels, RK3 hydro + multigrid gravity (L1 tol 1e-6)"
ZT_WORKLOAD = ("ZTWD binary: q=0.7, 5 levels, %d^3 bricks, PPM, Helmholtz EOS, BinaryDriver steps "
               "(RK3 hydro + multigrid gravity every substep, L1 tol 1e-7, regrid every 8 steps)")

# Bytes each kernel class must move per brick per launch (FP64, nx=8, BW=2,
# NF=6, PNX=10); the denominator-free "algorithmic" traffic of one launch.
NX, BW, NF, PNX = 8, 2, 6, 10
BYTES_PER_BRICK = {
    # read U on the cross of interior + 6 ghost slabs, write 3 face-flux arrays
    "flux": 8 * NF * (NX ** 3 + 6 * BW * NX ** 2) + 8 * 3 * NF * NX * NX * (NX + 1),
    # read 3 flux arrays + U + U0 interiors + 3 face-force arrays, write U
    "add_difs": 8 * 3 * NF * NX * NX * (NX + 1) + 8 * 3 * NF * NX ** 3 + 8 * 3 * PNX ** 3,
    # read dphi (with ghosts) and dphi1, write dphi; sweeps stay on chip
    "relax": 8 * (PNX ** 3 + 2 * NX ** 3),
    # read + write the six ghost slabs
    "ghost_fill": 8 * NF * 2 * 6 * BW * NX * NX,
    "dphi_boundaries": 8 * 2 * 6 * NX * NX,
}

# DRAM bytes (read + write) per launch of the persistent solve on the 5-level
# ZTWD binary, from ncu (dram__bytes_read.sum + dram__bytes_write.sum, caches
# flushed before each launch) on `bench.py --case ztwd_mixed_L5`: 8^3 bricks,
# the mean over the six solve launches of two BinaryDriver steps (2.72 GB of
# algorithmic bytes each); 12^3 bricks, the seventh solve launch of the case
# (7.93 GB of algorithmic bytes).  The solve's arrays stay in L2 across its
# V-cycles, so DRAM sees the cold fill, the per-launch zeroing of the tagged
# relaxation buffers and the dirty write-back.
ZT_SOLVE_DRAM_BYTES_PER_LAUNCH = {8: 16.69e6, 12: 185.0e6}


# the keys of the roofline object on the bench line (the rest of the solve's
# breakdown is written to the --json-out sidecar)
ROOFLINE_LINE_KEYS = ("bound", "kernel", "achieved", "peak", "unit", "frac", "peak_source", "traffic",
                      "algorithmic_bytes_per_launch", "ms_per_launch", "note", "traffic_note")


def load_amr():
    import importlib.util
    spec = importlib.util.spec_from_file_location("amr_b200", os.path.join(PKG, "amr.py"))
    amr = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(amr)
    spec = importlib.util.spec_from_file_location("amr_initial", os.path.join(PKG, "initial.py"))
    ini = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(ini)
    return amr, ini


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + q,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
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
        rows = []
        with open(self.path) as f:
            for line in f:
                parts = [x.strip() for x in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        smax = max(float(r[2]) for r in rows if r[2].replace(".", "").isdigit())
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        loaded = [s for s in sm if s > 0.5 * smax] or sm
        return {"sm_mhz": statistics.median(loaded), "sm_max_mhz": smax, "reasons": reasons,
                "samples": len(rows)}


def run_reference_steps(levels, threads, warm, steps, timeout=3000):
    """The reference's own CPU code (oracle/_ref, built from the reference
    sources, g++ -O3 -fopenmp) on the same workload: `warm` untimed RK3 steps
    (the first includes the initial solve from phi = 0), then `steps` timed
    steps.  Returns per-step seconds, leaf cells and bricks."""
    exe = os.path.join(ROOT, "oracle", "_ref", "g05_harness")
    if not os.path.exists(exe):
        return None
    env = dict(os.environ, OMP_NUM_THREADS=str(threads))
    try:
        r = subprocess.run([exe, "time_grav", "polytrope", str(levels), str(warm + steps), str(TOL), "-"],
                           env=env, capture_output=True, text=True, timeout=timeout)
    except subprocess.TimeoutExpired:
        return None
    if r.returncode != 0:
        return None
    rows = [json.loads(x) for x in r.stdout.strip().splitlines() if x.startswith("{")]
    per = [x for x in rows if "step" in x]
    summ = [x for x in rows if x.get("mode") == "grav"][-1]
    timed = per[warm:]
    return {"seconds": [x["seconds"] for x in timed], "vcycles": [x["vcycles"] for x in timed],
            "leaf_cells": [x.get("leaf_cells", summ["leaf_cells"]) for x in timed],
            "bricks": summ["bricks"], "threads": summ["threads"]}


def ztwd_harness(nx):
    """The reference's BINARY build for nx^3 bricks (oracle/_ref): the
    unpatched build (12^3) or the 8^3 variant."""
    return os.path.join(ROOT, "oracle", "_ref", "ztwd12_harness" if nx == 12 else "ztwd_harness")


def run_reference_ztwd(threads, warm, steps, nx=ZT_NX, timeout=1500):
    """The reference's BINARY build (oracle/_ref, g++ -O3 -fopenmp) on the
    headline workload: `warm` untimed BinaryDriver steps (the first solves
    from the initial potential), then `steps` timed ones."""
    exe = ztwd_harness(nx)
    if not os.path.exists(exe):
        return None
    helm_table = _load_module("helm_table", os.path.join(PKG, "helm_table.py"))
    tdir = tempfile.mkdtemp(prefix="ztwd_ref_")
    helm_table.ensure_table(tdir)
    env = dict(os.environ, OMP_NUM_THREADS=str(threads))
    try:
        r = subprocess.run([exe, "time_ztwd", str(ZT_LEVELS), str(warm + steps)], cwd=tdir, env=env,
                           capture_output=True, text=True, timeout=timeout)
        row = json.loads([x for x in r.stdout.splitlines() if x.startswith("{")][-1])
    except (subprocess.TimeoutExpired, IndexError, ValueError):
        return None
    finally:
        import shutil
        shutil.rmtree(tdir, ignore_errors=True)
    return {"seconds": row["seconds"][warm:], "leaf_cells": row["leaf_cells"][warm:], "bricks": row["bricks"],
            "threads": row["threads"]}


def reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    threads = os.cpu_count() or 1
    # a bounded sample: one untimed step (the initial solve) and at most two
    # timed steps (~20 s each on 16 host threads)
    s = run_reference_ztwd(threads, 1, min(args.steps, 2), nx=args.zt_nx)
    name = os.path.basename(ztwd_harness(args.zt_nx))
    if s is None or not s["seconds"]:
        print(json.dumps({"impl": "reference",
                          "unavailable": "oracle/_ref/%s missing, failed or timed out" % name}))
        return 0
    t = sum(s["seconds"])
    value = sum(s["leaf_cells"]) / t
    sample = ("reference BINARY build (oracle/_ref/%s, %s, %d threads): %d BinaryDriver steps of the 5-level "
              "binary on %d^3 bricks after 1 untimed step, %d bricks" %
              (name, REF_CXXFLAGS, s["threads"], len(s["seconds"]), args.zt_nx, s["bricks"]))
    out = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": len(s["seconds"]), "warmup": 1, "ms_per_step": 1000.0 * t / len(s["seconds"]),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": ZT_WORKLOAD % args.zt_nx, "levels": ZT_LEVELS, "nx": args.zt_nx,
                   "bricks": s["bricks"]},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": s["threads"], "kind": "reference",
                         "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out))
    return 0


def reference_arm_single_star(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    threads = os.cpu_count() or 1
    warm = max(1, args.warmup)
    s = run_reference_steps(LEVELS, threads, warm, args.steps)
    if s is None or not s["seconds"]:
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/g05_harness missing, failed or timed out"}))
        return 0
    t = sum(s["seconds"])
    value = sum(s["leaf_cells"]) / t
    sample = ("reference CPU code (oracle/_ref, g++ -O3 -fopenmp, %d threads): %d full RK3 steps after %d "
              "untimed (the first solves from phi = 0), %d bricks, %.1f V-cycles/step" %
              (s["threads"], len(s["seconds"]), warm, s["bricks"], sum(s["vcycles"]) / len(s["vcycles"])))
    out = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": len(s["seconds"]), "warmup": warm, "ms_per_step": 1000.0 * t / len(s["seconds"]),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "levels": LEVELS, "bricks": s["bricks"]},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": s["threads"], "kind": "reference",
                         "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out))
    return 0


def aggregate(ms_total, cells, world, dist, device="cuda"):
    """Whole-job figures over the replicas: the slowest rank's device time
    (max) and the cells of all ranks (sum); every rank gets both."""
    import torch
    t = torch.tensor([float(ms_total), float(cells)], dtype=torch.float64, device=device)
    if world > 1:
        dist.all_reduce(t[0:1], op=dist.ReduceOp.MAX)
        dist.all_reduce(t[1:2], op=dist.ReduceOp.SUM)
    return float(t[0]), float(t[1])


def run_form(amr, ini, form, args, world, local, torch, dist, e2e=False, profile=False):
    """Build the workload and time K steps of one form of our path.

    form: "fp64"  plain FP64, host-orchestrated (reference operation order)
          "graph" FP64, whole RK3 step replayed from a captured CUDA graph with
                  every loop decided on the device (bitwise equal to fp64)
          "persistent" the graph form with each solve's V-cycle loop as one
                  persistent cooperative kernel (bitwise equal to fp64)
          "mixed" the persistent form with the multigrid correction
                  (smoothing, restriction, prolongation of dphi) and the KT
                  flux in FP32; residual, potential and conserved update FP64
    """
    prec = amr.PREC_MIXED if form == "mixed" else amr.PREC_FP64
    a = amr.AMR(physics=amr.PHYSICS_EULER_GRAVITY, max_refine_level=LEVELS, grid_dim=0.5, z_reflect=0,
                max_bricks=8192, precision=prec, persistent_solve=2 if form in ("persistent", "mixed") else 0)
    ini.build_tree(a, "polytrope", 1.0e-6, 0.5, 0, LEVELS, device=True)
    stream = torch.cuda.ExternalStream(a.stream_handle())
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device="cuda")
    state = {"step": 0, "last_dt": 0.0}

    def one_step():
        st = state["step"]
        if form == "fp64":
            dt = a.max_dt()
            if st > 0:
                dt = min(1.25 * state["last_dt"], dt)
            state["last_dt"] = dt
            a.grav_step(dt, TOL, DYNAMIC_RANGE, st)
        else:
            a.graph_grav_step(TOL, DYNAMIC_RANGE, st)
        state["step"] = st + 1

    def barrier():
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()

    for _ in range(args.warmup):
        one_step()
    res = {"form": form}
    st0 = a.stats()
    persistent = form in ("persistent", "mixed")
    ph0 = a.solve_phases() if persistent else None
    w0 = a.solve_phase_waits() if persistent else None
    solve_ms = []
    k0 = a.launch_count()
    sampler = ClockSampler(local)
    barrier()
    sampler.start()
    times, cells = [], 0
    for _ in range(args.steps):
        with torch.cuda.stream(stream):
            flush.zero_()  # L2 flush between timed steps, outside the timed interval
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        n_cells = a.get_zone_cnt()
        torch.cuda.nvtx.range_push("timed_step")  # lets a profiler select the timed launches
        ev0.record(stream)
        one_step()
        ev1.record(stream)
        torch.cuda.nvtx.range_pop()
        ev1.synchronize()
        times.append(ev0.elapsed_time(ev1))
        if persistent:
            solve_ms.append(a.solve_last_ms())  # the step's last persistent solve kernel
        cells += n_cells
    barrier()
    res["clocks"] = sampler.stop()
    st1 = a.stats()
    res["gpu_launches"] = a.launch_count() - k0
    if persistent:
        ph1 = a.solve_phases()
        d = {k: {"ms": ph1[k]["ms"] - ph0[k]["ms"], "count": ph1[k]["count"] - ph0[k]["count"],
                 "bytes": ph1[k]["bytes"] - ph0[k]["bytes"]} for k in ph1}
        launches = 3 * args.steps  # one persistent solve per RK substep
        res["persistent"] = {"ms_per_launch": statistics.mean(solve_ms),
                             "bytes_per_launch": sum(v["bytes"] for v in d.values()) / launches,
                             "phase_ms_per_step": {k: round(v["ms"] / args.steps, 4) for k, v in d.items()},
                             "phases_per_step": {k: v["count"] / args.steps for k, v in d.items()}}
        w1 = a.solve_phase_waits()
        res["persistent"]["barrier_ms_per_step"] = {k: round((w1[k] - w0[k]) / args.steps, 4) for k in ph1}
        res["persistent"]["level_sum_ms_per_step"] = round((w1["level_sum"] - w0["level_sum"]) / args.steps, 4)
        res["persistent"]["level_sums_per_step"] = (w1["level_sum_count"] - w0["level_sum_count"]) / args.steps
    # state after warm-up + timed steps, for the error of one form against another
    res["final"] = {"U": a.download_state(), "phi": a.download_poisson()[0], "level": a.get_tree()["level"],
                    "loc": a.get_tree()["loc"]}
    t = aggregate(sum(times), cells, world, dist)
    res["ms_total"], res["cells"] = t
    res["value"] = res["cells"] / (res["ms_total"] / 1000.0)
    res["ms_per_step"] = res["ms_total"] / args.steps
    res["bricks"] = a.nbricks
    res["relax_calls_per_step"] = (st1["relax_calls"] - st0["relax_calls"]) / args.steps

    if e2e:
        # end to end through the public API: the state lives in pinned host
        # memory, is uploaded, stepped and read back every step
        cap = 8192 * a.nf * a.gnx ** 3
        hbuf = torch.empty(cap, dtype=torch.float64, pin_memory=True)
        U = a.download_state()
        hbuf[:U.size].copy_(torch.from_numpy(U.reshape(-1)))
        ptr = ctypes.cast(hbuf.data_ptr(), ctypes.POINTER(ctypes.c_double))
        barrier()
        e_times, e_cells, h2d, d2h = [], 0, 0, 0
        for _ in range(args.steps):
            ev0 = torch.cuda.Event(enable_timing=True)
            ev1 = torch.cuda.Event(enable_timing=True)
            n_in = a.nbricks * a.nf * a.gnx ** 3
            e_cells += a.get_zone_cnt()
            ev0.record(stream)
            a._check(a.lib.amr_upload_state(a.ctx, ptr))
            one_step()
            n_out = a.nbricks * a.nf * a.gnx ** 3
            a._check(a.lib.amr_download_state(a.ctx, ptr))
            ev1.record(stream)
            ev1.synchronize()
            e_times.append(ev0.elapsed_time(ev1))
            h2d += 8 * n_in
            d2h += 8 * n_out
        barrier()
        et = aggregate(sum(e_times), e_cells, world, dist)
        res["e2e"] = {"value": et[1] / (et[0] / 1000.0), "unit": UNIT,
                      "h2d_bytes_per_step": h2d // args.steps, "d2h_bytes_per_step": d2h // args.steps}

    if profile:
        # per-kernel-class device time over two profiled steps of the plain
        # launch sequence (event brackets need host-issued launches)
        a.profile(True)
        a.profile_reset()
        for _ in range(2):
            dt = a.max_dt()
            a.grav_step(min(dt, 1.25 * state["last_dt"]) if state["last_dt"] > 0 else dt, TOL, DYNAMIC_RANGE,
                        state["step"])
            state["step"] += 1
        a.synchronize()
        res["profile"] = a.profile_get()
        a.profile(False)
    a.close()
    return res


EOS_POINTS = 1 << 24
EOS_FLOPS_PER_POINT = 1000  # FP64 adds/muls of one helm_point call, counted in helm_kernels.cu
EOS_IO_BYTES = 56  # rho, T, abar, zbar in; p, e, cs out (FP64)
FP64_NOMINAL_TFLOPS = 37.0  # B200 FP64 (non-tensor), vendor figure: no measured FP64 peak exists here


def _load_module(name, path):
    import importlib.util
    spec = importlib.util.spec_from_file_location(name, path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def run_eos(torch, steps, warmup, cpu_sample):
    """Helmholtz EOS throughput: 2^24 points, forward (rho,T)->(p,e,cs) and
    inverse (rho,e)->T by Newton, each one launch over device arrays."""
    helm_table = _load_module("helm_table", os.path.join(PKG, "helm_table.py"))
    helm_mod = _load_module("helm_b200", os.path.join(PKG, "helm.py"))
    tdir = tempfile.mkdtemp(prefix="helm_table_")
    table = helm_table.ensure_table(tdir)
    h = helm_mod.Helm(table)
    n = EOS_POINTS
    g = torch.Generator(device="cpu").manual_seed(20261203)
    u = lambda lo, hi: lo + (hi - lo) * torch.rand(n, dtype=torch.float64, generator=g)
    rho_h = torch.pow(10.0, u(-2.0, 9.0))
    T_h = torch.pow(10.0, u(4.0, 9.0))
    abar_h = u(12.0, 16.0)
    guess_h = T_h * torch.pow(10.0, u(-0.5, 0.5))
    dev = lambda t: t.cuda()
    rho, T, abar, guess = dev(rho_h), dev(T_h), dev(abar_h), dev(guess_h)
    zbar = abar / 2
    p, e, cs = (torch.empty(n, dtype=torch.float64, device="cuda") for _ in range(3))
    status = torch.empty(n, dtype=torch.int32, device="cuda")
    Tout = torch.empty_like(T)
    iters = torch.empty(n, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream

    def fwd():
        h.eos_device(rho, T, abar, zbar, p, e, cs, status, stream=stream)

    def inv():
        Tout.copy_(guess)
        h.invert_T_device(rho, e_target, abar, zbar, Tout, status_i, iters=iters, stream=stream)

    def timed(fn):
        for _ in range(warmup):
            fn()
        ts = []
        for _ in range(steps):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            fn()
            b.record()
            b.synchronize()
            ts.append(a.elapsed_time(b))
        return statistics.median(ts)

    ms_f = timed(fwd)
    bad_f = int((status != 0).sum())
    e_target = e.clone()
    status_i = torch.empty_like(status)
    # the Newton launch starts from the guess each time (the copy is timed with it)
    ms_i = timed(inv)
    bad_i = int((status_i != 0).sum())
    it = iters.double()
    # accuracy against the oracle restatement on a sample
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import helm_oracle
    tab = helm_oracle.Table(table)
    idx = torch.arange(0, n, n // 4096)
    w = helm_oracle.eos(tab, rho_h[idx].numpy(), T_h[idx].numpy(), abar_h[idx].numpy(), abar_h[idx].numpy() / 2)
    err = {}
    for k, t in (("p", p), ("e", e), ("cs", cs)):
        got = t[idx.cuda()].cpu().numpy()
        err[k] = float((abs(got - w[k]) / abs(w[k])).max())
    Trel = float(((Tout - T).abs() / T).max())
    flops = EOS_FLOPS_PER_POINT * n / (ms_f * 1e-3) / 1e12
    res = {
        "points": n, "forward_ms": ms_f, "forward_points_per_s": n / (ms_f * 1e-3),
        "inverse_ms": ms_i, "inverse_points_per_s": n / (ms_i * 1e-3),
        "newton_iters_mean": float(it.mean()), "newton_iters_max": int(it.max()),
        "bad_status_forward": bad_f, "bad_status_inverse": bad_i,
        "forward_max_rel_err_vs_oracle": err, "inverse_max_rel_err_T_vs_true": Trel,
        "forward_fp64_tflops": flops, "fp64_peak_tflops": FP64_NOMINAL_TFLOPS, "fp64_peak_source": "nominal",
        "forward_fp64_frac": flops / FP64_NOMINAL_TFLOPS,
        "forward_io_gbs": EOS_IO_BYTES * n / (ms_f * 1e-3) / 1e9,
        "table": "synthetic closed-form free energy in the reference's table format (the real table is not shipped)",
    }
    if cpu_sample:
        exe = os.path.join(ROOT, "oracle", "_ref", "helm_harness")
        if os.path.exists(exe):
            import numpy as np
            m = 1 << 18
            with open(os.path.join(tdir, "in.bin"), "wb") as fh:
                np.array([m], np.int64).tofile(fh)
                np.stack([rho_h[:m].numpy(), T_h[:m].numpy(), abar_h[:m].numpy(), abar_h[:m].numpy() / 2],
                         1).tofile(fh)
            with open(os.path.join(tdir, "one.bin"), "wb") as fh:
                np.array([1], np.int64).tofile(fh)
                np.array([1e6, 1e6, 12.0, 6.0]).tofile(fh)
            t0 = time.time()
            subprocess.run([exe, "fwd", "in.bin", "out.bin"], cwd=tdir, check=True)
            t1 = time.time()
            subprocess.run([exe, "fwd", "one.bin", "out1.bin"], cwd=tdir, check=True)
            t2 = time.time()
            sec = max((t1 - t0) - (t2 - t1), 1e-9)  # minus process start + table read
            res["cpu_baseline"] = {"value": m / sec, "unit": "EOS points/s", "cores": 1, "kind": "reference",
                                   "sample": "reference helmholtz_eos (oracle/_ref/helm_harness, scalar) on the "
                                             "first 2^18 points of the same workload"}
    h.close()
    import shutil
    shutil.rmtree(tdir, ignore_errors=True)
    return res


def leaf_mask(t, nx):
    """[bricks, nx, nx, nx] True where the interior cell is not covered by a child."""
    n = t["level"].size
    half = nx // 2
    idx = np.arange(nx) // half
    oc = idx[None, None, :] | (idx[None, :, None] << 1) | (idx[:, None, None] << 2)  # [k][j][i]
    return ((t["child_mask"][:, None, None, None] >> oc[None]) & 1) == 0


def state_errors(fin, ref, bw):
    """Relative L2 of phi and relative L1 of density and energy over all bricks."""
    if not (np.array_equal(fin["level"], ref["level"]) and np.array_equal(fin["loc"], ref["loc"])):
        return {"comparable": False, "why": "the forms regridded to different trees"}
    sl = (slice(None), slice(bw, -bw), slice(bw, -bw), slice(bw, -bw))
    r0, r1 = fin["U"][:, 0][sl], ref["U"][:, 0][sl]
    e0, e1 = fin["U"][:, 4][sl], ref["U"][:, 4][sl]
    p0, p1 = fin["phi"][:, 1:-1, 1:-1, 1:-1], ref["phi"][:, 1:-1, 1:-1, 1:-1]
    return {"comparable": True,
            "phi_rel_l2": float(np.linalg.norm(p0 - p1) / np.linalg.norm(p1)),
            "rho_rel_l1": float(np.abs(r0 - r1).sum() / np.abs(r1).sum()),
            "energy_rel_l1": float(np.abs(e0 - e1).sum() / np.abs(e1).sum())}


def poisson_precision_check(amr, ini, rel_tol=1e-10):
    """Poisson solve of the initial star to L1 residual rel_tol x L1(4 pi G rho)
    in the FP64 graph form and the mixed form; potential error of the mixed
    form against FP64."""
    out = {}
    phis = {}
    for name, prec in (("fp64", amr.PREC_FP64), ("mixed", amr.PREC_MIXED)):
        a = amr.AMR(physics=amr.PHYSICS_EULER_GRAVITY, max_refine_level=LEVELS, grid_dim=0.5, z_reflect=0,
                    max_bricks=8192, precision=prec)
        t, U = ini.build_tree(a, "polytrope", 1.0e-6, 0.5, 0, LEVELS, device=True)
        bw, nx = a.bw, a.nx
        tt = a.get_tree()
        rho = U[:, 0, bw:-bw, bw:-bw, bw:-bw]
        l1_src = float((4.0 * np.pi * a.cfg.grav_g * np.abs(rho) * leaf_mask(tt, nx)).sum(axis=(1, 2, 3))
                       @ (tt["h"] ** 3))
        tol = rel_tol * l1_src
        t0 = time.time()
        err, cycles = a.graph_solve(tol, 100000)
        a.synchronize()
        out[name] = {"l1_residual": err, "tol": tol, "vcycles": cycles, "seconds": time.time() - t0}
        phis[name] = a.download_poisson()[0][:, 1:-1, 1:-1, 1:-1]
        a.close()
    p64, p32 = phis["fp64"], phis["mixed"]
    out["phi_rel_l2_mixed_vs_fp64"] = float(np.linalg.norm(p32 - p64) / np.linalg.norm(p64))
    out["relative_residual"] = rel_tol
    return out


FUSED_BYTES_PER_BRICK = 8 * NF * 3 * NX ** 3  # read U, U0, write U (interiors), FP64


def run_batched_substep(amr, ini, torch, steps, warmup, levels=5):
    """Uneven-brick KT substep on the synthetic random-field octree: one
    persistent fused launch per substep (ghost zones, limiter, flux,
    coarse-fine correction, RK combination), FP64 and FP32 flux, against the
    one-launch-per-step substep; an autotuning pass over the resident blocks
    per SM."""
    F = ini.random_field()
    thr = float(np.percentile(F, 90))
    out = {"levels": levels + 1, "threshold": "90th percentile of the density field", "seed": 20261203}
    ctxs = {}
    for name, prec in (("fp64", amr.PREC_FP64), ("fp32_flux", amr.PREC_MIXED)):
        a = amr.AMR(physics=amr.PHYSICS_EULER, max_refine_level=levels, grid_dim=0.5, z_reflect=0,
                    max_bricks=40000, precision=prec)
        t0 = time.time()
        t, _ = ini.build_tree(a, "random", thr, 0.5, 0, levels, device=True)
        out.setdefault("build_s", round(time.time() - t0, 1))
        out["bricks"] = a.nbricks
        out["per_level"] = np.bincount(t["level"]).tolist()
        out["leaf_cells"] = int(a.get_zone_cnt())
        ctxs[name] = a
    a64 = ctxs["fp64"]
    dt = a64.max_dt()
    stream = torch.cuda.ExternalStream(a64.stream_handle())

    def time_substeps(a, fn, k):
        for _ in range(warmup):
            fn(a)
        ts = []
        for _ in range(k):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            fn(a)
            e1.record(stream)
            e1.synchronize()
            ts.append(e0.elapsed_time(e1))
        return statistics.median(ts)

    # one-launch-per-step substep (ghost fill by level, flux, reflux, update)
    a64.store()
    plain_ms = time_substeps(a64, lambda a: a.sub_step(dt, 0.25), steps)
    # autotune the fused launch: resident blocks per SM
    tune = {}
    for bps in (1, 2, 0):
        tune[bps] = time_substeps(a64, lambda a: a.fused_sub_step(dt, 0.25, bps), steps)
    best = min(tune, key=tune.get)
    # fused kernel alone (profiled class: CUDA events around the launch)
    a64.profile(True)
    a64.profile_reset()
    for _ in range(steps):
        a64.fused_sub_step(dt, 0.25, best)
    a64.synchronize()
    pr = a64.profile_get()["fused_substep"]
    a64.profile(False)
    kms = pr["ms"] / pr["launches"]
    nb = out["bricks"]
    peak, peak_kind = peaks()
    achieved = FUSED_BYTES_PER_BRICK * nb / (kms * 1e-3) / 1e9
    # FP32 flux: speed and error against FP64 after one substep from the same state
    a32 = ctxs["fp32_flux"]
    a32.store()
    f32_ms = time_substeps(a32, lambda a: a.fused_sub_step(dt, 0.25, best), steps)
    errs = {}
    b64, b32 = a64, a32
    U0 = b64.download_state()
    b32.upload_state(U0)
    b32.store()
    b64.store()
    b64.fused_sub_step(dt, 1.0, best)
    b32.fused_sub_step(dt, 1.0, best)
    u64 = b64.download_state()[:, :, 2:-2, 2:-2, 2:-2]
    u32 = b32.download_state()[:, :, 2:-2, 2:-2, 2:-2]
    for f, nm in enumerate(("rho", "sx", "sy", "sz", "et", "tau")):
        errs[nm] = float(np.abs(u32[:, f] - u64[:, f]).sum() / max(np.abs(u64[:, f]).sum(), 1e-300))
    cells = nb * NX ** 3
    out.update({
        "dt": dt, "plain_substep_ms": plain_ms, "fused_substep_ms": tune[best], "fused_fp32_flux_substep_ms": f32_ms,
        "speedup_vs_plain": plain_ms / tune[best],
        "brick_cell_updates_per_s": cells / (tune[best] * 1e-3),
        "leaf_cell_updates_per_s": out["leaf_cells"] / (tune[best] * 1e-3),
        "autotune_ms_by_blocks_per_sm": {str(k): v for k, v in tune.items()}, "autotune_best": best,
        "roofline": {"bound": "hbm", "kernel": "k_substep_fused", "achieved": achieved, "peak": peak,
                     "unit": "GB/s", "frac": achieved / peak, "peak_source": peak_kind,
                     "algorithmic_bytes_per_launch": FUSED_BYTES_PER_BRICK * nb, "ms_per_launch": kms},
        "fp32_flux_rel_l1_vs_fp64": errs,
        "l2": "state (%.1f GB with the RK store) larger than L2, no flush" % (2 * nb * NF * (NX + 4) ** 3 * 8 / 1e9),
    })
    for a in ctxs.values():
        a.close()
    return out


def ztwd_context(amr, ini, helm_mod, table, levels, prec, persistent, nx=ZT_NX, max_bricks=4096):
    """A ZTWD binary context on the 5-level tree of the reference's two-polytrope
    initial data (binary/initialize.cpp), EOS units of Binary::set_units."""
    P = ini.binary_params()
    h = helm_mod.Helm(table)
    h.set_cgs_units(P["cm"], P["g"], P["s"], 1.0)
    a = amr.AMR(physics=amr.PHYSICS_ZTWD, nf=13, bw=3, nx=nx, reconstruction=amr.RECON_PPM, grid_dim=1.0,
                z_reflect=1, mirror_refine_y=1, max_refine_level=levels, rho_floor=ini.BINARY["rho_floor"], cfl=0.3,
                maxdtinc=1.25, max_bricks=max_bricks, precision=prec, persistent_solve=persistent)
    a.ztwd_set_eos(h)
    a.ztwd_set_frame(P["omega"], P["omega"], 0.0, 0.0)
    a.init()
    U = ini.evaluate("binary", a.get_tree(), a.bw, a.nx, 1.0, 1, levels, ghosts=False)
    thr = float(U[:, 0].max()) / DYNAMIC_RANGE  # min_refine_density from the root's first state
    ini.build_tree(a, "binary", thr, 1.0, 1, levels, device=True, ghosts=False)
    return a


def run_ztwd(amr, ini, torch, steps, warmup, cpu_sample, total=ZT_STEPS_TOTAL, nx=ZT_NX):
    """The 5-level ZTWD binary (q = 0.7, co-rotating frame, Helmholtz EOS):
    BinaryDriver steps (hydro + multigrid gravity every substep, regrid every
    8 steps) in the plain FP64 form, the persistent FP64 form and the mixed
    persistent form; `total` steps each, steps [warmup, warmup + steps) timed;
    the mixed form's potential, density and angular-momentum errors against
    the FP64 form after `total` steps."""
    helm_table = _load_module("helm_table", os.path.join(PKG, "helm_table.py"))
    helm_mod = _load_module("helm_b200", os.path.join(PKG, "helm.py"))
    tdir = tempfile.mkdtemp(prefix="ztwd_")
    table = helm_table.ensure_table(tdir)
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device="cuda")
    # "mixed" is the headline's form (FP32 multigrid correction, FP64 flux);
    # "mixed_flux32" adds the FP32 reconstruction and KT flux
    forms = (("fp64", amr.PREC_FP64, 0), ("fp64_persistent", amr.PREC_FP64, 2), ("mixed", ZT_PREC(amr), 2),
             ("mixed_flux32", amr.PREC_MIXED, 2))
    res = {"levels": ZT_LEVELS, "nx": nx, "tol_l1": ZT_TOL, "steps_total": total, "timed_steps": steps,
           "binary": dict(ini.BINARY), "regrid": "every 8 steps (binary_driver.cpp:426)"}
    finals = {}
    snaps = {}  # state after steps 1 and 10, for the growth of the mixed form's error
    layouts = {}  # the persistent forms' autotuned solve layouts
    for name, prec, pers in forms:
        a = ztwd_context(amr, ini, helm_mod, table, ZT_LEVELS, prec, pers, nx=nx)
        stream = torch.cuda.ExternalStream(a.stream_handle())
        times, cells, last = [], 0, 0.0
        k0 = a.launch_count()
        for s in range(total):
            dt = a.max_dt()
            if s > 0:
                dt = min(1.25 * last, dt)
            timed = warmup <= s < warmup + steps
            if s == warmup and pers:
                layouts[name] = autotune_solve(a)
            if s == warmup:
                ph0 = a.solve_phases() if pers else None
                w0 = a.solve_phase_waits() if pers else None
                st0 = a.stats()
            if timed:
                with torch.cuda.stream(stream):
                    flush.zero_()
                n = a.get_zone_cnt()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
            last = a.ztwd_step(dt, ZT_TOL, DYNAMIC_RANGE, s)
            if timed:
                e1.record(stream)
                e1.synchronize()
                times.append(e0.elapsed_time(e1))
                cells += n
            if s + 1 in (1, 10) and name in ("fp64", "mixed", "mixed_flux32"):
                t = a.get_tree()
                snaps[(name, s + 1)] = {"U": a.download_state(), "phi": a.download_poisson()[0], "level": t["level"],
                                        "loc": t["loc"], "h": t["h"], "child_mask": t["child_mask"]}
            if s == warmup + steps - 1:
                st1 = a.stats()
                if pers:
                    ph1, w1 = a.solve_phases(), a.solve_phase_waits()
                    phase_split = {
                        "phase_ms_per_step": {k: round((ph1[k]["ms"] - ph0[k]["ms"]) / steps, 3) for k in ph1},
                        "phases_per_step": {k: (ph1[k]["count"] - ph0[k]["count"]) / steps for k in ph1},
                        "barrier_ms_per_step": {k: round((w1[k] - w0[k]) / steps, 3) for k in ph1},
                        "level_sum_ms_per_step": round((w1["level_sum"] - w0["level_sum"]) / steps, 3)}
        t = a.get_tree()
        finals[name] = {"U": a.download_state(), "phi": a.download_poisson()[0], "level": t["level"],
                        "loc": t["loc"], "h": t["h"], "child_mask": t["child_mask"]}
        ms = sum(times) / len(times)
        res[name] = {"ms_per_step": ms, "value": cells / (sum(times) / 1000.0), "bricks": a.nbricks,
                     "leaf_cells": int(a.get_zone_cnt()), "gpu_launches_total": a.launch_count() - k0,
                     "relax_calls_per_step": (st1["relax_calls"] - st0["relax_calls"]) / steps}
        if pers:
            res[name]["persistent"] = phase_split
            res[name]["autotune"] = {k: layouts[name][k] for k in ("layout", "blocks_per_sm", "threads", "blocks")}
        a.close()
    res["metric_unit"] = UNIT
    res["speedup_mixed_vs_fp64"] = res["fp64"]["ms_per_step"] / res["mixed"]["ms_per_step"]
    def zt_errors(f64, f32, steps):
        if not (np.array_equal(f64["level"], f32["level"]) and np.array_equal(f64["loc"], f32["loc"])):
            return {"comparable": False, "steps": steps, "why": "the forms regridded to different trees"}
        bw = 3
        sl = (slice(None), slice(bw, -bw), slice(bw, -bw), slice(bw, -bw))
        leaf = leaf_mask({"level": f64["level"], "child_mask": f64["child_mask"]}, nx)
        vol = (f64["h"] ** 3)[:, None, None, None] * leaf
        r64, r32 = f64["U"][:, 0][sl], f32["U"][:, 0][sl]
        p64, p32 = f64["phi"][:, 1:-1, 1:-1, 1:-1], f32["phi"][:, 1:-1, 1:-1, 1:-1]
        lz64, lz32 = (f64["U"][:, 4][sl] * vol).sum(), (f32["U"][:, 4][sl] * vol).sum()
        return {"comparable": True, "steps": steps,
                "phi_rel_l2": float(np.linalg.norm(p32 - p64) / np.linalg.norm(p64)),
                "rho_rel_l1": float(np.abs(r32 - r64).sum() / np.abs(r64).sum()),
                "lz_total_rel": float(abs(lz32 - lz64) / abs(lz64))}

    res["errors_mixed_vs_fp64"] = zt_errors(finals["fp64"], finals["mixed"], total)
    res["errors_mixed_vs_fp64"]["against"] = "plain FP64 form (parity-tested against the reference's BINARY build)"
    res["errors_mixed_vs_fp64"]["growth"] = [zt_errors(snaps[("fp64", k)], snaps[("mixed", k)], k) for k in (1, 10)]
    res["errors_mixed_flux32_vs_fp64"] = zt_errors(finals["fp64"], finals["mixed_flux32"], total)
    res["errors_mixed_flux32_vs_fp64"]["growth"] = [zt_errors(snaps[("fp64", k)], snaps[("mixed_flux32", k)], k)
                                                    for k in (1, 10)]
    if cpu_sample:
        exe = ztwd_harness(nx)
        if os.path.exists(exe):
            threads = os.cpu_count() or 1
            env = dict(os.environ, OMP_NUM_THREADS=str(threads))
            try:
                r = subprocess.run([exe, "time_ztwd", str(ZT_LEVELS), "2"], cwd=tdir, env=env, capture_output=True,
                                   text=True, timeout=900)
                row = json.loads([x for x in r.stdout.splitlines() if x.startswith("{")][-1])
                sec = row["seconds"][-1]
                res["cpu_baseline"] = {
                    "value": row["leaf_cells"][-1] / sec, "unit": UNIT, "cores": row["threads"],
                    "kind": "reference", "seconds_per_step": sec,
                    "sample": "reference BINARY build (oracle/_ref/%s, %s): its second BinaryDriver step on "
                              "the same 5-level binary (the first solves from the initial phi), %d leaf cells" %
                              (os.path.basename(exe), REF_CXXFLAGS, row["leaf_cells"][-1])}
            except (subprocess.TimeoutExpired, IndexError, ValueError, KeyError):
                res["cpu_baseline"] = None
    import shutil
    shutil.rmtree(tdir, ignore_errors=True)
    return res


def run_error_study(amr, ini, torch, nx=ZT_NX, total=ZT_STEPS_TOTAL, snaps=(1, 10, 100)):
    """What the mixed forms' potential error means: trajectories of the binary
    over `total` steps in
      fp64          the plain FP64 result (persistent FP64 form, bitwise the
                    plain form) at the reference's tolerance ELL_TOLER
      fp64_perturbed the same with the initial density scaled by (1 + 1e-15):
                    how far round-off alone moves the trajectory
      fp64_tight    FP64 with the solve converged 10^4 times further (L1
                    tolerance ELL_TOLER / 1e4): the FP64 form's own solver
                    error at ELL_TOLER is fp64 against this one
      mixed         AMR_PREC_MIXED (FP32 flux and FP32 correction)
      mixed_solve   AMR_PREC_MIXED_SOLVE (FP32 correction, FP64 flux)
    and their potential relative L2 and density relative L1 differences at
    the snapshot steps.  ms per step is the mean device time per step."""
    helm_table = _load_module("helm_table", os.path.join(PKG, "helm_table.py"))
    helm_mod = _load_module("helm_b200", os.path.join(PKG, "helm.py"))
    tdir = tempfile.mkdtemp(prefix="ztwd_err_")
    table = helm_table.ensure_table(tdir)
    runs = (("fp64", amr.PREC_FP64, ZT_TOL, False), ("fp64_perturbed", amr.PREC_FP64, ZT_TOL, True),
            ("fp64_tight", amr.PREC_FP64, ZT_TOL * 1e-4, False), ("mixed", amr.PREC_MIXED, ZT_TOL, False),
            ("mixed_solve", amr.PREC_MIXED_SOLVE, ZT_TOL, False))
    out = {"nx": nx, "steps": total, "tol_l1": ZT_TOL, "runs": {}}
    shots = {}
    for name, prec, tol, perturb in runs:
        a = ztwd_context(amr, ini, helm_mod, table, ZT_LEVELS, prec, 2, nx=nx)
        if perturb:
            U = a.download_state()
            U[:, 0] *= 1.0 + 1e-15
            a.upload_state(U)
        stream = torch.cuda.ExternalStream(a.stream_handle())
        last, ms = 0.0, []
        for s in range(total):
            dt = a.max_dt()
            if s > 0:
                dt = min(1.25 * last, dt)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            last = a.ztwd_step(dt, tol, DYNAMIC_RANGE, s)
            e1.record(stream)
            e1.synchronize()
            ms.append(e0.elapsed_time(e1))
            if s + 1 in snaps:
                t = a.get_tree()
                b = a.bw
                shots[(name, s + 1)] = {"rho": a.download_state()[:, 0, b:-b, b:-b, b:-b].copy(),
                                        "phi": a.download_poisson()[0][:, 1:-1, 1:-1, 1:-1].copy(),
                                        "level": t["level"], "loc": t["loc"]}
        out["runs"][name] = {"tol_l1": tol, "ms_per_step": statistics.mean(ms[3:]) if total > 3 else None,
                             "bricks": a.nbricks}
        a.close()
    import shutil
    shutil.rmtree(tdir, ignore_errors=True)

    def diff(x, y):
        if not (np.array_equal(x["level"], y["level"]) and np.array_equal(x["loc"], y["loc"])):
            return None
        return {"phi_rel_l2": float(np.linalg.norm(x["phi"] - y["phi"]) / np.linalg.norm(y["phi"])),
                "rho_rel_l1": float(np.abs(x["rho"] - y["rho"]).sum() / np.abs(y["rho"]).sum())}

    pairs = {"mixed_vs_fp64": ("mixed", "fp64"), "mixed_solve_vs_fp64": ("mixed_solve", "fp64"),
             "fp64_vs_fp64_tight": ("fp64", "fp64_tight"), "mixed_vs_fp64_tight": ("mixed", "fp64_tight"),
             "fp64_perturbed_vs_fp64": ("fp64_perturbed", "fp64")}
    out["differences"] = {k: {str(s): diff(shots[(x, s)], shots[(y, s)]) for s in snaps}
                          for k, (x, y) in pairs.items()}
    return out


def autotune_solve(a):
    """Runs the persistent solve's autotuner on a representative solve of the
    binary -- from the potential of the step's start (phi0) to the current
    density, as the third substep solves -- and keeps the fastest layout;
    returns the trials and the choice."""
    P = a.download_poisson()
    Pk = P.copy()
    Pk[0] = P[1]
    a.upload_poisson(Pk)
    ms, best = a.autotune_solve(ZT_TOL, reps=2)
    a.upload_poisson(P)
    lay = a.solve_layout()
    return {"trials_ms": [None if m is None else round(m, 4) for m in ms], "best_trial": best,
            "layout": lay[0], "blocks_per_sm": lay[1], "threads": lay[2], "blocks": lay[3], "layouts": lay[4],
            "trial": "layout = trial // 3, blocks per SM = (1, 2, all)[trial % 3]; one persistent solve from the "
                     "step's starting potential, mean of 2 after 1 untimed"}


def run_ztwd_headline(amr, ini, args, world, local, torch, dist):
    """The headline: W untimed then K timed BinaryDriver steps of the 5-level
    ZTWD binary in the mixed persistent form (L2 flushed between timed steps,
    outside the timed interval); then, on a second context that replays the
    same W warm-up steps, the same K steps end to end through the C ABI with
    the state copied from and to pinned host memory every step."""
    helm_table = _load_module("helm_table", os.path.join(PKG, "helm_table.py"))
    helm_mod = _load_module("helm_b200", os.path.join(PKG, "helm.py"))
    tdir = tempfile.mkdtemp(prefix="ztwd_head_")
    table = helm_table.ensure_table(tdir)
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device="cuda")

    def barrier():
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()

    tuned = {}

    def warmed():
        """A fresh context of the workload after the W warm-up steps, and its
        step function (dt from max_dt with the MAXDTINC clamp); the first
        one runs the solve autotuner after its warm-up, the second takes its
        choice."""
        a = ztwd_context(amr, ini, helm_mod, table, ZT_LEVELS, ZT_PREC(amr), 2, nx=args.zt_nx)
        state = {"step": 0, "last": 0.0}

        def one_step():
            s = state["step"]
            dt = a.max_dt()
            if s > 0:
                dt = min(1.25 * state["last"], dt)
            state["last"] = a.ztwd_step(dt, ZT_TOL, DYNAMIC_RANGE, s)
            state["step"] = s + 1

        for _ in range(args.warmup):
            one_step()
        if not tuned and not args.no_autotune:
            tuned.update(autotune_solve(a))
        elif tuned:
            a.set_solve_layout(tuned["layout"], tuned["blocks_per_sm"])
        return a, one_step

    a, one_step = warmed()
    stream = torch.cuda.ExternalStream(a.stream_handle())
    ph0, w0, tot0 = a.solve_phases(), a.solve_phase_waits(), a.solve_totals()
    rp0 = a.relax_passes()
    rs0 = a.solve_relax_split()
    rl0 = a.solve_relax_level_ms()
    k0 = a.launch_count()
    sampler = ClockSampler(local)
    barrier()
    sampler.start()
    times, cells = [], 0
    for _ in range(args.steps):
        with torch.cuda.stream(stream):
            flush.zero_()
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        n = a.get_zone_cnt()
        torch.cuda.nvtx.range_push("timed_step")
        ev0.record(stream)
        one_step()
        ev1.record(stream)
        torch.cuda.nvtx.range_pop()
        ev1.synchronize()
        times.append(ev0.elapsed_time(ev1))
        cells += n
    barrier()
    res = {"clocks": sampler.stop(), "gpu_launches": a.launch_count() - k0, "bricks": a.nbricks, "autotune": tuned,
           "ms_steps": [round(x, 3) for x in times]}
    ph1, w1, tot1 = a.solve_phases(), a.solve_phase_waits(), a.solve_totals()
    launches = max(tot1[1] - tot0[1], 1)
    d = {k: {"ms": ph1[k]["ms"] - ph0[k]["ms"], "count": ph1[k]["count"] - ph0[k]["count"],
             "bytes": ph1[k]["bytes"] - ph0[k]["bytes"]} for k in ph1}
    res["persistent"] = {
        "ms_per_launch": (tot1[0] - tot0[0]) / launches, "launches": launches,
        "bytes_per_launch": sum(v["bytes"] for v in d.values()) / launches,
        "phase_ms_per_step": {k: round(v["ms"] / args.steps, 4) for k, v in d.items()},
        "phases_per_step": {k: v["count"] / args.steps for k, v in d.items()},
        "barrier_ms_per_step": {k: round((w1[k] - w0[k]) / args.steps, 4) for k in ph1},
        "level_sum_ms_per_step": round((w1["level_sum"] - w0["level_sum"]) / args.steps, 4)}
    rs1 = a.solve_relax_split()
    res["persistent"]["relax_split_per_step"] = {k: round((rs1[k] - rs0[k]) / args.steps, 3) for k in rs1}
    lv = a.get_tree()["level"]
    nl = int(lv.max()) + 1
    res["persistent"]["bricks_by_level"] = [int((lv == l).sum()) for l in range(nl)]
    res["persistent"]["relax_passes_per_step_by_level"] = [
        round(float(x) / args.steps, 1) for x in (a.relax_passes() - rp0)[:nl]]
    res["persistent"]["relax_ms_per_step_by_level"] = [
        round(float(x) / args.steps, 3) for x in (a.solve_relax_level_ms() - rl0)[:nl]]
    a.close()
    t = aggregate(sum(times), cells, world, dist)
    res["ms_total"], res["cells"] = t
    res["value"] = res["cells"] / (res["ms_total"] / 1000.0)
    res["ms_per_step"] = res["ms_total"] / args.steps
    res["leaf_cells_per_step"] = cells / args.steps
    # end to end through the public API, host buffers, the same K steps
    a, one_step = warmed()
    stream = torch.cuda.ExternalStream(a.stream_handle())
    cap = 3 * a.nbricks * a.nf * a.gnx ** 3  # room for the tree to grow during the K steps
    hbuf = torch.empty(cap, dtype=torch.float64, pin_memory=True)
    U = a.download_state()
    hbuf[:U.size].copy_(torch.from_numpy(U.reshape(-1)))
    ptr = ctypes.cast(hbuf.data_ptr(), ctypes.POINTER(ctypes.c_double))
    barrier()
    e_times, e_cells, h2d, d2h = [], 0, 0, 0
    for _ in range(args.steps):
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        n_in = a.nbricks * a.nf * a.gnx ** 3
        e_cells += a.get_zone_cnt()
        ev0.record(stream)
        a._check(a.lib.amr_upload_state(a.ctx, ptr))
        one_step()
        n_out = a.nbricks * a.nf * a.gnx ** 3
        if n_out > cap:
            raise RuntimeError("e2e host buffer too small for the regridded tree")
        a._check(a.lib.amr_download_state(a.ctx, ptr))
        ev1.record(stream)
        ev1.synchronize()
        e_times.append(ev0.elapsed_time(ev1))
        h2d += 8 * n_in
        d2h += 8 * n_out
    barrier()
    a.close()
    et = aggregate(sum(e_times), e_cells, world, dist)
    res["e2e"] = {"value": et[1] / (et[0] / 1000.0), "unit": UNIT,
                  "h2d_bytes_per_step": h2d // args.steps, "d2h_bytes_per_step": d2h // args.steps,
                  "ms_per_step": et[0] / args.steps, "ms_steps": [round(x, 3) for x in e_times]}
    import shutil
    shutil.rmtree(tdir, ignore_errors=True)
    return res


def run_case(case, nx=ZT_NX, layout=None):
    """One small run of a single kernel family, for profiler captures:
    solve_L3      one Poisson solve (L1 tol 1e-6) of the 3-level star, mixed
                  persistent form (k_solve_persistent)
    substep_L4    two fused substeps on the 5-level random-field octree
                  (k_substep_fused, FP64)
    eos_1M        2^20 points, forward and inverse Helmholtz EOS
    ztwd_L5       two BinaryDriver steps of the 5-level ZTWD binary, plain FP64
                  (k_zt_flux, k_zt_add_difs, k_zt_max_dt, ... as separate launches)
    ztwd_mixed_L5 four steps of the same binary in the headline's mixed
                  persistent form (FP32 correction, FP64 hydro), the last two
                  inside the NVTX range timed_step
    single_fp64_L4, single_mixed_L4
                  the 4-level single star, plain FP64 / mixed persistent form:
                  3 warm-up steps, then 2 steps inside timed_step"""
    import torch
    amr, ini = load_amr()
    if case == "solve_L3":
        a = amr.AMR(physics=amr.PHYSICS_EULER_GRAVITY, max_refine_level=3, grid_dim=0.5, z_reflect=0,
                    max_bricks=2048, precision=amr.PREC_MIXED, persistent_solve=2)
        ini.build_tree(a, "polytrope", 1.0e-6, 0.5, 0, 3, device=True)
        err, cyc = a.graph_solve(1e-6, 1000)
        a.synchronize()
        print(json.dumps({"case": case, "bricks": a.nbricks, "vcycles": cyc, "l1": err}))
        a.close()
    elif case == "substep_L4":
        F = ini.random_field()
        a = amr.AMR(physics=amr.PHYSICS_EULER, max_refine_level=4, grid_dim=0.5, z_reflect=0, max_bricks=8192)
        ini.build_tree(a, "random", float(np.percentile(F, 90)), 0.5, 0, 4, device=True)
        dt = a.max_dt()
        a.store()
        for beta in (1.0, 0.25):
            a.fused_sub_step(dt, beta)
        a.synchronize()
        print(json.dumps({"case": case, "bricks": a.nbricks, "dt": dt}))
        a.close()
    elif case == "eos_1M":
        helm_table = _load_module("helm_table", os.path.join(PKG, "helm_table.py"))
        helm_mod = _load_module("helm_b200", os.path.join(PKG, "helm.py"))
        tdir = tempfile.mkdtemp(prefix="helm_table_")
        h = helm_mod.Helm(helm_table.ensure_table(tdir))
        n = 1 << 20
        g = torch.Generator(device="cpu").manual_seed(5)
        rho = torch.pow(10.0, -2 + 11 * torch.rand(n, dtype=torch.float64, generator=g)).cuda()
        T = torch.pow(10.0, 4 + 5 * torch.rand(n, dtype=torch.float64, generator=g)).cuda()
        abar = (12 + 4 * torch.rand(n, dtype=torch.float64, generator=g)).cuda()
        zbar = abar / 2
        p, e, cs = (torch.empty_like(rho) for _ in range(3))
        st = torch.empty(n, dtype=torch.int32, device="cuda")
        h.eos_device(rho, T, abar, zbar, p, e, cs, st)
        Tg = T * 1.5
        h.invert_T_device(rho, e, abar, zbar, Tg, st)
        torch.cuda.synchronize()
        print(json.dumps({"case": case, "points": n, "bad": int((st != 0).sum())}))
        h.close()
        import shutil
        shutil.rmtree(tdir, ignore_errors=True)
    elif case in ("single_fp64_L4", "single_mixed_L4"):
        # the single star's timed steps (NVTX range timed_step), 3 warm-up
        import types
        form = "mixed" if case == "single_mixed_L4" else "fp64"
        r = run_form(amr, ini, form, types.SimpleNamespace(steps=2, warmup=3), 1, 0, torch, None)
        print(json.dumps({"case": case, "bricks": r["bricks"], "ms_per_step": r["ms_per_step"],
                          "gpu_launches": r["gpu_launches"]}))
    elif case in ("ztwd_L5", "ztwd_mixed_L5"):
        helm_table = _load_module("helm_table", os.path.join(PKG, "helm_table.py"))
        helm_mod = _load_module("helm_b200", os.path.join(PKG, "helm.py"))
        tdir = tempfile.mkdtemp(prefix="ztwd_")
        mixed = case == "ztwd_mixed_L5"
        # a pool of 640 bricks (the tree has about 320): a few GB on the
        # device, so that a profiler's save and restore stay small
        a = ztwd_context(amr, ini, helm_mod, helm_table.ensure_table(tdir), ZT_LEVELS,
                         ZT_PREC(amr) if mixed else amr.PREC_FP64, 2 if mixed else 0, nx=nx, max_bricks=640)
        if mixed and layout is not None:
            a.set_solve_layout(*layout)
        last = 0.0
        nsteps = 4 if mixed else 2
        solve = {}
        for s in range(nsteps):
            dt = a.max_dt()
            dt = min(1.25 * last, dt) if s else dt
            if mixed and s == 2:
                tot0, ph0 = a.solve_totals(), a.solve_phases()
            if mixed and s >= 2:
                torch.cuda.nvtx.range_push("timed_step")
            last = a.ztwd_step(dt, ZT_TOL, DYNAMIC_RANGE, s)
            if mixed and s >= 2:
                a.synchronize()
                torch.cuda.nvtx.range_pop()
        a.synchronize()
        if mixed:
            # the persistent solve launches inside the timed_step ranges:
            # algorithmic bytes per launch, to set beside a profiler's DRAM bytes
            tot1, ph1 = a.solve_totals(), a.solve_phases()
            n = max(tot1[1] - tot0[1], 1)
            solve = {"solve_launches": tot1[1] - tot0[1], "solve_ms_per_launch": (tot1[0] - tot0[0]) / n,
                     "solve_algorithmic_bytes_per_launch":
                         sum(ph1[k]["bytes"] - ph0[k]["bytes"] for k in ph1) / n}
        print(json.dumps({"case": case, "bricks": a.nbricks, "dt": last, **solve}))
        a.close()
        import shutil
        shutil.rmtree(tdir, ignore_errors=True)
    else:
        raise SystemExit("unknown case " + case)
    return 0


def roofline_persistent(res, traffic=None):
    """Roofline of the persistent solve kernel, the step's dominant kernel:
    algorithmic bytes per launch (the arrays each phase must read and write
    once, summed by the kernel over its phases) over the launch's duration
    from CUDA events on the launching stream; `traffic` the measured DRAM
    bytes per launch where a capture of this workload exists."""
    p = res["persistent"]
    peak, peak_kind = peaks()
    achieved = p["bytes_per_launch"] / (p["ms_per_launch"] * 1e-3) / 1e9
    return {"bound": "hbm", "kernel": "k_solve_persistent", "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak, "peak_source": peak_kind, "traffic": traffic,
            "algorithmic_bytes_per_launch": p["bytes_per_launch"], "ms_per_launch": p["ms_per_launch"],
            "phase_ms_per_step": p["phase_ms_per_step"], "phases_per_step": p["phases_per_step"],
            "barrier_ms_per_step": p.get("barrier_ms_per_step"),
            "level_sum_ms_per_step": p.get("level_sum_ms_per_step"),
            "bricks_by_level": p.get("bricks_by_level"),
            "relax_passes_per_step_by_level": p.get("relax_passes_per_step_by_level"),
            "relax_split_per_step": p.get("relax_split_per_step"),
            "relax_ms_per_step_by_level": p.get("relax_ms_per_step_by_level"),
            "note": "latency-bound: the reference's V-cycle is a chain of dependent per-level steps "
                    "(%d grid barriers per step here); the relaxation sweeps run in shared memory"
                    % round(sum(p["phases_per_step"].values()))}


def roofline_of(prof):
    known = {k: v for k, v in prof.items() if k in BYTES_PER_BRICK and v["launches"] > 0}
    dom = max(prof.items(), key=lambda kv: kv[1]["ms"])[0]
    peak, peak_kind = peaks()
    name = dom if dom in known else max(known.items(), key=lambda kv: kv[1]["ms"])[0]
    pr = prof[name]
    bytes_per_launch = BYTES_PER_BRICK[name] * pr["units"] / pr["launches"]
    ms_per_launch = pr["ms"] / pr["launches"]
    achieved = bytes_per_launch / (ms_per_launch * 1e-3) / 1e9
    total = sum(x["ms"] for x in prof.values())
    return {"bound": "hbm", "kernel": name, "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak, "peak_source": peak_kind, "traffic": None,
            "algorithmic_bytes_per_launch": bytes_per_launch, "ms_per_launch": ms_per_launch,
            "dominant_class": dom,
            "class_share": {k: round(v["ms"] / max(total, 1e-9), 4) for k, v in prof.items() if v["ms"] > 0}}


def run_single_star(amr, ini, args, world, local, torch, dist):
    """The single star (4 levels, Euler state): mixed persistent form with its
    e2e and kernel-class profile, the plain / graph / persistent FP64 forms,
    the mixed form's errors, a tight Poisson solve, the reference CPU code."""
    head = run_form(amr, ini, "mixed", args, 1, local, torch, dist, e2e=True, profile=True)
    plain = run_form(amr, ini, "fp64", args, 1, local, torch, dist)
    graph64 = run_form(amr, ini, "graph", args, 1, local, torch, dist)
    pers64 = run_form(amr, ini, "persistent", args, 1, local, torch, dist)
    errors = state_errors(head["final"], plain["final"], 2)
    errors["steps"] = args.warmup + args.steps
    errors["against"] = "plain FP64 form (parity-tested against the reference CPU code)"
    cpu = None
    if not args.no_cpu_baseline:
        s = run_reference_steps(LEVELS, os.cpu_count() or 1, 1, 1, timeout=1200)
        if s is not None and s["seconds"]:
            cpu = {"value": sum(s["leaf_cells"]) / sum(s["seconds"]), "unit": UNIT, "cores": s["threads"],
                   "kind": "reference",
                   "sample": "reference CPU code (oracle/_ref): one full RK3 step of this workload after one "
                             "untimed step (which solves from phi = 0), %d bricks, %d V-cycles" %
                             (s["bricks"], s["vcycles"][0])}
    form = lambda r: {"value": r["value"], "ms_per_step": r["ms_per_step"], "gpu_launches": r["gpu_launches"]}
    return {"workload": WORKLOAD, "levels": LEVELS, "bricks": head["bricks"],
            "mixed_persistent": dict(form(head), e2e=head["e2e"], clocks=head["clocks"],
                                     relax_calls_per_step=head["relax_calls_per_step"]),
            "roofline": roofline_persistent(head), "class_roofline": roofline_of(head["profile"]),
            "fp64_plain": form(plain), "fp64_graph": form(graph64), "fp64_persistent": form(pers64),
            "speedup_vs_fp64_plain": plain["ms_per_step"] / head["ms_per_step"],
            "errors_vs_fp64": errors, "poisson_precision": poisson_precision_check(amr, ini), "cpu_baseline": cpu}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=8,
                    help="timed steps (the default 8 covers one regrid cadence of the binary)")
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--zt-nx", type=int, default=ZT_NX, choices=[8, 12],
                    help="interior cells per brick edge of the binary (12: the reference's BINARY build)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-autotune", action="store_true", help="keep the solve's default block layout")
    ap.add_argument("--solve-layout", default=None,
                    help="LAYOUT:BLOCKS_PER_SM of the persistent solve for --case runs (amr_set_solve_layout)")
    ap.add_argument("--no-compare", action="store_true",
                    help="skip the FP64 forms and the 100-step error comparison of the binary")
    ap.add_argument("--sections", action="store_true",
                    help="also run the secondary sections (single star, random-field octree substep, Helmholtz "
                         "EOS) and write them with the binary's details to the --json-out sidecar")
    ap.add_argument("--error-study", action="store_true",
                    help="also run the binary's error study (FP64 at a tight tolerance, round-off perturbation, "
                         "both mixed forms over 100 steps) into the --json-out sidecar")
    ap.add_argument("--json-out", default=None,
                    help="sidecar JSON file: the headline line plus the binary's per-form details and, with "
                         "--sections, the secondary sections")
    ap.add_argument("--case", default=None,
                    choices=["solve_L3", "substep_L4", "eos_1M", "ztwd_L5", "ztwd_mixed_L5", "single_fp64_L4",
                             "single_mixed_L4"],
                    help="run one small case for a profiler capture and exit")
    args = ap.parse_args()
    if args.case:
        return run_case(args.case, args.zt_nx,
                        tuple(int(x) for x in args.solve_layout.split(":")) if args.solve_layout else None)
    if args.impl == "reference":
        return reference_arm(args)

    import torch
    import torch.distributed as dist

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
    amr, ini = load_amr()
    nx = args.zt_nx
    head = run_ztwd_headline(amr, ini, args, world, local, torch, dist)
    ztwd = None
    if rank == 0 and not args.no_compare:
        ztwd = run_ztwd(amr, ini, torch, args.steps, max(args.warmup, 3), not args.no_cpu_baseline, nx=nx)
    sections = {}
    if rank == 0 and args.error_study:
        sections["error_study"] = run_error_study(amr, ini, torch, nx=nx)
    if rank == 0 and args.sections:
        sections["single_star"] = run_single_star(amr, ini, args, world, local, torch, dist)
        sections["batched_substep"] = run_batched_substep(amr, ini, torch, max(args.steps, 3), max(args.warmup, 3))
        sections["helmholtz_eos"] = run_eos(torch, max(args.steps, 3), max(args.warmup, 3),
                                            not args.no_cpu_baseline)
    if rank == 0:
        cpu = ztwd.get("cpu_baseline") if ztwd else None
        traffic = ZT_SOLVE_DRAM_BYTES_PER_LAUNCH.get(nx)
        # the line keeps the roofline's figures; the solve's per-phase and
        # per-level splits go to the sidecar
        roofline = dict(roofline_persistent(head, traffic),
                        traffic_note=None if traffic is None else
                        "ncu DRAM read+write per solve launch on this workload (L2-resident arrays: far "
                        "below the algorithmic bytes)")
        out = {
            "metric": METRIC, "value": head["value"], "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": head["ms_per_step"], "ms_steps": head["ms_steps"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64+f32",
            "data": "synthetic",
            "config": {"workload": ZT_WORKLOAD % nx, "form": ZT_FORM, "levels": ZT_LEVELS, "nx": nx,
                       "bricks": head["bricks"], "leaf_cells_per_step": head["leaf_cells_per_step"],
                       "tol_l1": ZT_TOL, "binary": dict(ini.BINARY),
                       "l2": "flushed between timed steps (256 MiB write)", "parallelism": "replicas",
                       "timed_steps": [args.warmup, args.warmup + args.steps - 1],
                       "regrids_in_timed_steps": sum(1 for q in range(args.warmup, args.warmup + args.steps)
                                                     if q % 8 == 0)},
            "roofline": {k: v for k, v in roofline.items() if k in ROOFLINE_LINE_KEYS},
            "cpu_baseline": cpu, "e2e": head["e2e"],
            "autotune": {k: head["autotune"].get(k) for k in ("layout", "blocks_per_sm", "threads", "blocks",
                                                            "trials_ms")} if head.get("autotune") else None,
            "clocks": head["clocks"], "gpu_launches": head["gpu_launches"],
        }
        if ztwd is not None:
            out["fp64_plain"] = {k: ztwd["fp64"][k] for k in ("value", "ms_per_step", "gpu_launches_total")}
            out["fp64_persistent"] = {k: ztwd["fp64_persistent"][k] for k in ("value", "ms_per_step")}
            out["mixed_100_steps"] = {k: ztwd["mixed"][k] for k in ("value", "ms_per_step")}
            out["speedup_vs_fp64_plain"] = ztwd["fp64"]["ms_per_step"] / head["ms_per_step"]
            # the errors after the 100 steps (their growth after 1 and 10 steps
            # is in the sidecar's ztwd_binary)
            out["errors_vs_fp64"] = {k: v for k, v in ztwd["errors_mixed_vs_fp64"].items() if k != "growth"}
            f32 = ztwd["errors_mixed_flux32_vs_fp64"]
            out["mixed_flux32_100_steps"] = dict({k: ztwd["mixed_flux32"][k] for k in ("value", "ms_per_step")},
                                                 phi_rel_l2=f32.get("phi_rel_l2"), rho_rel_l1=f32.get("rho_rel_l1"))
        line = json.dumps(out)
        print(line)
        if args.json_out:
            side = dict(out, ztwd_binary=ztwd, **sections)
            side["roofline"] = roofline
            with open(args.json_out, "w") as f:
                f.write(json.dumps(side) + "\n")
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
