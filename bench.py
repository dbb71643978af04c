#!/usr/bin/env python
"""Benchmark: cell-updates/s of the self-gravitating hydro step on one B200.

Workload (the reference's single-star configuration): n=1.5 Lane-Emden
polytrope, central density 1, radius 0.25, unit cube [-0.5,0.5]^3, ambient
floor 1e-10, at rest; 4 refinement levels (8^3-cell bricks, BW=2,
minmod-theta 1.3, CFL 0.4, gamma 5/3); regrid every 8 steps at
rho_max/1e6; one RK3 step = 3 substeps, each hydro (KT fluxes, coarse-fine
correction, RK combine, gravity sources) followed by a multigrid Poisson
solve to an L1 error <= 1e-6 (the reference's single-star ELL_TOLER).
A step's work is the leaf cells it advances (GridNode::get_zone_cnt).

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

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "3d-eulerian-amr_b200")

LEVELS = 4
TOL = 1.0e-6
DYNAMIC_RANGE = 1.0e6
METRIC = "cell-updates/s (hydro+gravity step), 1 B200: mixed+batched vs FP64 at set error"
UNIT = "cell-updates/s"
WORKLOAD = "single star: n=1.5 polytrope, 4 levels, RK3 hydro + multigrid gravity (L1 tol 1e-6)"

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
    sources, g++ -O2 -fopenmp) on the same workload: `warm` untimed RK3 steps
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


def reference_arm(args):
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
    sample = ("reference CPU code (oracle/_ref, g++ -O2 -fopenmp, %d threads): %d full RK3 steps after %d "
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


def run_form(amr, ini, form, args, world, local, torch, dist, e2e=False, profile=False):
    """Build the workload and time K steps of one form of our path.

    form: "fp64"  plain FP64, host-orchestrated (reference operation order)
          "graph" FP64, whole RK3 step replayed from a captured CUDA graph with
                  every loop decided on the device (bitwise equal to fp64)
    """
    a = amr.AMR(physics=amr.PHYSICS_EULER_GRAVITY, max_refine_level=LEVELS, grid_dim=0.5, z_reflect=0,
                max_bricks=8192, precision=amr.PREC_FP64)
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
        cells += n_cells
    barrier()
    res["clocks"] = sampler.stop()
    st1 = a.stats()
    res["gpu_launches"] = a.launch_count() - k0
    t = torch.tensor([sum(times), float(cells)], dtype=torch.float64, device="cuda")
    if world > 1:
        dist.all_reduce(t[0:1], op=dist.ReduceOp.MAX)
        dist.all_reduce(t[1:2], op=dist.ReduceOp.SUM)
    res["ms_total"], res["cells"] = float(t[0]), float(t[1])
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
        et = torch.tensor([sum(e_times), float(e_cells)], dtype=torch.float64, device="cuda")
        if world > 1:
            dist.all_reduce(et[0:1], op=dist.ReduceOp.MAX)
            dist.all_reduce(et[1:2], op=dist.ReduceOp.SUM)
        res["e2e"] = {"value": float(et[1]) / (float(et[0]) / 1000.0), "unit": UNIT,
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


def roofline_of(prof):
    known = {k: v for k, v in prof.items() if k in BYTES_PER_BRICK and v["launches"] > 0}
    dom = max(prof.items(), key=lambda kv: kv[1]["ms"])[0]
    peak, peak_kind = peaks()
    name = dom if dom in known else max(known.items(), key=lambda kv: kv[1]["ms"])[0]
    pr = prof[name]
    bytes_per_launch = BYTES_PER_BRICK[name] * pr["units"] / pr["launches"]
    ms_per_launch = pr["ms"] / pr["launches"]
    achieved = bytes_per_launch / (ms_per_launch * 1e-3) / 1e9
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tpath):
        with open(tpath) as f:
            traffic = json.load(f).get(name)
    total = sum(x["ms"] for x in prof.values())
    return {"bound": "hbm", "kernel": name, "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak, "peak_source": peak_kind, "traffic": traffic,
            "algorithmic_bytes_per_launch": bytes_per_launch, "ms_per_launch": ms_per_launch,
            "dominant_class": dom,
            "class_share": {k: round(v["ms"] / max(total, 1e-9), 4) for k, v in prof.items() if v["ms"] > 0}}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--form", default="graph", choices=["fp64", "graph"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-compare", action="store_true", help="skip the plain FP64 comparison run")
    ap.add_argument("--json-out", default=None)
    args = ap.parse_args()
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
    head = run_form(amr, ini, args.form, args, world, local, torch, dist, e2e=True, profile=True)
    plain = None
    if not args.no_compare and args.form != "fp64":
        plain = run_form(amr, ini, "fp64", args, world, local, torch, dist)
    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        s = run_reference_steps(LEVELS, threads, 1, 1, timeout=1200)
        if s is not None and s["seconds"]:
            cpu = {"value": sum(s["leaf_cells"]) / sum(s["seconds"]), "unit": UNIT, "cores": s["threads"],
                   "kind": "reference",
                   "sample": "reference CPU code (oracle/_ref): one full RK3 step of this workload after one "
                             "untimed step (which solves from phi = 0), %d bricks, %d V-cycles" %
                             (s["bricks"], s["vcycles"][0])}
    if rank == 0:
        out = {
            "metric": METRIC, "value": head["value"], "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": head["ms_per_step"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "form": args.form, "levels": LEVELS, "bricks": head["bricks"],
                       "leaf_cells_per_step": head["cells"] / args.steps / world, "tol_l1": TOL,
                       "l2": "flushed between timed steps (256 MiB write)", "parallelism": "replicas"},
            "roofline": roofline_of(head["profile"]), "cpu_baseline": cpu, "e2e": head.get("e2e"),
            "clocks": head["clocks"], "gpu_launches": head["gpu_launches"],
            "relax_calls_per_step": head["relax_calls_per_step"],
            "fp64_plain": None if plain is None else {"value": plain["value"], "ms_per_step": plain["ms_per_step"],
                                                       "gpu_launches": plain["gpu_launches"]},
        }
        line = json.dumps(out)
        print(line)
        if args.json_out:
            with open(args.json_out, "w") as f:
                f.write(line + "\n")
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
