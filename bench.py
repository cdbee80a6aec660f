#!/usr/bin/env python
"""Benchmark of the time-step engine on the closed-channel DNS workload.

Workload (default): 192 x 192 x 96 closed channel on 4pi x 2pi x 2, nu = 1/180,
unit pressure-gradient forcing, SSP-RK33 with dt = 1e-4, seeded laminar profile
plus Gaussian noise.  One "step" = one SSP-RK33 step (3 right-hand sides +
3 pressure projections) of the whole member.  Metric: grid-point updates/s
(n1 * n2 * n3 points advanced one step per second).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

Under torchrun (N > 1) each rank advances its own member (replicas, weak
scaling); the value is all ranks' updates over the max-over-ranks device time.
`--impl reference` times the CPU restatement of the reference's path (the test
oracle) on the host cores for the same workload.
"""

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(REPO, "boundarylayerdynamics.jl_b200"))

METRIC = "grid-pt updates/s (plain FP64 vs mixed) @192^2x96"
UNIT = "grid-pt updates/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--config", default="dns192")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--error-steps", type=int, default=1000, help="steps of the mixed-vs-FP64 error run")
    ap.add_argument("--cpu-budget", type=float, default=150.0, help="seconds for the reference arm")
    return ap.parse_args()


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


# ------------------------------------------------------------------- clock sampling
class Clocks:
    """Samples nvidia-smi every 200 ms on one GPU while the timed region runs."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index, self.rows, self.proc = index, [], None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                self.rows.append(parts)

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        smax = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({n for r in self.rows for n, v in zip(names, r[5:9]) if v.lower().startswith("active")})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": reasons, "samples": len(self.rows)}


def peaks():
    p = os.path.join(REPO, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# --------------------------------------------------------------------- bytes model
def state_bytes(model):
    """Bytes of one member's spectral state (3 fields) in FP64: the S of B_alg = 8 S per step."""
    return (2 * model.n3 + (model.n3 - 1)) * model.K1 * model.K2 * 16


def phase_bytes(model, prec):
    """Algorithmic bytes per launch of each kernel kind of the advection space (DNS workload)."""
    cs = 8 if prec == "mixed" else 16
    P1, P2, K1, n3 = model.info.adv_p1, model.info.adv_p2, model.K1, model.n3
    layer = P2 * K1 * cs
    cin = 3 * n3 + 3 * (n3 - 1)          # u, v, vort3 on C; w, vort1, vort2 on I
    cout = 2 * n3 + (n3 - 1)             # adv1, adv2 on C; adv3 on I
    S = state_bytes(model)
    return {
        "inv_y": S + cin * layer,                    # read state, write 6 mixed terms
        "adv_x": (cin + cout) * layer,               # read 6 mixed terms, write 3
        "fwd_y": cout * layer + 2 * S,               # read 3 mixed terms and the state, write du
        "project": 2 * S,                            # read the stage inputs, write the projected state
    }


# ------------------------------------------------------------------------ B200 arm
def run_b200(args):
    import ctypes
    import numpy as np
    import torch
    import BoundaryLayerDynamics as BLD
    from BoundaryLayerDynamics import workloads, _capi

    ws, rank, local = dist_env()
    torch.cuda.set_device(local)
    dist = None
    if ws > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    spec = workloads.CONFIGS[args.config]
    dt = spec["dt"]
    W, K = max(3, args.warmup), args.steps
    u0, v0, w0 = workloads.initial_fields(spec, seed=spec["seed"] + rank)
    npts = spec["resolution"][0] * spec["resolution"][1] * spec["resolution"][2]
    lib = _capi.load()

    def barrier():
        if dist is not None:
            t = torch.ones(1, device="cuda")
            dist.all_reduce(t)
        torch.cuda.synchronize()

    def max_over_ranks(x):
        if dist is None:
            return x
        t = torch.tensor([x], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    res = {}
    models = {}
    for prec in ("fp64", "mixed"):
        m = workloads.build(spec, BLD, precision=prec, device=local)
        BLD.initialize(m, vel1=u0, vel2=v0, vel3=w0)
        m.prepare()
        sp = ctypes.c_void_p()
        _capi.check(lib.bld_get_stream(m._h, ctypes.byref(sp)))
        stream = torch.cuda.ExternalStream(sp.value)
        m.step(W, dt)
        pt = _capi.BldPhaseTimes()
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with Clocks(local) as clk:
            e0.record(stream)
            _capi.check(lib.bld_step_async(m._h, K, dt, _capi.SSPRK33))
            e1.record(stream)
            e1.synchronize()
        m.sync()
        ms = max_over_ranks(e0.elapsed_time(e1))
        barrier()
        _capi.check(lib.bld_time_phases(m._h, 20, _capi.SSPRK33, ctypes.byref(pt)))
        res[prec] = dict(ms_total=ms, ms_per_step=ms / K, clocks=clk.summary(),
                         phases=dict(inv_y=pt.inv_y_ms[0], adv_x=pt.x_ms[0], fwd_y=pt.fwd_y_ms[0],
                                     project=pt.project_ms),
                         launches_per_step=pt.launches_per_step)
        models[prec] = (m, stream)

    # mixed-vs-FP64 velocity error after `error_steps` steps from the same initial state
    err = None
    if args.error_steps > 0 and rank == 0:
        fin = {}
        for prec in ("fp64", "mixed"):
            m, _ = models[prec]
            BLD.initialize(m, vel1=u0, vel2=v0, vel3=w0)
            m.evolve(args.error_steps * dt, dt)
            fin[prec] = m.state
        num = sum(np.linalg.norm((fin["mixed"][f] - fin["fp64"][f]).ravel()) ** 2 for f in fin["fp64"])
        den = sum(np.linalg.norm(fin["fp64"][f].ravel()) ** 2 for f in fin["fp64"])
        mf = models["fp64"][0]
        err = {"steps": args.error_steps, "rel_velocity_l2": math.sqrt(num / den),
               "max_abs_divergence_mixed": divergence_max(fin["mixed"], mf, spec),
               "max_abs_divergence_fp64": divergence_max(fin["fp64"], mf, spec)}

    # end to end: every step uploads the state from pinned host memory, runs
    # evolve!(model, dt) (initial projection + rates, one step) and reads the state back
    m, stream = models["fp64"]
    BLD.initialize(m, vel1=u0, vel2=v0, vel3=w0)
    host = {f: torch.empty(m.zeros(f).shape, dtype=torch.complex128, pin_memory=True) for f in BLD.FIELDS}
    st = m.state
    for f in BLD.FIELDS:
        host[f].numpy()[...] = st[f]
    ptrs = [host[f].data_ptr() for f in BLD.FIELDS]
    Ke = max(3, min(K, 20))
    for _ in range(2):
        _capi.check(lib.bld_set_state(m._h, 0, *ptrs))
        _capi.check(lib.bld_evolve(m._h, 0.0, dt, dt, _capi.SSPRK33))
        _capi.check(lib.bld_get_state(m._h, 0, *ptrs))
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(Ke):
        _capi.check(lib.bld_set_state(m._h, 0, *ptrs))
        _capi.check(lib.bld_evolve(m._h, 0.0, dt, dt, _capi.SSPRK33))
        _capi.check(lib.bld_get_state(m._h, 0, *ptrs))
    e1.record(stream)
    e1.synchronize()
    e2e_ms = max_over_ranks(e0.elapsed_time(e1)) / Ke
    sbytes = state_bytes(m)

    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return None

    fp, mx = res["fp64"], res["mixed"]
    value = ws * npts / (fp["ms_per_step"] / 1e3)
    peak, peak_kind = peaks()
    # dominant kernel of the FP64 form by time share per step
    lps = fp["launches_per_step"]
    ph = fp["phases"]
    counts = {"inv_y": 3, "adv_x": 3, "fwd_y": 3, "project": 3}
    share = {k: ph[k] * counts[k] for k in ph}
    dom = max(share, key=share.get)
    pb = phase_bytes(m, "fp64")
    ach = pb[dom] / (ph[dom] * 1e-3) / 1e9
    step_ach = 8 * sbytes / (fp["ms_per_step"] * 1e-3) / 1e9
    out = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": K, "warmup": W,
        "ms_per_step": fp["ms_per_step"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded laminar profile + Gaussian noise)",
        "config": {"workload": "closed-channel DNS 192x192x96, 4pi x 2pi x 2, nu=1/180, SSPRK33 dt=1e-4",
                   "padding": f"{m.info.adv_p1}x{m.info.adv_p2} (reference {m.info.adv_ref_p1}x{m.info.adv_ref_p2})",
                   "l2": "working set (~0.5 GB per step) larger than the 126 MB L2; no flush",
                   "parallelism": f"replicas x{ws}"},
        "mixed": {"value": ws * npts / (mx["ms_per_step"] / 1e3), "ms_per_step": mx["ms_per_step"],
                  "speedup_vs_fp64": fp["ms_per_step"] / mx["ms_per_step"], "dtype": "f32 transforms/products, f64 state+pressure",
                  "error_vs_fp64": err, "clocks": mx["clocks"]},
        "roofline": {"bound": "hbm", "kernel": f"k_{dom}" if dom != "project" else "k_project",
                     "achieved": ach, "peak": peak, "unit": "GB/s", "frac": ach / peak, "peak_kind": peak_kind,
                     "algorithmic_bytes_per_launch": pb[dom], "avg_launch_ms": ph[dom], "traffic": None},
        "roofline_step": {"bound": "hbm", "algorithmic_bytes_per_step": 8 * sbytes, "achieved": step_ach,
                          "peak": peak, "unit": "GB/s", "frac": step_ach / peak},
        "phases_ms_fp64": ph, "phases_ms_mixed": mx["phases"],
        "e2e": {"value": ws * npts / (e2e_ms / 1e3), "unit": UNIT, "ms_per_step": e2e_ms,
                "h2d_bytes_per_step": sbytes, "d2h_bytes_per_step": sbytes,
                "path": "bld_set_state(pinned host) + bld_evolve(one step: projection, rates, SSPRK33 step) + bld_get_state"},
        "gpu_launches": lps * K,
        "clocks": fp["clocks"],
    }
    return out


def divergence_max(state, model, spec):
    """max |D1 u + D2 v + d3 w| over all modes (spectral, FP64 on the host)."""
    import numpy as np
    L1, L2, L3 = spec["size"]
    n3 = model.n3
    k1 = np.arange(model.K1)
    k2 = np.concatenate([np.arange(model.k2max + 1), np.arange(-model.k2max, 0)])
    D1 = (1j * k1 * 2 * math.pi / L1)[None, None, :]
    D2 = (1j * k2 * 2 * math.pi / L2)[None, :, None]
    w = state["vel3"]
    zero = np.zeros_like(w[:1])
    wext = np.concatenate([zero, w, zero])
    dz = L3 / n3
    div = D1 * state["vel1"] + D2 * state["vel2"] + (wext[1:] - wext[:-1]) / dz
    return float(np.abs(div).max())


# ------------------------------------------------------------------ reference arm
def cpu_reference(spec, budget, steps, warmup):
    """Time SSP-RK33 steps of the oracle (the CPU restatement of the reference's path)."""
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import bld_oracle as O
    from BoundaryLayerDynamics import workloads
    cores = os.cpu_count() or 1
    O.set_fft_workers(cores)
    m = workloads.build(spec, O)
    u, v, w = workloads.initial_fields(spec)
    m.initialize(vel1=u, vel2=v, vel3=w)
    st = [m.state[f] for f in m.fields]
    prob = O.ODEProblem(m.rate(), m.projection(), st, (0.0, 1e9))
    step = O.SSPRK33(prob)
    dt = spec["dt"]
    t0 = time.perf_counter()
    step(dt)
    prob._rate(prob.du, prob.u, dt)
    first = time.perf_counter() - t0
    nw = min(max(0, warmup - 1), int(budget / 3 / max(first, 1e-3)))
    for _ in range(nw):
        step(dt)
        prob._rate(prob.du, prob.u, dt)
    nk = max(1, min(steps, int((budget - first * (1 + nw)) / max(first, 1e-3))))
    t0 = time.perf_counter()
    for _ in range(nk):
        step(dt)
        prob._rate(prob.du, prob.u, dt)
    el = time.perf_counter() - t0
    n = spec["resolution"]
    return n[0] * n[1] * n[2] * nk / el, nk, el, cores


def run_reference(args):
    from BoundaryLayerDynamics import workloads
    ws, rank, _ = dist_env()
    if rank != 0:
        return None
    spec = workloads.CONFIGS[args.config]
    value, nk, el, cores = cpu_reference(spec, args.cpu_budget, args.steps, args.warmup)
    sample = f"{nk} full SSPRK33 steps of the {spec['resolution']} workload ({el:.1f} s)"
    return {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
        "steps_timed": nk, "warmup": args.warmup, "ms_per_step": el / nk * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "closed-channel DNS 192x192x96, 4pi x 2pi x 2, nu=1/180, SSPRK33 dt=1e-4"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def main():
    args = parse()
    if args.impl == "reference":
        out = run_reference(args)
    else:
        out = run_b200(args)
        if out is not None and not args.no_cpu_baseline:
            from BoundaryLayerDynamics import workloads
            spec = workloads.CONFIGS[args.config]
            value, nk, el, cores = cpu_reference(spec, 25.0, 3, 1)
            out["cpu_baseline"] = {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                                   "sample": f"{nk} full SSPRK33 steps of the {spec['resolution']} workload ({el:.1f} s)"}
    if out is not None:
        print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
