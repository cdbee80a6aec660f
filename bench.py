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

# DRAM bytes per launch (dram__bytes_read.sum + dram__bytes_write.sum) of the x-pass
# kernel the autotuner picks at 192^2x96, from one ncu capture of a step
# (profiles/step_kernels_dns192_fp64.md, profiles/step_kernels_dns192_mixed.md)
TRAFFIC = {("dns192", "k_adv_x2<double, 16, 18, wide>"): (254.4 + 95.5) * 1e6,
           ("dns192", "k_adv_x2<double, 16, 18>"): (254.1 + 95.65) * 1e6,
           ("dns192", "k_adv_x2<float, 16, 18>"): (128.6 + 34.7) * 1e6}
TRAFFIC_SOURCE = "ncu capture of one step in profiles/ (a fixed figure, not measured in this run)"
UNIT = "grid-pt updates/s"
# the workload both arms report under "config" (identical dicts); how the engine
# runs it goes under "config_notes"
CONFIG = {"workload": "closed-channel DNS 192x192x96, 4pi x 2pi x 2, nu=1/180, SSPRK33 dt=1e-4"}
# seconds of the same step loop run untimed before and after the timed steps,
# inside the clock-sampling window (nvidia-smi samples every 200 ms)
CLOCK_WINDOW_S = 2.5


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
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the ensemble, serving, tridiagonal and LES lines (run at N=1 only)")
    ap.add_argument("--only", default="", help="comma list of extras to run (ensemble,serving,tridiag,les64,les512)")
    ap.add_argument("--serve-budget-gb", type=float, default=16.0, help="HBM budget of the served stream")
    ap.add_argument("--serve-seconds", type=float, default=30.0, help="target length of the served stream")
    ap.add_argument("--profile", action="store_true",
                    help="profiler mode: set up the workload, then run --profile-steps steps between "
                         "cudaProfilerStart/Stop (for ncu --profile-from-start off) and exit")
    ap.add_argument("--profile-steps", type=int, default=1)
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"], help="precision of --profile")
    return ap.parse_args()


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


# ------------------------------------------------------------------- clock sampling
class Clocks:
    """Samples nvidia-smi every 200 ms on one GPU over a window that holds the
    timed steps and CLOCK_WINDOW_S seconds of the same step loop on either side."""

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
            # nvidia-smi takes a moment to print its first sample: start the
            # sampled work only once it does (at most 10 s)
            t0 = time.time()
            while not self.rows and self.proc.poll() is None and time.time() - t0 < 10:
                time.sleep(0.05)
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
                "reasons": reasons, "samples": len(self.rows),
                "window": f"the timed steps plus {CLOCK_WINDOW_S} s of the same step loop before and after"}


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

    from BoundaryLayerDynamics import replicas

    def max_over_ranks(x):
        return replicas.reduce_max(x, dist, device="cuda")

    res = {}
    models = {}
    for prec in ("fp64", "mixed"):
        m = workloads.build(spec, BLD, precision=prec, device=local)
        BLD.initialize(m, vel1=u0, vel2=v0, vel3=w0)
        m.prepare()
        sp = ctypes.c_void_p()
        _capi.check(lib.bld_get_stream(m._h, ctypes.byref(sp)))
        stream = torch.cuda.ExternalStream(sp.value)
        # warm-up steps, timed only to size the untimed roll before and after the timed steps
        w0e, w1e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        w0e.record(stream)
        m.step(W, dt)
        w1e.record(stream)
        w1e.synchronize()
        roll = max(1, int(CLOCK_WINDOW_S * 1e3 / max(w0e.elapsed_time(w1e) / W, 1e-3)))
        pt = _capi.BldPhaseTimes()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        # the clock sampler covers the timed steps and the same step loop before
        # and after them, so that it sees the load for several seconds
        with Clocks(local) as clk:
            m.step(roll, dt)
            barrier()
            e0.record(stream)
            _capi.check(lib.bld_step_async(m._h, K, dt, _capi.SSPRK33))
            e1.record(stream)
            e1.synchronize()
            m.sync()
            m.step(roll, dt)
            m.sync()
        ms = max_over_ranks(e0.elapsed_time(e1))
        barrier()
        _capi.check(lib.bld_time_phases(m._h, 20, _capi.SSPRK33, ctypes.byref(pt)))
        res[prec] = dict(ms_total=ms, ms_per_step=ms / K, clocks=clk.summary(), kernels=m.kernels(),
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
    extras = {} if (args.no_extras or ws > 1) else run_extras(args, local)

    fp, mx = res["fp64"], res["mixed"]
    value = ws * npts / (fp["ms_per_step"] / 1e3)
    peak, peak_kind = peaks()
    lps = fp["launches_per_step"]
    ph = fp["phases"]
    names ={"inv_y": "inv_y", "adv_x": "x", "fwd_y": "fwd_y"}

    def kname(kern, phase):
        return kern["projection"] if phase == "project" else kern["advection"][names[phase]]

    def roofline(prec, phases):
        """The dominant kernel against the HBM roofline.  `achieved` divides the
        algorithmic bytes of one SSP-RK stage, B_alg / 3 = 8 S / 3 (the stage reads
        its input and u^n and writes its output; S = the FP64 state), by one launch
        of that kernel (one launch per stage): the fraction of the step's
        compulsory traffic this kernel would need at the device's peak.  The
        kernel's own input and output bytes (intermediates included) divided by
        the same time are kept as `own_bytes_*`."""
        share = {k: phases[k] for k in phases}
        d = max(share, key=share.get)
        mm = models[prec][0]
        b_alg = 8 * state_bytes(mm) / 3
        own = phase_bytes(mm, prec)[d]
        t = phases[d] * 1e-3
        a = b_alg / t / 1e9
        kn = kname(res[prec]["kernels"], d)
        tr = TRAFFIC.get((args.config, kn))
        return {"bound": "hbm", "kernel": kn, "achieved": a, "peak": peak, "unit": "GB/s", "frac": a / peak,
                "peak_kind": peak_kind, "algorithmic_bytes_per_launch": b_alg, "avg_launch_ms": phases[d],
                "own_bytes_per_launch": own, "own_bytes_achieved": own / t / 1e9,
                "own_bytes_frac": own / t / 1e9 / peak,
                "traffic": tr, "traffic_source": (TRAFFIC_SOURCE if tr is not None else None)}
    step_ach = 8 * sbytes / (fp["ms_per_step"] * 1e-3) / 1e9
    out = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": K, "warmup": W,
        "ms_per_step": fp["ms_per_step"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded laminar profile + Gaussian noise)",
        "config": dict(CONFIG),
        "config_notes": {"padding": f"{m.info.adv_p1}x{m.info.adv_p2} (reference {m.info.adv_ref_p1}x{m.info.adv_ref_p2})",
                         "l2": "working set (~0.5 GB per step) larger than the 126 MB L2; no flush",
                         "parallelism": f"replicas x{ws}"},
        "mixed": {"value": ws * npts / (mx["ms_per_step"] / 1e3), "ms_per_step": mx["ms_per_step"],
                  "speedup_vs_fp64": fp["ms_per_step"] / mx["ms_per_step"], "dtype": "f32 transforms/products, f64 state+pressure",
                  "error_vs_fp64": err, "clocks": mx["clocks"]},
        "roofline": roofline("fp64", ph),
        "roofline_mixed": roofline("mixed", mx["phases"]),
        "kernels": {"fp64": fp["kernels"], "mixed": mx["kernels"]},
        "roofline_step": {"bound": "hbm", "algorithmic_bytes_per_step": 8 * sbytes, "achieved": step_ach,
                          "peak": peak, "unit": "GB/s", "frac": step_ach / peak},
        "phases_ms_fp64": ph, "phases_ms_mixed": mx["phases"],
        "e2e": {"value": ws * npts / (e2e_ms / 1e3), "unit": UNIT, "ms_per_step": e2e_ms,
                "h2d_bytes_per_step": sbytes, "d2h_bytes_per_step": sbytes,
                "path": "bld_set_state(pinned host) + bld_evolve(one step: projection, rates, SSPRK33 step) + bld_get_state"},
        "gpu_launches": lps * K,
        "clocks": fp["clocks"],
    }
    out.update(extras)
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


# ------------------------------------------------------------------ extra workloads
def _event_time(stream, fn):
    """Device time (ms) of fn() bracketed by CUDA events on `stream`."""
    import torch
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    fn()
    e1.record(stream)
    e1.synchronize()
    return e0.elapsed_time(e1)


def run_les(name, precisions, steps, warmup, local):
    """Single-member LES at one of the LES sizes: updates/s per precision."""
    import ctypes
    import torch
    import BoundaryLayerDynamics as BLD
    from BoundaryLayerDynamics import workloads, _capi
    spec = workloads.CONFIGS[name]
    u0, v0, w0 = workloads.initial_fields(spec)
    n = spec["resolution"]
    npts = n[0] * n[1] * n[2]
    out = {"workload": f"half-channel LES {n[0]}x{n[1]}x{n[2]}, rough wall z0=1e-4 / free slip, "
                       f"Smagorinsky Cs=0.1, nu=1e-5, SSPRK33 dt=1e-4"}
    for prec in precisions:
        m = workloads.build(spec, BLD, precision=prec, device=local)
        BLD.initialize(m, vel1=u0, vel2=v0, vel3=w0)
        m.prepare()
        stream = torch.cuda.ExternalStream(m.stream)
        m.step(warmup, spec["dt"])
        m.sync()
        ms = _event_time(stream, lambda: m.step_async(steps, spec["dt"]))
        m.sync()
        sb = state_bytes(m)
        peak, _ = peaks()
        ach = 8 * sb / (ms / steps * 1e-3) / 1e9
        # device time per launch of each phase (index 0: advection space, 1: SGS space)
        pt = _capi.BldPhaseTimes()
        _capi.check(m._lib.bld_time_phases(m._h, 5, _capi.SSPRK33, ctypes.byref(pt)))
        phases = {"inv_y": list(pt.inv_y_ms), "x": list(pt.x_ms), "fwd_y": list(pt.fwd_y_ms),
                  "project": pt.project_ms, "launches_per_step": pt.launches_per_step}
        out[prec] = {"value": npts * steps / (ms * 1e-3), "unit": UNIT, "ms_per_step": ms / steps, "steps": steps,
                     "device_bytes": m.info.device_bytes, "kernels": m.kernels(), "phases_ms": phases,
                     "roofline_step": {"algorithmic_bytes_per_step": 8 * sb, "achieved": ach, "unit": "GB/s",
                                       "frac": ach / peak}}
        del m
    return out


def run_ensemble(steps, warmup, local):
    """64 uneven LES members (24 x 64^2x32, 24 x 96^2x48, 16 x 128^2x64), mixed form,
    per-member z0 and Cs; one parent-graph launch per step for all three classes."""
    import ctypes
    import torch
    from BoundaryLayerDynamics import _capi
    from BoundaryLayerDynamics import workloads
    from BoundaryLayerDynamics.ensemble import Ensemble
    groups = workloads.ensemble_members()
    ens = Ensemble.from_groups(groups, precision="mixed", device=local)
    ens.initialize(groups, seed=100)
    ens.prepare()
    dt = 1e-4
    ens.step(warmup, dt)
    stream = torch.cuda.ExternalStream(ens.models[0].stream)
    ms = _event_time(stream, lambda: ens.step(steps, dt))
    # the same steps with the classes one after the other (one graph per class)
    def serial():
        for m in ens.models:
            m.step_async(steps, dt)
            m.sync()
    ms_serial = _event_time(stream, serial)
    sb = sum(state_bytes(m) * m.members for m in ens.models)
    peak, _ = peaks()
    ach = 8 * sb / (ms / steps * 1e-3) / 1e9
    # kernel launches inside one step's graph, summed over the classes
    kernels_per_step = 0
    for m in ens.models:
        pt = _capi.BldPhaseTimes()
        _capi.check(m._lib.bld_time_phases(m._h, 1, _capi.SSPRK33, ctypes.byref(pt)))
        kernels_per_step += pt.launches_per_step
    return {"workload": "ensemble of 64 LES members: 24 x 64^2x32, 24 x 96^2x48, 16 x 128^2x64; "
                        "z0 ~ logU[1e-5,1e-3], Cs ~ U[0.08,0.16]; SSPRK33 dt=1e-4",
            "dtype": "f32 transforms/products, f64 state+pressure",
            "members": ens.members, "points_per_step": ens.points,
            "value": ens.points * steps / (ms * 1e-3), "unit": UNIT, "ms_per_step": ms / steps, "steps": steps,
            "ms_per_step_classes_serial": ms_serial / steps,
            "launches_per_step": kernels_per_step, "graph_launches_per_step": 1,
            "device_bytes": sum(m.info.device_bytes for m in ens.models),
            "roofline_step": {"algorithmic_bytes_per_step": 8 * sb, "achieved": ach, "unit": "GB/s",
                              "frac": ach / peak}}


def run_serving(budget_gb, seconds, local):
    """Served stream: Poisson arrivals at 80% of the measured batched capacity,
    sizes {64^2x32, 128^2x64, 192^2x96, 256^2x128} with p {0.4, 0.3, 0.2, 0.1},
    500 SSPRK33 steps each, seeded z0 and forcing; pools are created and released
    against the HBM budget as requests come and go (admission by free HBM), and
    every request's initial field is generated on the device at admission."""
    from BoundaryLayerDynamics import serving as S
    srv = S.ElasticServer.create(int(budget_gb * 2**30), precision="mixed", device=local, tick=10)
    rate, per_req = S.calibrate_rate_elastic(srv, steps=500, load=0.8)
    n = int(min(64, max(16, round(rate * seconds))))
    reqs = S.make_requests(n, rate, seed=2024, steps=500, materialize=False)
    st = srv.run(reqs)
    st.update({
        "workload": "served LES stream: sizes 64^2x32/128^2x64/192^2x96/256^2x128 (p .4/.3/.2/.1), "
                    "500 SSPRK33 steps each, z0 ~ logU[1e-5,1e-3], forcing ~ U[0.5,1.5]",
        "dtype": "f32 transforms/products, f64 state+pressure",
        "admission": "pools created on demand and released when idle against the HBM budget; "
                     "initial fields generated on the device at admission",
        "arrival_rate_per_s": rate, "load": 0.8,
        "service_s_per_request_at_full_pool": {f"{s[0]}^2x{s[1]}": v for s, v in per_req.items()},
        "unit_latency": "s", "unit": UNIT, "tick_steps": 10,
    })
    return st


def run_tridiag(iters, local):
    """Batched tridiagonal pressure systems of the 512x512x256 LES alone:
    (i) 256 x 511 = 130 816 complex systems of 256 (the pressure solve's shape),
    (ii) 512 x 512 = 262 144 real systems of 256; staggered second-difference
    matrix with the horizontal wavenumber shift, random right-hand sides."""
    import numpy as np
    import torch
    from BoundaryLayerDynamics import _capi
    lib = _capi.load()
    n, L1, L2 = 256, 8 * math.pi, 4 * math.pi
    alpha = float(n)                     # uniform grid on [0, 1]: N3 / (dx3/dzeta)
    out = {}
    peak, _ = peaks()
    for kind, nk1, nk2, ebytes in (("complex", 256, 511, 16), ("real", 512, 512, 8)):
        nsys = nk1 * nk2
        rng = np.random.default_rng(5)
        k1 = np.arange(nsys) % nk1
        k2 = np.arange(nsys) // nk1 - nk2 // 2
        shift = 4 * math.pi ** 2 * ((k1 / L1) ** 2 + (k2 / L2) ** 2) / alpha
        diag = np.full((nsys, n), -2.0 * alpha)
        diag[:, 0] = diag[:, -1] = -alpha
        diag -= shift[:, None]
        diag[(nk2 // 2) * nk1, -1] = -3 * alpha          # the k = (0, 0) system
        beta = np.full(n - 1, alpha)
        gam = np.empty((n, nsys))
        g = 1.0 / diag[:, 0]
        gam[0] = g
        for z in range(1, n):
            g = 1.0 / (diag[:, z] - g * beta[z - 1] ** 2)
            gam[z] = g
        g_d = torch.tensor(gam, device="cuda")
        b_d = torch.tensor(np.concatenate([beta, [0.0]]), device="cuda")
        if kind == "complex":
            r0 = torch.tensor(rng.uniform(-1, 1, (n, nsys)) + 1j * rng.uniform(-1, 1, (n, nsys)), device="cuda")
            fn = lib.bld_ldlt_solve_device
        else:
            r0 = torch.tensor(rng.uniform(-1, 1, (n, nsys)), device="cuda")
            fn = lib.bld_ldlt_solve_real_device
        bufs = [r0.clone() for _ in range(2)]          # alternate buffers: 2 x 0.5-1 GB, beyond L2
        stream = torch.cuda.current_stream()
        for b in bufs:
            _capi.check(fn(g_d.data_ptr(), b_d.data_ptr(), b.data_ptr(), nsys, n, stream.cuda_stream))
        def launches():
            for i in range(iters):
                b = bufs[i % 2]
                _capi.check(fn(g_d.data_ptr(), b_d.data_ptr(), b.data_ptr(), nsys, n, stream.cuda_stream))
        ms = _event_time(stream, launches) / iters
        alg = nsys * n * (8 + 2 * ebytes)                 # gamma once, rhs read + solution written
        ach = alg / (ms * 1e-3) / 1e9
        out[kind] = {"systems": nsys, "n": n, "ms_per_solve": ms, "algorithmic_bytes": alg,
                     "achieved": ach, "unit": "GB/s", "peak": peak, "frac": ach / peak,
                     "unknowns_per_s": nsys * n / (ms * 1e-3)}
        del g_d, b_d, r0, bufs
    out["kernel"] = "k_ldlt_seg"
    return out


def run_extras(args, local):
    want = set(filter(None, args.only.split(","))) or {"ensemble", "serving", "tridiag", "les64", "les512"}
    out = {}
    if "tridiag" in want:
        out["tridiag"] = run_tridiag(20, local)
    if "les64" in want:
        out["les64"] = run_les("les64", ("fp64", "mixed"), 100, 5, local)
    if "ensemble" in want:
        out["ensemble"] = run_ensemble(max(args.steps // 2, 10), max(3, args.warmup), local)
    if "les512" in want:
        out["les512"] = run_les("les512", ("mixed",), 10, 3, local)
    if "serving" in want:
        out["serving"] = run_serving(args.serve_budget_gb, args.serve_seconds, local)
    return out


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
        "config": dict(CONFIG),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def run_profile(args):
    """The workload's setup (model, autotuning, initial projection, warm-up) outside
    the profiled range; then --profile-steps steps inside cudaProfilerStart/Stop."""
    import torch
    import BoundaryLayerDynamics as BLD
    from BoundaryLayerDynamics import workloads
    if args.config == "ensemble":
        # the 64-member uneven LES ensemble (mixed form), one parent-graph step per step
        from BoundaryLayerDynamics.ensemble import Ensemble
        groups = workloads.ensemble_members()
        ens = Ensemble.from_groups(groups, precision="mixed")
        ens.initialize(groups, seed=100)
        ens.prepare()
        ens.step(max(3, args.warmup), 1e-4)
        torch.cuda.synchronize()
        torch.cuda.profiler.start()
        ens.step(args.profile_steps, 1e-4)
        torch.cuda.synchronize()
        torch.cuda.profiler.stop()
        return {"profile": "ensemble", "precision": "mixed", "steps": args.profile_steps,
                "kernels": [m.kernels() for m in ens.models]}
    spec = workloads.CONFIGS[args.config]
    m = workloads.build(spec, BLD, precision=args.precision)
    u0, v0, w0 = workloads.initial_fields(spec)
    BLD.initialize(m, vel1=u0, vel2=v0, vel3=w0)
    m.prepare()
    m.step(max(3, args.warmup), spec["dt"])
    m.sync()
    torch.cuda.profiler.start()
    m.step(args.profile_steps, spec["dt"])
    m.sync()
    torch.cuda.profiler.stop()
    return {"profile": args.config, "precision": args.precision, "steps": args.profile_steps,
            "adv_p": [m.info.adv_p1, m.info.adv_p2], "sgs_p": [m.info.sgs_p1, m.info.sgs_p2],
            "kernels": m.kernels()}


def main():
    args = parse()
    if args.profile:
        print(json.dumps(run_profile(args)), flush=True)
        return
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
