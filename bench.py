#!/usr/bin/env python
"""Benchmark of the B200 phase-field step: cell-updates/s of the 3D
three-variant martensite at 256^3, FP32, Philox noise (the headline workload).

  python bench.py [--gpus N --steps K --warmup W] [--impl ours|reference]

One process per GPU (torchrun for N > 1).  The path does not shard a single
simulation: every rank advances its own replica (sim_id = rank) with no data
collective, so `value` is the whole-job aggregate of N replicas ("weak").

value   -- device time of K steps on resident HBM data, CUDA events on the
           launching stream, max over ranks.
e2e     -- the same metric through the C ABI with host buffers: every step
           uploads the field set from pinned host memory
           (gs_sim_set_field_async), steps once (gs_sim_step) and reads the
           field set back into pinned host memory (gs_sim_copy_field_async +
           gs_sim_copy_field_wait), so that step k's download overlaps step
           k+1's upload on the two directions of the host link; every copy
           is waited for inside the timed region; host clock.  The
           one-at-a-time variant (gs_sim_set_field, gs_sim_step,
           gs_sim_get_field) is reported beside it as "serial".
roofline-- the dominant pass, timed live with CUDA events between passes
           (gs_sim_profile_step), algorithmic bytes / time vs measured HBM.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "general-simulator_b200"))

METRIC = "cell-updates/s at 256³ martensite, % HBM roofline; adjoint:forward; sims/s"
UNIT = "cell-updates/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--n", type=int, default=256)
    ap.add_argument("--e2e-steps", type=int, default=20)
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-tune", action="store_true", help="keep the launchers' default tile sizes")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the comparator, adjoint and ensemble measurements (1 GPU only)")
    return ap.parse_args()


def workload_config(n: int, steps: int, extra: dict | None = None) -> dict:
    cfg = {
        "workload": f"martensite TDGL + Khachaturyan elasticity, 3D {n}^3, 3 variants, FP32 fields, "
                    "Philox noise 1e-3, dt 0.005, sigma_zz 0.005",
        "grid": [n, n, n], "variants": 3, "dtype": "fp32", "timed_steps": steps,
        "l2": "inputs larger than L2 (field set + spectrum = 2 x 201 MB > 126 MB L2); no flush",
        "initial": "eta ~ U[-0.01, 0.01], numpy PCG64 seed 1",
    }
    if extra:
        cfg.update(extra)
    return cfg


# ---------------------------------------------------------------------------
# distributed plumbing
# ---------------------------------------------------------------------------
def dist_setup(gpus: int):
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import datetime

        import torch.distributed as dist

        backend = "nccl"
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
    return ws, rank, local


def max_over_ranks(x: float, ws: int) -> float:
    if ws == 1:
        return x
    import torch
    import torch.distributed as dist

    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(ws: int) -> None:
    if ws > 1:
        import torch.distributed as dist

        dist.barrier()


# ---------------------------------------------------------------------------
# clocks sampled during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, uuid: str | None):
        self.uuid = uuid
        self.proc = None
        self.lines: list[str] = []

    def start(self):
        cmd = ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "50"]
        if self.uuid:
            cmd += ["-i", self.uuid]
        try:
            self.proc = subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except FileNotFoundError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.12)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.t.join(timeout=2)
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[0]))
                smax = float(parts[1])
            except ValueError:
                continue
            for nm, v in zip(names, parts[4:8]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peaks() -> dict:
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return {"hbm_gbs": d["hbm_gbs"], "source": "measured"}
    return {"hbm_gbs": 6650.0, "source": "fallback"}


def committed_traffic() -> dict | None:
    """DRAM bytes per launch of the dominant pass from the committed ncu
    summary (profiles/dram_traffic.json), or None."""
    path = os.path.join(ROOT, "profiles", "dram_traffic.json")
    if not os.path.exists(path):
        return None
    with open(path) as f:
        return json.load(f)


# ---------------------------------------------------------------------------
# secondary measurements of the metric (1 GPU): cuFFT comparator, adjoint,
# batched ensemble; device time with CUDA events on the launching stream
# ---------------------------------------------------------------------------
def _timed(stream, fn) -> float:
    import torch

    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    fn()
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1)


def _comparator_ms(p, kind: str, steps: int) -> float:
    import torch

    import gs_b200 as gb

    sim = gb.Sim(p, plain=kind == "plain", cufft=kind == "cufft")
    sim.set_field("eta", gb.initial_eta(p, 1).astype(np.float32))
    stream = torch.cuda.Stream()
    with torch.cuda.stream(stream):
        sim.step(5, stream.cuda_stream)
        ms = min(_timed(stream, lambda: sim.step(steps, stream.cuda_stream)) for _ in range(2)) / steps
    sim.close()
    return ms


def extra_comparator(n: int, ours_ms: float, steps: int = 50) -> dict:
    """The same step with cuFFT: (1) the comparator of the hand-written FFT
    passes -- cufftExecR2C / C2R batched over the variants, one contraction
    sweep with the octant B table, and this project's fused update without
    its z transforms; (2) the reference's structure (cuFFT C2C on complex
    copies, B streamed from a [V][V][N] array, unfused sweeps)."""
    import gs_b200 as gb

    p = gb.mart3d_params(n, dtype=gb.GS_DTYPE_F32, noise=1e-3)
    cu = _comparator_ms(p, "cufft", steps)
    pl = _comparator_ms(p, "plain", steps)
    return {"what": "cuFFT R2C/C2R batched over V (planned once) + octant-B-table contraction sweep + this "
                    "project's fused update kernel without its z transforms",
            "ms_per_step": cu, "ours_ms_per_step": ours_ms, "speedup": cu / ours_ms, "steps": steps,
            "comparator_reference_structure": {
                "what": "cuFFT C2C batch V on complex copies, B(n) streamed from a [V][V][N] array, unfused sweeps "
                        "(the reference's structure)",
                "ms_per_step": pl, "speedup": pl / ours_ms}}


def extra_adjoint(steps_fwd: int = 200) -> dict:
    """Calibration workload: 96^3, 3 variants, FP32, 200 steps, checkpoint
    every 20, noise off.  forward = 200 plain steps (gs_sim_step); backward
    = gs_adjoint_backward (segment recompute + adjoint sweeps + gradient
    sums), both device time on one stream, both replaying captured graphs
    (the forward also timed with direct launches)."""
    import ctypes as C

    import torch

    import gs_b200 as gb
    import gs_torch as gt

    run, th0, eta0, target, et = gt.calibration_setup(96, steps_fwd, gb.GS_DTYPE_F32, 20)
    a = run.adj
    p = run.params_for(th0)
    a.set_params(p)
    a.set_loss(target, 0.1, et)
    stream = torch.cuda.Stream()
    sh = stream.cuda_stream
    L = gb.lib()
    loss = (C.c_double * 3)()
    g = (C.c_double * 6)()

    def back():
        gb.check(L.gs_adjoint_backward(a.h, None, 0, 0.0, loss, g, None, 0, C.c_void_p(sh)), "backward")

    with torch.cuda.stream(stream):
        a.forward(eta0, sh)
        back()  # first run direct; later ones replay captured graphs
        bwd = []
        for _ in range(4):
            a.forward(eta0, sh)
            bwd.append(_timed(stream, back))
        bwd = min(bwd)
        launches = a.launch_count()
        fwd = {}
        for graph in (False, True):
            sim = gb.Sim(p)
            sim.use_graph(graph)
            sim.set_field("eta", eta0.astype(np.float32))
            sim.step(20, sh)
            fwd[graph] = min(_timed(stream, lambda: sim.step(steps_fwd, sh)) for _ in range(3))
            sim.close()
    mem = a.device_bytes()
    run.close()
    return {"workload": "96^3, 3 variants, FP32, 200 steps, checkpoint every 20, noise off",
            "forward_ms": fwd[True], "forward_direct_ms": fwd[False], "backward_ms": bwd,
            "adjoint_to_forward": bwd / fwd[True],
            "backward_launches": launches, "device_bytes": mem,
            "note": "backward includes recomputing every segment from its checkpoint"}


def extra_ensemble(steps: int = 100, total_steps: int = 2000) -> dict:
    """64 uneven simulations in grouped launches with CUDA-graph replay
    against the same simulations run one after another with the plain
    (cuFFT) step and with the hand-written single-simulation step."""
    import torch

    import gs_b200 as gb

    ps = gb.ensemble_params(gb.GS_DTYPE_F32)
    b = gb.Batch(ps)
    for i, p in enumerate(ps):
        b.set_eta(i, gb.initial_eta(p, 200 + i).astype(np.float32))
    b.use_graph(True)
    stream = torch.cuda.Stream()
    sh = stream.cuda_stream
    with torch.cuda.stream(stream):
        scheds = b.autotune(reps=3, stream=sh)
        b.step(4, sh)
        ms = _timed(stream, lambda: b.step(steps, sh)) / steps
    groups = b.groups()
    b.close()
    cells = sum(p.ncells for p in ps)
    shapes = {}
    for p in ps:
        shapes.setdefault((p.nx, p.ny, p.nz, p.nvariants), []).append(p)
    seq = {"cufft": 0.0, "plain": 0.0, "ours": 0.0}
    per_shape = {}
    with torch.cuda.stream(stream):
        for key, plist in shapes.items():
            row = {}
            for kind in ("cufft", "plain", "ours"):
                sim = gb.Sim(plist[0], plain=kind == "plain", cufft=kind == "cufft")
                sim.set_field("eta", gb.initial_eta(plist[0], 7).astype(np.float32))
                sim.step(3, sh)
                t = _timed(stream, lambda: sim.step(20, sh)) / 20
                sim.close()
                row[kind] = t
                seq[kind] += t * len(plist)
            per_shape["x".join(map(str, key[:3])) + f"/V{key[3]}"] = {**row, "count": len(plist)}
    sims_s = len(ps) / (ms * total_steps / 1e3)
    return {"workload": "64 sims: 32 x 128^2 + 16 x 256^2 (V=2), 12 x 64^3 + 4 x 128^3 (V=3), FP32, "
                        f"noise 1e-3, {total_steps} steps each",
            "batched_ms_per_step": ms, "groups": groups, "group_schedules": scheds, "sims_per_s": sims_s,
            "cell_updates_per_s": cells * 1e3 / ms,
            "sequential_plain_sims_per_s": len(ps) / (seq["cufft"] * total_steps / 1e3),
            "sequential_ours_sims_per_s": len(ps) / (seq["ours"] * total_steps / 1e3),
            "vs_sequential_plain": seq["cufft"] / ms, "vs_sequential_ours": seq["ours"] / ms,
            "sequential_plain_note": "plain = the cuFFT R2C/C2R comparator step run one simulation after another",
            "sequential_reference_structure_sims_per_s": len(ps) / (seq["plain"] * total_steps / 1e3),
            "vs_sequential_reference_structure": seq["plain"] / ms,
            "per_shape_ms_per_step": per_shape, "timed_steps": steps}


def precip_pass_bytes(names: list, p) -> dict:
    """Algorithmic HBM bytes of each pass of the precipitate step (FP32, V
    variants, F1 = V + 1 chain-1 fields with the concentration's misfit;
    chain 2 transforms V + 2 fields: c, mu and u_p = eta_p - dt L g_p; the
    last sweep also writes the next step's chain-1 z spectra): every field or
    spectrum a pass must read or write once.  At V = 4 a steady-state step
    moves 376 N bytes."""
    V, N = p.nvariants, p.ncells
    F1 = V + (1 if p.c_elastic else 0)
    F2 = V + 2
    f = 4 * N
    table = {"z_forward": 2 * F1 * f, "y_forward": 2 * F1 * f, "x_contraction": 2 * F1 * f,
             "y_inverse": 2 * F1 * f, "precip_mid": (F1 + (V + 1) + F2) * f,
             "z_inverse_potential": 2 * F1 * f, "precip_local": (F1 + (V + 1) + (V + 1)) * f,
             "z_forward_update_fields": 2 * F2 * f, "y_forward_update_fields": 2 * F2 * f,
             "x_kspace_update": (F2 + (V + 1)) * f, "y_inverse_update_fields": 2 * (V + 1) * f,
             "z_inverse_c_eta": 2 * (V + 1) * f, "z_inverse_c_eta_next_z_forward": (2 * (V + 1) + F1) * f}
    return {nm: table[nm] for nm in names}


def extra_configs() -> dict:
    """The other workloads of the step, timed the same way: the 2D FP64
    martensite (128^2, 2 variants, 1000-step runs), the headline martensite
    at 128^3 and the 3D precipitate
    (256^3, concentration + 4 variants, FP32, semi-implicit, FP64 mass
    projection) with its relative mass drift over the timed steps."""
    import torch

    import gs_b200 as gb

    out = {}
    stream = torch.cuda.Stream()
    sh = stream.cuda_stream
    with torch.cuda.stream(stream):
        p = gb.mart2d_params(128, dtype=gb.GS_DTYPE_F64)
        sim = gb.Sim(p)
        sim.set_field("eta", gb.initial_eta(p, 0, 0.01))
        sim.use_graph(True)
        sim.step(10, sh)
        steps = 1000
        ms = _timed(stream, lambda: sim.step(steps, sh)) / steps
        sim.close()
        out["mart2d_fp64_128"] = {"ms_per_step": ms, "cell_updates_per_s": p.ncells * 1e3 / ms, "steps": steps,
                                  "note": "graph replay; a 1000-step run of this workload takes 1000 x ms_per_step"}
        # the headline workload at its smaller size (fields of 25 MB: L2-resident)
        p = gb.mart3d_params(128, dtype=gb.GS_DTYPE_F32, noise=1e-3)
        sim = gb.Sim(p)
        sim.set_field("eta", gb.initial_eta(p, 1))
        sim.autotune(reps=3, stream=sh)
        sim.use_graph(True)
        sim.step(10, sh)
        steps = 500
        ms = _timed(stream, lambda: sim.step(steps, sh)) / steps
        sim.close()
        out["mart3d_fp32_128"] = {"ms_per_step": ms, "cell_updates_per_s": p.ncells * 1e3 / ms, "steps": steps,
                                  "note": "autotuned, graph replay; fields and spectra (50 MB) fit in L2"}
        p = gb.precip3d_params(256, dtype=gb.GS_DTYPE_F32)
        sim = gb.Sim(p)
        sim.set_field("concentration", gb.initial_c(p, 2))
        sim.set_field("eta", gb.initial_eta(p, 3, 0.01))
        psched = sim.autotune(reps=3, stream=sh)  # on a kept copy of the state
        sim.step(3, sh)
        m0 = sim.stats(sh)["mass"]
        steps = 20
        ms = _timed(stream, lambda: sim.step(steps, sh)) / steps
        m1 = sim.stats(sh)["mass"]
        launches = sim.launch_count()
        # the statistics ran the first chain on the spectrum buffer: one step
        # to get back to the steady state (fused z forward), then the passes
        sim.step(1, sh)
        passes = [sim.profile_step(sh) for _ in range(3)]
        names = sim.pass_names()
        sim.close()
        pass_ms = np.median(np.array(passes), axis=0)
        algo = precip_pass_bytes(names, p)
        dom = int(np.argmax(pass_ms))
        peak = measured_peaks()
        step_bytes = sum(algo.values())
        out["precipitate_fp32_256"] = {
            "ms_per_step": ms, "cell_updates_per_s": p.ncells * 1e3 / ms, "steps": steps, "tile_schedule": psched,
            "launches_per_step": launches / steps, "mass_drift_relative": abs(m1 - m0) / abs(m0),
            "step_bytes_algorithmic": step_bytes,
            "step_gbs_algorithmic": step_bytes / (ms / 1e3) / 1e9,
            "roofline": {"bound": "hbm", "kernel": names[dom], "launch_ms": float(pass_ms[dom]),
                         "algorithmic_bytes_per_launch": algo[names[dom]],
                         "achieved": algo[names[dom]] / (pass_ms[dom] / 1e3) / 1e9, "peak": peak["hbm_gbs"],
                         "unit": "GB/s", "frac": algo[names[dom]] / (pass_ms[dom] / 1e3) / 1e9 / peak["hbm_gbs"],
                         "peak_source": peak["source"],
                         "pass_ms": {nm: float(t) for nm, t in zip(names, pass_ms)},
                         "pass_bytes": algo}}
    return out


def extra_precip_adjoint(n: int = 256, steps: int = 100, K: int = 10) -> dict:
    """Adjoint of the precipitate run: 256^3, concentration + 4 variants,
    FP32, 100 steps, noise off, a checkpoint every 10 steps.  plain = 100
    steps of gs_sim_step; forward = the adjoint's forward run (the same
    steps, checkpoints and the last segment kept on the device); backward =
    gs_precip_adjoint_backward (the earlier segments recomputed from their
    checkpoints, all reverse steps and the nine parameter sums, replayed as a
    captured graph), seeds already on the device.  Device time on one
    stream."""
    import torch

    import gs_b200 as gb

    p = gb.precip3d_params(n, dtype=gb.GS_DTYPE_F32)
    p.noise_amp = 0.0
    c0 = gb.initial_c(p, 2)
    e0 = gb.initial_eta(p, 3, 0.3)
    rng = np.random.default_rng(0)
    stream = torch.cuda.Stream()
    sh = stream.cuda_stream
    with torch.cuda.stream(stream):
        sim = gb.Sim(p)
        sim.set_field("concentration", c0)
        sim.set_field("eta", e0)
        sim.step(3, sh)
        plain = min(_timed(stream, lambda: sim.step(steps, sh)) for _ in range(2))
        sim.close()
        a = gb.PrecipAdjoint(p, steps, K)
        a.forward(c0, e0, sh, outputs=False)
        a.set_seed(rng.standard_normal(c0.shape), rng.standard_normal(e0.shape))
        a.backward(stream=sh, outputs=False)  # direct; the next ones replay the captured sweep
        a.backward(stream=sh, outputs=False)
        fwd = min(_timed(stream, lambda: a.forward(stream=sh, outputs=False)) for _ in range(2))
        bwd = min(_timed(stream, lambda: a.backward(stream=sh, outputs=False)) for _ in range(2))
        mem = a.device_bytes()
        a.close()
    return {"workload": f"{n}^3, concentration + 4 variants, FP32, {steps} steps, noise off, checkpoint every {K}",
            "plain_ms": plain, "forward_ms": fwd, "backward_ms": bwd, "adjoint_to_plain": bwd / plain,
            "device_bytes": mem,
            "note": "backward includes recomputing every segment but the last from its checkpoint"}


def extra_slab(n: int = 256, nranks: int = 2, steps: int = 20) -> dict:
    """The slab-decomposed step on one GPU: nranks slabs of the headline grid
    in one process, the transposes and halos as device copies (the exchange
    a multi-GPU run does over NVLink), device time per step against the
    one-device step.  Measures the decomposition's own cost (packing, the
    x-pencil passes on kz sub-ranges); the cross-GPU exchange itself is not
    measured here (one GPU)."""
    import torch

    import gs_b200 as gb
    import gs_slab

    p = gb.mart3d_params(n, dtype=gb.GS_DTYPE_F32, noise=1e-3)
    eta0 = gb.initial_eta(p, 1).astype(np.float32)
    slabs = [gs_slab.Slab(p, r, nranks) for r in range(nranks)]
    try:
        for r, sl in enumerate(slabs):
            sl.set_eta(eta0[:, sl.plan.x_range(r)])
        stream = torch.cuda.current_stream()
        gs_slab.step_local(slabs, 3)
        ms = min(_timed(stream, lambda: gs_slab.step_local(slabs, steps)) for _ in range(2)) / steps
        xfer = 2 * sum(int(sl.geom.a2a_bytes) for sl in slabs) + sum(int(sl.geom.halo_bytes) for sl in slabs)
    finally:
        for sl in slabs:
            sl.close()
    return {"workload": f"{n}^3, 3 variants, FP32, noise 1e-3, {nranks} x-slabs on one GPU",
            "ms_per_step": ms, "exchange_bytes_per_step": xfer,
            "note": "all-to-all and halo exchanges as device copies on the same GPU; a multi-GPU run replaces "
                    "them with NCCL collectives (unmeasured on hardware: one GPU in this run)"}


# ---------------------------------------------------------------------------
# CPU baseline: the FP64 oracle on the host cores
# ---------------------------------------------------------------------------
def cpu_model() -> str:
    """The host CPU's model name (/proc/cpuinfo), or the platform's string."""
    try:
        with open("/proc/cpuinfo") as f:
            for ln in f:
                if ln.lower().startswith("model name"):
                    return ln.split(":", 1)[1].strip()
    except OSError:
        pass
    import platform

    return platform.processor() or "unknown"


def cpu_baseline(n: int, seconds: float) -> dict:
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import gs_b200 as gb
    import oracle_py as orc

    cores = os.cpu_count() or 1
    orc.set_threads(cores)
    p = gb.mart3d_params(n, noise=1e-3, host_only=True)
    eta = gb.initial_eta(p, 1)
    steps = 0
    t0 = time.perf_counter()
    while True:
        eta = orc.mart_run(p, eta, 1, step0=steps)
        steps += 1
        if time.perf_counter() - t0 >= seconds:
            break
    dt = time.perf_counter() - t0
    return {"value": n ** 3 * steps / dt, "unit": UNIT, "cores": orc.get_threads(), "kind": "port",
            "cpu_model": cpu_model(),
            "sample": f"{steps} FP64 oracle step(s) of the {n}^3 3-variant workload, {dt:.1f} s "
                      f"({orc.get_threads()} OpenMP threads on {cpu_model()})"}


def run_reference(args, ws, rank):
    """The reference arm: the reference has no CPU implementation of the
    step (its kernels are device-only), so this times the FP64 CPU port of
    the same discretisation on all host cores.  Nothing here loads the
    product library: the parameters are filled in Python (host_only) and
    only oracle/liboracle.so is mapped."""
    if rank != 0:
        return
    cores = os.cpu_count() or 1
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import gs_b200 as gb
    import oracle_py as orc

    orc.set_threads(cores)
    p = gb.mart3d_params(args.n, noise=1e-3, host_only=True)
    eta = gb.initial_eta(p, 1)
    budget = 150.0
    t0 = time.perf_counter()
    warm = 0
    for i in range(args.warmup):
        eta = orc.mart_run(p, eta, 1, step0=i)
        warm += 1
        if time.perf_counter() - t0 > 60.0:
            break
    done = 0
    ts = time.perf_counter()
    for i in range(args.steps):
        eta = orc.mart_run(p, eta, 1, step0=warm + i)
        done += 1
        if time.perf_counter() - ts > budget:
            break
    dt = time.perf_counter() - ts
    v = args.n ** 3 * done / dt
    model = cpu_model()
    sample = (f"{done} of {args.steps} requested steps (time budget {budget:.0f} s) after {warm} warm-up "
              f"step(s), FP64 oracle port, {orc.get_threads()} threads on {model}")
    line = {"metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus, "steps": done,
            "warmup": warm, "ms_per_step": 1e3 * dt / max(done, 1), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "impl": "reference", "config": workload_config(args.n, done),
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": orc.get_threads(), "cpu_model": model,
                             "kind": "port", "sample": sample},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------
def run_ours(args, ws, rank, local):
    import torch

    import gs_b200 as gb

    torch.cuda.set_device(local)
    dev_uuid = None
    try:
        dev_uuid = "GPU-" + str(torch.cuda.get_device_properties(local).uuid)
    except Exception:
        pass
    n = args.n
    p = gb.mart3d_params(n, dtype=gb.GS_DTYPE_F32, noise=1e-3)
    p.sim_id = rank
    eta0 = gb.initial_eta(p, 1).astype(np.float32)
    V, N = p.nvariants, p.ncells
    sim = gb.Sim(p)
    sim.set_field("eta", eta0)
    stream = torch.cuda.Stream()
    sh = stream.cuda_stream
    with torch.cuda.stream(stream):
        # tile schedule from the library's autotuner (trial steps leave the state as it was)
        schedule = sim.autotune(reps=8, stream=sh) if not args.no_tune else sim.schedule()
        sim.step(args.warmup, sh)
        launches_per_step = sim.launch_count() / max(args.warmup, 1)
        torch.cuda.synchronize()
        barrier(ws)
        torch.cuda.synchronize()
        clk = ClockSampler(dev_uuid)
        clk.start()
        time.sleep(0.15)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        sim.step(args.steps, sh)
        e1.record(stream)
        torch.cuda.synchronize()
        clocks = clk.stop()
        ms = e0.elapsed_time(e1)
        barrier(ws)
    ms_max = max_over_ranks(ms, ws)
    value = N * args.steps * ws / (ms_max / 1e3)
    launches = int(round(launches_per_step * args.steps))

    # the same steps replayed from a captured CUDA graph (gs_sim_use_graph)
    with torch.cuda.stream(stream):
        sim.use_graph(True)
        sim.step(4, sh)
        torch.cuda.synchronize()
        g0 = torch.cuda.Event(enable_timing=True)
        g1 = torch.cuda.Event(enable_timing=True)
        g0.record(stream)
        sim.step(args.steps, sh)
        g1.record(stream)
        torch.cuda.synchronize()
        graph_ms = g0.elapsed_time(g1) / args.steps
        sim.use_graph(False)

    # per-pass device times of one step (live, on the launching stream)
    with torch.cuda.stream(stream):
        passes = [sim.profile_step(sh) for _ in range(5)]
    pass_ms = np.median(np.array(passes), axis=0)
    # algorithmic HBM bytes of each pass, FP32, V fields of N cells.  In steady
    # state the update also runs the next step's z forward (4 passes a step);
    # a step whose spectra were not ready runs the z forward on its own (5).
    f = 4 * V * N
    if len(pass_ms) == 4:
        names = ["y_forward", "x_fwd_contract_inv", "y_inverse", "z_inverse_update_z_forward"]
        algo = [2 * f, 2 * f, 2 * f, 4 * f]
    else:
        names = ["z_forward_r2c_eta2", "y_forward", "x_fwd_contract_inv", "y_inverse", "z_inverse_c2r_update"]
        algo = [2 * f, 2 * f, 2 * f, 2 * f, 3 * f]
    dom = int(np.argmax(pass_ms))
    peaks = measured_peaks()
    achieved = algo[dom] / (pass_ms[dom] / 1e3) / 1e9
    tr = committed_traffic()
    traffic = None
    if tr and tr.get("kernel_pass") == names[dom] and tr.get("n") == n:
        traffic = tr.get("dram_bytes_per_launch")
    step_bytes = sum(algo)
    step_gbs = step_bytes * args.steps / (ms / 1e3) / 1e9

    # e2e through the C ABI with host buffers
    pinned = torch.empty(V * N, dtype=torch.float32).pin_memory()
    pinned.numpy()[:] = eta0.ravel()
    out_pinned = torch.empty(V * N, dtype=torch.float32).pin_memory()
    import ctypes as C

    L = gb.lib()
    ptr_in = C.c_void_p(pinned.data_ptr())
    ptr_out = C.c_void_p(out_pinned.data_ptr())
    with torch.cuda.stream(stream):
        for _ in range(2):
            gb.check(L.gs_sim_set_field(sim.h, b"eta", ptr_in, V * N, 0), "set_field")
            sim.step(1, sh)
            gb.check(L.gs_sim_get_field(sim.h, b"eta", ptr_out, V * N, 0), "get_field")
        torch.cuda.synchronize()
        barrier(ws)
        t0 = time.perf_counter()
        for _ in range(args.e2e_steps):
            gb.check(L.gs_sim_set_field(sim.h, b"eta", ptr_in, V * N, 0), "set_field")
            sim.step(1, sh)
            gb.check(L.gs_sim_get_field(sim.h, b"eta", ptr_out, V * N, 0), "get_field")
        torch.cuda.synchronize()
        serial_s = time.perf_counter() - t0
        # pipelined: two page-locked output buffers, step k's download in
        # flight while step k+1 uploads and runs
        out2 = [out_pinned, torch.empty(V * N, dtype=torch.float32).pin_memory()]
        tk = C.c_int(0)

        def pipelined(k):
            prev = None
            for i in range(k):
                gb.check(L.gs_sim_set_field_async(sim.h, b"eta", ptr_in, V * N, 0, C.c_void_p(sh)), "upload")
                sim.step(1, sh)
                gb.check(L.gs_sim_copy_field_async(sim.h, b"eta", C.c_void_p(sh),
                                                   C.c_void_p(out2[i % 2].data_ptr()), C.byref(tk)), "download")
                if prev is not None:
                    gb.check(L.gs_sim_copy_field_wait(sim.h, prev, None, 0, 0), "download wait")
                prev = tk.value
            gb.check(L.gs_sim_copy_field_wait(sim.h, prev, None, 0, 0), "download wait")

        pipelined(2)
        torch.cuda.synchronize()
        barrier(ws)
        t0 = time.perf_counter()
        pipelined(args.e2e_steps)
        torch.cuda.synchronize()
        piped_s = time.perf_counter() - t0

        # staged: step k+1's upload goes to a staging buffer on the upload
        # stream while step k runs and step k's download goes the other way
        def staged(k):
            prev = None
            gb.check(L.gs_sim_stage_field_async(sim.h, b"eta", ptr_in, V * N, 0), "stage")
            for i in range(k):
                sim.step(1, sh)  # waits for the staged field set and swaps it in
                gb.check(L.gs_sim_copy_field_async(sim.h, b"eta", C.c_void_p(sh),
                                                   C.c_void_p(out2[i % 2].data_ptr()), C.byref(tk)), "download")
                if i + 1 < k:
                    gb.check(L.gs_sim_stage_field_async(sim.h, b"eta", ptr_in, V * N, 0), "stage")
                if prev is not None:
                    gb.check(L.gs_sim_copy_field_wait(sim.h, prev, None, 0, 0), "download wait")
                prev = tk.value
            gb.check(L.gs_sim_copy_field_wait(sim.h, prev, None, 0, 0), "download wait")

        staged(2)
        torch.cuda.synchronize()
        barrier(ws)
        t0 = time.perf_counter()
        staged(args.e2e_steps)
        torch.cuda.synchronize()
        e2e_s = time.perf_counter() - t0
    e2e_s = max_over_ranks(e2e_s, ws)
    piped_s = max_over_ranks(piped_s, ws)
    serial_s = max_over_ranks(serial_s, ws)
    e2e = {"value": N * args.e2e_steps * ws / e2e_s, "unit": UNIT, "h2d_bytes_per_step": 4 * V * N,
           "d2h_bytes_per_step": 4 * V * N, "steps": args.e2e_steps,
           "how": "per step: gs_sim_step(1) (swaps in the field set staged from pinned host memory) + "
                  "gs_sim_copy_field_async(eta, into pinned host) + gs_sim_stage_field_async(next step's eta, "
                  "from pinned host) + gs_sim_copy_field_wait of the previous step's download: step k+1's upload, "
                  "step k and step k's download run at once; every copy is waited for inside the timed region; "
                  "host clock",
           "overlapped": {"value": N * args.e2e_steps * ws / piped_s,
                          "how": "per step: gs_sim_set_field_async(eta, pinned host) + gs_sim_step(1) + "
                                 "gs_sim_copy_field_async + gs_sim_copy_field_wait of the previous download "
                                 "(the upload waits for the step before it)"},
           "serial": {"value": N * args.e2e_steps * ws / serial_s,
                      "how": "per step: gs_sim_set_field + gs_sim_step(1) + gs_sim_get_field, one after the other"}}
    sim.close()

    if rank != 0:
        return
    extras = {}
    if ws == 1 and not args.no_extras:
        extras["comparator"] = extra_comparator(n, ms / args.steps)
        extras["adjoint"] = extra_adjoint()
        extras["ensemble"] = extra_ensemble()
        extras["other_workloads"] = extra_configs()
        extras["precip_adjoint"] = extra_precip_adjoint()
        extras["slab"] = extra_slab(n)
    cpu = None
    if ws == 1 and not args.no_cpu:
        cpu = cpu_baseline(n, args.cpu_seconds)
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": workload_config(n, args.steps, {"parallelism": f"replicas x{ws}" if ws > 1 else "single GPU",
                                                   "tile_schedule": schedule,
                                                   "step_bytes_algorithmic": step_bytes,
                                                   "step_gbs_algorithmic": step_gbs}),
        "roofline": {"bound": "hbm", "kernel": names[dom], "achieved": achieved, "peak": peaks["hbm_gbs"],
                     "unit": "GB/s", "frac": achieved / peaks["hbm_gbs"], "traffic": traffic,
                     "peak_source": peaks["source"], "algorithmic_bytes_per_launch": algo[dom],
                     "launch_ms": float(pass_ms[dom]),
                     "pass_ms": {nm: float(t) for nm, t in zip(names, pass_ms)}},
        "cpu_baseline": cpu,
        "e2e": e2e,
        "gpu_launches": launches,
        "clocks": clocks,
        "graph_replay": {"ms_per_step": graph_ms,
                         "note": "the timed steps again, replayed from a captured CUDA graph (gs_sim_use_graph): "
                                 "the captured kernels read the step constants from device memory (the noise "
                                 "counter advances between replays), which costs more than the launches it saves"},
        **extras,
    }
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    if args.impl == "reference":
        # no device work: rank 0 times the CPU implementation, others exit
        run_reference(args, int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")))
        return
    ws, rank, local = dist_setup(args.gpus)
    try:
        run_ours(args, ws, rank, local)
    finally:
        if ws > 1:
            import torch.distributed as dist

            dist.destroy_process_group()


if __name__ == "__main__":
    main()
