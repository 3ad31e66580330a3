#!/usr/bin/env python3
"""Benchmark of the fused MUSCL-Hancock step on Kelvin-Helmholtz 2048^2.

Workload: 2-D Cartesian KH on [0,1]^2, 2048x2048 cells, periodic, gamma=1.4,
van Leer slopes, HLLC, CFL 0.4 (synthetic seeded initial state).  A "step" is
one time step of the whole grid.  The headline arm is the FP32-mixed fused
step; the plain FP64 and the fast FP64 fused steps are measured in the same
run, and the relative L1 and L-infinity errors of every stored field of the
mixed (and fast FP64) result against the FP64 result after the config's 1000
steps (same dt sequence) are reported.

Metric: Mcell-updates/s = steps x interior cells / time (src/main.cpp:570-581).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

With --gpus N > 1 under torchrun each rank runs an independent replica of the
single-domain step ("replicas only"); value is the sum over ranks, timing the
max over ranks.  --impl reference times the reference's own FP64 array code
(compiled from its sources against host Kokkos/MPI stand-ins, OpenMP on the
host cores; the C oracle where that build is absent) on a bounded sample.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

NX = 2048
CELLS = NX * NX
BYTES_PER_CELL = 2 * (2 + 2) * 8  # one FP64 read + one FP64 write of (rho, rhou_x, rhou_y, E)
WORKLOAD = "kelvin_helmholtz_2d_2048x2048_vanleer_hllc_cfl0.4_periodic"


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=1000)
    p.add_argument("--warmup", type=int, default=20)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--e2e-chunk", type=int, default=100, help="steps per C-ABI call in the end-to-end arm")
    p.add_argument("--cpu-budget", type=float, default=20.0, help="seconds of CPU oracle work for cpu_baseline")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-adjoint", action="store_true", help="skip the adjoint cost measurement")
    p.add_argument("--no-ensemble", action="store_true", help="skip the batched ensemble measurement")
    p.add_argument("--no-stage-loop", action="store_true",
                   help="skip the passive-scalar (stage-composed loop) measurement")
    p.add_argument("--no-rt3d", action="store_true", help="skip the 3-D Rayleigh-Taylor measurement")
    p.add_argument("--rt3d-steps", type=int, default=500, help="steps of the 3-D Rayleigh-Taylor measurement")
    p.add_argument("--accuracy-steps", type=int, default=1000,
                   help="KH steps over which the mixed step is compared with the FP64 step (the config's 1000)")
    return p.parse_args()


# HBM3e of an HGX B200 (7.7 TB/s nominal), beside the measured copy peak
HBM_SPEC_GBS = 7700.0
# Algorithmic HBM bytes per cell and step of one gradient (forward with
# checkpoints, recomputation, reverse sweep): the forward step reads and writes
# the 32-byte state (64 B), the recomputation repeats it (64 B), the reverse
# step reads the state and the incoming adjoint and writes the outgoing one
# (96 B); the checkpoints add 64 B per cell every k steps.
ADJ_BYTES_PER_CELL_STEP = 64 + 64 + 96


def kh_domain(precision):
    from heraclespp_b200 import Domain, setups

    d = Domain(2, [NX, NX], gamma=1.4, limiter="VanLeer", riemann="HLLC", bc=["Periodic"] * 4, precision=precision)
    grid = setups.Grid.from_domain(d)
    prim = setups.kelvin_helmholtz(grid)
    return d, prim


class ClockSampler:
    """SM clock, power and clock-event (throttle) reasons of this GPU, sampled
    from a thread through NVML every millisecond or so (read-only queries),
    with nvidia-smi every 200 ms where NVML is not importable.  `window(t0, t1)`
    marks the timed region on the host clock; the summary keeps the samples
    inside it (the nearest one on each side when the region is shorter than
    the sampling period)."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    REASONS = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")

    def __init__(self, gpu_index, pci_bus_id=None):
        self.gpu = gpu_index
        self.pci = pci_bus_id
        self.samples = []  # (host time, sm MHz, max sm MHz, power W, set of reasons)
        self.source = None
        self._win = None
        self._stop = threading.Event()
        self._t = None

    def _nvml(self):
        import pynvml as nv

        nv.nvmlInit()
        h = nv.nvmlDeviceGetHandleByPciBusId(self.pci.encode()) if self.pci else nv.nvmlDeviceGetHandleByIndex(self.gpu)
        bits = {"hw_slowdown": nv.nvmlClocksEventReasonHwSlowdown,
                "hw_thermal_slowdown": nv.nvmlClocksEventReasonHwThermalSlowdown,
                "sw_thermal_slowdown": nv.nvmlClocksEventReasonSwThermalSlowdown,
                "sw_power_cap": nv.nvmlClocksEventReasonSwPowerCap}
        smax = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
        self.source = "nvml"
        try:
            while not self._stop.is_set():
                sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
                r = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
                pw = nv.nvmlDeviceGetPowerUsage(h) * 1e-3
                self.samples.append((time.perf_counter(), float(sm), float(smax), pw,
                                     {k for k, b in bits.items() if r & b}))
                self._stop.wait(0.001)
        finally:
            nv.nvmlShutdown()

    def _smi(self):
        self.source = "nvidia-smi"
        gid = self.pci if self.pci else str(self.gpu)
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", f"--id={gid}", f"--query-gpu={self.FIELDS}",
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True, timeout=5)
                if out.returncode == 0 and out.stdout.strip():
                    f = [x.strip() for x in out.stdout.strip().split(",")]
                    num = lambda x: float(x) if x.replace(".", "").isdigit() else None  # noqa: E731
                    rs = {nm for k, nm in enumerate(self.REASONS) if len(f) > 5 + k and f[5 + k].lower().startswith("active")}
                    self.samples.append((time.perf_counter(), num(f[1]), num(f[2]), num(f[3]), rs))
            except Exception:
                pass
            self._stop.wait(0.2)

    def _run(self):
        try:
            import pynvml  # noqa: F401
        except ImportError:
            self._smi()
            return
        try:
            self._nvml()
        except Exception:
            self._smi()

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        # let the first samples arrive before the caller's timed region
        t_end = time.perf_counter() + 0.5
        while not self.samples and time.perf_counter() < t_end:
            time.sleep(0.005)
        return self

    def __exit__(self, *a):
        # a few samples after the region, then stop
        time.sleep(0.01)
        self._stop.set()
        self._t.join(timeout=10)

    def window(self, t0, t1):
        self._win = (t0, t1)

    def summary(self):
        samples = list(self.samples)
        if self._win is not None and samples:
            t0, t1 = self._win
            inside = [s for s in samples if t0 <= s[0] <= t1]
            if not inside:
                before = [s for s in samples if s[0] < t0][-1:]
                after = [s for s in samples if s[0] > t1][:1]
                inside = before + after
            samples = inside
        if not samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0,
                    "source": self.source}
        sm = [s[1] for s in samples if s[1] is not None]
        smax = [s[2] for s in samples if s[2] is not None]
        pw = [s[3] for s in samples if s[3] is not None]
        reasons = set().union(*[s[4] for s in samples])
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "power_w_median": round(float(np.median(pw)), 1) if pw else None,
                "reasons": sorted(reasons), "samples": len(samples), "source": self.source}


def pci_bus_id(torch, dev):
    """NVML's PCI bus id string of a CUDA device (the same GPU whatever
    CUDA_VISIBLE_DEVICES renumbers)."""
    try:
        p = torch.cuda.get_device_properties(dev)
        return f"{p.pci_domain_id:08X}:{p.pci_bus_id:02X}:{p.pci_device_id:02X}.0"
    except Exception:
        return None


def time_fused(torch, d, steps, warmup, clk=None):
    """Device time of `steps` fused steps (CUDA events on the library's stream).
    The warm-up runs at least `warmup` steps, rounded up to a multiple of 6, so
    that the timed steps start where the library's step graphs start (their
    control slots repeat every 6 steps) and replay graphs, not single launches;
    its first call also captures those graphs."""
    stream = torch.cuda.ExternalStream(d.stream_handle())
    d.run(cfl=0.4, nsteps=(warmup + 5) // 6 * 6)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    t0 = time.perf_counter()
    e0.record(stream)
    r = d.run(cfl=0.4, nsteps=steps)
    e1.record(stream)
    e1.synchronize()
    t1 = time.perf_counter()
    torch.cuda.synchronize()
    if clk is not None:
        clk.window(t0, t1)
    return e0.elapsed_time(e1) * 1e-3, r


def field_errors(mixed, ref, ng):
    """Error of the FP32-mixed state against the FP64 one, per stored field,
    over the interior cells: relative L1 (sum |a-b| / sum |b|), relative
    L-infinity (max |a-b| / max |b|) and the largest per-cell relative error
    of the positive fields (rho, E)."""
    rho_a, m_a, E_a = mixed
    rho_b, m_b, E_b = ref
    nd = m_a.shape[0]
    inner = tuple(slice(ng, -ng) if n > 1 else slice(None) for n in rho_a.shape)
    pairs = [("rho", rho_a, rho_b)] + [(f"rhou_{k}", m_a[k], m_b[k]) for k in range(nd)] + [("E", E_a, E_b)]
    out = {}
    for name, a, b in pairs:
        a = a[inner]
        b = b[inner]
        diff = np.abs(a - b)
        e = {"rel_l1": float(np.sum(diff) / np.sum(np.abs(b))),
             "rel_linf": float(np.max(diff) / np.max(np.abs(b)))}
        if name in ("rho", "E"):
            e["max_cell_rel"] = float(np.max(diff / np.abs(b)))
        out[name] = e
    return out


def kh_accuracy(prim, steps):
    """KH 2048^2 over `steps` steps: the FP32-mixed step with its own CFL dts,
    then the FP64 step with the same dt sequence; errors per field."""
    dm, _ = kh_domain("fp32_mixed")
    dm.set_state_from_prim(*prim)
    dm.run(cfl=0.4, nsteps=steps)
    dts = dm.dt_log()[:steps]
    mixed = dm.get_state()
    dm.close()
    d64, _ = kh_domain("fp64")
    d64.set_state_from_prim(*prim)
    d64.run(nsteps=steps, dts=dts)
    ref = d64.get_state()
    d64.close()
    dfast, _ = kh_domain("fp64_fast")
    dfast.set_state_from_prim(*prim)
    dfast.run(nsteps=steps, dts=dts)
    fast = dfast.get_state()
    dfast.close()
    return {"steps_compared": int(len(dts)), "reference": "FP64 fused step (bit-equal to the oracle), same dts",
            "fields": field_errors(mixed, ref, 2), "fp64_fast_fields": field_errors(fast, ref, 2)}


def read_traffic():
    """DRAM bytes per launch of the fused mixed kernel, from the committed ncu summary."""
    f = ROOT / "profiles" / "fused_step_mixed_kh2048.txt"
    if not f.exists():
        return None
    for line in f.read_text().splitlines():
        if line.startswith("traffic_bytes_per_launch:"):
            try:
                return float(line.split(":", 1)[1].strip())
            except ValueError:
                return None
    return None


def measured_peaks():
    f = ROOT / "MEASURED_PEAKS.json"
    if f.exists():
        try:
            return json.loads(f.read_text()), "measured"
        except Exception:
            pass
    return {"hbm_gbs": 6650.0}, "fallback"


def cpu_baseline(budget_s, cells_full=CELLS):
    """The reference's FP64 CPU path on the full KH 2048^2 grid, on all host
    cores, for as many steps as fit in budget_s.  Kind "reference": the
    reference's own array code (hydro/, mesh/, boundary*, analysis/ compiled
    from its sources against the host Kokkos/MPI stand-ins, OpenMP loops;
    oracle/_ref/libref_step_2d_cart.so) driven in the order of its time loop.
    Kind "port" (when that library is absent): the oracle, the same algorithm
    restated in C with OpenMP."""
    from heraclespp_b200 import setups
    from oracle import Oracle, RefStep, ref_step_path

    ncores = os.cpu_count() or 1
    kw = dict(gamma=1.4, limiter="VanLeer", riemann="HLLC", bc=["Periodic"] * 4)
    if ref_step_path(2).exists():
        RefStep.set_threads(2, "Cartesian", ncores)
        o = RefStep(2, [NX, NX], **kw)
        kind, what = "reference", "the reference's own array code on the host Kokkos/MPI stand-ins"
        threads = o.threads()
    else:
        Oracle.set_threads(ncores)
        o = Oracle(2, [NX, NX], **kw)
        kind, what = "port", "the FP64 oracle (C restatement)"
        threads = Oracle.get_threads()
    init = Oracle(2, [NX, NX], **kw)
    grid = setups.Grid.from_domain(init)
    rho, rhou, E, fx = init.init_from_prim(*setups.kelvin_helmholtz(grid))
    t0 = time.perf_counter()
    o.run(rho, rhou, E, fx, cfl=0.4, max_iter=1)
    one = time.perf_counter() - t0
    n = max(1, int(budget_s / max(one, 1e-3)))
    t0 = time.perf_counter()
    o.run(rho, rhou, E, fx, cfl=0.4, max_iter=n)
    el = time.perf_counter() - t0
    return {"value": n * cells_full / el * 1e-6, "unit": "Mcell-updates/s", "cores": threads, "kind": kind,
            "sample": f"{n} full steps of KH 2048^2 with {what}, {threads} OpenMP threads, {el:.1f} s"}


def adjoint_cost(torch, nsteps=400, n=512, k=32):
    """Gresho 512^2, 400 steps, checkpoint every 32: device time of one
    gradient (adjoint forward + backward) against one forward run."""
    from heraclespp_b200 import Domain, setups

    kw = dict(gamma=5.0 / 3.0, limiter="VanLeer", riemann="HLLC", bc=["Periodic"] * 4)
    out = {"config": f"gresho_vortex_2d_{n}x{n}_{nsteps}steps_checkpoint{k}", "buffers": "device"}
    for prec in ("fp64", "fp32_mixed"):
        d = Domain(2, [n, n], precision=prec, **kw)
        prim = setups.gresho_vortex(setups.Grid.from_domain(d))
        d.set_state_from_prim(*prim)
        d.run(cfl=0.4, nsteps=nsteps)
        dts = d.dt_log()[:nsteps]
        # the final adjoint and the gradient stay on the device, as the state
        # does in the forward run it is compared with
        lam = torch.zeros((4,) + d.shape3, dtype=torch.float64, device="cuda")
        lam[0] = 1.0
        grad = torch.zeros_like(lam)
        stream = torch.cuda.ExternalStream(d.stream_handle())

        def timed(fn):
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            fn()
            e1.record(stream)
            e1.synchronize()
            return e0.elapsed_time(e1)

        d.set_state_from_prim(*prim)
        d.run(nsteps=nsteps, dts=dts)  # warm the graphs
        d.set_state_from_prim(*prim)
        fwd = timed(lambda: d.run(nsteps=nsteps, dts=dts))
        def gradient():
            d.adjoint_forward(nsteps, dts=dts, precision=prec, checkpoint_every=k)
            d.adjoint_backward(lam, grad, device=True)

        d.set_state_from_prim(*prim)
        gradient()  # warm: checkpoint and segment buffers, the second stream
        d.set_state_from_prim(*prim)
        adj = timed(gradient)
        cells = n * n
        algo = cells * (nsteps * ADJ_BYTES_PER_CELL_STEP + (nsteps // k) * 64)
        out[prec] = {"forward_ms": fwd, "gradient_ms": adj, "adj_over_fwd": adj / fwd,
                     "gradient_algorithmic_gb": algo * 1e-9, "gradient_achieved_gbs": algo / (adj * 1e-3) * 1e-9,
                     "schedule": d.schedule()}
        d.close()
    return out


def stage_loop_cost(torch, steps=20):
    """KH 2048^2 with one passive scalar: the fused tile kernel carrying the
    scalar (FP64 and FP32-mixed) against the fused FP64 step without it and
    against hcl_run composed of the FP64 stage entry points (the reference's
    per-stage kernels, dt and health readbacks each step; hcl_set_stage_loop).
    Device time per step."""
    from heraclespp_b200 import Domain, setups

    kw = dict(gamma=1.4, limiter="VanLeer", riemann="HLLC", bc=["Periodic"] * 4)
    out = {"config": f"kelvin_helmholtz_2d_{NX}x{NX}_nfx1_{steps}steps"}
    runs = (("stage_loop_nfx1_fp64", 1, "fp64", True), ("fused_nfx1_fp64", 1, "fp64", False),
            ("fused_nfx1_fp32_mixed", 1, "fp32_mixed", False), ("fused_nfx0_fp64", 0, "fp64", False))
    for name, nfx, prec, staged in runs:
        d = Domain(2, [NX, NX], nfx=nfx, precision=prec, stage_loop=staged, **kw)
        grid = setups.Grid.from_domain(d)
        prim = setups.kelvin_helmholtz(grid)
        fx = None
        if nfx:
            s3, (X, Y, Z), _ = grid.interior()
            fx = np.zeros((nfx,) + prim[0].shape)
            fx[0][s3] = np.broadcast_to((np.abs(Y - 0.5) < 0.25).astype(float), fx[0][s3].shape)
        d.set_state_from_prim(*prim, fx=fx)
        d.run(cfl=0.4, nsteps=2)
        stream = torch.cuda.ExternalStream(d.stream_handle())
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        d.run(cfl=0.4, nsteps=steps)
        e1.record(stream)
        e1.synchronize()
        out[name] = {"ms_per_step": e0.elapsed_time(e1) / steps}
        if prec == "fp32_mixed":
            out[name]["schedule"] = d.schedule()
        d.close()
    fused = out["fused_nfx1_fp64"]["ms_per_step"]
    out["stage_over_fused_nfx1"] = out["stage_loop_nfx1_fp64"]["ms_per_step"] / fused
    out["fused_nfx1_over_nfx0"] = fused / out["fused_nfx0_fp64"]["ms_per_step"]
    return out


def rt3d_cost(torch, steps=500, nx=(256, 256, 512)):
    """3-D Rayleigh-Taylor 256x256x512 on [0,0.5]^2 x [0,1], g_z = -0.1,
    reflecting z walls, periodic x/y, HLL, Minmod: FP32-mixed run with its
    CFL dts, then the FP64 and fast FP64 steps with the same dts (device time
    of each, and the errors of mixed and fast FP64 against FP64 per field)."""
    from heraclespp_b200 import Domain, setups

    kw = dict(gamma=1.4, limiter="Minmod", riemann="HLL",
              bc=["Periodic", "Periodic", "Periodic", "Periodic", "Reflexive", "Reflexive"],
              g=(0.0, 0.0, -0.1), xmax=(0.5, 0.5, 1.0))
    cells = nx[0] * nx[1] * nx[2]
    out = {"config": f"rayleigh_taylor_3d_{nx[0]}x{nx[1]}x{nx[2]}_minmod_hll_{steps}steps", "cells": cells,
           "bytes_per_cell": 80}
    dm = Domain(3, list(nx), precision="fp32_mixed", **kw)
    prim = setups.rayleigh_taylor_3d(setups.Grid.from_domain(dm))
    dm.set_state_from_prim(*prim)
    dm.run(cfl=0.4, nsteps=3)  # warm-up (tuning, graphs)
    dm.set_state_from_prim(*prim)
    stream = torch.cuda.ExternalStream(dm.stream_handle())
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    dm.run(cfl=0.4, nsteps=steps)
    e1.record(stream)
    e1.synchronize()
    t_mixed = e0.elapsed_time(e1) * 1e-3
    dts = dm.dt_log()[:steps]
    st_m = dm.get_state()
    dm.close()
    d64 = Domain(3, list(nx), precision="fp64", **kw)
    d64.set_state_from_prim(*prim)
    d64.run(nsteps=3, dts=dts[:3])
    d64.set_state_from_prim(*prim)
    stream = torch.cuda.ExternalStream(d64.stream_handle())
    torch.cuda.synchronize()
    e0.record(stream)
    d64.run(nsteps=steps, dts=dts)
    e1.record(stream)
    e1.synchronize()
    t_64 = e0.elapsed_time(e1) * 1e-3
    st_64 = d64.get_state()
    d64.close()
    dfa = Domain(3, list(nx), precision="fp64_fast", **kw)
    dfa.set_state_from_prim(*prim)
    dfa.run(nsteps=3, dts=dts[:3])
    dfa.set_state_from_prim(*prim)
    stream = torch.cuda.ExternalStream(dfa.stream_handle())
    torch.cuda.synchronize()
    e0.record(stream)
    dfa.run(nsteps=steps, dts=dts)
    e1.record(stream)
    e1.synchronize()
    t_fa = e0.elapsed_time(e1) * 1e-3
    st_fa = dfa.get_state()
    dfa.close()
    out["fp32_mixed"] = {"mcups": steps * cells / t_mixed * 1e-6, "ms_per_step": t_mixed / steps * 1e3,
                         "achieved_gbs": 80 * cells / (t_mixed / steps) * 1e-9}
    out["fp64"] = {"mcups": steps * cells / t_64 * 1e-6, "ms_per_step": t_64 / steps * 1e3,
                   "achieved_gbs": 80 * cells / (t_64 / steps) * 1e-9}
    out["fp64_fast"] = {"mcups": steps * cells / t_fa * 1e-6, "ms_per_step": t_fa / steps * 1e3,
                        "achieved_gbs": 80 * cells / (t_fa / steps) * 1e-9}
    out["speedup_mixed_vs_fp64"] = t_64 / t_mixed
    out["speedup_mixed_vs_fp64_fast"] = t_fa / t_mixed
    out["accuracy"] = {"steps_compared": int(len(dts)), "reference": "FP64 fused step, same dts",
                       "fields": field_errors(st_m, st_64, 2), "fp64_fast_fields": field_errors(st_fa, st_64, 2)}
    return out


ENSEMBLE_SIDES = (128, 256, 512, 1024)


def ensemble_cost(torch, nprob=96, nsteps=300, k=20, seed=2024, rank=0, world=1):
    """96 independent 2-D four-quadrant Riemann problems (sides drawn from
    {128, 256, 512, 1024}, seeded), outflow, Minmod, HLLC, FP32-mixed,
    300 steps: one persistent graph-replayed launch against looping the
    single-problem step (each problem's own hcl_run), then the adjoint of
    the sum of the final total energies.  Wall-clock of synchronous calls.
    With world > 1 the problems are sharded over the ranks (cost-balanced),
    times are the maximum over ranks and the objective is summed."""
    from heraclespp_b200 import Domain, Ensemble, setups
    from heraclespp_b200.sharding import partition, problem_cost, torch_reducers, total_energy

    rng = np.random.default_rng(seed)
    sides = [(int(rng.choice(ENSEMBLE_SIDES)), int(rng.choice(ENSEMBLE_SIDES))) for _ in range(nprob)]
    cells = sum(a * b for a, b in sides)
    mine = partition([problem_cost(s, nsteps) for s in sides], world)[rank]
    if world > 1:
        rsum, rmax = torch_reducers(device="cuda")
    else:
        rsum = rmax = (lambda x: x)  # noqa: E731
    my_sides = [sides[p] for p in mine]
    kw = dict(gamma=1.4, limiter="Minmod", riemann="HLLC", bc=["NullGradient"] * 4)
    ens = Ensemble([dict(nx=list(s), **kw) for s in my_sides])
    prims = [setups.four_quadrant(setups.Grid.from_domain(d), seed=1000 + p) for p, d in zip(mine, ens.domains)]

    def reset(doms):
        for d, prim in zip(doms, prims):
            d.set_state_from_prim(*prim)

    def wall(fn):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        out = fn()
        torch.cuda.synchronize()
        return rmax(time.perf_counter() - t0), out

    reset(ens.domains)
    ens.run(nsteps)  # autotune, capture
    reset(ens.domains)
    t_ens, r = wall(lambda: ens.run(nsteps))
    energy = rsum(sum(total_energy(d) for d in ens.domains))
    out = {"config": f"{nprob} four-quadrant problems, sides from {list(ENSEMBLE_SIDES)} (seed {seed}), "
                     f"{cells} cells, {nsteps} steps, Minmod, HLLC, outflow, fp32_mixed",
           "cells": cells, "ranks": world, "problems_on_rank0": len(mine),
           "final_total_energy": energy,
           "ensemble": {"ms": t_ens * 1e3, "mcups": cells * nsteps / t_ens * 1e-6, "strip_rows": r.strip_rows,
                        "blocks_per_sm": r.blocks_per_sm, "warps_per_cta": r.warps_per_cta, "grid": r.grid,
                        "launches": r.launches,
                        "graph": bool(r.graph)}}
    # looping the single-problem step (each problem graph-replays its own steps)
    doms = [Domain(2, list(s), precision="fp32_mixed", **kw) for s in my_sides]
    reset(doms)
    for d in doms:
        d.run(cfl=0.4, nsteps=nsteps)  # autotune, capture
    reset(doms)
    t_loop, _ = wall(lambda: [d.run(cfl=0.4, nsteps=nsteps) for d in doms])
    out["loop"] = {"ms": t_loop * 1e3, "mcups": cells * nsteps / t_loop * 1e-6}
    out["ensemble_over_loop"] = t_loop / t_ens
    # adjoint of J = sum_p sum_cells E dV
    lams = []
    for d in ens.domains:
        lam = torch.zeros((4,) + d.shape3, dtype=torch.float64, device="cuda")
        dv = torch.from_numpy(d.grid()["dv"]).cuda()
        lam[3, :, 2:-2, 2:-2] = dv[:, 2:-2, 2:-2]
        lams.append(lam)
    grads = [torch.empty_like(x) for x in lams]
    torch.cuda.synchronize()
    for prec in ("fp64", "fp32_mixed"):
        reset(ens.domains)
        ens.run(nsteps, checkpoint_every=k, adjoint_precision=prec)
        ens.adjoint(lams, grads)  # allocate the sweep buffers
        reset(ens.domains)
        t_f, _ = wall(lambda: ens.run(nsteps, checkpoint_every=k, adjoint_precision=prec))
        t_b, _ = wall(lambda: ens.adjoint(lams, grads))
        out[f"adjoint_{prec}"] = {"forward_ckpt_ms": t_f * 1e3, "backward_ms": t_b * 1e3,
                                  "adj_over_fwd": (t_f + t_b) / t_ens, "checkpoint_every": k}
    ens.close()
    # looping the single-problem adjoint (FP32 sweep) over the same problems
    def loop_adjoint():
        for d, lam, gr in zip(doms, lams, grads):
            d.adjoint_forward(nsteps, cfl=0.4, checkpoint_every=k, precision="fp32_mixed")
            d.adjoint_backward(lam, gr, device=True)

    reset(doms)
    loop_adjoint()  # allocate
    reset(doms)
    t_la, _ = wall(loop_adjoint)
    out["loop_adjoint_fp32_mixed_ms"] = t_la * 1e3
    ens_adj = out["adjoint_fp32_mixed"]
    out["adjoint_ensemble_over_loop"] = t_la * 1e3 / (ens_adj["forward_ckpt_ms"] + ens_adj["backward_ms"])
    for d in doms:
        d.close()
    return out


def dist_setup(args):
    import torch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch.distributed as dist

        backend = "nccl" if args.impl == "ours" else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
    return world, rank, local


def run_reference(args):
    world, rank, local = dist_setup(args)
    if rank != 0:
        if world > 1:
            import torch.distributed as dist

            dist.barrier()
            dist.destroy_process_group()
        return
    base = cpu_baseline(min(args.cpu_budget * 3, 60.0))
    line = {"metric": "Mcell-updates/s", "value": base["value"], "unit": "Mcell-updates/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "impl": "reference",
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "cells": CELLS, "precision": "fp64"},
            "cpu_baseline": base,
            "e2e": {"value": base["value"], "unit": "Mcell-updates/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist

        dist.barrier()
        dist.destroy_process_group()


def run_ours(args):
    import torch

    world, rank, local = dist_setup(args)
    import heraclespp_b200 as hb

    dev_index = local
    os.environ.setdefault("CUDA_DEVICE_ORDER", "PCI_BUS_ID")
    torch.cuda.set_device(dev_index)
    peaks, peaks_kind = measured_peaks()
    hbm_peak = float(peaks.get("hbm_gbs", 6650.0))

    # ---- FP32-mixed headline --------------------------------------------
    d, prim = kh_domain("fp32_mixed")
    d.h  # noqa: B018
    d.set_state_from_prim(*prim)
    launches0 = hb.kernel_launch_count()
    if world > 1:
        import torch.distributed as dist

        dist.barrier()
    with ClockSampler(int(os.environ.get("HCL_NVSMI_INDEX", dev_index)), pci_bus_id(torch, dev_index)) as clk:
        el_mixed, r_mixed = time_fused(torch, d, args.steps, args.warmup, clk)
    launches = hb.kernel_launch_count() - launches0 - args.warmup

    # ---- FP64 fused step, same workload ---------------------------------------
    d64, _ = kh_domain("fp64")
    d64.set_state_from_prim(*prim)
    el_64, _ = time_fused(torch, d64, args.steps, args.warmup)
    d64.close()
    dfast, _ = kh_domain("fp64_fast")
    dfast.set_state_from_prim(*prim)
    el_fast, _ = time_fused(torch, dfast, args.steps, args.warmup)
    dfast.close()
    # accuracy of mixed vs FP64 over the config's step count, every field
    accuracy = kh_accuracy(prim, args.accuracy_steps)

    # ---- end to end through the C ABI with host buffers ----------------------
    pinned = [torch.empty(s, dtype=torch.float64).pin_memory() for s in (d.shape3, (2,) + d.shape3, d.shape3)]
    host = d.get_state()
    for t_, h_ in zip(pinned, host):
        t_.numpy()[...] = h_
    chunk = args.e2e_chunk
    reps = max(1, args.steps // chunk)
    torch.cuda.synchronize()
    stream = torch.cuda.ExternalStream(d.stream_handle())
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(reps):
        d.set_state(*[t_.numpy() for t_ in pinned])
        d.run(cfl=0.4, nsteps=chunk)
        d.get_state(out=tuple(t_.numpy() for t_ in pinned))
    e1.record(stream)
    e1.synchronize()
    el_e2e = e0.elapsed_time(e1) * 1e-3
    state_bytes = sum(int(np.prod(t_.shape)) * 8 for t_ in pinned)
    # the same with the whole state copied in and out around every single step
    n1 = max(1, min(args.steps, 10))
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(n1):
        d.set_state(*[t_.numpy() for t_ in pinned])
        d.run(cfl=0.4, nsteps=1)
        d.get_state(out=tuple(t_.numpy() for t_ in pinned))
    e1.record(stream)
    e1.synchronize()
    el_e2e1 = e0.elapsed_time(e1) * 1e-3

    # ---- cross-rank aggregation -------------------------------------------
    el_max, el64_max, e2e_max, e2e1_max, elf_max = el_mixed, el_64, el_e2e, el_e2e1, el_fast
    if world > 1:
        import torch.distributed as dist

        t = torch.tensor([el_mixed, el_64, el_e2e, el_e2e1, el_fast], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        el_max, el64_max, e2e_max, e2e1_max, elf_max = (float(v) for v in t.tolist())

    value = world * args.steps * CELLS / el_max * 1e-6
    value64 = world * args.steps * CELLS / el64_max * 1e-6
    value_fast = world * args.steps * CELLS / elf_max * 1e-6
    e2e_val = world * reps * chunk * CELLS / e2e_max * 1e-6
    ms_per_step = el_max / args.steps * 1e3
    achieved = BYTES_PER_CELL * CELLS / (el_mixed / args.steps) * 1e-9  # GB/s per launch
    traffic = read_traffic()
    line = {
        "metric": "Mcell-updates/s", "value": value, "unit": "Mcell-updates/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "fp32-mixed (f32 fluxes, f64 state)", "data": "synthetic",
        "config": {"workload": WORKLOAD, "cells": CELLS, "precision": "fp32_mixed", "parallelism": "replicas",
                   "l2": "inputs larger than L2 (state 134 MB read + 134 MB written per step)",
                   "e2e_steps_per_call": chunk, "schedule": d.schedule(),
                   "warmup_steps_run": (args.warmup + 5) // 6 * 6},
        "fp64": {"value": value64, "ms_per_step": el64_max / args.steps * 1e3, "unit": "Mcell-updates/s"},
        "fp64_fast": {"value": value_fast, "ms_per_step": elf_max / args.steps * 1e3, "unit": "Mcell-updates/s",
                      "what": "all FP64, FMA contraction, perfect gas without the temperature round trip"},
        "speedup_mixed_vs_fp64": value / value64,
        "speedup_mixed_vs_fp64_fast": value / value_fast,
        "accuracy": accuracy,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm_peak, "unit": "GB/s",
                     "frac": achieved / hbm_peak, "traffic": traffic,
                     "peak_spec": HBM_SPEC_GBS, "frac_of_spec": achieved / HBM_SPEC_GBS,
                     "peak_source": f"{peaks_kind} (MEASURED_PEAKS.json hbm_gbs)" if peaks_kind == "measured"
                     else "fallback 6.65 TB/s",
                     "bytes_per_cell": BYTES_PER_CELL, "cells_per_launch": CELLS},
        "e2e": {"value": e2e_val, "unit": "Mcell-updates/s", "h2d_bytes_per_step": state_bytes / chunk,
                "d2h_bytes_per_step": state_bytes / chunk + 96},
        "e2e_state_copied_every_step": {"value": world * n1 * CELLS / e2e1_max * 1e-6, "unit": "Mcell-updates/s",
                                        "steps": n1, "h2d_bytes_per_step": state_bytes,
                                        "d2h_bytes_per_step": state_bytes + 96},
        "gpu_launches": int(launches),
        "clocks": clk.summary(),
    }
    if rank == 0 and not args.no_adjoint:
        line["adjoint"] = adjoint_cost(torch)
    if not args.no_ensemble:
        ens = ensemble_cost(torch, rank=rank, world=world)
        if rank == 0:
            line["ensemble"] = ens
    if rank == 0 and not args.no_rt3d:
        line["rt3d"] = rt3d_cost(torch, steps=args.rt3d_steps)
    if rank == 0 and not args.no_stage_loop:
        line["stage_loop"] = stage_loop_cost(torch)
    if rank == 0 and not args.no_cpu_baseline and world == 1:
        line["cpu_baseline"] = cpu_baseline(args.cpu_budget)
    d.close()
    if world > 1:
        import torch.distributed as dist

        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
