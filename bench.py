#!/usr/bin/env python
"""Benchmark: 2D radial acoustics, FP64, 4096^2 cells, t_final = 0.6.

One "step" is one claw2 call over one output interval (dtout = t_final/20,
the unit in which claw2ez hands the state back to the host), i.e. ~137
time steps of the fused step2 kernel at 4096^2.  --steps 20 times the whole
run from t=0 to t=0.6.  The metric is cell-updates/s: accepted time steps x
cells / device time.

  value    : state resident in HBM, frames driven through the library's
             claw_advance (device-side dt control, CUDA-graph time loop)
  e2e      : the same frames through claw_advance_host, i.e. with the
             host->device copy of q (pinned) before and the device->host copy
             after every frame inside the timed region
  roofline : the step kernel's algorithmic bytes (read q + write q,
             48 B per cell-update) / its time per executed step (CUDA events
             on the library's stream over the timed frames / accepted +
             rejected steps); traffic from the kernel's ncu capture
  variants : the same frames on the reference-order FP64 kernel (bit-identical
             to the CPU restatement) and on the FP32 path
  cpu_baseline : the CPU restatement of step2/flux2 (the oracle) timed on
             this host on a bounded sample (whole 4096^2 steps; one core as
             the reference's serial step2, and all cores threaded beside it)
  other_configs : the other workloads (1D, 2D 1024^2, 3D 256^3 / 512^3, the
             split steps, one 2048^2 Euler grid, the Euler ensemble, the
             learned corrector, the time to an L1 error per precision), each
             with its roofline and, where the reference has a CPU path, a
             CPU baseline

The headline arithmetic is FP64 with fused multiply-adds in characteristic
variables (precision "fp64_fma"): the same algorithm and dt sequence as the
reference-order path, within 1e-12 relative of it over the full run.

--impl reference times that CPU restatement alone on the same metric, on every
host thread the process may use (the slices of a sweep spread over them; the
reference's own 2D step is serial, and its one-core figure is reported beside).
Under torchrun with N > 1 each rank runs an independent replica (the
workload fits one GPU and does not shard), value = all ranks' cell-updates /
max time over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_CELLS = 4096
NOUT = 20
TFINAL = 0.6
PEAKS_FALLBACK = {"hbm_gbs": 6650.0, "source": "fallback"}


def traffic_per_launch(precision, cells):
    """DRAM bytes (read + write) per launch of the step kernel, scaled from
    the ncu capture summarised in profiles/ (bytes per cell-update at a size
    larger than L2); None when no capture is recorded."""
    key = {"fp64_fma": "step2_char_kernel_fp64_fma", "fp64": "step2_kernel_fp64",
           "fp32": "step2_char_kernel_fp32"}[precision]
    bpc, _ = kernel_stats(key)
    return bpc * cells if bpc is not None else None


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return {"hbm_gbs": float(d["hbm_gbs"]), "source": "measured"}
    return PEAKS_FALLBACK


class ClockSampler:
    """SM clocks, power and clock-event (throttle) reasons sampled during the
    timed region: NVML read in-process every 10 ms (the GPU this process runs
    on, mapped through CUDA_VISIBLE_DEVICES), else `nvidia-smi -lms 200`.
    Only reads; changes no setting."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    # NVML clock-event reason bits (nvml.h): SwPowerCap 0x4, HwSlowdown 0x8,
    # SwThermalSlowdown 0x20, HwThermalSlowdown 0x40
    BITS = (("hw_slowdown", 0x8), ("hw_thermal_slowdown", 0x40),
            ("sw_thermal_slowdown", 0x20), ("sw_power_cap", 0x4))

    def __init__(self, device):
        self.device = device
        self.rows = []  # (sm MHz, max sm MHz, power W, reason bits)
        self.proc = None
        self.thread = None
        self.nvml = None
        self.halt = threading.Event()
        self.first = threading.Event()

    def _nvml_start(self):
        import pynvml
        import torch
        pynvml.nvmlInit()
        try:
            idx = torch.cuda._get_nvml_device_index(self.device)
        except Exception:
            idx = self.device
        h = pynvml.nvmlDeviceGetHandleByIndex(idx)
        reasons = getattr(pynvml, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
            pynvml.nvmlDeviceGetCurrentClocksThrottleReasons
        smax = float(pynvml.nvmlDeviceGetMaxClockInfo(h, pynvml.NVML_CLOCK_SM))
        self.nvml = pynvml

        def loop():
            while not self.halt.is_set():
                try:
                    sm = float(pynvml.nvmlDeviceGetClockInfo(h, pynvml.NVML_CLOCK_SM))
                    pw = pynvml.nvmlDeviceGetPowerUsage(h) / 1000.0
                    self.rows.append((sm, smax, pw, int(reasons(h))))
                except pynvml.NVMLError:
                    pass
                self.first.set()
                self.halt.wait(0.01)

        self.thread = threading.Thread(target=loop, daemon=True)
        self.thread.start()
        self.first.wait(2.0)

    def start(self):
        try:
            self._nvml_start()
            return
        except Exception:
            self.nvml = None
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except (FileNotFoundError, OSError):
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9 and parts[1].replace(".", "").isdigit():
                bits = 0
                for k, (_, bit) in enumerate(self.BITS):
                    if "Active" in parts[5 + k] and "Not" not in parts[5 + k]:
                        bits |= bit
                pw = float(parts[3]) if parts[3].replace(".", "").isdigit() else float("nan")
                self.rows.append((float(parts[1]), float(parts[2]), pw, bits))

    def stop(self):
        if self.nvml is not None:
            self.halt.set()
            self.thread.join(timeout=2)
            try:
                self.nvml.nvmlShutdown()
            except Exception:
                pass
            source = "nvml, 10 ms"
        elif self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            if self.thread:
                self.thread.join(timeout=2)
            source = "nvidia-smi, 200 ms"
        else:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["clock sampling unavailable"]}
        rows = list(self.rows)
        reasons = sorted({n for r in rows for n, bit in self.BITS if r[3] & bit})
        pw = [r[2] for r in rows if r[2] == r[2]]
        return {"sm_mhz": float(np.median([r[0] for r in rows])) if rows else None,
                "sm_max_mhz": max(r[1] for r in rows) if rows else None,
                "power_w": float(np.median(pw)) if pw else None,
                "reasons": reasons, "samples": len(rows), "source": source}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def reduce_over_ranks(x, op, world, device):
    """max or sum of a float over the ranks (NCCL on the GPU run; any
    initialised process group works, gloo with device 'cpu')."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX if op == "max" else dist.ReduceOp.SUM)
    return float(t.item())


def whole_job_rate(updates_local, ms_local, world, device):
    """Replicas (weak scaling): the cell-updates of all ranks over the
    slowest rank's device time.  Returns (rate, max ms, total updates)."""
    ms_max = reduce_over_ranks(ms_local, "max", world, device)
    total = reduce_over_ranks(updates_local, "sum", world, device)
    return total / (ms_max * 1e-3), ms_max, total


def host_cpu():
    """The host's CPU model and logical core count (lscpu / os.cpu_count)."""
    model = None
    try:
        out = subprocess.run(["lscpu"], capture_output=True, text=True, timeout=10).stdout
        for line in out.splitlines():
            if line.startswith("Model name:"):
                model = line.split(":", 1)[1].strip()
                break
    except (OSError, subprocess.SubprocessError):
        pass
    return {"model": model, "nproc": os.cpu_count()}


def cpu_reference_sample(n, nsteps, threads=1):
    """Time the CPU restatement (oracle, speed build) on nsteps whole n^2
    steps of the workload with `threads` host threads (the slices of a sweep
    spread over them); returns (cell-updates/s, seconds, threads)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from classic_b200 import problems
    from pyoracle import OracleGrid
    rd, solver, params, q0, _ = problems.radial_acoustics_2d(n=n)
    g = OracleGrid(rd.clawdata, solver, params, variant="fast")
    g.lib.orc_set_threads(threads)
    try:
        g.set_q(q0)
        dt = 0.9 * (2.0 / n) / 2.0
        t0 = time.perf_counter()
        for _ in range(nsteps):
            g.step(dt)
        sec = time.perf_counter() - t0
    finally:
        g.lib.orc_set_threads(1)
    return n * n * nsteps / sec, sec, threads


def host_threads():
    """Host threads this process may run on."""
    try:
        return len(os.sched_getaffinity(0))
    except (AttributeError, OSError):
        return os.cpu_count() or 1


def run_reference_arm(args):
    world, rank, local = dist_setup()
    if rank != 0:
        return 0
    n = N_CELLS
    nt = host_threads()
    for _ in range(args.warmup):
        cpu_reference_sample(n, 1, nt)
    rates, secs = [], 0.0
    for _ in range(args.steps):
        r, s, cores = cpu_reference_sample(n, 1, nt)
        rates.append(r)
        secs += s
    value = n * n * args.steps / secs
    r1, s1, _ = cpu_reference_sample(n, 1, 1)  # the reference's own serial step, for scale
    line = {
        "metric": "cell-updates/s", "value": value, "unit": "cell-updates/s",
        "impl": "reference", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * secs / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"2D radial acoustics FP64 {n}^2, MC, transverse 2",
                   "step": f"one whole {n}^2 time step (bounded sample of a frame)"},
        "cpu_baseline": {"value": value, "unit": "cell-updates/s", "cores": nt, "kind": "port",
                         "sample": f"{args.steps} whole {n}^2 steps of the CPU restatement with "
                                   f"the slices of each sweep spread over {nt} host threads (the "
                                   "reference's 2D step itself is serial)", "host": host_cpu(),
                         "one_core": {"value": r1, "cores": 1,
                                      "sample": f"1 whole {n}^2 step on one core ({s1:.1f} s)"}},
        "e2e": {"value": value, "unit": "cell-updates/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def kernel_stats(key):
    """DRAM bytes and FP64 thread-operations per cell-update of one kernel
    (one step), scaled from the ncu captures summarised in profiles/ (sizes
    larger than L2); (None, None) when no capture is recorded."""
    p = os.path.join(ROOT, "profiles", "dram_bytes_per_cell.txt")
    if not os.path.exists(p):
        return None, None
    for line in open(p):
        parts = line.split()
        if len(parts) >= 2 and not line.startswith("#") and parts[0] == key:
            fp64 = float(parts[2]) if len(parts) >= 3 and parts[2] != "-" else None
            return float(parts[1]), fp64
    return None, None


def roofline_entry(rate, alg_bytes, peaks, key=None, fp64_peak=None):
    """Roofline of a side workload from its cell-update rate: algorithmic
    bytes per cell x rate against the measured HBM copy bandwidth; the DRAM
    traffic and FP64 operations per cell from the kernel's ncu capture when
    one is recorded, and then the FP64 fraction against the probed FMA peak."""
    achieved = rate * alg_bytes / 1e9
    out = {"bound": "hbm", "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
           "frac": achieved / peaks["hbm_gbs"], "algorithmic_bytes_per_cell": alg_bytes,
           "traffic_bytes_per_cell": None, "peak_source": peaks["source"]}
    if key:
        tb, fp64 = kernel_stats(key)
        out["traffic_bytes_per_cell"] = tb
        if fp64 is not None and fp64_peak:
            # FP64 pipe: thread-instructions per second against the probe's
            # (an FMA is one instruction and two flops)
            out["fp64_inst_per_cell"] = fp64
            out["fp64_tinst_per_s"] = rate * fp64 / 1e12
            out["fp64_tinst_peak"] = fp64_peak / 2.0
            out["fp64_frac"] = rate * fp64 / 1e12 / (fp64_peak / 2.0)
            if out["fp64_frac"] > out["frac"]:
                out["bound"] = "fp64"
    return out


def cpu_rate(make, steps, threads, dt):
    """cell-updates/s of the CPU restatement (speed build, `threads` host
    threads) over `steps` whole steps of one grid; returns (rate, seconds)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from pyoracle import OracleGrid
    rd, solver, params, q0, aux = make()
    g = OracleGrid(rd.clawdata, solver, params, variant="fast")
    g.lib.orc_set_threads(threads)
    try:
        g.set_q(q0)
        if aux is not None:
            g.set_aux(aux)
        cells = int(np.prod(rd.clawdata.num_cells))
        t0 = time.perf_counter()
        for _ in range(steps):
            g.step(dt)
        sec = time.perf_counter() - t0
    finally:
        g.lib.orc_set_threads(1)
    return cells * steps / sec, sec


def other_configs(peaks, cpu=True):
    """The other workloads of the suite, measured once each after the
    headline (device time from CUDA events inside the library), each with
    its roofline and a CPU baseline of the restatement on this host (a
    bounded sample; one core, and all cores where the reference's path is
    threaded -- its 3D step is OpenMP-parallel, its 1D and 2D steps serial):
    1D acoustics (800 cells, 10 frames to t=1), 2D radial acoustics at
    1024^2 (first frame), 3D heterogeneous acoustics (256^3 and 512^3, the
    first frame t=0..0.1; FP64 reference order, contracted FP64, FP32), the
    dimensionally split steps (2D radial 4096^2 to t=0.03, Godunov and
    Strang; 3D 256^3 Godunov, first frame) and the batched 2D Euler ensemble
    (256 instances, sides log-uniform in 128..1024, to t=0.25)."""
    from classic_b200 import _lib, problems
    from classic_b200.solver import BatchSolver, Solver
    import ctypes
    out = {}
    nproc = os.cpu_count() or 1
    fp64_peak = None
    try:
        tf, msb = ctypes.c_double(0.0), ctypes.c_double(0.0)
        if _lib.load().claw_probe_fp64(ctypes.byref(tf), ctypes.byref(msb)) == 0:
            fp64_peak = tf.value
            out["fp64_fma_probe"] = {"tflops": tf.value, "ms": msb.value,
                                     "what": "independent FP64 FMA chains, 2 flops per FMA"}
    except Exception as e:
        out["fp64_fma_probe"] = {"error": str(e)}
    try:
        rd, solver, params, q0, _ = problems.acoustics_1d_config()
        s = Solver(rd.clawdata, solver, params)
        s.set_q(q0)
        t, dt, steps, ms = 0.0, float(rd.clawdata.dt_initial), 0, 0.0
        for _ in range(10):
            info, st = s.advance(t, t + 0.1, dt)
            t, dt = st["t_reached"], st["dt_next"]
            steps += st["steps_taken"]
            ms += st["device_ms"]
        s.close()
        rate = 800 * steps / (ms * 1e-3)
        e = {"cell_updates_per_s": rate, "steps": steps, "device_ms": ms,
             "note": "one CTA runs the whole claw1 loop per frame (latency-bound, one SM); "
                     "q (12.8 KB) stays on chip, so no DRAM traffic figure applies",
             "roofline": roofline_entry(rate, 32, peaks)}
        if cpu:
            sys.path.insert(0, os.path.join(ROOT, "oracle"))
            from pyoracle import OracleGrid
            o = OracleGrid(rd.clawdata, solver, params, variant="fast")
            o.set_q(q0)
            t0 = time.perf_counter()
            t, dt, osteps = 0.0, float(rd.clawdata.dt_initial), 0
            for _ in range(10):
                info, so = o.advance(t, t + 0.1, dt)
                t, dt = so["t_reached"], so["dt_next"]
                osteps += so["steps_taken"]
            sec = time.perf_counter() - t0
            e["cpu_baseline"] = {"value": 800 * osteps / sec, "unit": "cell-updates/s", "cores": 1,
                                 "kind": "port", "sample": f"the whole run ({osteps} steps, {sec:.2f} s)"}
        out["acoustics_1d_800"] = e
    except Exception as e:  # a failed side measurement must not hide the headline
        out["acoustics_1d_800"] = {"error": str(e)}
    # 2D radial acoustics at 1024^2: the first frame (t = 0 .. 0.03)
    for prec in ("fp64", "fp64_fma", "fp32"):
        key = f"radial_2d_1024_{prec}"
        try:
            rd, solver, params, q0, _ = problems.radial_acoustics_2d(n=1024)
            s = Solver(rd.clawdata, solver, params, precision=prec)
            s.set_q(q0)
            s.advance(0.0, 0.03, 0.01)  # warm-up frame
            s.set_q(q0)
            info, st = s.advance(0.0, 0.03, 0.01)
            s.close()
            ex = st["steps_taken"] + st["steps_rejected"]
            rate = 1024 ** 2 * ex / (st["device_ms"] * 1e-3)
            es = 4 if prec == "fp32" else 8
            kern = {"fp64": "step2_kernel_fp64", "fp64_fma": "step2_char_kernel_fp64_fma",
                    "fp32": "step2_char_kernel_fp32"}[prec]
            e = {"cell_updates_per_s": rate, "steps": st["steps_taken"], "device_ms": st["device_ms"],
                 "l2": "q (25 MB per FP64 buffer) fits in L2: the rate is not HBM-bound at this size",
                 "roofline": roofline_entry(rate, 6 * es, peaks, kern, fp64_peak)}
            if cpu and prec == "fp64":
                mk = lambda: problems.radial_acoustics_2d(n=1024)[:4] + (None,)
                r1, s1 = cpu_rate(mk, 5, 1, 0.0008)
                rn, sn = cpu_rate(mk, 10, nproc, 0.0008)
                e["cpu_baseline"] = {"value": r1, "unit": "cell-updates/s", "cores": 1, "kind": "port",
                                     "sample": f"5 whole 1024^2 steps from the initial data ({s1:.1f} s); "
                                               "the reference's 2D step is serial",
                                     "threaded": {"value": rn, "cores": nproc,
                                                  "sample": f"10 steps ({sn:.1f} s), every third slice in parallel"}}
            out[key] = e
        except Exception as e:
            out[key] = {"error": str(e)}
    for n in (256, 512):
        for prec in ("fp64", "fp64_fma", "fp32"):
            key = f"hetero_acoustics_3d_{n}_{prec}"
            try:
                rd, solver, params, q0, aux = problems.heterogeneous_acoustics_3d(n=n)
                s = Solver(rd.clawdata, solver, params, precision=prec)
                s.set_q(q0)
                s.set_aux(aux)
                info, st = s.advance(0.0, 0.1, 0.01)
                s.close()
                n3 = n ** 3
                upd = n3 * (st["steps_taken"] + st["steps_rejected"])
                es = 4 if prec == "fp32" else 8
                rate = upd / (st["device_ms"] * 1e-3)
                kern = {"fp64": "sweep3p_fp64", "fp64_fma": "sweep3f_fp64_fma",
                        "fp32": "sweep3f_fp32"}[prec]
                e = {"cell_updates_per_s": rate, "steps": st["steps_taken"],
                     "device_ms": st["device_ms"],
                     "roofline": roofline_entry(rate, 10 * es, peaks, kern, fp64_peak)}
                if cpu and prec == "fp64" and n == 256:
                    mk_s = lambda: problems.heterogeneous_acoustics_3d(n=96)
                    mk_n = lambda: problems.heterogeneous_acoustics_3d(n=256)
                    r1, s1 = cpu_rate(mk_s, 1, 1, 0.002)
                    rn, sn = cpu_rate(mk_n, 1, nproc, 0.002)
                    e["cpu_baseline"] = {
                        "value": rn, "unit": "cell-updates/s", "cores": nproc, "kind": "port",
                        "sample": f"1 whole 256^3 step on {nproc} threads ({sn:.1f} s): the reference's "
                                  "step3 is OpenMP-parallel over 2x2 colour blocks, restated the same way",
                        "one_core": {"value": r1, "cores": 1,
                                     "sample": f"1 whole step of the same problem at 96^3 ({s1:.1f} s)"}}
                out[key] = e
            except Exception as e:
                out[key] = {"error": str(e)}
    # other methods of the same workload on the characteristic kernel: transverse
    # 1; minmod, superbee and van Leer compiled in (FP64 contracted and FP32);
    # MC / van Leer on the two waves (a compiled pair) and MC / none (read at
    # run time).  4096^2; a first frame
    # (t 0 -> 0.02) warms up, the next (0.02 -> 0.05) is timed.
    char_kern = "step2_char_kernel"
    for key, trans, lims, prec, kern, tkey in (
            ("radial_2d_4096_trans1_fp64_fma", 1, ["mc", "mc"], "fp64_fma", char_kern + " (order 2, transverse 1)",
             "step2_char_kernel_fp64_fma_trans1"),
            ("radial_2d_4096_minmod_fp64_fma", 2, ["minmod", "minmod"], "fp64_fma", char_kern,
             "step2_char_kernel_fp64_fma_minmod"),
            ("radial_2d_4096_superbee_fp64_fma", 2, ["superbee", "superbee"], "fp64_fma", char_kern,
             "step2_char_kernel_fp64_fma_superbee"),
            ("radial_2d_4096_vanleer_fp64_fma", 2, ["vanleer", "vanleer"], "fp64_fma", char_kern,
             "step2_char_kernel_fp64_fma_vanleer"),
            ("radial_2d_4096_vanleer_fp32", 2, ["vanleer", "vanleer"], "fp32", char_kern,
             "step2_char_kernel_fp32_vanleer"),
            ("radial_2d_4096_mixed_limiters_fp64_fma", 2, ["mc", "vanleer"], "fp64_fma",
             char_kern + " (MC on wave 1, van Leer on wave 2, compiled in)", "step2_char_kernel_fp64_fma_mc_vanleer"),
            ("radial_2d_4096_runtime_limiters_fp64_fma", 2, ["mc", "none"], "fp64_fma",
             char_kern + " (limiters read at run time)", "step2_char_kernel_fp64_fma_runtime")):
        try:
            rd, solver, params, q0, _ = problems.radial_acoustics_2d(n=4096)
            rd.clawdata.transverse_waves = trans
            rd.clawdata.limiter = lims
            s = Solver(rd.clawdata, solver, params, precision=prec)
            s.set_q(q0)
            info, st = s.advance(0.0, 0.02, 0.01)
            info, st = s.advance(0.02, 0.05, st["dt_next"])
            s.close()
            rate = 4096 ** 2 * (st["steps_taken"] + st["steps_rejected"]) / (st["device_ms"] * 1e-3)
            out[key] = {"cell_updates_per_s": rate, "steps": st["steps_taken"], "device_ms": st["device_ms"],
                        "kernel": kern, "limiters": lims,
                        "roofline": roofline_entry(rate, 48 if prec != "fp32" else 24, peaks, tkey,
                                                   fp64_peak)}
        except Exception as e:
            out[key] = {"error": str(e)}
    # dimensionally split steps (dimsp2 / dimsp3): FP64 reference order, and the
    # 2D splits in characteristic variables (contracted FP64)
    for key, dim, split, sprec in (("radial_2d_4096_godunov_split_fp64", 2, "godunov", "fp64"),
                                   ("radial_2d_4096_godunov_split_fp64_fma", 2, "godunov", "fp64_fma"),
                                   ("radial_2d_4096_strang_split_fp64", 2, "strang", "fp64"),
                                   ("radial_2d_4096_strang_split_fp64_fma", 2, "strang", "fp64_fma"),
                                   ("hetero_acoustics_3d_256_split_fp64", 3, "godunov", "fp64")):
        try:
            if dim == 2:
                rd, solver, params, q0, aux = problems.radial_acoustics_2d(n=4096)
                t1, dt0, cells, nbytes = 0.03, 0.01, 4096 ** 2, 48
            else:
                rd, solver, params, q0, aux = problems.heterogeneous_acoustics_3d(n=256)
                t1, dt0, cells, nbytes = 0.1, 0.01, 256 ** 3, 80
            rd.clawdata.dimensional_split = split
            s = Solver(rd.clawdata, solver, params, precision=sprec)
            s.set_q(q0)
            if aux is not None:
                s.set_aux(aux)
            info, st = s.advance(0.0, t1, dt0)
            s.close()
            rate = cells * (st["steps_taken"] + st["steps_rejected"]) / (st["device_ms"] * 1e-3)
            if dim == 3:
                kern = "split3_fp64"
            elif split == "godunov":
                kern = "split2_kernel_fp64" if sprec == "fp64" else "step2s_char_kernel_fp64_fma"
            else:
                kern = "split2_kernel_fp64_strang" if sprec == "fp64" else "step2s_char_kernel_fp64_fma_strang"
            out[key] = {"cell_updates_per_s": rate, "steps": st["steps_taken"],
                        "device_ms": st["device_ms"],
                        "roofline": roofline_entry(rate, nbytes, peaks, kern, fp64_peak)}
        except Exception as e:
            out[key] = {"error": str(e)}
    # one 2048^2 Euler grid (four-quadrant data, seed 7) on the generic kernel:
    # reference order and the contracted build; t 0 -> 0.02 warms up, the next
    # 0.02 is timed
    for prec in ("fp64", "fp64_fma"):
        key = "euler_2d_2048_" + prec
        try:
            rd, solver, params, q0, _ = problems.euler_quadrants(n=2048, seed=7)
            s = Solver(rd.clawdata, solver, params, precision=prec)
            s.set_q(q0)
            info, st = s.advance(0.0, 0.02, float(rd.clawdata.dt_initial))
            info, st = s.advance(0.02, 0.04, st["dt_next"])
            s.close()
            rate = 2048 ** 2 * (st["steps_taken"] + st["steps_rejected"]) / (st["device_ms"] * 1e-3)
            out[key] = {"cell_updates_per_s": rate, "steps": st["steps_taken"], "device_ms": st["device_ms"],
                        "kernel": "step2_kernel (Euler Roe, MC, transverse 2)",
                        "roofline": roofline_entry(rate, 64, peaks, "step2_kernel_euler_" + prec, fp64_peak)}
        except Exception as e:
            out[key] = {"error": str(e)}
    sizes = problems.euler_ensemble_sizes(256, seed=0)
    for prec in ("fp64", "fp64_fma"):
        key = "euler_batch_256" if prec == "fp64" else "euler_batch_256_fp64_fma"
        try:
            insts = [problems.euler_quadrants(n=nn, seed=1000 + k) for k, nn in enumerate(sizes)]
            b = BatchSolver([i[0] for i in insts], "euler_roe_2d", {"gamma": 1.4}, precision=prec)
            for k, inst in enumerate(insts):
                b.set_q(k, inst[3])
            shape = b.autotune(repeats=2)  # launch shape chosen before the timed run
            info, st = b.advance(0.0, 0.25)
            b.close()
            upd = sum(nn * nn * (x["steps_taken"] + x["steps_rejected"]) for nn, x in zip(sizes, st))
            ms = st[0]["device_ms"]
            rate = upd / (ms * 1e-3)
            kern = "step2_batch_kernel_euler" + ("_fp64_fma" if prec == "fp64_fma" else "")
            e = {"cell_updates_per_s": rate, "cell_updates": upd, "precision": prec,
                 "device_ms": ms, "launches": st[0]["launches"],
                 "steps_min_max": [min(x["steps_taken"] for x in st),
                                   max(x["steps_taken"] for x in st)],
                 "autotuned_shape": {"min_rows": shape["min_rows"],
                                     "ctas_per_sm": shape["ctas_per_sm"]},
                 "roofline": roofline_entry(rate, 64, peaks, kern, fp64_peak)}
            if cpu and prec == "fp64":
                nn = 512
                mk = lambda: problems.euler_quadrants(n=nn, seed=7)[:4] + (None,)
                r1, s1 = cpu_rate(mk, 20, 1, 2e-4)
                rn, sn = cpu_rate(mk, 40, nproc, 2e-4)
                e["cpu_baseline"] = {"value": r1, "unit": "cell-updates/s", "cores": 1, "kind": "port",
                                     "sample": f"20 whole steps of one 512^2 instance from its initial data "
                                               f"({s1:.1f} s); the reference advances one grid per claw2 "
                                               "call, serially",
                                     "threaded": {"value": rn, "cores": nproc,
                                                  "sample": f"40 steps ({sn:.1f} s), every third slice in parallel"}}
            out[key] = e
        except Exception as e:
            out[key] = {"error": str(e)}
    # time to an L1 error (the metric's second half): 2D radial acoustics at
    # 512^2 / 1024^2 / 2048^2 in each precision against a 4096^2 truth; the
    # batched Euler ensemble against one claw2 call per instance (32 instances)
    try:
        from classic_b200 import accuracy
        out["time_to_l1_radial_2d"] = accuracy.radial_time_to_l1()
    except Exception as e:
        out["time_to_l1_radial_2d"] = {"error": str(e)}
    try:
        from classic_b200 import accuracy
        out["euler_ensemble_batched_vs_serial"] = accuracy.ensemble_batched_vs_serial(32)
    except Exception as e:
        out["euler_ensemble_batched_vs_serial"] = {"error": str(e)}
    # the learned corrector (the shipped network) on two unseen seeds: coarse
    # 256^2 corrected / plain against the block-averaged 1024^2 FP64 run
    try:
        from classic_b200 import corrector as C
        net, norm, alpha, interval = C.load_trained(
            os.path.join(ROOT, "classic_b200", "data", "corrector_euler_256.npz"))
        pl, co, tf_, tk_ = [], [], 0.0, 0.0
        C.corrected_run(net, norm, 61999, n=256, alpha=alpha, interval=interval)  # warm-up
        for seed in (61000, 61001):
            qc, _, _ = C.plain_run(seed, 256)
            qk, _, _, tk = C.corrected_run(net, norm, seed, n=256, alpha=alpha, interval=interval)
            qf, _, tf = C.plain_run(seed, 1024)
            ref = C.block_average(qf, 4)
            pl.append(C.l1_error(qc, ref))
            co.append(C.l1_error(qk, ref))
            tf_ += tf
            tk_ += tk
        out["corrector_euler_256"] = {
            "l1_vs_fine_plain": float(np.mean(pl)), "l1_vs_fine_corrected": float(np.mean(co)),
            "wall_fine_over_corrected": tf_ / tk_, "alpha": alpha, "interval": interval,
            "note": "2 unseen seeds; 200 held-out seeds in profiles/corrector_euler_256.md"}
    except Exception as e:
        out["corrector_euler_256"] = {"error": str(e)}
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=NOUT)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--n", type=int, default=N_CELLS)
    ap.add_argument("--precision", default="fp64_fma", choices=["fp64_fma", "fp64", "fp32"])
    ap.add_argument("--cpu-steps", type=int, default=2)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-variants", action="store_true")
    ap.add_argument("--no-configs", action="store_true", help="skip the other workloads")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference_arm(args)

    world, rank, local = dist_setup()
    import torch
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))

    def barrier():
        if world > 1:
            torch.distributed.barrier()

    def max_over_ranks(x):
        return reduce_over_ranks(x, "max", world, "cuda")

    def sum_over_ranks(x):
        return reduce_over_ranks(x, "sum", world, "cuda")

    from classic_b200 import problems
    from classic_b200.solver import Solver

    n = args.n
    rd, solver, params, q0, _ = problems.radial_acoustics_2d(n=n, nout=NOUT, tfinal=TFINAL)
    cd = rd.clawdata
    s = Solver(cd, solver, params, precision=args.precision)
    cells = n * n
    dtout = (TFINAL - 0.0) / float(np.float32(NOUT))

    def frames(k, host_q=None):
        """k claw2 calls (frames) from t=0; returns (accepted steps, kernel ms,
        launches, executed steps = accepted + rejected)."""
        t, dt = 0.0, float(cd.dt_initial)
        steps = launches = executed = 0
        kms = 0.0
        for _ in range(k):
            if host_q is None:
                info, st = s.advance(t, t + dtout, dt)
            else:
                info, st = s.advance_host(host_q, t, t + dtout, dt)
            if info != 0:
                raise RuntimeError(f"advance info={info}")
            t, dt = st["t_reached"], st["dt_next"]
            steps += st["steps_taken"]
            executed += st["steps_taken"] + st["steps_rejected"]
            kms += st["device_ms"]
            launches += st["launches"]
        return steps, kms, launches, executed

    # ---- warm-up (then reset to the initial data)
    s.set_q(q0)
    frames(args.warmup)
    s.set_q(q0)
    torch.cuda.synchronize()
    barrier()

    # ---- timed region: device-resident state
    clocks = ClockSampler(local)
    clocks.start()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    ev0.record()
    steps, kms, launches, executed = frames(args.steps)
    ev1.record()
    torch.cuda.synchronize()
    clk = clocks.stop()
    ms = ev0.elapsed_time(ev1)
    barrier()
    value, ms_max, total_updates = whole_job_rate(float(cells) * steps, ms, world, "cuda")

    # ---- e2e: same frames with host q in / out per frame (pinned)
    e2e = None
    if not args.no_e2e:
        host = torch.empty(s.q_shape, dtype=torch.float64, pin_memory=True).numpy()
        host[...] = q0
        torch.cuda.synchronize()
        barrier()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        esteps, _, _, _ = frames(args.steps, host_q=host)
        e1.record()
        torch.cuda.synchronize()
        ems = max_over_ranks(e0.elapsed_time(e1))
        qbytes = 3 * cells * 8
        e2e = {"value": sum_over_ranks(float(cells) * esteps) / (ems * 1e-3),
               "unit": "cell-updates/s", "h2d_bytes_per_step": qbytes, "d2h_bytes_per_step": qbytes,
               "ms_per_step": ems / args.steps}

    # ---- roofline of the step kernel (algorithmic bytes per launch).  The
    # device time of the frames (CUDA events around each claw2 call on the
    # library's stream, host checks between rounds included) is divided by
    # the steps the kernel executed (accepted + rejected), not by launches:
    # a launch issued after a frame is done returns at once.
    es = 4 if args.precision == "fp32" else 8
    bytes_per_launch = 2 * 3 * es * cells
    per_launch_ms = kms / max(executed, 1)
    achieved = bytes_per_launch / (per_launch_ms * 1e-3) / 1e9
    peaks = load_peaks()
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                "frac": achieved / peaks["hbm_gbs"], "traffic": traffic_per_launch(args.precision, cells),
                "peak_source": peaks["source"],
                "kernel": "step2_char_kernel" if args.precision != "fp64" else "step2_kernel",
                "algorithmic_bytes_per_launch": bytes_per_launch,
                "avg_launch_ms": per_launch_ms,
                "avg_launch_ms_basis": "device ms of the timed frames / executed steps",
                "executed_steps": executed, "launches": launches}

    # ---- the other arithmetic variants on the same frames (kernel-level rate)
    variants = {}
    if not args.no_variants:
        for prec in ("fp64", "fp64_fma", "fp32"):
            if prec == args.precision:
                continue
            v = Solver(cd, solver, params, precision=prec)
            v.set_q(q0)
            t, dt, vsteps, vms, vl = 0.0, float(cd.dt_initial), 0, 0.0, 0
            for _ in range(2):
                info, st = v.advance(t, t + dtout, dt)
                t, dt = st["t_reached"], st["dt_next"]
                vsteps += st["steps_taken"]
                vms += st["device_ms"]
                vl += st["steps_taken"] + st["steps_rejected"]
            v.close()
            ves = 4 if prec == "fp32" else 8
            vpl = vms / max(vl, 1)
            variants[prec] = {"cell_updates_per_s": cells * vsteps / (vms * 1e-3),
                              "avg_launch_ms": vpl,
                              "hbm_frac": 2 * 3 * ves * cells / (vpl * 1e-3) / 1e9 / peaks["hbm_gbs"],
                              "parity": {"fp64": "bit-identical to the CPU restatement",
                                         "fp64_fma": "within 1e-12 relative of fp64, same dt sequence",
                                         "fp32": "within 1e-5 relative of fp64"}[prec]}

    configs = None
    if rank == 0 and world == 1 and not args.no_configs:
        configs = other_configs(peaks, cpu=args.cpu_steps > 0)
        # the step kernel's FP64 pipe beside its HBM fraction: FP64
        # thread-instructions per cell (ncu) at the timed rate against the probe
        probe = configs.get("fp64_fma_probe", {}).get("tflops")
        _, fp64_per_cell = kernel_stats({"fp64_fma": "step2_char_kernel_fp64_fma",
                                         "fp64": "step2_kernel_fp64"}.get(args.precision, ""))
        if probe and fp64_per_cell:
            rate = cells / (per_launch_ms * 1e-3)
            roofline["fp64_inst_per_cell"] = fp64_per_cell
            roofline["fp64_frac"] = rate * fp64_per_cell / (probe / 2.0 * 1e12)

    cpu = None
    if rank == 0 and world == 1 and args.cpu_steps > 0:
        rate, sec, cores = cpu_reference_sample(n, args.cpu_steps)
        nproc = os.cpu_count() or 1
        mk = lambda: problems.radial_acoustics_2d(n=n)[:4] + (None,)
        rn, sn = cpu_rate(mk, max(1, args.cpu_steps), nproc, 0.9 * (2.0 / n) / 2.0)
        cpu = {"value": rate, "unit": "cell-updates/s", "cores": cores, "kind": "port",
               "sample": f"{args.cpu_steps} whole {n}^2 steps of the CPU restatement from the "
                         f"initial data ({sec:.1f} s); the reference's 2D step is serial",
               "host": host_cpu(),
               "threaded": {"value": rn, "cores": nproc,
                            "sample": f"{max(1, args.cpu_steps)} whole steps ({sn:.1f} s), every "
                                      "third slice in parallel (not the reference's scheme)"}}

    if rank == 0:
        line = {
            "metric": "cell-updates/s", "value": value, "unit": "cell-updates/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32" if args.precision == "fp32" else "f64",
            "data": "synthetic",
            "config": {"workload": f"2D radial acoustics {n}^2, MC limiter, transverse 2, "
                                   "extrap BCs, t_final 0.6",
                       "arithmetic": {"fp64_fma": "FP64, fused multiply-add, characteristic variables",
                                      "fp64": "FP64, reference operation order",
                                      "fp32": "FP32 update, FP64 CFL/dt/time"}[args.precision],
                       "step": f"one claw2 call over dtout = {dtout:g} (~{steps / args.steps:.0f} "
                               "time steps)",
                       "time_steps_timed": steps, "cells": cells,
                       "l2": "inputs larger than L2 (403 MB q per buffer)",
                       "parallelism": "replicas" if world > 1 else "single GPU"},
            "roofline": roofline,
            "cpu_baseline": cpu,
            "e2e": e2e,
            "gpu_launches": launches,
            "clocks": clk,
            "variants": variants,
            "other_configs": configs,
        }
        print(json.dumps(line), flush=True)
    s.close()
    if world > 1:
        torch.distributed.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
