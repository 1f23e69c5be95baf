"""Benchmark of the RTM propagation hot path (Gpts/s per time step).

Workload (default `vti_cfd`): the VTI pseudo-acoustic single-shot RTM forward
pass on a 512 x 512 x 400 grid (10 m, 32-cell PML, compact FD, seeded smooth
layered velocity 1500-4500 m/s, eps 0-0.25, delta 0-0.1, 20 Hz Ricker), with
the reference's default COMPRESS_16 snapshot store every 8 steps.  One bench
step = one time step of the forward migration loop (operator with PML,
update, source injection, snapshot when due), inputs resident in HBM.
Every volume is 419 MB > the 126 MB L2, so no flush is needed between steps.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl cuda|reference]

N > 1 runs N independent replicas (one shot per GPU, no collective; shots are
independent in RTM), launched by torch.distributed.run.
"""
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

from konglong_b200 import replicas as R  # noqa: E402

# algorithmic HBM bytes per cell-step (each array read / written once per step)
#   VTI core: R w1, w0, vel, eps, del; W w0 = 24 B; PML memory 48 B x fraction
#   of cells in PML slabs (3 first derivatives x 2 rounds x q r/w).
ALG_BYTES = {"vti_cfd": None, "iso128": None, "tti_q": None}


def pml_fraction(spec):
    f = 0.0
    for n, a, b in ((spec.nx, spec.nbnd[0], spec.nbnd[1]), (spec.ny, spec.nbnd[2], spec.nbnd[3]),
                    (spec.nz, spec.nbnd[4], spec.nbnd[5])):
        f += (a + b) / n
    return f


def alg_bytes_per_cell(spec, snap_fmt, interval):
    from konglong_b200.spec import ISO, TTI, VTI
    m = pml_fraction(spec)
    if spec.model_type == ISO and spec.engine == 0:
        core, pml = 16.0, 16.0 * m
    elif spec.model_type == VTI:
        core, pml = 24.0, 48.0 * m
    else:
        core, pml = 32.0, 48.0 * m
    if spec.use_q:
        core += 4.0 + 3 * 4.0 * spec.q_order
    if getattr(spec, "state_fp16", False):
        core -= 3 * 2.0  # w1 read, w0 read and write in 2 bytes (3s with s = 2)
    if spec.use_q and getattr(spec, "q_bf16", False):
        core -= 3 * 2.0 * spec.q_order  # Q memory d0 / d1 read, d0 write in 2 bytes
    snap = {0: 4.0, 1: 2.0, 2: 2.0, 3: 33 * 4.0 / 512}[snap_fmt] / interval
    return core + pml + snap, core, pml


def kernel_alg_bytes(spec, m):
    """Compulsory HBM bytes per cell of one launch of each kernel kind (inputs
    read once, outputs written once, PML memory of the cells in PML slabs)."""
    aniso = 8.0 * (spec.model_type >= 2) + 8.0 * (spec.model_type == 3)
    q = (4.0 + 3 * 4.0 * spec.q_order) if spec.use_q else 0.0
    return {"iso_fd8_step": 16.0 + 16.0 * m,
            "grad_fd8": 4.0 + aniso + 12.0 + 24.0 * m,
            "div_fd8": 12.0 + 12.0 + 4.0 + 24.0 * m,
            "cfd_z": 8.0, "cfd_x": 8.0, "cfd_y": 8.0,
            # segment-parallel pipeline: a line solve with one first-derivative
            # PML component round (Z, X), the fused y kernel (w1, gx, gz and the
            # anisotropy parameters in; px, pz, dy out; two PML rounds), the fused
            # x kernel (px, dz, dy, vel, w0, w1 in; w0 out; one PML round)
            "cfd_z_seg": 8.0 + 8.0 * m, "cfd_x_seg": 8.0 + 8.0 * m,
            "cfd_y_fused": 4.0 + 8.0 + aniso + 12.0 + 16.0 * m,
            "cfd_x_fused": 24.0 + 4.0 + 8.0 * m + q,
            "cfd_grad_epilogue": 24.0 + aniso + 24.0 * m,
            "cfd_div_epilogue": 28.0 + 24.0 * m,
            "fused_io": 6.0, "slab_max": 4.0}


# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) per cell of one
# launch, from ncu captures of the same kernels on the 0.75-scale grid of the
# vti_cfd workload.  The PML slabs scale with the grid, so bytes per cell carry
# over to the full grid.  Each entry records the SHA-256 prefix of the kernel
# source it was captured on; when the source has changed since, the figure no
# longer describes the kernel that runs and the bench reports traffic as null.
MEASURED_DRAM_B_PER_CELL = {"vti_cfd": {"cfd_div_epilogue": 37.9, "cfd_grad_epilogue": 38.7,
                                        "cfd_x": 6.75, "cfd_y": 6.83, "cfd_z": 6.83}}
MEASURED_DRAM_SOURCE = {"vti_cfd": ("konglong_b200/csrc/kernels_cfd.cu", "f002906f4d2b116c")}


def measured_traffic_current(workload):
    """True when the kernel source behind MEASURED_DRAM_B_PER_CELL[workload] is unchanged."""
    import hashlib
    src = MEASURED_DRAM_SOURCE.get(workload)
    if not src:
        return False
    try:
        with open(os.path.join(os.path.dirname(os.path.abspath(__file__)), src[0]), "rb") as f:
            return hashlib.sha256(f.read()).hexdigest()[:16] == src[1]
    except OSError:
        return False


class ClockSampler:
    """SM clock and clock-event reasons sampled during the timed region: NVML read
    every 5 ms from a thread (the timed regions here last 0.1-1 s), nvidia-smi
    every 200 ms when NVML is not importable.  Reads only; changes no setting."""

    NAMES = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]

    def __init__(self, index=0):
        self.index = index
        self.rows = []   # (sm_mhz, max_mhz, reasons set)
        self.proc = None
        self.stop = threading.Event()
        self.th = None

    def _nvml_handle(self, nv):
        try:  # the CUDA device this process uses, matched by UUID (indices may differ)
            import torch
            u = str(torch.cuda.get_device_properties(self.index).uuid)
            return nv.nvmlDeviceGetHandleByUUID(u if u.startswith("GPU-") else "GPU-" + u)
        except Exception:
            return nv.nvmlDeviceGetHandleByIndex(self.index)

    def __enter__(self):
        try:
            import pynvml as nv
            nv.nvmlInit()
            h = self._nvml_handle(nv)
            bits = [getattr(nv, "nvmlClocksEventReason" + k, getattr(nv, "nvmlClocksThrottleReason" + k, 0))
                    for k in ("HwSlowdown", "HwThermalSlowdown", "SwThermalSlowdown", "SwPowerCap")]
            reasons_fn = getattr(nv, "nvmlDeviceGetCurrentClocksEventReasons",
                                 getattr(nv, "nvmlDeviceGetCurrentClocksThrottleReasons", None))
            mx = float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM))

            def run():
                while not self.stop.is_set():
                    try:
                        sm = float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM))
                        r = reasons_fn(h) if reasons_fn else 0
                        self.rows.append((sm, mx, {self.NAMES[k] for k in range(4) if bits[k] and r & bits[k]}))
                    except Exception:
                        pass
                    self.stop.wait(0.005)
            self.th = threading.Thread(target=run, daemon=True)
            self.th.start()
            return self
        except Exception:
            pass
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.th = threading.Thread(target=self._read, daemon=True)
            self.th.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            r = [x.strip() for x in line.split(",")]
            if len(r) >= 9 and r[1].replace(".", "").isdigit() and r[2].replace(".", "").isdigit():
                self.rows.append((float(r[1]), float(r[2]),
                                  {self.NAMES[k] for k in range(4) if r[5 + k].lower() == "active"}))

    def __exit__(self, *a):
        self.stop.set()
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        if self.th:
            self.th.join(timeout=5)

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [r[0] for r in self.rows]
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": max(r[1] for r in self.rows),
                "reasons": sorted(set().union(*[r[2] for r in self.rows])), "samples": len(self.rows)}


def build_workload(name, steps_total, scale=1.0):
    from konglong_b200 import workloads as W
    if name == "vti_cfd":
        return W.vti_cfd(scale=scale, nt=steps_total)
    if name == "iso128":
        return W.iso128(scale=scale, nt=steps_total)
    if name == "tti_q":
        return W.tti_q(scale=scale, nt=steps_total)
    if name == "iso512":
        shot = W.vti_cfd(scale=scale, nt=steps_total)
        shot.spec.engine, shot.spec.model_type = 0, 1
        shot.eps = shot.dl = None
        shot.name = "iso512"
        return shot
    if name == "vti_fd8":
        shot = W.vti_cfd(scale=scale, nt=steps_total)
        shot.spec.engine = 0
        shot.name = "vti_fd8"
        return shot
    if name in ("vti_r2c", "vti_r2r"):  # the compact-FD model and shot through the pseudo-spectral engines
        shot = W.vti_cfd(scale=scale, nt=steps_total)
        shot.spec.engine = 2 if name == "vti_r2c" else 3
        shot.name = name
        return shot
    raise SystemExit(f"unknown workload {name}")


def config_of(shot, snap_fmt, steps):
    s = shot.spec
    return {"workload": f"{shot.name}: {s.nx}x{s.ny}x{s.nz} {['FD8', 'CFD', 'FFTWR2C', 'FFTWR2R'][s.engine]} "
                        f"{['', 'ISO', 'VTI', 'TTI'][s.model_type]}{'+Q' if s.use_q else ''}, PML {s.nbnd[0]}, "
                        f"dt {s.dt * 1e3:.4f} ms, forward RTM step, snapshots every {shot.interval} steps",
            "grid": [s.nx, s.ny, s.nz], "cells": s.n, "snapshot_format": ["fp32", "c16", "fp16s"][snap_fmt],
            "l2": f"inputs larger than L2 ({s.n * 4 / 1e6:.0f} MB per volume), no flush", "dt_s": s.dt}


def run_cuda(args, rank, world):
    import ctypes as C
    from konglong_b200 import workloads as W
    from konglong_b200.propagator import Propagator, spread_coeffs
    from konglong_b200.spec import FORWARD, SNAP_C16

    K, Wm = args.steps, args.warmup
    shot = build_workload(args.workload, 2 * K + Wm + 8, args.scale)
    s = shot.spec
    s.state_fp16 = bool(args.state_fp16)
    s.q_bf16 = bool(args.q_bf16)
    s.kernel_variant = args.kernel_variant
    snap_fmt = {"c16": SNAP_C16, "fp32": 0, "fp16s": 2}[args.snap]
    k1, k2 = W.spread_band(s)
    src = W.make_traceset([shot.src_pos], s.nx, s.ny, s.nz, 10, k1, k2, spread_coeffs)
    rcv = W.make_traceset(shot.rcv_pos, s.nx, s.ny, s.nz, 10, k1, k2, spread_coeffs)
    p = Propagator(s)
    if s.use_q:
        p.set_q_coeffs(*W.q_coefficients(s.dt, shot.fpeak))
    p.set_model(**shot.model_arrays())
    nslots = (2 * K + Wm) // shot.interval + 2
    p.snapshot_setup(snap_fmt, nslots)
    if args.snap_offload:
        p.snapshot_offload(args.snap_offload)
    p.set_injection(src, shot.wavelet[None, :], s.dt_dxyz)
    tuned = p.autotune(3) if not args.no_autotune else None
    p.reset()
    ranks = R.Ranks.from_env()
    # warm-up steps (untimed), then K timed steps continuing the same shot
    p.migration(FORWARD, 0, Wm, -1, shot.interval)
    R.barrier(ranks)
    with ClockSampler(ranks.local_rank) as clk:
        p.migration(FORWARD, Wm, Wm + K, -1, shot.interval)
    ms = R.max_over_ranks(ranks, p.last_loop_ms, device="cuda")
    R.barrier(ranks)
    cells = s.n
    value = R.aggregate_gpts(world, cells, K, ms)
    ms_step = ms / K

    launches = p.launch_count()
    # per-kernel device times: the same loop run eagerly with CUDA events
    # around every launch on the engine's stream (after the timed region)
    p.profile(True)
    p.migration(FORWARD, Wm + K, Wm + 2 * K, -1, shot.interval)
    prof = p.profile_read()
    p.profile(False)
    alg, core, pml = alg_bytes_per_cell(s, snap_fmt, shot.interval)
    peak, peak_src = 6650.0, "fallback"
    try:
        peak = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))["hbm_gbs"]
        peak_src = "measured"
    except Exception:
        pass
    kbytes = kernel_alg_bytes(s, pml_fraction(s))
    if "cfd_y_fused" in prof:  # segment-parallel pipeline: its Z / X launches carry a PML round
        kbytes["cfd_z"], kbytes["cfd_x"] = kbytes["cfd_z_seg"], kbytes["cfd_x_seg"]
    dom = max(prof, key=lambda k: prof[k][0])
    dom_ms = prof[dom][0] / prof[dom][1]
    dom_bytes = kbytes.get(dom, 8.0) * cells
    roof = {"bound": "hbm", "kernel": dom, "achieved": dom_bytes / (dom_ms * 1e-3) / 1e9, "peak": peak,
            "unit": "GB/s", "frac": None, "traffic": None, "peak_source": peak_src,
            "alg_bytes_per_cell_kernel": kbytes.get(dom, 8.0), "avg_launch_ms": dom_ms,
            "share_of_step": prof[dom][0] / sum(v[0] for v in prof.values()),
            "step": {"alg_bytes_per_cell": round(alg, 2), "achieved_gbs": alg * cells / (ms_step * 1e-3) / 1e9,
                     "frac": alg * cells / (ms_step * 1e-3) / 1e9 / peak},
            "kernels_ms_per_step": {k: round(v[0] / K, 4) for k, v in prof.items()}}
    roof["frac"] = roof["achieved"] / peak
    bpc = MEASURED_DRAM_B_PER_CELL.get(args.workload, {}).get(dom)
    if bpc is not None and measured_traffic_current(args.workload):
        roof["traffic"] = bpc * cells
        roof["traffic_source"] = "ncu DRAM bytes per cell at 0.75 scale x cells of one launch"
    elif bpc is not None:
        roof["traffic_source"] = "stale: the kernel source changed since the ncu capture"

    # end to end through the public API with host buffers: modelling run of K
    # steps with the receiver samples read back (set_injection H2D of the
    # source trace, modelling, D2H of every extracted sample)
    e2e = None
    if not args.no_e2e:
        q = Propagator(s)
        if s.use_q:
            q.set_q_coeffs(*W.q_coefficients(s.dt, shot.fpeak))
        q.set_model(**shot.model_arrays())
        q.set_extraction(rcv, K)
        q.reset()
        q.set_injection(src, shot.wavelet[None, :K + 1].copy(), s.dt_dxyz)
        q.modelling(2, -1, 1)  # warm the graph path
        q.reset()
        wav = np.ascontiguousarray(shot.wavelet[None, :K + 1])
        R.barrier(ranks)
        t0 = time.perf_counter()
        q.set_injection(src, wav, s.dt_dxyz)
        q.modelling(K, -1, 1)
        tr = q.traces()
        t1 = time.perf_counter()
        wall = R.max_over_ranks(ranks, t1 - t0, device="cuda")
        e2e = {"value": R.aggregate_gpts(world, cells, K, wall * 1e3), "unit": "Gpts/s",
               "h2d_bytes_per_step": int(wav.nbytes // K), "d2h_bytes_per_step": int(tr.nbytes // K),
               "what": "Propagator.modelling via the C ABI: traces H2D, K steps with receiver extraction, "
                       "receiver samples D2H; wall clock"}
        q.close()
    p.close()
    cfg = config_of(shot, snap_fmt, K)
    cfg["autotuned_shape"] = tuned
    cfg["kernel_variant"] = args.kernel_variant
    cfg["state"] = "fp16 per-slab scale" if s.state_fp16 else "fp32"
    if s.use_q:
        cfg["q_memory"] = "bf16" if s.q_bf16 else "fp32"
    if args.snap_offload:
        cfg["snapshots"] = f"pinned host memory, {args.snap_offload} device staging slots"
    return dict(value=value, ms=ms, ms_step=ms_step, roofline=roof, e2e=e2e, clocks=clk.summary(),
                config=cfg, shot=shot, launches=launches)


def run_small_shots(args, ranks):
    """Batched small-shot workload (64 seeded shots, grids 96-256 per axis,
    500-2000 steps, receivers every step; ISO, or VTI with per-layer Thomsen
    parameters for small_shots_vti): every shot's full modelling run, once per
    shot with its own CUDA-graph loop (per-shot launches) and once for all
    shots together (persistent launches per step over every shot, batched
    I/O).  Metric: shots per second of the batched run."""
    from konglong_b200 import workloads as W
    from konglong_b200.propagator import Batch, Propagator, spread_coeffs
    from konglong_b200.spec import ISO, VTI
    vti = args.workload == "small_shots_vti"
    shots = W.small_shots(nshots=64, seed=4 + ranks.rank, model=VTI if vti else ISO)

    def setup(sh):
        s = sh.spec
        p = Propagator(s)
        p.set_model(**sh.model_arrays())
        k1, k2 = W.spread_band(s)
        src = W.make_traceset([sh.src_pos], s.nx, s.ny, s.nz, 10, k1, k2, spread_coeffs)
        rcv = W.make_traceset(sh.rcv_pos, s.nx, s.ny, s.nz, 10, k1, k2, spread_coeffs)
        p.set_injection(src, sh.wavelet[None, :], s.dt_dxyz)
        p.set_extraction(rcv, sh.nt)
        p.reset()
        return p

    ps = [setup(sh) for sh in shots]
    nts = [sh.nt for sh in shots]
    cell_steps = sum(sh.spec.n * sh.nt for sh in shots)
    # per-shot launches: each shot's own modelling loop, back to back
    per_ms = 0.0
    for p, n in zip(ps, nts):
        p.modelling(n, -1, 1)
        per_ms += p.last_loop_ms
    for p in ps:
        p.reset()
    b = Batch(ps)
    choice = b.autotune(3)
    for p in ps:
        p.reset()
    R.barrier(ranks)
    with ClockSampler(ranks.local_rank) as clk:
        b.modelling(nts, -1, 1)
    ms = R.max_over_ranks(ranks, b.last_ms, device="cuda")
    # e2e: one more batched run through the API with the traces read back
    for p in ps:
        p.reset()
    t0 = time.perf_counter()
    b.modelling(nts, -1, 1)
    tr_bytes = sum(p.traces().nbytes for p in ps)
    wall = R.max_over_ranks(ranks, time.perf_counter() - t0, device="cuda")
    b.close()
    m = [sum(2 * w / n for w, n in zip(sh.spec.nbnd[0::2], (sh.spec.nx, sh.spec.ny, sh.spec.nz))) for sh in shots]
    core, pml = (24.0, 48.0) if vti else (16.0, 16.0)
    alg = sum((core + pml * mm) * sh.spec.n * sh.nt for mm, sh in zip(m, shots))
    peak, peak_src = 6650.0, "fallback"
    try:
        peak = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))["hbm_gbs"]
        peak_src = "measured"
    except Exception:
        pass
    achieved = alg / (ms * 1e-3) / 1e9
    nshots = len(shots) * ranks.world
    return {"metric": "shots/s", "value": nshots / (ms * 1e-3), "unit": "shots/s", "ms": ms,
            "per_shot": {"value": len(shots) / (per_ms * 1e-3), "ms": per_ms,
                         "what": "the same shots, one rtm_modelling (own CUDA-graph loop) per shot"},
            "gpts": R.aggregate_gpts(ranks.world, cell_steps, 1, ms),
            "roofline": {"bound": "hbm",
                         "kernel": ("grad_fd8_batch + div_fd8_batch" if vti else "iso_fd8_batch") +
                                   " (whole batched step)", "achieved": achieved,
                         "peak": peak, "unit": "GB/s", "frac": achieved / peak, "traffic": None,
                         "peak_source": peak_src,
                         "alg_bytes": ("24 + 48 m per cell-step (VTI FD8)" if vti else
                                       "16 + 16 m per cell-step (ISO FD8)") + ", m = PML slab fraction per shot"},
            "e2e": {"value": nshots / wall, "unit": "shots/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": int(tr_bytes / max(nts)),
                    "what": "batched modelling through the C ABI, all receiver traces read back; wall clock"},
            "clocks": clk.summary(), "tuned_shape": choice,
            "config": {"workload": f"{args.workload}: 64 {'VTI' if vti else 'ISO'} FD8 shots, grids uniform "
                                   "96-256 per axis, 500-2000 steps, 3-5 layers"
                                   f"{' (epsilon 0-0.2, delta 0-0.1 per layer, CFL dt)' if vti else ''}, "
                                   "10-25 Hz Ricker, 16x16 receivers, PML 16",
                       "cell_steps": cell_steps, "shots": nshots}}


RTM_FORMS = {
    # plain FP32 GPU form: FP32 state, Q memory and snapshots
    "plain": dict(q_bf16=False, snap="fp32"),
    # the same with the reference's default snapshot codec (COMPRESS_16)
    "plain_c16": dict(q_bf16=False, snap="c16"),
    # mixed precision: BF16 Q memory, FP16 snapshots with a per-slab scale
    "mixed": dict(q_bf16=True, snap="fp16s"),
    # mixed precision + learned compression: BF16 Q memory, learned 8^3-block
    # snapshots (16:1) with the FP16 store of their 5 % highest-energy blocks
    "chosen": dict(q_bf16=True, snap="ae"),
}


def train_compressor(seed=5, nblocks=20000, steps=3000):
    """The learned snapshot code trained as the workload describes: about 20k
    8^3 blocks of forward wavefields of the compact-FD VTI model family, Adam
    on the GPU by the project's own kernels."""
    from konglong_b200 import compressor as CP
    from konglong_b200 import workloads as W
    from konglong_b200.propagator import Propagator, spread_coeffs
    shot = W.vti_cfd(scale=0.25, seed=seed, nt=400)
    blocks, scales = CP.training_blocks(shot, Propagator, spread_coeffs, nblocks=nblocks, every=20, seed=seed)
    ae = CP.AutoEncoder(seed=seed)
    ae.fit(blocks, steps=steps, weights=scales ** 2)
    return ae, int(blocks.shape[0])


def rtm_form_propagator(shot, form, ae=None):
    import dataclasses
    from konglong_b200 import workloads as W
    from konglong_b200.propagator import Propagator
    from konglong_b200.spec import SNAP_AE, SNAP_C16, SNAP_FP16S, SNAP_FP32
    f = RTM_FORMS[form]
    s = dataclasses.replace(shot.spec, q_bf16=f["q_bf16"])
    p = Propagator(s)
    p.set_q_coeffs(*W.q_coefficients(s.dt, shot.fpeak))
    p.set_model(**shot.model_arrays())
    fmt = {"fp32": SNAP_FP32, "c16": SNAP_C16, "fp16s": SNAP_FP16S, "ae": SNAP_AE}[f["snap"]]
    if fmt == SNAP_AE:
        p.set_compressor(ae)
        p.set_compressor_fallback(1e-3, 0.05)
    return p, fmt


def rtm_schedule(p, fmt, nt, interval, reserve_bytes):
    """Store / recompute plan of one shot on this GPU: the snapshot slots and
    checkpoints that fit the HBM left after the engine's own arrays (less
    reserve_bytes).  Returns the plan and the figures behind it."""
    import torch
    from konglong_b200.propagator import checkpoint_plan, checkpoint_slots_for_budget
    nsnap = (nt - 1) // interval + 1
    slot_b = p.snapshot_slot_bytes(fmt)
    ckpt_b = p.checkpoint_setup(0)
    free = torch.cuda.mem_get_info()[0]
    budget = free - reserve_bytes
    s = checkpoint_slots_for_budget(nt, interval, slot_b, ckpt_b, budget)
    if s == 0:
        raise SystemExit("rtm_schedule: not even one snapshot slot and its checkpoints fit")
    seg = checkpoint_plan(nt, interval, s)
    return {"snapshots": nsnap, "slot_bytes": slot_b, "snapshot_gb_per_shot": nsnap * slot_b / 1e9,
            "hbm_budget_gb": budget / 1e9, "fits": s >= nsnap, "seg_slots": s, "segments": len(seg),
            "checkpoint_gb": ckpt_b / 1e9, "recomputed_steps": sum(b - a for a, b in seg[:-1])}


def run_rtm_shot(args, ranks):
    """RTM s/shot of the TTI + Q workload (640 x 640 x 512, PML 32, 5000 steps,
    a snapshot every 8 steps: 625 snapshots) in the plain FP32 form, the
    plain form with COMPRESS_16 snapshots, and the mixed and chosen forms
    (RTM_FORMS).  A form whose snapshots do not fit the GPU's memory runs
    store / recompute (Propagator.rtm_shot_checkpointed): checkpoints of the
    propagation state at segment starts, each earlier segment's snapshots
    recomputed in the backward pass.  Each form runs K forward steps
    (snapshots stored) and K backward steps (128 x 128 receiver traces
    injected, imaging condition fused into the step) on the full grid, timed
    with CUDA events, and one checkpoint save + load;
      s/shot = forward ms/step x (5000 + recomputed steps)
             + backward ms/step x 5000 + 4 checkpoint copies per extra segment.
    --full-shot runs the whole checkpointed shot instead and reports its
    measured time.  Image NRMSE of each form against the plain form: the same
    shot at 0.08 scale (51 x 51 x 41, 160 steps)."""
    import torch
    from konglong_b200 import workloads as W
    from konglong_b200.propagator import spread_coeffs
    from konglong_b200.spec import BACKWARD, FORWARD
    K, Wm = args.steps, args.warmup
    forms = ["plain", "plain_c16", "mixed", "chosen"]
    ae, ntrain = train_compressor()
    interval, NT = 8, 5000
    res = {}
    shot = W.tti_q(scale=args.scale, nt=NT if args.full_shot else 2 * (K + Wm) + 8)
    s = shot.spec
    k1, k2 = W.spread_band(s)
    src = W.make_traceset([shot.src_pos], s.nx, s.ny, s.nz, 10, k1, k2, spread_coeffs)
    rcv = W.make_traceset(shot.rcv_pos, s.nx, s.ny, s.nz, 10, k1, k2, spread_coeffs)
    data = (np.random.default_rng(7).standard_normal((rcv.ntr, shot.nt)) * 1e3).astype(np.float32)
    clk_all = []
    for form in forms:
        p, fmt = rtm_form_propagator(shot, form, ae)
        p.image_setup(3, 4, 1)  # the image volumes are allocated before the budget is taken
        reserve = (1 << 30) + (s.n * 4 if fmt == 3 else 0)  # 1 GiB margin (+ the learned decode scratch)
        plan = rtm_schedule(p, fmt, NT, interval, reserve)
        if args.full_shot:
            with ClockSampler(ranks.local_rank) as clk:
                img, ms = p.rtm_shot_checkpointed(src, shot.wavelet[None, :], rcv, data, NT, NT, interval,
                                                  plan["seg_slots"], snap_fmt=fmt, ntaper_t=3, ntaper_z=4)
            clk_all.append(clk.summary())
            p.close()
            res[form] = {"plan": plan, "measured_ms": ms, "s_per_shot": sum(ms.values()) / 1e3}
            continue
        p.snapshot_setup(fmt, min(plan["seg_slots"], (Wm + K) // interval + 2))
        p.reset()
        p.set_injection(src, shot.wavelet[None, :], s.dt_dxyz)
        p.migration(FORWARD, 0, Wm, -1, interval)          # warm-up (graph capture, first launches)
        with ClockSampler(ranks.local_rank) as clk:
            p.migration(FORWARD, Wm, Wm + K, -1, interval)
            fwd = p.last_loop_ms
            p.reset()
            p.image_setup(3, 4, 1)
            p.set_injection(rcv, data, s.dt_dxyz)
            p.migration(BACKWARD, Wm + K - 1, Wm - 1, -1, interval)
            bwd = p.last_loop_ms
        clk_all.append(clk.summary())
        copy_ms = 0.0
        if plan["segments"] > 1:
            p.snapshot_setup(fmt, 0)
            p.checkpoint_setup(1)
            p.checkpoint_save(0), p.checkpoint_load(0)  # warm
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            p.checkpoint_save(0), p.checkpoint_load(0)
            torch.cuda.synchronize()
            copy_ms = (time.perf_counter() - t0) * 1e3 / 2
        p.close()
        fwd_step, bwd_step = fwd / K, bwd / K
        total = fwd_step * (NT + plan["recomputed_steps"]) + bwd_step * NT + copy_ms * 4 * (plan["segments"] - 1)
        res[form] = {"plan": plan, "forward_ms_per_step": fwd_step, "backward_ms_per_step": bwd_step,
                     "checkpoint_copy_ms": copy_ms, "s_per_shot": total / 1e3}
    # image error of each form against the plain FP32 form on the same shot at
    # 0.08 scale (160 steps); the tests state both against the FP64 oracle
    small = W.tti_q(scale=0.08, nt=160)
    ss = small.spec
    k1, k2 = W.spread_band(ss)
    s_src = W.make_traceset([small.src_pos], ss.nx, ss.ny, ss.nz, 10, k1, k2, spread_coeffs)
    s_rcv = W.make_traceset(small.rcv_pos, ss.nx, ss.ny, ss.nz, 10, k1, k2, spread_coeffs)
    s_data = (np.random.default_rng(7).standard_normal((s_rcv.ntr, 160)) * 1e3).astype(np.float32)
    imgs = {}
    for form in forms:
        p, fmt = rtm_form_propagator(small, form, ae)
        imgs[form] = p.rtm_shot(s_src, small.wavelet[None, :], s_rcv, s_data, 160, 112, 4, snap_fmt=fmt,
                                ntaper_t=3, ntaper_z=4)[0]
        p.close()
    ref = imgs["plain"].astype(np.float64).ravel()
    for form in forms:
        res[form]["image_nrmse_vs_plain"] = float(np.linalg.norm(imgs[form].astype(np.float64).ravel() - ref) /
                                                  max(np.linalg.norm(ref), 1e-300))
    ae.close()
    return {"forms": res, "clocks": clk_all, "ntrain": ntrain, "shot": shot}


def run_ae_codec(args, ranks):
    """The learned compressor's fused encoder and decoder on one snapshot of
    the C3 grid (640 x 640 x 512 at scale 1): K timed calls each after W
    warm-up calls, CUDA events on the default stream.  Reports ms per
    snapshot, TFLOP/s (61440 FLOP per 8^3 block each way: the four layers'
    MACs x 2) against bf16_tflops_sustained, and GB/s of the volume and the
    codes read and written."""
    import torch
    from konglong_b200 import _lib
    from konglong_b200 import compressor as AE
    from konglong_b200 import workloads as W
    s = W.tti_q(scale=args.scale, nt=8).spec
    nx, ny, nz = s.nx, s.ny, s.nz
    L = _lib.lib()
    ae = AE.AutoEncoder(seed=5)
    g = torch.Generator(device="cuda").manual_seed(5)
    w = torch.randn(ny, nx, nz, device="cuda", generator=g)
    nb = ((nx + 7) // 8) * ((ny + 7) // 8) * ((nz + 7) // 8)
    lat = torch.zeros(nb * AE.LATENT, device="cuda", dtype=torch.bfloat16)
    sc = torch.zeros(nb, device="cuda")
    out = torch.zeros_like(w)
    enc = lambda: _lib.check(L.rtm_ae_compress_volume(ae.a, w.data_ptr(), nx, ny, nz, lat.data_ptr(), sc.data_ptr(),
                                                       None), "rtm_ae_compress_volume")
    dec = lambda: _lib.check(L.rtm_ae_decompress_volume(ae.a, lat.data_ptr(), sc.data_ptr(), nx, ny, nz,
                                                         out.data_ptr(), None), "rtm_ae_decompress_volume")
    res = {}
    with ClockSampler(ranks.local_rank) as clk:
        for name, f in (("encode", enc), ("decode", dec)):
            for _ in range(args.warmup):
                f()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record()
            for _ in range(args.steps):
                f()
            e1.record()
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1) / args.steps
            res[name] = {"ms": ms, "tflops": nb * 61440 / (ms * 1e-3) / 1e12,
                         "gbs": (s.n * 4 + nb * (AE.LATENT * 2 + 4)) / (ms * 1e-3) / 1e9}
    ae.close()
    peak = {}
    try:
        peak = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    return {"res": res, "clocks": clk.summary(), "grid": [nx, ny, nz], "blocks": nb,
            "tflops_peak": peak.get("bf16_tflops_sustained", 1400.0), "hbm_peak": peak.get("hbm_gbs", 6650.0)}


def cpu_baseline(shot, max_seconds=20.0):
    """The reference's own CPU kernels (oracle/_ref) on the full grid, all host
    threads, a bounded number of time steps."""
    from oracle import pyoracle as O
    if not O.ref_available():
        return None, "port"
    s = shot.spec
    if s.use_q or s.engine not in (0, 1):  # the FFT engines' FFTW calls are answered by DFT sums here
        return None, "reference"
    threads = os.cpu_count() or 1
    r = O.Reference(s, nthreads=threads)
    r.set_model(shot.vel, shot.eps, shot.dl, shot.pjx, shot.pjy)
    r.reset()
    first = r.run(1, 1)
    n = max(1, min(50, int(max_seconds / max(first, 1e-3))))
    t = r.run(2, n)
    r.close()
    return {"value": s.n * n / t / 1e9, "unit": "Gpts/s", "cores": threads, "kind": "reference",
            "sample": f"{n} full time steps ({s.nx}x{s.ny}x{s.nz}) of bgprtm KernelCPU "
                      f"({'CFD' if s.engine else 'FD8'}) + update2nd + source injection, "
                      f"OMP {threads} threads, {t:.1f} s"}, "reference"


def run_reference(args, rank, world):
    """--impl reference: the reference's CPU path (oracle/_ref, else the oracle
    port) timed on this host's cores on the same workload."""
    from oracle import pyoracle as O
    shot = build_workload(args.workload, args.steps + args.warmup + 8, args.scale)
    s = shot.spec
    threads = os.cpu_count() or 1
    if s.engine not in (0, 1):
        return {"unavailable": "the reference's FFT engines call FFTW, absent from this image; the harness answers "
                               "those calls with plain DFT sums, which would time the stand-in, not the reference"}
    if O.ref_available() and not s.use_q:
        r = O.Reference(s, nthreads=threads)
        r.set_model(shot.vel, shot.eps, shot.dl, shot.pjx, shot.pjy)
        kind = "reference"
    else:
        r = O.Oracle(s)
        r.set_model(**shot.model_arrays())
        kind = "port"
    r.reset()
    # warm-up (bounded)
    t_first = None
    for w in range(min(args.warmup, 1)):
        t0 = time.perf_counter()
        r.kernel(), r.update2nd(), r.swap()
        t_first = time.perf_counter() - t0
    budget = 150.0
    k = args.steps
    if t_first and t_first * k > budget:
        k = max(1, int(budget / t_first))
    t0 = time.perf_counter()
    for _ in range(k):
        r.kernel(), r.update2nd(), r.swap()
    t = time.perf_counter() - t0
    val = s.n * k / t / 1e9
    return {"value": val, "k": k, "kind": kind, "threads": threads, "t": t, "shot": shot}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=40)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="cuda", choices=["cuda", "reference"])
    ap.add_argument("--workload", default="vti_cfd",
                    choices=["vti_cfd", "iso128", "tti_q", "vti_fd8", "iso512", "vti_r2c", "vti_r2r", "small_shots",
                             "small_shots_vti", "tti_q_rtm", "ae_codec"])
    ap.add_argument("--scale", type=float, default=1.0,
                    help="grid scale of the workload (1.0 = the configuration the metric is quoted on; "
                         "smaller values are for profiler captures)")
    ap.add_argument("--state-fp16", action="store_true",
                    help="FP16 wavefield state with per-slab scales (FD8 VTI / TTI workloads)")
    ap.add_argument("--snap", default="c16", choices=["c16", "fp32", "fp16s"],
                    help="snapshot format of the forward step workloads (default: the reference's COMPRESS_16)")
    ap.add_argument("--q-bf16", action="store_true",
                    help="Q memory variables stored as bfloat16 (TTI + Q workloads)")
    ap.add_argument("--kernel-variant", type=int, default=0, choices=[0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10],
                    help="rtm_config.kernel_variant (0 auto; the autotuner then picks among its shapes)")
    ap.add_argument("--no-autotune", action="store_true",
                    help="keep the default launch shapes (profiler runs: timings under a profiler mislead the tuner)")
    ap.add_argument("--snap-offload", type=int, default=0,
                    help="keep the snapshots in pinned host memory with this many device staging slots")
    ap.add_argument("--full-shot", action="store_true",
                    help="tti_q_rtm: run every form's whole 5000-step checkpointed shot instead of timed samples")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    ranks = R.Ranks.from_env()
    world, rank = ranks.world, ranks.rank
    if args.impl == "reference":
        if not R.runs_reference_arm(ranks):
            return
        r = run_reference(args, rank, world)
        if "unavailable" in r:
            print(json.dumps({"impl": "reference", "unavailable": r["unavailable"]}), flush=True)
            return
        shot = r["shot"]
        line = {"metric": "Gpts/s per step", "value": r["value"], "unit": "Gpts/s", "n_gpus": args.gpus,
                "steps": r["k"], "warmup": min(args.warmup, 1), "ms_per_step": r["t"] / r["k"] * 1e3,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic (seeded model)", "impl": "reference",
                "config": config_of(shot, 1, r["k"]),
                "cpu_baseline": {"value": r["value"], "unit": "Gpts/s", "cores": r["threads"], "kind": r["kind"],
                                 "sample": f"{r['k']} full time steps on the full grid, {r['t']:.1f} s"},
                "e2e": {"value": r["value"], "unit": "Gpts/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return
    if world > 1:
        import torch
        torch.cuda.set_device(ranks.local_rank)
        R.init(ranks, "nccl", timeout_s=300)
    else:
        try:
            import torch
            torch.cuda.set_device(0)
        except Exception:
            pass
    if args.workload in ("small_shots", "small_shots_vti"):
        r = run_small_shots(args, ranks)
        if rank == 0:
            line = {"metric": r["metric"], "value": r["value"], "unit": r["unit"], "n_gpus": world,
                    "steps": None, "warmup": args.warmup, "ms_per_step": None, "ms_total": r["ms"],
                    "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                    "data": "synthetic (seeded models)", "config": r["config"], "per_shot_launches": r["per_shot"],
                    "speedup_vs_per_shot": r["value"] / r["per_shot"]["value"] if world == 1 else None,
                    "gpts": r["gpts"], "roofline": r["roofline"], "cpu_baseline": None, "e2e": r["e2e"],
                    "clocks": r["clocks"], "tuned_shape": r["tuned_shape"]}
            print(json.dumps(line), flush=True)
        R.finish(ranks)
        return
    if args.workload == "ae_codec":
        r = run_ae_codec(args, ranks)
        if rank == 0:
            e = r["res"]["encode"]
            line = {"metric": "learned snapshot codec ms per snapshot (encode)", "value": e["ms"], "unit": "ms",
                    "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "higher_is_better": False,
                    "scaling": "weak", "vs_baseline": None, "dtype": "bf16 operands, fp32 accumulation",
                    "data": "synthetic (random volume)",
                    "config": {"workload": "ae_codec: fused encoder / decoder of one {}x{}x{} snapshot ({} 8^3 blocks)"
                               .format(*r["grid"], r["blocks"])},
                    "codec": r["res"],
                    "roofline": {"bound": "hbm", "achieved": e["gbs"], "peak": r["hbm_peak"], "unit": "GB/s",
                                 "frac": e["gbs"] / r["hbm_peak"], "traffic": None,
                                 "tensor": {"achieved_tflops": e["tflops"], "peak_tflops": r["tflops_peak"],
                                            "frac": e["tflops"] / r["tflops_peak"]}},
                    "clocks": r["clocks"]}
            print(json.dumps(line), flush=True)
        R.finish(ranks)
        return
    if args.workload == "tti_q_rtm":
        r = run_rtm_shot(args, ranks)
        if rank == 0:
            f = r["forms"]
            s = r["shot"].spec
            line = {"metric": "RTM s/shot", "value": f["chosen"]["s_per_shot"], "unit": "s/shot", "n_gpus": world,
                    "steps": args.steps, "warmup": args.warmup, "higher_is_better": False, "scaling": "weak",
                    "vs_baseline": None, "dtype": "f32 arithmetic; bf16 Q memory and learned / fp16 snapshots "
                                                  "in the mixed and chosen forms",
                    "data": "synthetic (seeded model)",
                    "config": {"workload": f"tti_q RTM shot: {s.nx}x{s.ny}x{s.nz} FD8 TTI+Q, PML {s.nbnd[0]}, "
                                           f"dt {s.dt * 1e3:.4f} ms, 5000 steps, snapshots every 8 steps",
                               "timing": ("the whole checkpointed shot run and timed (device ms of its loops)"
                                          if args.full_shot else
                                          f"{args.steps} forward + {args.steps} backward full-grid steps timed; "
                                          "s/shot = forward ms/step x (5000 + recomputed steps) + backward ms/step "
                                          "x 5000 + 4 checkpoint copies per extra segment"),
                               "memory": "snapshots that do not fit the HBM left after the engine's arrays run "
                                         "store / recompute (checkpoints at segment starts, earlier segments "
                                         "recomputed in the backward pass); the host (196 GB on these boxes) "
                                         "cannot hold 524 GB of FP32 snapshots either",
                               "image_nrmse": "each form's image vs the plain FP32 form's on the same shot at "
                                              "0.08 scale (51x51x41, 160 steps)",
                               "compressor_training_blocks": r["ntrain"],
                               "forms": {k: RTM_FORMS[k] for k in f}},
                    "s_per_shot": {k: v["s_per_shot"] for k, v in f.items()},
                    "speedup_vs_plain": {k: f["plain"]["s_per_shot"] / v["s_per_shot"] for k, v in f.items()},
                    "image_nrmse_vs_plain": {k: v["image_nrmse_vs_plain"] for k, v in f.items()},
                    "ms_per_step": {k: {"forward": v.get("forward_ms_per_step"),
                                        "backward": v.get("backward_ms_per_step")} for k, v in f.items()},
                    "measured_ms": {k: v["measured_ms"] for k, v in f.items() if "measured_ms" in v},
                    "store_recompute_plan": {k: v["plan"] for k, v in f.items()},
                    "cpu_baseline": None, "clocks": r["clocks"]}
            print(json.dumps(line), flush=True)
        R.finish(ranks)
        return
    r = run_cuda(args, rank, world)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu, _ = cpu_baseline(r["shot"])
    if rank == 0:
        line = {"metric": "Gpts/s per step", "value": r["value"], "unit": "Gpts/s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": r["ms_step"],
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic (seeded model)", "config": r["config"], "roofline": r["roofline"],
                "cpu_baseline": cpu, "e2e": r["e2e"], "clocks": r["clocks"],
                "gpu_launches": r["launches"]}
        print(json.dumps(line), flush=True)
    R.finish(ranks)


if __name__ == "__main__":
    main()
