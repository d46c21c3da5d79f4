#!/usr/bin/env python
"""Benchmark: frames/s aligned + corrected at 4096^2.

Workload (one step = one movie): 60 synthetic float32 frames of 4096x4096,
5x5 patches, -Iter 10 -Bft 500 150 -Tol 0.1, 0.8 e/px/frame (FmDose 1.161
e/A^2 at 0.83 A/px, 300 kV, dose weighting on), gain uniform in [0.9, 1.1],
global random-walk drift plus a smooth local field of up to 2 px.  The data
are generated on the GPU from a fixed seed (no dataset is needed).

`value`: frames/s with the raw frames already in HBM (device timing with
CUDA events on the work stream, max over ranks).  `e2e`: the same through
the C ABI with pinned host buffers (H2D of the raw frames and D2H of the
sums inside the timed region).  Inputs (4 GB per movie) exceed L2, so no
flush is needed between steps.  Multi-GPU runs are independent replicas
(one movie per GPU, no collective on the data path).

`--impl reference` times the FP64 CPU restatement of the reference path (the
reference has no CPU implementation of its own) on all host cores, on a
bounded sample of the same workload (3 frames of 4096x4096 per step).

`--gpus N` without an outside launcher starts N replica processes itself
(torch.distributed.run, one per GPU, rendezvous on 127.0.0.1).

Accuracy: the CPU-baseline leg (rank 0, one GPU) also writes the timed movie
as an MRC file and runs the reference program built from the reference's
sources (oracle/_ref/MotionCor3, when present) on it with the same options:
the line reports the timed run's shifts and sums against the reference's,
and the reference's own shift error against the generator's drift beside
ours.
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
sys.path.insert(0, ROOT)

METRIC = "frames/s aligned+corrected at 4096^2 vs plain GPU path; shift err <=0.05 px"
CPU_SAMPLE_FRAMES = 3


def workload(cfg: str):
    if cfg == "cfg1":
        return dict(nx=1024, ny=1024, nz=40, dose=1.0, gain=False, local=False,
                    params=dict(patch=(0, 0), iter=7, tol=0.5, bft=(150, 100), pix_size=1.0),
                    name="40x1024^2 global only, -Iter 7 -Tol 0.5 -Bft 150, 1 e/px/frame")
    return dict(nx=4096, ny=4096, nz=60, dose=0.8, gain=True, local=True,
                params=dict(patch=(5, 5), iter=10, tol=0.1, bft=(500, 150), fm_dose=1.161,
                            pix_size=0.83, kv=300),
                name="60x4096^2 float32, -Patch 5 5 -Iter 10 -Bft 500 150, dose-weighted (DW+DWS), gain")


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.samples = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                self.samples.append(parts)

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        mx = [float(s[2]) for s in self.samples if s[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for s in self.samples:
            for i, n in enumerate(names):
                if s[5 + i].lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": sorted(reasons),
                "samples": len(self.samples)}


def measured_peak_hbm():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def max_over_ranks(value: float, dist=None, device="cpu") -> float:
    """The largest value over all ranks (timings are reported as the slowest
    rank's); the value itself without a process group."""
    if dist is None:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def aggregate_rate(ms_local: float, world: int, units_per_rank: int, dist=None,
                   device="cpu"):
    """(slowest rank's milliseconds, units of all ranks per second): replicas
    each process units_per_rank units in ms_local milliseconds."""
    ms = max_over_ranks(ms_local, dist, device)
    return ms, world * units_per_rank / (ms / 1000.0)


def spawn_replicas(args, argv) -> int:
    """Re-runs this script under torch.distributed.run with one process per GPU."""
    import socket
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1",
           f"--nproc-per-node={args.gpus}", "--master-addr", "127.0.0.1", "--master-port",
           str(port), os.path.abspath(__file__)] + list(argv)
    return subprocess.run(cmd).returncode


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def cpu_run(frames, gain, params, steps=1):
    """Oracle (FP64 restatement) on the sample; returns seconds per step."""
    from oracle import oracle as O
    kw = dict(params)
    O.lib()
    ts = []
    for _ in range(steps):
        t0 = time.perf_counter()
        O.process_movie(frames, gain=gain, **kw)
        ts.append(time.perf_counter() - t0)
    return ts


def run_reference(args, wl, world, rank):
    """CPU arm: the FP64 restatement of the reference path on all host cores."""
    if rank != 0:
        return 0
    import numpy as np
    from motioncor3_b200 import synthetic as S
    n = CPU_SAMPLE_FRAMES
    try:
        import torch
        if torch.cuda.is_available():
            mv = S.make_movie(wl["nx"], wl["ny"], n, dose=wl["dose"], seed=7, gain=wl["gain"],
                              local=wl["local"], backend="torch")
            frames = mv.frames.cpu().numpy()
            gain = mv.gain.cpu().numpy() if mv.gain is not None else None
        else:
            raise RuntimeError
    except Exception:
        mv = S.make_movie(wl["nx"], wl["ny"], n, dose=wl["dose"], seed=7, gain=wl["gain"],
                          local=False)
        frames, gain = mv.frames, mv.gain
    params = dict(wl["params"])
    for _ in range(args.warmup):
        cpu_run(frames, gain, params)
    ts = cpu_run(frames, gain, params, steps=args.steps)
    total = sum(ts)
    value = n * args.steps / total
    cores = os.cpu_count() or 1
    sample = f"{n} frames of {wl['nx']}x{wl['ny']} per step, same options"
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "frames/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1000.0 * total / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": wl["name"], "sample": sample, "l2_flush": "inputs > L2"},
        "cpu_baseline": {"value": value, "unit": "frames/s", "cores": cores, "kind": "port",
                         "sample": sample},
        "e2e": {"value": value, "unit": "frames/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def _read_log(path):
    rows = []
    for line in open(path):
        if line.startswith("#") or not line.strip():
            continue
        rows.append([float(v) for v in line.split()])
    return np.asarray(rows, np.float64)


def _sum_agreement(r, o, frac=1e-3):
    """Relative RMS over all pixels; fraction of pixels apart by more than
    `frac` of the RMS (a local-correction gather that moved to the
    neighbouring pixel); relative RMS over the other pixels."""
    r = np.asarray(r, np.float64)
    o = np.asarray(o, np.float64)
    d = o - r
    rms = np.sqrt(np.mean(r * r))
    big = np.abs(d) > frac * rms
    rest = ~big
    return (float(np.sqrt(np.mean(d * d)) / rms), float(big.mean()),
            float(np.sqrt(np.mean(d[rest] ** 2) / np.mean(r[rest] ** 2))))


def reference_check(frames, gain, wl, res, sums, drift, rerun_at=None):
    """Runs the reference program (built from the reference's sources into
    oracle/_ref) on the timed movie with the workload's options; returns the
    timed run's differences from it and both programs' shift errors against
    the generator's drift.  rerun_at(centres) -> (result, sums) processes the
    movie again with given patch centres: used when the reference's centres
    still differ from ours after three runs, so that the patch shifts and
    sums are compared patch for patch."""
    import tempfile
    from motioncor3_b200 import mrcio
    exe = os.path.join(ROOT, "oracle", "_ref", "MotionCor3")
    if not os.path.exists(exe):
        return {"skipped": "reference program not built"}
    pr = wl["params"]
    tags = ["-Patch", str(pr["patch"][0]), str(pr["patch"][1]), "-Iter", str(pr["iter"]),
            "-Tol", str(pr["tol"]), "-Bft", str(pr["bft"][0]), str(pr["bft"][1]),
            "-PixSize", str(pr["pix_size"]), "-Cs", "0"]
    if pr.get("fm_dose"):
        tags += ["-FmDose", str(pr["fm_dose"]), "-kV", str(pr.get("kv", 300))]
    nz = frames.shape[0]
    with tempfile.TemporaryDirectory() as td:
        mvp = os.path.join(td, "movie.mrc")
        if float(frames.max()) <= 255 and np.array_equal(frames, np.round(frames)):
            mrcio.write(mvp, frames.astype(np.uint8))  # Poisson counts: exact in mode 0
        else:
            mrcio.write(mvp, frames)
        args = [exe, "-InMrc", mvp, "-OutMrc", os.path.join(td, "sum.mrc"), "-LogDir", td + "/",
                "-Gpu", "0"] + tags
        if gain is not None:
            mrcio.write(os.path.join(td, "gain.mrc"), gain.astype(np.float32))
            args += ["-Gain", os.path.join(td, "gain.mrc")]
        env = dict(os.environ)
        env["LD_LIBRARY_PATH"] = "/usr/local/cuda/lib64:" + env.get("LD_LIBRARY_PATH", "")
        patch = res.n_patches > 0
        # The reference's feature map is normalised in place while neighbouring
        # threads still read it (Align/GNormByStd2D.cu), so its patch centres
        # can move between runs; it runs up to three times, until its centres
        # equal ours, before the shifts and sums are compared.
        for attempt in range(1, 4):
            p = subprocess.run(args, capture_output=True, text=True, env=env, timeout=900, cwd=td)
            if p.returncode != 0:
                return {"error": "reference program exit " + str(p.returncode)}
            if not patch:
                break
            pp = _read_log(os.path.join(td, "movie-Patch-Patch.log"))
            cen = pp[:, 1:3].reshape(res.n_patches, nz, 2)[:, 0]
            if np.array_equal(cen, res.patch_centers):
                break
        full = _read_log(os.path.join(td, "movie-Patch-Full.log" if patch else "movie-Full.log"))
        ref_g = full[:, 1:3]
        out = {"program": "reference MotionCor3 built from its sources (oracle/_ref)",
               "reference_runs": attempt,
               "global_shift_diff_px_max": float(np.abs(ref_g - res.global_shifts).max())}
        if patch:
            P = res.n_patches
            ref_p = pp[:, 3:5].reshape(P, nz, 2).transpose(1, 0, 2)
            same = bool(np.array_equal(cen, res.patch_centers))
            out["patch_centres_identical"] = same
            if not same and rerun_at is not None:
                out["patch_centres_diff_px_max"] = float(np.abs(cen - res.patch_centers).max())
                res, sums = rerun_at(cen)
                out["compared_at_reference_centres"] = bool(np.array_equal(cen, res.patch_centers))
            out["patch_shift_diff_px_max"] = float(np.abs(ref_p - res.patch_shifts).max())
        for k, suf in enumerate(("", "_DW", "_DWS")[: sums.shape[0]]):
            r = mrcio.read(os.path.join(td, f"sum{suf}.mrc"))[0]
            rel, moved, rest = _sum_agreement(r, sums[k])
            out[f"sum{suf or '_plain'}"] = {"rel_rms": rel, "moved_gather_pixels": moved,
                                            "rel_rms_other_pixels": rest}
    ref_f = nz // 2
    true = -(np.asarray(drift, np.float64) - np.asarray(drift, np.float64)[ref_f])
    for name, g in (("reference", ref_g), ("ours", np.asarray(res.global_shifts, np.float64))):
        d = np.abs((g - g[ref_f]) - true)
        out[f"{name}_err_vs_truth_px_rms"] = float(np.sqrt(np.mean(d ** 2)))
    return out


def run_ours(args, wl, world, rank, local):
    import numpy as np
    import torch
    from motioncor3_b200 import api
    from motioncor3_b200 import synthetic as S

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    nx, ny, nz = wl["nx"], wl["ny"], wl["nz"]
    mv = S.make_movie(nx, ny, nz, dose=wl["dose"], seed=1000 + rank, gain=wl["gain"],
                      local=wl["local"], backend="torch", device=f"cuda:{local}")
    params = api.Params(gpu=local, **wl["params"])
    mc = api.MotionCor3(params)
    stream = torch.cuda.current_stream()
    mc.set_stream(stream.cuda_stream)
    if mv.gain is not None:
        mc.set_gain(mv.gain)
    frames = mv.frames
    info = mc.plan(nx, ny, nz)
    sums = torch.empty((info["n_sums"], ny, nx), dtype=torch.float32, device="cuda")

    def barrier():
        if dist is not None:
            dist.barrier()

    # ---- device-resident timing ----
    for _ in range(args.warmup):
        mc.process(frames, sums_out=sums)
    api.profile_enable(True)
    api.profile_read(reset=True)
    launches0 = api.kernel_launches()
    clocks = ClockSampler(local)
    clocks.start()
    barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    last = None
    for _ in range(args.steps):
        last = mc.process(frames, sums_out=sums)
    e1.record(stream)
    torch.cuda.synchronize()
    barrier()
    clk = clocks.stop()
    ms = e0.elapsed_time(e1)
    launches = (api.kernel_launches() - launches0) // max(args.steps, 1)
    prof = api.profile_read(reset=True)
    api.profile_enable(False)
    ms, value = aggregate_rate(ms, world, nz * args.steps, dist, "cuda")

    # ---- end to end through the C ABI with pinned host buffers ----
    host_frames = frames.cpu().pin_memory()
    host_sums = torch.empty((info["n_sums"], ny, nx), dtype=torch.float32).pin_memory()
    hf, hs = host_frames.numpy(), host_sums.numpy()
    mc.prefetch(hf)
    mc.process(hf, sums_out=hs)
    barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    f0 = torch.cuda.Event(enable_timing=True)
    f1 = torch.cuda.Event(enable_timing=True)
    f0.record(stream)
    # every step copies its movie host->device and its sums back; the copy of
    # movie k+1 runs on the copy stream while movie k is processed
    mc.prefetch(hf)
    for i in range(args.steps):
        if i + 1 < args.steps:
            mc.prefetch(hf)
        mc.process(hf, sums_out=hs)
    f1.record(stream)
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    e2e_ms = max(f0.elapsed_time(f1), wall * 1000.0)
    e2e_ms, e2e = aggregate_rate(e2e_ms, world, nz * args.steps, dist, "cuda")
    h2d = hf.nbytes
    d2h = hs.nbytes

    # ---- roofline of the dominant kernel ----
    peak, peak_kind = measured_peak_hbm()
    top = max(prof.items(), key=lambda kv: kv[1][1]) if prof else None
    roof = None
    if top:
        name, (n_launch, tot_ms, tot_bytes) = top
        achieved = (tot_bytes / n_launch) / ((tot_ms / n_launch) / 1000.0) / 1e9
        # DRAM traffic per launch: the ncu-measured ratio of DRAM bytes to
        # algorithmic bytes for this kernel (profiles/traffic.json, captured
        # on a smaller case of the same launch shape), scaled to this launch
        traffic, traffic_src = None, None
        tp = os.path.join(ROOT, "profiles", "traffic.json")
        if os.path.exists(tp):
            ent = json.load(open(tp)).get(name)
            if ent:
                traffic = ent["dram_over_algorithmic"] * tot_bytes / n_launch
                traffic_src = ent["capture"]
        roof = {"bound": "hbm", "kernel": name, "achieved": achieved, "peak": peak,
                "peak_kind": peak_kind, "unit": "GB/s", "frac": achieved / peak,
                "traffic": traffic, "traffic_source": traffic_src,
                "launches_per_step": n_launch / args.steps,
                "share_of_step": tot_ms / ms if ms else None,
                "algorithmic_bytes_per_launch": tot_bytes / n_launch}

    # ---- accuracy of the timed run: full-frame shifts against the drift the
    #      generator applied (relative to the central frame; the reference's
    #      two smoothings follow a jittery random walk only to about a pixel) ----
    accuracy = None
    try:
        est = np.asarray(last.global_shifts, np.float64)
        ref_f = nz // 2
        est = est - est[ref_f]
        true = -(np.asarray(mv.drift, np.float64) - np.asarray(mv.drift, np.float64)[ref_f])
        d = np.abs(est - true)
        accuracy = {"shift_err_vs_truth_px_max": float(d.max()),
                    "shift_err_vs_truth_px_rms": float(np.sqrt(np.mean(d ** 2))),
                    "iterations_global": int(last.iterations[0])}
    except Exception as exc:  # the report never fails on this extra
        accuracy = {"error": str(exc)}

    # ---- form (1) beside the plain path: the same movie with the patch
    #      transforms' row pass as split-BF16 DFT GEMMs on the tensor cores ----
    forms = None
    if wl["params"].get("patch", (0, 0))[0] > 0 and not args.no_forms:
        try:
            mg = api.MotionCor3(api.Params(gpu=local, dft_gemm=1, **wl["params"]))
            mg.set_stream(stream.cuda_stream)
            if mv.gain is not None:
                mg.set_gain(mv.gain)
            sums_g = torch.empty_like(sums)
            for _ in range(max(args.warmup, 1)):
                mg.process(frames, sums_out=sums_g)
            g0 = torch.cuda.Event(enable_timing=True)
            g1 = torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            g0.record(stream)
            for _ in range(args.steps):
                lg = mg.process(frames, sums_out=sums_g)
            g1.record(stream)
            torch.cuda.synchronize()
            gms = g0.elapsed_time(g1) / args.steps
            dg = float(np.abs(lg.global_shifts - last.global_shifts).max())
            dp = float(np.abs(lg.patch_shifts - last.patch_shifts).max()) if last.n_patches else 0.0
            rel = float(torch.sqrt(torch.mean((sums_g - sums) ** 2) / torch.mean(sums ** 2)))
            mg.close()
            forms = {"split_bf16_dft_gemm": {
                "what": "patch transforms' row pass (408 reals) as 3 BF16 tcgen05 products "
                        "with FP32 accumulation in tensor memory",
                "ms_per_step": gms, "value": nz / gms * 1e3, "unit": "frames/s",
                "max_global_shift_diff_vs_fp32_px": dg, "max_patch_shift_diff_vs_fp32_px": dp,
                "sums_rel_rms_vs_fp32": rel}}
        except Exception as exc:  # the report never fails on this extra
            forms = {"error": str(exc)[-300:]}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        n = CPU_SAMPLE_FRAMES
        sf = host_frames[:n].numpy().copy()
        g = mv.gain.cpu().numpy() if mv.gain is not None else None
        ts = cpu_run(sf, g, dict(wl["params"]))
        cpu = {"value": n / ts[0], "unit": "frames/s", "cores": os.cpu_count() or 1,
               "kind": "port",
               "sample": f"{n} frames of {nx}x{ny} with the same options (FP64 oracle, all cores)"}
        # checker: the reference program on the timed movie
        try:
            def rerun_at(centres):
                mc.set_patch_centers(centres)
                r = mc.process(frames, sums_out=sums)
                mc.set_patch_centers(None)
                return r, sums.cpu().numpy()

            chk = reference_check(host_frames.numpy(), g, wl, last, sums.cpu().numpy(), mv.drift,
                                  rerun_at)
        except Exception as exc:  # the report never fails on this extra
            chk = {"error": str(exc)[-300:]}
        if accuracy is not None:
            accuracy["vs_reference_program"] = chk

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "frames/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic",
            "config": {"workload": wl["name"], "frames_per_step": nz,
                       "parallelism": f"replicas x{world}", "l2_flush": "inputs 4 GB > L2",
                       "iterations_global": int(last.iterations[0]),
                       "iterations_patch_max": int(last.iterations[1:].max()) if last.n_patches else 0},
            "e2e": {"value": e2e, "unit": "frames/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h},
            "gpu_launches": int(launches),
            "clocks": clk,
            "roofline": roof,
            "cpu_baseline": cpu,
            "accuracy": accuracy,
            "forms": forms,
            "kernels": {k: {"launches_per_step": v[0] / args.steps, "ms_per_step": v[1] / args.steps,
                            "GBps": (v[2] / v[1] / 1e6) if v[1] else None}
                        for k, v in sorted(prof.items(), key=lambda kv: -kv[1][1])},
        }
        print(json.dumps(line), flush=True)
    mc.close()
    if dist is not None:
        dist.destroy_process_group()
    return 0


def run_batch(args, world, rank, local):
    """Uneven movies through the movie queue (mc3_submit / mc3_wait): 64
    movies drawn from 2048^2, 4096^2 and 5760x4092 with 20-80 frames each
    (uint8 counts in pinned host memory, 5x5 patches), each size autotuned
    first.  Reports aggregate frames/s and per-movie latency percentiles."""
    import torch
    from motioncor3_b200 import api
    from motioncor3_b200 import synthetic as S
    torch.cuda.set_device(local)
    sizes = [(2048, 2048), (4096, 4096), (5760, 4092)]
    n_movies, max_nz = args.movies, 80
    rng = np.random.default_rng(3 + rank)
    base = {}
    for k, (nx, ny) in enumerate(sizes):
        mv = S.make_movie(nx, ny, max_nz, dose=1.0, seed=300 + 10 * rank + k, local=True,
                          backend="torch", device=f"cuda:{local}")
        base[(nx, ny)] = torch.clamp(mv.frames, 0, 255).to(torch.uint8).cpu().pin_memory()
        del mv
    torch.cuda.empty_cache()
    jobs = [(sizes[int(rng.integers(0, 3))], int(rng.integers(20, max_nz + 1)))
            for _ in range(n_movies)]
    params = api.Params(gpu=local, patch=(5, 5), iter=10, tol=0.1, bft=(500, 150), pix_size=1.0)
    mc = api.MotionCor3(params)
    tuning = {}
    for nx, ny in sizes:
        tuning[f"{nx}x{ny}"] = mc.autotune(nx, ny, 50, args.tuning_json)
    for (nx, ny), nz in jobs[:3]:  # warm-up
        mc.wait(mc.submit(base[(nx, ny)][:nz].numpy()))
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    tickets = [mc.submit(base[(nx, ny)][:nz].numpy()) for (nx, ny), nz in jobs]
    done = [mc.wait(t) for t in tickets]
    wall = time.perf_counter() - t0
    frames = sum(nz for _, nz in jobs)
    lat = np.array([d[1] for d in done])
    dev = np.array([d[0].time_ms for d in done])
    value = frames / wall
    mc.close()
    if rank == 0:
        line = {
            "metric": "frames/s aligned+corrected, uneven movie batch (movie queue)",
            "value": value, "unit": "frames/s", "n_gpus": world, "movies": n_movies,
            "frames": frames, "higher_is_better": True, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "64 movies from {2048^2, 4096^2, 5760x4092} x 20-80 frames, "
                                   "uint8 counts in pinned host memory, -Patch 5 5 -Iter 10 "
                                   "-Bft 500 150", "sizes": [f"{nx}x{ny}x{nz}" for (nx, ny), nz in jobs]},
            "latency_ms_submit_to_done": {"p50": float(np.percentile(lat, 50)),
                                          "p99": float(np.percentile(lat, 99))},
            "device_ms_per_movie": {"p50": float(np.percentile(dev, 50)),
                                    "p99": float(np.percentile(dev, 99))},
            "autotuned_ms_per_movie_at_50_frames": tuning,
            "wall_s": wall,
        }
        print(json.dumps(line), flush=True)
    return 0


def run_dft_rows(args):
    """Form (1) in isolation: the row pass of the patch transforms (rows of
    408 reals, the benchmark's patch width) as the FP32 FFT and as the
    split-BF16 DFT GEMM on the tensor cores, on the same rows (inputs above
    L2), timed with CUDA events; a small fixed case for profiler captures."""
    import torch
    from motioncor3_b200 import api
    rows, nx = args.rows, 408
    x = torch.rand((rows, nx + 2), dtype=torch.float32, device="cuda")
    y = torch.empty((rows, nx // 2 + 1), dtype=torch.complex64, device="cuda")
    out = {"case": "dft_rows", "rows": rows, "points": nx}
    for method, name in ((0, "fp32_fft"), (1, "split_bf16_dft_gemm")):
        for _ in range(args.warmup):
            api.rfft_rows(x, y, nx, method)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(args.steps):
            api.rfft_rows(x, y, nx, method)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / args.steps
        gb = rows * (nx * 4 + (nx // 2 + 1) * 8) / 1e9
        out[name] = {"ms_per_launch": ms, "GBps_algorithmic": gb / ms * 1e3}
        if method == 1:
            out[name]["TFLOPs_3_bf16_products"] = rows * 3 * 2.0 * 416 * 416 / ms / 1e9
    print(json.dumps(out), flush=True)
    return 0


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--config", choices=["cfg2", "cfg1", "cfg3"], default="cfg2")
    ap.add_argument("--movies", type=int, default=64, help="cfg3: movies in the batch")
    ap.add_argument("--tuning-json", default=None, help="cfg3: write the autotuner's choices here")
    ap.add_argument("--case", choices=["movie", "dft_rows"], default="movie",
                    help="dft_rows: the patch row transform alone (FP32 FFT and DFT GEMM)")
    ap.add_argument("--rows", type=int, default=300000, help="dft_rows: rows of 408 reals")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU-baseline sample")
    ap.add_argument("--no-forms", action="store_true",
                    help="skip the split-BF16 DFT GEMM rerun of the timed movie")
    ap.add_argument("--frames", type=int, default=0,
                    help="override the frame count (small cases for profiling; not a bench line)")
    args = ap.parse_args(argv)
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        return spawn_replicas(args, sys.argv[1:] if argv is None else argv)
    world, rank, local = dist_setup()
    if args.case == "dft_rows":
        return run_dft_rows(args)
    if args.config == "cfg3":
        return run_batch(args, world, rank, local) if args.impl == "ours" else 0
    wl = workload(args.config)
    if args.frames > 0:
        wl["nz"] = args.frames
        wl["name"] = wl["name"].replace(f"{workload(args.config)['nz']}x", f"{args.frames}x", 1)
    if args.impl == "reference":
        return run_reference(args, wl, world, rank)
    return run_ours(args, wl, world, rank, local)


if __name__ == "__main__":
    sys.exit(main())
