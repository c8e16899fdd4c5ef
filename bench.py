#!/usr/bin/env python
"""Frames/s of the KinectFusion frame step on B200 (one JSON line on rank 0).

Workload (default): the single-session precision form at 512^3 over a 3 m cube, FP16
TSDF + uint16 weight, split-BF16 J^T J, FP64 solve, ICP {10,5,4}, 512x424 uint16 depth of
a seeded analytic scene (8 spheres + 2 boxes, ground plane) on an orbit; marching cubes
every 100 frames.  A step is one frame of src/kinect.cpp:654-695: depth ingest + pyramid,
ICP, integrate, (recover), raycast.

  value  frames/s with the depth frames already resident in HBM (device timed)
  e2e    frames/s through the C ABI from pinned host frames: every step copies the
         uint16 frame host->device and reads the pose/flags back device->host
Multi-GPU: independent sessions, one per rank (replicas, no collective on the data
path); value is the total over ranks divided by the slowest rank's time.
`--impl reference` times the FP64 CPU port of the reference algorithm (the oracle) on
this host's cores for the same workload.
"""
from __future__ import annotations

import argparse
import glob
import faulthandler
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)


TUNE_FRAME = 15  # the warm-up frame after which the plain form autotunes its launch shapes
PLAIN_WARM = 5  # untimed single-session frames (the ring of frame graphs is captured) before a plain pass


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=200)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--no-autotune", action="store_true",
                   help="keep the default launch shapes instead of autotuning them during warm-up")
    p.add_argument("--launch-shape", default=None, metavar="ZC,ROWS",
                   help="fix the plain form's launch shapes (integrate z-chunk, raycast tile rows; "
                        "rows 1 = persistent sweep) instead of autotuning them")
    p.add_argument("--impl", choices=["ours", "reference"], default="ours")
    p.add_argument("--workload", choices=["c2", "c1"], default="c2",
                   help="plain form's workload: c2 = the 512^3 precision form (default line); "
                        "c1 = the 128^3 FP32 plain form (storage and J^T J from the workload)")
    p.add_argument("--size", type=int, default=512)
    p.add_argument("--storage", choices=["f16u16", "f32f32", "rg16i"], default="f16u16")
    p.add_argument("--jtj", choices=["bf16", "fp32"], default="bf16")
    p.add_argument("--cpu-frames", type=int, default=4, help="oracle frames timed for cpu_baseline")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-reference-quirks", action="store_true",
                   help="skip the pass with the reference's own quirk set")
    p.add_argument("--no-forms", action="store_true",
                   help="skip the batched and served sub-records of the default line")
    p.add_argument("--form", choices=["plain", "batched", "served", "large"], default="plain",
                   help="plain: the single-session frame step (default line); batched: config 3; "
                        "served: config 4; large: config 5")
    p.add_argument("--sessions", type=int, default=64, help="batched form: sessions per batch")
    p.add_argument("--duration", type=float, default=30.0, help="served form: seconds of arrivals")
    p.add_argument("--slots", type=int, default=128, help="served form: resident session slots")
    return p.parse_args()


def workload(args, n_frames):
    from oglfusionkinectv2_b200 import synth, _lib as L
    if getattr(args, "workload", "c2") == "c1":
        return synth.plain_c1(n_frames=n_frames)
    storage = {"f16u16": L.KF_STORAGE_F16U16, "f32f32": L.KF_STORAGE_F32F32, "rg16i": L.KF_STORAGE_RG16I}[args.storage]
    jtj = L.KF_JTJ_SPLIT_BF16 if args.jtj == "bf16" else L.KF_JTJ_FP32
    return synth.precision_c2(n_frames=n_frames, storage=storage, jtj=jtj, size=args.size)


def _gen(args_tuple):
    name, size, storage, jtj, n, idx = args_tuple
    from oglfusionkinectv2_b200 import synth
    if name.startswith("c1"):
        w = synth.plain_c1(n_frames=n)
    else:
        w = synth.precision_c2(n_frames=n, storage=storage, jtj=jtj, size=size)
    return idx, w.frame(idx)


def gen_frames(w, indices, procs):
    """Render frames in a spawn pool (started before any CUDA call)."""
    import multiprocessing as mp
    c = w.config
    jobs = [(w.name, c.volumeSize[0], c.storage, c.jtj, w.n_frames, i) for i in indices]
    if procs <= 1 or len(jobs) < 4:
        return {i: w.frame(i) for i in indices}
    ctx = mp.get_context("spawn")
    with ctx.Pool(procs) as pool:
        return dict(pool.map(_gen, jobs, chunksize=4))


class ClockSampler:
    """Samples SM clock and throttle reasons through NVML while the timed region runs."""

    REASONS = {0x1: "gpu_idle", 0x2: "applications_clocks_setting", 0x4: "sw_power_cap",
               0x8: "hw_slowdown", 0x20: "sw_thermal_slowdown", 0x40: "hw_thermal_slowdown",
               0x80: "hw_power_brake_slowdown", 0x100: "display_clock_setting"}

    def __init__(self, device_index: int):
        self.samples, self.reasons = [], set()
        self.max_mhz = None
        self._stop = threading.Event()
        self._h = None
        try:
            import pynvml as N
            N.nvmlInit()
            self.N = N
            import torch
            props = torch.cuda.get_device_properties(device_index)
            uuid = getattr(props, "uuid", None)
            self._h = None
            if uuid is not None:
                try:
                    self._h = N.nvmlDeviceGetHandleByUUID(("GPU-" + str(uuid)).encode())
                except Exception:
                    self._h = None
            if self._h is None:
                # by PCI address (NVML indices ignore CUDA_VISIBLE_DEVICES)
                bus = getattr(props, "pci_bus_id", None)
                dom = getattr(props, "pci_domain_id", 0) or 0
                dv = getattr(props, "pci_device_id", 0) or 0
                if bus is not None:
                    try:
                        self._h = N.nvmlDeviceGetHandleByPciBusId(f"{dom:08x}:{bus:02x}:{dv:02x}.0".encode())
                    except Exception:
                        self._h = None
            if self._h is None:
                self.error = "nvml device not matched (no UUID or PCI bus id match)"
                return
            self.max_mhz = N.nvmlDeviceGetMaxClockInfo(self._h, N.NVML_CLOCK_SM)
        except Exception as e:  # NVML unavailable: report what we could not sample
            self.error = str(e)

    def _run(self):
        N = self.N
        while not self._stop.is_set():
            try:
                self.samples.append(N.nvmlDeviceGetClockInfo(self._h, N.NVML_CLOCK_SM))
                mask = N.nvmlDeviceGetCurrentClocksEventReasons(self._h)
                for bit, name in self.REASONS.items():
                    if mask & bit and bit != 0x1:
                        self.reasons.add(name)
            except Exception:
                pass
            time.sleep(0.05)

    def __enter__(self):
        if self._h is not None:
            self._t = threading.Thread(target=self._run, daemon=True)
            self._t.start()
        return self

    def __exit__(self, *exc):
        self._stop.set()
        if self._h is not None:
            self._t.join()

    def summary(self):
        if self._h is None:
            return {"sm_mhz": None, "sm_max_mhz": None,
                    "reasons": [getattr(self, "error", None) or "nvml unavailable"]}
        s = sorted(self.samples)
        return {"sm_mhz": s[len(s) // 2] if s else None, "sm_max_mhz": self.max_mhz,
                "reasons": sorted(self.reasons), "samples": len(s)}


def measured_traffic(workload: str, stage: str):
    """DRAM bytes (read + write) per launch of the stage's kernel from the committed ncu capture
    of this workload (profiles/*_traffic.txt: "<kernel> <workload> dram_bytes_per_launch <n>"),
    or None when none was captured."""
    kernel = {"integrate": "integrate_kernel", "raycast": "raycast_kernel", "track": "icp_kernel"}.get(stage)
    for path in glob.glob(os.path.join(os.path.dirname(os.path.abspath(__file__)), "profiles", "*_traffic.txt")):
        for line in open(path):
            f = line.split()
            if len(f) == 4 and f[0] == kernel and f[1] == workload and f[2] == "dram_bytes_per_launch":
                return int(f[3])
    return None


def measured_peak_hbm():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def algorithmic_bytes(cfg, stage):
    """Per-launch algorithmic bytes of a stage (the per-unit byte model times the units)."""
    n = int(np.prod(cfg.volumeSize))
    bv = 8 if cfg.storage == 0 else 4          # bytes per voxel (value + weight)
    p0 = 512 * 424
    if stage == "integrate":                   # read + write every voxel, depth in
        return 2 * bv * n + 4 * p0
    if stage == "raycast":                     # value plane read once, vertex + normal out
        return (bv // 2) * n + 32 * p0
    if stage == "track":                       # per ICP iteration at level l: 4 float4 maps read
        return sum(int(it) * 64 * (p0 >> (2 * l)) for l, it in enumerate(cfg.iterations))
    raise ValueError(stage)


def stage_rooflines(w, per, peak):
    out = {}
    for stage in ("integrate", "raycast", "track"):
        ms = per.get(stage) or 0.0
        if ms <= 0:
            continue
        algo = algorithmic_bytes(w.config, stage)
        gbs = algo / (ms / 1000.0) / 1e9
        traffic = measured_traffic(w.name, stage)
        out[stage] = {"algorithmic_bytes": algo, "ms": ms, "achieved": gbs, "frac": gbs / peak,
                      "traffic": traffic,
                      "traffic_frac": (traffic / (ms / 1000.0) / 1e9 / peak if traffic else None)}
    return out


CPU_WARM_FRAMES = 2  # untimed oracle frames before the timed cpu_baseline sample


def cpu_baseline(args, w, frames_by_idx):
    """Time the FP64 oracle (CPU port of the reference algorithm) on a bounded sample: frames
    0 .. CPU_WARM_FRAMES + cpu_frames - 1 of the sequence from the first ground-truth pose.
    Returns the baseline record, the oracle's pose after every frame, and the oracle's final
    volume (raw bytes) for the accuracy comparison."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import kf_oracle as O
    O.Oracle.set_threads(0)
    o = O.Oracle(w.config, w.intrinsics)
    o.Reset(w.poses[0])
    warm = CPU_WARM_FRAMES
    n = max(1, args.cpu_frames)
    poses = []
    for i in range(warm):
        o.frameStep(frames_by_idx[i])
        poses.append(o.getPose())
    t0 = time.perf_counter()
    for i in range(warm, warm + n):
        o.frameStep(frames_by_idx[i])
        poses.append(o.getPose())
    dt = time.perf_counter() - t0
    cores = O.Oracle.threads()
    vol = o.getVolumeRaw()
    o.close()
    rec = {"value": n / dt, "unit": "frames/s", "cores": cores, "kind": "port",
           "sample": f"frames {warm}-{warm + n - 1} of the same {w.config.volumeSize[0]}^3 sequence "
                     f"after {warm} untimed frames (FP64 oracle, OpenMP, {cores} threads)"}
    return rec, poses, vol


def tsdf_error(raw_gpu, raw_oracle, cfg):
    """TSDF value error (in units of the truncation mu: values are stored divided by mu)
    between two raw volumes, over the voxels either side has touched."""
    from oglfusionkinectv2_b200.gfusion import decode_volume
    Fg, Wg = decode_volume(raw_gpu, cfg)
    Fo, Wo = decode_volume(raw_oracle, cfg)
    touched = (Wg > 0) | (Wo > 0)
    d = np.abs(Fg - Fo)[touched]
    n = int(touched.sum())
    return {"voxels_touched": n,
            "max_abs": float(d.max()) if n else 0.0,
            "p99_99_abs": float(np.percentile(d, 99.99)) if n else 0.0,
            "frac_above_1e-3": float(np.mean(d > 1e-3)) if n else 0.0,
            "weight_mismatch_frac": float(np.mean((Wg != Wo)[touched])) if n else 0.0,
            "unit": "TSDF value (fraction of mu)"}


def accuracy_pass(w, base, fbytes, n_steps, prefix, final_pose_ref, shape):
    """A second session steps frames 0 .. n_steps-1 from the first ground-truth pose, one
    synchronous frame at a time, with the timed session's launch shapes (every computation
    is deterministic, so it retraces the timed session: its pose after the last frame is
    compared with the timed session's, bit for bit).  Returns its per-frame poses and its
    raw volume after `prefix` frames."""
    from oglfusionkinectv2_b200 import GFusion
    ga = GFusion(w.config, w.intrinsics)
    ga.Reset(w.poses[0])
    ga.setLaunchShape(*shape)
    poses, vol_prefix = [], None
    for i in range(n_steps):
        ga.frameStepDevice(base + i * fbytes)
        poses.append(ga.getPose())
        if i + 1 == prefix:
            vol_prefix = ga.getVolumeRaw()
    same = bool(np.array_equal(poses[-1], final_pose_ref)) if final_pose_ref is not None else None
    ga.close()
    return poses, vol_prefix, same


def rmse_translation(est, gt) -> float:
    d = np.array([np.linalg.norm(np.asarray(a)[:3, 3] - np.asarray(b)[:3, 3]) for a, b in zip(est, gt)])
    return float(np.sqrt(np.mean(d * d))) if len(d) else 0.0


def run_batched(args, sub=False):
    """Config 3: sessions of uneven volume sizes stepped together (one launch per stage),
    against the same sessions stepped one at a time through the single-session path.
    sub: a bounded pass (20 steps after 5 warm-up steps) whose record is returned for the
    default line instead of printed."""
    import torch
    from oglfusionkinectv2_b200 import GFusion, GFusionBatch, synth
    K, W = (20, 5) if sub else (args.steps, max(3, args.warmup))
    K_plain = min(K, 20)
    n_frames = W + K + PLAIN_WARM + K_plain
    ws = synth.batched_c3(args.sessions, n_frames=n_frames)
    torch.cuda.set_device(0)
    log(f"rendering {len(ws)} x {n_frames} frames on the device")
    frames = [w.frames_torch(range(n_frames), "cuda") for w in ws]
    torch.cuda.synchronize()
    fbytes = 512 * 424 * 2
    gs = []
    for w in ws:
        g = GFusion(w.config, w.intrinsics)
        g.Reset(w.poses[0])
        gs.append(g)
    batch = GFusionBatch(len(gs))
    ptr = lambda i: [f.data_ptr() + i * fbytes for f in frames]
    est = [[] for _ in gs]
    tuned = None
    for i in range(W):
        if i == W - 1 and not args.no_autotune:
            # brick and tile shapes for this mix (scratch copies; the sessions are untouched);
            # one more untimed step rebuilds the batch tables with them
            shape, tms = batch.autotune(gs, repeats=3)
            tuned = {"integrate_z_chunk": shape[0], "raycast_rows": shape[1], "candidates_ms": tms}
        batch.frameStepDevice(gs, ptr(i))
        for j, P in enumerate(batch.poses(len(gs))):
            est[j].append(P)
    torch.cuda.synchronize()
    lat, stage = [], np.zeros(5)
    launches0 = batch.launchCount()
    def collect(t_enqueued):
        # the results of the step enqueued at t_enqueued are on the host now
        lat.append(1000 * (time.perf_counter() - t_enqueued))
        nonlocal stage
        stage = stage + batch.stageTimes()
        for j, P in enumerate(batch.poses(len(gs))):
            est[j].append(P)

    with ClockSampler(0) as clk:
        t0 = time.perf_counter()
        # asynchronous steps: each call enqueues a step and reads the previous one's results,
        # so the device runs a step while the host prepares the next
        t_prev = None
        for i in range(W, W + K):
            ts = time.perf_counter()
            batch.frameStepDeviceAsync(gs, ptr(i))
            if t_prev is not None:
                collect(t_prev)
            t_prev = ts
        batch.sync()
        collect(t_prev)
        wall = time.perf_counter() - t0
    launches = batch.launchCount() - launches0
    # the plain path: the same sessions, one frame step at a time (PLAIN_WARM untimed frames
    # capture each session's ring of frame graphs)
    for i in range(W + K, W + K + PLAIN_WARM):
        for j, g in enumerate(gs):
            g.frameStepDevice(frames[j].data_ptr() + i * fbytes)
            est[j].append(g.getPose())
    tp = time.perf_counter()
    for i in range(W + K + PLAIN_WARM, W + K + PLAIN_WARM + K_plain):
        for j, g in enumerate(gs):
            g.frameStepDevice(frames[j].data_ptr() + i * fbytes)
    plain_wall = time.perf_counter() - tp
    # the plain configuration (FP32 TSDF + weight, FP32 J^T J), same scenes and sizes, one
    # session at a time through the single-session frame step
    from oglfusionkinectv2_b200 import _lib as L
    g32 = []
    for w in ws:
        c = w.config
        c32 = type(c)(**{**c.__dict__, "storage": L.KF_STORAGE_F32F32, "jtj": L.KF_JTJ_FP32})
        g = GFusion(c32, w.intrinsics)
        g.Reset(w.poses[0])
        g32.append(g)
    W32 = max(W, PLAIN_WARM)
    for i in range(W32):
        for j, g in enumerate(g32):
            g.frameStepDevice(frames[j].data_ptr() + i * fbytes)
    tq = time.perf_counter()
    for i in range(W32, W32 + K_plain):
        for j, g in enumerate(g32):
            g.frameStepDevice(frames[j].data_ptr() + i * fbytes)
    plain32_wall = time.perf_counter() - tq
    del g32
    ate = [rmse_translation(e, w.poses[:len(e)]) for e, w in zip(est, ws)]
    sizes = [w.config.volumeSize[0] for w in ws]
    value = len(gs) * K / wall
    plain = len(gs) * K_plain / plain_wall
    line = {"metric": f"aggregate frames/s, batched form ({len(gs)} sessions, 128-384^3 F16U16)",
            "value": value, "unit": "frames/s", "n_gpus": 1, "steps": K, "warmup": W,
            "ms_per_step": 1000 * wall / K, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "c3_batched", "sessions": len(gs),
                       "sizes": {str(z): sizes.count(z) for z in sorted(set(sizes))},
                       "storage": "f16u16", "jtj": "bf16", "depth": "512x424 uint16 (device-resident)",
                       "l2": "volumes 0.5 GB-5 GB total > L2",
                       "launch_shape": tuned or {"integrate_z_chunk": 16, "raycast_rows": 4, "autotune": "off"}},
            "latency_ms": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99)),
                           "from": "enqueue of a step to its results on the host (steps pipelined one deep)"},
            "stage_ms_per_step": dict(zip(["pyramid", "track", "integrate", "recover", "raycast"],
                                          (stage / K).tolist())),
            "plain_one_at_a_time": {"value": plain, "unit": "frames/s", "steps": K_plain,
                                    "form": "same sessions (F16U16, split-BF16), single-session frame step",
                                    "ratio_batched_over_plain": value / plain},
            "plain_fp32_one_at_a_time": {"value": len(ws) * K_plain / plain32_wall, "unit": "frames/s",
                                         "steps": K_plain,
                                         "form": "same scenes and sizes, FP32 TSDF + FP32 J^T J, single-session frame step",
                                         "ratio_batched_over_plain": value / (len(ws) * K_plain / plain32_wall)},
            "ate_mm": {"mean": 1000 * float(np.mean(ate)), "max": 1000 * float(np.max(ate))},
            "gpu_launches": launches, "clocks": clk.summary()}
    for g in gs:
        g.close()
    batch.close()
    del frames
    torch.cuda.empty_cache()
    if sub:
        return line
    print(json.dumps(line), flush=True)
    return 0


def run_large(args):
    """Config 5: a 768^3 TSDF over 4 m, direct SDF tracking along a room walk (500 frames),
    then full histoPyramid and scan marching cubes."""
    import torch
    from oglfusionkinectv2_b200 import GFusion, MCubes, synth, _lib as L
    K, W = args.steps, max(3, args.warmup)
    w = synth.large_c5(W + K)
    torch.cuda.set_device(0)
    log(f"rendering {W + K} frames of the room on the device")
    frames = w.frames_torch(range(W + K), "cuda")
    torch.cuda.synchronize()
    fbytes = 512 * 424 * 2
    g = GFusion(w.config, w.intrinsics)
    g.Reset(w.poses[0])
    est = []
    for i in range(W):
        g.frameStepDevice(frames.data_ptr() + i * fbytes)
        est.append(g.getPose())
    g.resetStageStats()
    stream = torch.cuda.ExternalStream(g.stream())
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    lost = 0
    with ClockSampler(0) as clk:
        e0.record(stream)
        for i in range(W, W + K):
            lost += 0 if g.frameStepDevice(frames.data_ptr() + i * fbytes) else 1
            est.append(g.getPose())
        e1.record(stream)
        torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    stage_mean, _ = g.stageStats()
    mc = MCubes(g)
    mc.generateMarchingCubes(L.KF_MC_HISTOPYRAMID)  # allocates
    n_hp = mc.generateMarchingCubes(L.KF_MC_HISTOPYRAMID)
    t_hp = float(g.getTimes()[5])
    n_scan = mc.generateMarchingCubes(L.KF_MC_SCAN)
    n_scan = mc.generateMarchingCubes(L.KF_MC_SCAN)
    t_scan = float(g.getTimes()[5])
    ate = rmse_translation(est, w.poses[:len(est)])
    line = {"metric": "frames/s at 768^3 TSDF, SDF tracking (large-volume form)", "value": K / (ms / 1000.0),
            "unit": "frames/s", "n_gpus": 1, "steps": K, "warmup": W, "ms_per_step": ms / K,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (device-rendered room walk, 5% dropouts, flying pixels)",
            "config": {"workload": "c5_large_768", "volume": [768, 768, 768], "dim_m": 4.0, "storage": "f16u16",
                       "tracking": "sdf", "depth": "512x424 uint16 (device-resident)"},
            "stage_ms": dict(zip(["pyramid", "track", "integrate", "recover", "raycast"],
                                 [float(x) for x in stage_mean[:5]])),
            "frames_not_tracked": lost, "ate_mm": 1000 * ate,
            "marching_cubes": {"histopyramid": {"triangles": n_hp, "ms": t_hp},
                               "scan": {"triangles": n_scan, "ms": t_scan}},
            "clocks": clk.summary()}
    print(json.dumps(line), flush=True)
    return 0


def serve_pass(server, arrivals, seqs, gt, duration, fbytes, max_slots):
    """Drive `server` in real time for `duration` seconds: sessions arrive per `arrivals`,
    stream their frames at 30 Hz from the device-resident sequences, and are closed when
    done.  Returns (frames stepped, sessions admitted, max admission wait, per-session
    translation errors)."""
    L_seq = seqs[0].shape[0]
    waiting = list(arrivals)
    active = {}  # sid -> [arrival, t_admit, frames, scene, submitted, errs]
    errs_done = []
    max_wait = 0.0
    t0 = server.now()
    frames = 0
    admitted = 0
    while True:
        t = server.now() - t0
        if t > duration:
            break
        while waiting and waiting[0].t <= t:
            a = waiting[0]
            cfg = gt[a.scene][1]
            cfg.volumeSize = (a.size, a.size, a.size)
            sid = server.open(cfg, gt[a.scene][2], gt[a.scene][0][0])
            if sid is None:
                break
            waiting.pop(0)
            max_wait = max(max_wait, t - a.t)
            active[sid] = [a, t, a.frames, a.scene, 0, []]
            admitted += 1
        for sid, st in active.items():
            a, ta, n, sc, sub, _ = st
            due = min(n, int((t - ta) * 30.0) + 1)
            while sub < due:
                p = sub % (2 * L_seq - 2)
                idx = p if p < L_seq else 2 * L_seq - 2 - p
                server.submit_device(sid, seqs[sc].data_ptr() + idx * fbytes)
                sub += 1
            st[4] = sub
        # asynchronous steps: the device runs this step while the loop admits and queues
        n_done = server.step_async()
        frames += n_done
        if n_done:
            ids, poses, _ = server.last_step(max_slots)
            for sid, P in zip(ids.tolist(), poses):
                a, ta, n, sc, sub, errs = active[sid]
                done = len(errs) + 1
                p = (done - 1) % (2 * L_seq - 2)
                idx = p if p < L_seq else 2 * L_seq - 2 - p
                errs.append(float(np.linalg.norm(P[:3, 3] - gt[sc][0][idx][:3, 3])))
                if done >= n:
                    errs_done.append(errs)
                    server.close_session(sid)
                    del active[sid]
    server.sync()  # the step in flight (its frames are past the measured duration)
    errs_all = errs_done + [st[5] for st in active.values()]
    for sid in list(active):
        server.close_session(sid)
    return frames, admitted, max_wait, errs_all


def run_served(args, sub=False):
    """Config 4: Poisson session arrivals, 30 Hz frame streams, admission by slots and free
    device memory, continuous batching; against the same arrival process stepped one
    session at a time.  sub: a bounded pass (10 s of arrivals) whose record is returned for
    the default line instead of printed."""
    import torch
    from oglfusionkinectv2_b200 import GFusionServer, synth
    torch.cuda.set_device(0)
    duration = 10.0 if sub else args.duration
    n_scenes, L_seq = 16, 300
    arrivals = synth.served_c4(duration, n_scenes=n_scenes)
    scenes = [synth.session_scene(L_seq, splitmix(0xC0FFEE + 4000 + k), 128, phase_deg=22.5 * k,
                                  deg_per_frame=0.5 if k % 2 else -0.5) for k in range(n_scenes)]
    log(f"rendering {n_scenes} x {L_seq} frames on the device; {len(arrivals)} arrivals in {duration} s")
    seqs = [w.frames_torch(range(L_seq), "cuda") for w in scenes]
    torch.cuda.synchronize()
    gt = [(w.poses, w.config, w.intrinsics) for w in scenes]
    fbytes = 512 * 424 * 2
    slots, batch_max = args.slots, min(args.slots, 128)
    sizes = sorted({a.size for a in arrivals})
    results = {}
    for name, max_batch in (("served", batch_max), ("plain_one_at_a_time", 1)):
        server = GFusionServer(max_sessions=slots, max_batch=max_batch)
        # a warm pool: sessions of every volume size created before the arrivals start
        cfg = gt[0][1]
        per = -(-slots // len(sizes)) + 1
        for z in sizes:
            cfg.volumeSize = (z, z, z)
            server.prewarm(cfg, gt[0][2], per)
        with ClockSampler(0) as clk:
            frames, admitted, max_wait, errs = serve_pass(server, arrivals, seqs, gt, duration, fbytes, slots)
        st = server.stats()
        server.close()
        flat = [e for es in errs for e in es]
        results[name] = {"frames_per_s": frames / duration, "frames": frames, "p50_ms": st["p50_ms"],
                         "p99_ms": st["p99_ms"], "max_ms": st["max_ms"], "sessions_admitted": admitted,
                         "max_admission_wait_s": max_wait, "busy_fraction": st["busy_s"] / duration,
                         "pose_err_mm": {"median": 1000 * float(np.median(flat)) if flat else None,
                                         "p99": 1000 * float(np.percentile(flat, 99)) if flat else None},
                         "clocks": clk.summary()}
        log(f"{name}: {results[name]['frames_per_s']:.0f} frames/s p50 {st['p50_ms']:.1f} ms p99 {st['p99_ms']:.1f} ms")
    sv, pl = results["served"], results["plain_one_at_a_time"]
    line = {"metric": "aggregate frames/s, served form (Poisson 20 sessions/s, 30 Hz streams, 128-512^3)",
            "value": sv["frames_per_s"], "unit": "frames/s", "n_gpus": 1, "steps": sv["frames"], "warmup": 0,
            "ms_per_step": 1000.0 / sv["frames_per_s"] if sv["frames_per_s"] else None,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic",
            "config": {"workload": "c4_served", "duration_s": duration, "arrivals": len(arrivals),
                       "slots": slots, "max_batch": batch_max, "storage": "f16u16", "jtj": "bf16",
                       "warm_pool": "sessions of every volume size created before the arrivals",
                       "scenes": f"{n_scenes} seeded sequences of {L_seq} frames, replayed back and forth"},
            "latency_ms": {"p50": sv["p50_ms"], "p99": sv["p99_ms"], "max": sv["max_ms"]},
            "served": sv, "plain_one_at_a_time": pl,
            "ratio_served_over_plain": sv["frames_per_s"] / pl["frames_per_s"] if pl["frames_per_s"] else None}
    del seqs
    torch.cuda.empty_cache()
    if sub:
        return line
    print(json.dumps(line), flush=True)
    return 0


def splitmix(x: int) -> int:
    from oglfusionkinectv2_b200 import synth
    return synth.splitmix64(x) & 0xFFFFFFFF


PLAIN_METRIC = "frames/s at 512^3 TSDF (single session, plain frame step)"


def plain_metric(w):
    n = w.config.volumeSize[0]
    return PLAIN_METRIC if n == 512 else PLAIN_METRIC.replace("512^3", f"{n}^3")


def plain_config(w, args, world):
    """The workload description both arms report for the plain line."""
    from oglfusionkinectv2_b200 import _lib as L
    storage = {L.KF_STORAGE_F16U16: "f16u16", L.KF_STORAGE_F32F32: "f32f32", L.KF_STORAGE_RG16I: "rg16i"}[w.config.storage]
    jtj = "bf16" if w.config.jtj == L.KF_JTJ_SPLIT_BF16 else "fp32"
    return {"workload": w.name, "volume": list(w.config.volumeSize), "dim_m": float(w.config.volumeDimensions[0]),
            "storage": storage, "jtj": jtj, "solve": "f64 cholesky",
            "depth": "512x424 uint16", "icp_iterations": [10, 5, 4],
            "quirks": hex(w.config.quirks), "parallelism": f"replicas x{world}", "mc_every": w.mc_every}


def max_over_ranks(values, world, device):
    """Elementwise maximum of per-rank timings over all ranks (every rank calls it, in the
    same order); the slowest replica sets the job's time."""
    import torch
    t = torch.tensor(values, dtype=torch.float64, device=device)
    if world > 1:
        import torch.distributed as dist
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(x) for x in t]


def aggregate_value(world, steps, ms_max):
    """Whole-job frames/s: every rank steps its own session `steps` frames (replicas)."""
    return world * steps / (ms_max / 1000.0)


def run_reference(args):
    """--impl reference: the reference algorithm's CPU port on this host, same workload."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    steps = max(1, min(args.steps, 12))   # a bounded sample of the workload
    warm = max(1, min(args.warmup, 3))
    w = workload(args, warm + steps)
    frames = {i: w.frame(i) for i in range(warm + steps)}
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import kf_oracle as O
    O.Oracle.set_threads(0)
    o = O.Oracle(w.config, w.intrinsics)
    o.Reset(w.poses[0])
    for i in range(warm):
        o.frameStep(frames[i])
    t0 = time.perf_counter()
    for i in range(warm, warm + steps):
        o.frameStep(frames[i])
    dt = time.perf_counter() - t0
    v = steps / dt
    cores = O.Oracle.threads()
    line = {"impl": "reference", "metric": plain_metric(w), "value": v,
            "unit": "frames/s", "n_gpus": args.gpus, "steps": steps, "warmup": warm,
            "ms_per_step": 1000 * dt / steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {**plain_config(w, args, 1), "sample": "the oracle steps frames only (no marching cubes)"},
            "cpu_baseline": {"value": v, "unit": "frames/s", "cores": cores, "kind": "port",
                             "sample": f"{steps} frames after {warm} untimed (requested {args.steps})"},
            "e2e": {"value": v, "unit": "frames/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def log(msg):
    print(f"[bench {time.strftime('%H:%M:%S')}] {msg}", file=sys.stderr, flush=True)


def main():
    faulthandler.enable()
    args = parse()
    if args.form == "batched" and args.impl == "ours":
        return run_batched(args)
    if args.form == "served" and args.impl == "ours":
        return run_served(args)
    if args.form == "large" and args.impl == "ours":
        return run_large(args)
    if args.impl == "reference":
        return run_reference(args)
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    # the autotuner times its candidates after warm-up frame TUNE_FRAME, on a volume that has
    # fused several views (after the first frame it holds one view's thin shell, on which the
    # raycast's tile shapes rank differently); four more frames then capture the ring of
    # frame graphs
    fixed = tuple(int(x) for x in args.launch_shape.split(",")) if args.launch_shape else None
    if fixed:
        args.no_autotune = True
    K, W = args.steps, max(3 if args.no_autotune else TUNE_FRAME + 5, args.warmup)
    n_e2e = 0 if args.no_e2e else K
    n_lat = 0 if args.no_e2e else max(K, 50)
    n_frames = W + K + n_e2e + 1 + n_lat
    w = workload(args, n_frames)
    ncpu = os.cpu_count() or 1
    log(f"rendering {n_frames} frames")
    frames = gen_frames(w, range(n_frames), max(1, min(16, ncpu // max(1, world))))
    log("frames ready")

    import torch
    torch.cuda.set_device(local)
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600), device_id=torch.device("cuda", local))
    from oglfusionkinectv2_b200 import GFusion, MCubes, _lib as L
    import ctypes as C

    g = GFusion(w.config, w.intrinsics)
    g.Reset(w.poses[0])
    if fixed:
        g.setLaunchShape(*fixed)
    log("session created")
    mc = MCubes(g)
    stream = torch.cuda.ExternalStream(g.stream())
    stack = np.stack([frames[i] for i in range(n_frames)]).view(np.int16)
    dframes = torch.from_numpy(stack).cuda()
    fbytes = 512 * 424 * 2
    base = dframes.data_ptr()
    mc_calls = 0
    mc_ms = []

    def maybe_mc(i):
        nonlocal mc_calls
        if w.mc_every and (i + 1) % w.mc_every == 0:
            mc.generateMarchingCubes(L.KF_MC_HISTOPYRAMID)
            mc_ms.append(float(g.getTimes()[5]))  # device time of the extraction (CUDA events)
            mc_calls += 1

    tuned = None
    for i in range(W):
        g.frameStepDevice(base + i * fbytes, sync=False)
        if i == TUNE_FRAME and not args.no_autotune:
            # brick and tile shapes for this volume and frame (scratch copies; the session is
            # untouched); the following warm-up frames capture the frame graphs with them
            shape, tms = g.autotune(repeats=5)
            tuned = {"integrate_z_chunk": shape[0], "raycast_rows": shape[1], "candidates_ms": tms}
    mc_warm_ms = None
    if w.mc_every:
        mc.generateMarchingCubes(L.KF_MC_HISTOPYRAMID)  # first extraction allocates its buffers
        mc.generateMarchingCubes(L.KF_MC_HISTOPYRAMID)  # a warm one, timed on the device
        mc_warm_ms = float(g.getTimes()[5])
    torch.cuda.synchronize()
    log("warm-up done")
    if world > 1:
        dist.barrier()
    g.resetStageStats()
    launches0 = g.launchCount()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        torch.cuda.synchronize()
        ev0.record(stream)
        for i in range(W, W + K):
            g.frameStepDevice(base + i * fbytes, sync=False)
            maybe_mc(i - W)
        ev1.record(stream)
        torch.cuda.synchronize()
    dev_ms = ev0.elapsed_time(ev1)
    log(f"timed pass {dev_ms:.1f} ms")
    launches = g.launchCount() - launches0
    stage_mean, stage_frames = g.stageStats()
    pose_timed_last = g.getPose()                 # after frame W + K - 1
    tracked_ok = g.frameStepDevice(base + (W + K) * fbytes)  # a synchronised step: state readable

    # end to end: pinned host frames through kf_frame_step_u16_async (H2D frame + D2H
    # pose/flags); each call's result is the previous frame's pose
    e2e = None
    e2e_poses = []
    lib = L.load()
    t = C.c_int()
    if n_e2e:
        pinned = torch.empty((n_e2e + n_lat, 424, 512), dtype=torch.int16).pin_memory()
        pinned.copy_(torch.from_numpy(stack[W + K + 1:W + K + 1 + n_e2e + n_lat]))
        hp = pinned.data_ptr()
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        g.resetStageStats()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        t0 = time.perf_counter()
        # pipelined steps: each call uploads its frame and reads the previous frame's result
        # (pose and flags, 144 B), so the device runs a frame while the host prepares the next
        pose = (C.c_double * 16)()
        for i in range(n_e2e):
            st = lib.kf_frame_step_u16_async(g.handle, C.c_void_p(hp + i * fbytes))
            if st:
                raise L.KfError(st, "kf_frame_step_u16_async")
            if i:
                lib.kf_get_last_result(g.handle, pose, C.byref(t))
                e2e_poses.append(np.array(pose[:]).reshape(4, 4, order="F"))
            maybe_mc(i)
        st = lib.kf_frame_sync(g.handle, C.byref(t))
        if st:
            raise L.KfError(st, "kf_frame_sync")
        e1.record(stream)
        torch.cuda.synchronize()
        wall = time.perf_counter() - t0
        lib.kf_get_last_result(g.handle, pose, C.byref(t))
        e2e_poses.append(np.array(pose[:]).reshape(4, 4, order="F"))
        e2e_ms = e0.elapsed_time(e1)
        log(f"e2e pass {e2e_ms:.1f} ms")
        # the device's own stage times over the same frames: what the end-to-end rate adds
        # to them is host and copy time
        e2e_stage, _ = g.stageStats()
        e2e = {"ms": e2e_ms, "wall_s": wall, "device_ms": float(np.sum(e2e_stage[:5]))}

        # frame latency: synchronous steps from pinned host frames, the host clock from the
        # call to the frame's pose on the host (the session continues the same sequence)
        lat_ms = []
        for i in range(n_e2e, n_e2e + n_lat):
            t1 = time.perf_counter()
            st = lib.kf_frame_step_u16(g.handle, C.c_void_p(hp + i * fbytes), C.byref(t))
            lib.kf_get_pose(g.handle, pose)
            lat_ms.append(1000 * (time.perf_counter() - t1))
            if st:
                raise L.KfError(st, "kf_frame_step_u16")
        e2e["latency_ms"] = {"p50": float(np.percentile(lat_ms, 50)), "p99": float(np.percentile(lat_ms, 99)),
                             "max": float(np.max(lat_ms)), "frames": n_lat,
                             "from": "kf_frame_step_u16 call (pinned host frame) to the frame's pose on the host"}

    # max over ranks of the timed durations
    dev_ms_max, e2e_ms_max = max_over_ranks([dev_ms, e2e["ms"] if e2e else 0.0], world, "cuda")

    out = None
    if rank == 0:
        value = aggregate_value(world, K, dev_ms_max)
        stages = ["pyramid", "track", "integrate", "recover", "raycast"]
        per = {s: float(stage_mean[i]) for i, s in enumerate(stages)}
        dom = "integrate" if per["integrate"] >= per["raycast"] else "raycast"
        peak, peak_kind = measured_peak_hbm()
        algo = algorithmic_bytes(w.config, dom)
        achieved = algo / (per[dom] / 1000.0) / 1e9 if per[dom] > 0 else None
        traffic = measured_traffic(w.name, dom)
        out = {
            "metric": plain_metric(w),
            "value": value, "unit": "frames/s", "n_gpus": world, "steps": K, "warmup": W,
            "ms_per_step": dev_ms_max / K, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {**plain_config(w, args, world),
                       "l2": "volume > L2 (126 MB); inputs resident",
                       "mc_calls": mc_calls, "mc_ms_mean": (float(np.mean(mc_ms)) if mc_ms else None),
                       "launch_shape": tuned or {"integrate_z_chunk": (fixed or (16, 4))[0],
                                                 "raycast_rows": (fixed or (16, 4))[1], "autotune": "off"}},
            "stage_ms": per, "stage_frames": stage_frames,
            "roofline": {"kernel": dom, "bound": "hbm", "achieved": achieved, "peak": peak,
                         "unit": "GB/s", "frac": (achieved / peak if achieved else None),
                         "peak_source": peak_kind, "algorithmic_bytes": algo,
                         "traffic": traffic,
                         # the DRAM bytes the kernel really moves (ncu capture) over its time
                         "traffic_gbs": (traffic / (per[dom] / 1000.0) / 1e9 if traffic and per[dom] > 0 else None),
                         "traffic_frac": (traffic / (per[dom] / 1000.0) / 1e9 / peak if traffic and per[dom] > 0 else None),
                         "traffic_source": "profiles/*_traffic.txt (ncu dram__bytes_read.sum + dram__bytes_write.sum)",
                         # the same figures for the three frame kernels (byte model over the
                         # stage's event-timed mean; ncu DRAM bytes where captured)
                         "stages": stage_rooflines(w, per, peak)},
            "gpu_launches": launches,
            "clocks": clk.summary(),
            "tracked_last": bool(tracked_ok),
        }
        if mc_warm_ms is not None:
            # marching cubes every mc_every frames, amortised over the frames between extractions
            out["mc_every"] = w.mc_every
            out["mc_warm_ms"] = mc_warm_ms
            out["ms_per_step_with_mc"] = dev_ms_max / K + mc_warm_ms / w.mc_every
        if e2e:
            out["e2e"] = {"value": world * n_e2e / (e2e_ms_max / 1000.0), "unit": "frames/s",
                          "h2d_bytes_per_step": fbytes, "d2h_bytes_per_step": 144,
                          "wall_frames_per_s": n_e2e / e2e["wall_s"],
                          "api": "kf_frame_step_u16_async from pinned host frames, each call reading "
                                 "the previous frame's pose and flags",
                          "latency_ms": e2e["latency_ms"],
                          "device_stage_ms_per_frame": e2e["device_ms"]}
    shape_used = g.launchShape()  # the timed session's launch shapes, for the passes below
    g.close()

    if rank == 0 and world == 1 and not args.no_reference_quirks:
        try:
            out["reference_quirks"] = reference_quirks_pass(w, base, fbytes, W, K, shape_used)
        except Exception as e:  # noqa: BLE001
            out["reference_quirks"] = {"error": f"{type(e).__name__}: {e}"}
    if rank == 0 and world == 1:
        # accuracy: ground truth over the timed frames (a deterministic re-run of the same
        # frames) and over the end-to-end frames (that pass's own results); the FP64 oracle
        # over the cpu_baseline prefix, poses and TSDF
        prefix = CPU_WARM_FRAMES + max(1, args.cpu_frames)
        acc = {}
        acc_poses = vol_prefix = None
        try:
            log("accuracy pass")
            acc_poses, vol_prefix, same = accuracy_pass(w, base, fbytes, W + K, prefix, pose_timed_last, shape_used)
            acc["ate_vs_ground_truth_mm"] = {
                "timed_frames": 1000 * rmse_translation(acc_poses[W:W + K], w.poses[W:W + K]),
                "all_frames_to_timed_end": 1000 * rmse_translation(acc_poses, w.poses[:W + K]),
                "rerun_matches_timed_session": same}
            if e2e_poses:
                e2e_gt = w.poses[W + K + 1:W + K + 1 + len(e2e_poses)]
                acc["ate_vs_ground_truth_mm"]["e2e_frames"] = 1000 * rmse_translation(e2e_poses, e2e_gt)
        except Exception as e:  # noqa: BLE001
            acc["error"] = f"{type(e).__name__}: {e}"
        if not args.no_cpu_baseline:
            log("cpu baseline")
            out["cpu_baseline"], o_poses, o_vol = cpu_baseline(args, w, frames)
            if acc_poses is not None:
                try:
                    n = len(o_poses)
                    acc["vs_fp64_oracle"] = {
                        "frames": f"0-{n - 1} (the cpu_baseline frames, same start pose)",
                        "ate_mm": 1000 * rmse_translation(acc_poses[:n], o_poses),
                        "max_translation_diff_mm": 1000 * max(float(np.linalg.norm(a[:3, 3] - b[:3, 3]))
                                                              for a, b in zip(acc_poses[:n], o_poses)),
                        "tsdf_after_prefix": tsdf_error(vol_prefix, o_vol, w.config)}
                except Exception as e:  # noqa: BLE001
                    acc["vs_fp64_oracle"] = {"error": f"{type(e).__name__}: {e}"}
        out["accuracy"] = acc
    if rank == 0 and world == 1 and not args.no_forms:
        # the batched and served forms beside the plain line; a failure there is recorded,
        # it does not lose the plain line
        for key, fn in (("batched", run_batched), ("served", run_served)):
            log(f"{key} form")
            try:
                out[key] = fn(args, sub=True)
            except Exception as e:  # noqa: BLE001
                out[key] = {"error": f"{type(e).__name__}: {e}"}
    if rank == 0:
        print(json.dumps(out), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def reference_quirks_pass(w, base, fbytes, W, K, shape):
    """The same frames with the reference's own behaviour (every quirk bit set: same-pixel
    ICP association and the narrow TSDF band among them), timed like the main pass, with
    its launch shapes."""
    import torch
    from oglfusionkinectv2_b200 import GFusion, _lib as L
    c = w.config
    cq = type(c)(**{**c.__dict__, "quirks": L.KF_QUIRKS_REFERENCE})
    g = GFusion(cq, w.intrinsics)
    g.Reset(w.poses[0])
    g.setLaunchShape(*shape)
    for i in range(W):
        g.frameStepDevice(base + i * fbytes, sync=False)
    torch.cuda.synchronize()
    stream = torch.cuda.ExternalStream(g.stream())
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for i in range(W, W + K):
        g.frameStepDevice(base + i * fbytes, sync=False)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    P = g.getPose()
    g.close()
    return {"value": K / (ms / 1000.0), "unit": "frames/s", "ms_per_step": ms / K,
            "quirks": hex(L.KF_QUIRKS_REFERENCE), "steps": K,
            "translation_error_last_frame_mm": 1000 * float(np.linalg.norm(P[:3, 3] - w.poses[W + K - 1][:3, 3]))}


if __name__ == "__main__":
    sys.exit(main())
