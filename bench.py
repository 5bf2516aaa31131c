"""Benchmark of the Diff-FVR hot path on B200.

Workload (one "step"): batched candidate screening with the pose adjoint on a
seeded 128^3 ellipsoid volume (1 mm spacing, zero-padded 2x -> 256^3
spectrum): 64 candidate poses x 2 orthogonal parallel views (AP, lateral),
128 x 128 detector, zero-IFFT high-passed spectral NCC loss and its gradient
with respect to the 6-DOF pose.  A pose-eval is one candidate x both views,
loss + 6-DOF gradient.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

Prints one JSON line (rank 0).  Multi-GPU runs are independent replicas (the
path has no exchange step): each rank screens its own 64 candidates; the step
time is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

REPO = Path(__file__).resolve().parent
sys.path.insert(0, str(REPO / "diff-fvr_b200"))
sys.path.insert(0, str(REPO))

METRIC = "pose-evals/sec (fwd+grad) BF16 vs FP32 path at ≤1e-3 rel err; % HBM roofline"
UNIT = "pose-evals/s"
VOL_N, CANDIDATES, OUT_RES, SEED = 128, 64, 128, 0
WORKLOAD = ("batched candidate screening with pose adjoint: seeded 128^3 ellipsoid volume (1 mm) -> 256^3 "
            "spectrum, 64 candidates x 2 parallel views (AP, lateral), 128x128 detector, high-passed zero-IFFT "
            "spectral NCC + 6-DOF pose gradient")
FALLBACK_HBM_GBS = 6650.0


def _dist():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def _max_over_ranks(torch, dist, ws, dev, ms):
    """The slowest rank's time (every rank takes this collective in the same
    order); the local time itself on one rank."""
    if ws <= 1:
        return float(ms)
    t = torch.tensor([float(ms)], device=dev, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def _peak_hbm():
    p = REPO / "MEASURED_PEAKS.json"
    try:
        v = float(json.loads(p.read_text())["hbm_gbs"])
        return v, "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


_SAMPLER = r"""
import sys, time
import pynvml
pynvml.nvmlInit()
ident = sys.argv[1]
h = pynvml.nvmlDeviceGetHandleByUUID(ident) if ident.startswith("GPU-") else pynvml.nvmlDeviceGetHandleByIndex(int(ident))
print("max", pynvml.nvmlDeviceGetMaxClockInfo(h, pynvml.NVML_CLOCK_SM), flush=True)
get_r = getattr(pynvml, "nvmlDeviceGetCurrentClocksEventReasons", None) or pynvml.nvmlDeviceGetCurrentClocksThrottleReasons
while True:
    t = time.time()
    print(f"{t:.6f} {pynvml.nvmlDeviceGetClockInfo(h, pynvml.NVML_CLOCK_SM)} {int(get_r(h))}", flush=True)
    time.sleep(0.002)
"""

_REASONS = {0x4: "sw_power_cap", 0x8: "hw_slowdown", 0x20: "sw_thermal_slowdown", 0x40: "hw_thermal_slowdown",
            0x80: "hw_power_brake_slowdown"}


class ClockSampler:
    """SM clock and clock-event reasons sampled by NVML every ~2 ms in a
    separate process; only the samples inside the marked window are kept."""

    def __init__(self, torch, dev):
        try:
            ident = "GPU-" + str(torch.cuda.get_device_properties(dev).uuid)
        except Exception:
            ident = str(dev.index or 0)
        self.ident = ident
        self.proc = None
        self.t0 = self.t1 = None

    def start(self):
        try:
            self.proc = subprocess.Popen([sys.executable, "-c", _SAMPLER, self.ident], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            line = self.proc.stdout.readline()  # "max <MHz>": the sampler is running
            self.max_mhz = float(line.split()[1]) if line.startswith("max") else None
        except Exception:
            self.proc = None

    def mark(self, begin):
        if begin:
            self.t0 = time.time()
        else:
            self.t1 = time.time()

    def stop(self):
        if self.proc is None:
            return None
        time.sleep(0.01)
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except Exception:
            self.proc.kill()
            out, _ = self.proc.communicate()
        rows = []
        for line in out.splitlines():
            f = line.split()
            if len(f) == 3:
                rows.append((float(f[0]), float(f[1]), int(f[2])))
        inside = [r for r in rows if self.t0 is not None and self.t0 <= r[0] <= self.t1]
        window = "timed region"
        if len(inside) < 3:  # timed region shorter than a few sampling periods
            inside = [r for r in rows if self.t0 - 0.05 <= r[0] <= self.t1 + 0.05]
            window = "timed region +- 50 ms"
        if not inside:
            return None
        reasons = sorted({name for _, _, m in inside for bit, name in _REASONS.items() if m & bit})
        return {"sm_mhz": statistics.median(r[1] for r in inside), "sm_max_mhz": self.max_mhz, "reasons": reasons,
                "samples": len(inside), "window": window, "source": "NVML, 2 ms polling"}


def _setup(torch, dev):
    import fvr
    from fvr import synthetic

    vol = synthetic.make_ellipsoid_volume(VOL_N, SEED)
    poses = synthetic.make_poses(CANDIDATES, SEED + 1)
    tpose = synthetic.make_poses(1, SEED + 2)
    eng = fvr.TorchDiffFVREngine(torch.from_numpy(vol), spacing=(1.0, 1.0, 1.0), pad_factor=2.0, device=dev)
    with torch.no_grad():
        t_ap = eng(torch.from_numpy(tpose).to(dev), view="ap", out_res=OUT_RES)
        t_lat = eng(torch.from_numpy(tpose).to(dev), view="lateral", out_res=OUT_RES)
    f_ap = eng.prepare_spectral_target(t_ap)
    f_lat = eng.prepare_spectral_target(t_lat)
    return vol, poses, eng, f_ap, f_lat


def _time_steps(torch, fn, steps, flush, timer=None, name=None):
    """Per-step device time with CUDA events; L2 flushed (256 MiB write) before
    each step.  With a LaunchTimer the named kernel's launches are timed too."""
    step_ms, kern_ms = [], []
    for _ in range(steps):
        flush.add_(1)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        fn()
        b.record()
        b.synchronize()
        step_ms.append(a.elapsed_time(b))
        if timer is not None:
            kern_ms.extend(timer.durations_ms(name))
    return step_ms, kern_ms


def run_b200(args, torch):
    import torch.distributed as dist
    from fvr import autotune, profiling
    from fvr.graphs import BiplanarSpectralNCCStep

    ws, rank, local = _dist()
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    if ws > 1:
        import datetime

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=dev)
    vol, poses_np, eng, f_ap, f_lat = _setup(torch, dev)
    flush = torch.zeros(64 * 1024 * 1024, dtype=torch.float32, device=dev)  # 256 MiB > 126 MB L2
    poses = torch.from_numpy(poses_np).to(dev)
    sub = torch.from_numpy(poses_np[:4]).to(dev)
    K, W = args.steps, args.warmup
    out = {}

    # FP32 single-candidate eager path through the reference API (the plain baseline)
    def eager_step(p):
        pp = p.detach().requires_grad_(True)
        loss = eng.forward_spectral_ncc(pp, f_ap, view="ap") + eng.forward_spectral_ncc(pp, f_lat, view="lateral")
        loss.backward()
        return loss, pp.grad

    p1 = poses[:1].clone()
    for _ in range(W):
        eager_step(p1)
    t_single, _ = _time_steps(torch, lambda: eager_step(p1), K, flush)

    # batched, graph-captured, per storage precision; the headline (16-bit
    # brick-scaled f16) last, with the hot kernel timed inside the graph
    results = {}
    for name, dt in (("f32", torch.float32), ("bf16", torch.bfloat16), ("f16", torch.float16)):
        if name != "f32":
            eng.to_precision(dt) if name == "bf16" else _f16_from_f32(eng, vol, dev, torch)
        # the measured step is the product graph; a second capture of the same
        # step with CUDA-event nodes around the kernels times them for the
        # roofline (the event nodes add a few microseconds to a replay, so
        # the step time does not come from that graph)
        step = BiplanarSpectralNCCStep(eng, f_ap, f_lat, CANDIDATES, warmup=W)
        timer = profiling.LaunchTimer(["tc_sncc_moments"], capacity=4)
        tstep = BiplanarSpectralNCCStep(eng, f_ap, f_lat, CANDIDATES, warmup=1, capture_context=timer)
        loss, grad = step(poses)
        res = {"loss": float(loss), "grad": grad.detach().cpu().numpy().copy(),
               "img": {v: eng(sub, view=v, out_res=OUT_RES).cpu().numpy() for v in ("ap", "lateral")},
               "kernels_per_step": step._g.kernels_per_replay}
        for _ in range(W):
            step._g.replay()
        if name == "f16":
            clocks = ClockSampler(torch, dev)
            clocks.start()
            if ws > 1:
                dist.barrier()
            torch.cuda.synchronize()
            clocks.mark(True)
        st, _ = _time_steps(torch, step._g.replay, K, flush)
        torch.cuda.synchronize()
        if name == "f16":
            clocks.mark(False)
            if ws > 1:
                dist.barrier()
            res["clocks"] = clocks.stop()
            res["step_obj"] = step
        tstep(poses)  # the same candidate poses in the timing graph's input buffer
        for _ in range(W):
            tstep._g.replay()
        _, km = _time_steps(torch, tstep._g.replay, K, flush, timer, "tc_sncc_moments")
        res["step_ms"], res["kern_ms"] = st, km
        results[name] = res

    f16 = results["f16"]
    total_ms = _max_over_ranks(torch, dist, ws, dev, sum(f16["step_ms"]))
    value = ws * CANDIDATES * K / (total_ms / 1e3)
    step16 = f16.pop("step_obj")

    # e2e through the public step API: host poses in, host (loss, grad) out;
    # one graph replay holds the pinned-host read of the poses and both kernels,
    # the epilogue writing loss and gradient straight into pinned host memory
    h_poses = torch.from_numpy(poses_np).pin_memory()
    h_loss = torch.empty((), dtype=torch.float32).pin_memory()
    h_grad = torch.empty((CANDIDATES, 6), dtype=torch.float32).pin_memory()
    step_io = BiplanarSpectralNCCStep(eng, f_ap, f_lat, CANDIDATES, warmup=W, host_io=True)
    step_io.host_poses.copy_(h_poses)

    def e2e_step():  # the events around it close once the host writes have landed
        step_io(step_io.host_poses, sync=False)

    for _ in range(W):
        e2e_step()
    t_e2e, _ = _time_steps(torch, e2e_step, K, flush)
    e2e_ms = _max_over_ranks(torch, dist, ws, dev, statistics.mean(t_e2e))
    h_loss.copy_(step_io.host_loss)
    h_grad.copy_(step_io.host_grad)
    e2e_grad_match = bool(torch.equal(h_grad, step16(h_poses.to(dev))[1].cpu()))

    def e2e_eager():
        lo, gr = eager_step(h_poses.to(dev, non_blocking=True))
        h_loss.copy_(lo.detach(), non_blocking=True)
        h_grad.copy_(gr, non_blocking=True)

    for _ in range(W):
        e2e_eager()
    t_eager, _ = _time_steps(torch, e2e_eager, K, flush)

    pou = _pou_leg(torch, dev, flush, max(3, min(W, 5)), max(5, min(K, 20)))
    pou8 = _pou_eight_block_leg(torch, dev, flush, max(3, min(W, 5)), max(5, min(K, 20)))
    fwd_only = _sncc_forward_leg(torch, dev, flush, max(3, min(W, 5)), max(5, min(K, 20)))
    npl = _numpy_leg(torch, dev, max(3, min(W, 5)), max(5, min(K, 20)), rank == 0)
    reg = _registration_leg(torch, dev)
    large = _large_volume_leg(torch, dev, flush, max(3, min(W, 5)), max(5, min(K, 20)))
    mine = {"screening": {"graph_f16": value / ws, "eager_api_f16": CANDIDATES / (statistics.mean(t_eager) / 1e3)},
            "forward_one_view": {R: v["ms_per_call"] for R, v in fwd_only["bf16"].items()},
            "pou": {"grid4_P128_det0.8mm": {k: pou[k]["ms_per_step"] for k in ("f32", "bf16")},
                    "grid2_P128_det1.0mm": {k: pou8[k]["forward_backward"]["ms_per_step"] for k in ("f32", "bf16")}}}
    # the reference's own GPU path, single-GPU runs only (its set-up takes longer than the
    # process group's timeout would allow the other ranks to wait)
    ref_gpu = _reference_gpu_leg(torch, dev, flush, max(3, min(W, 5)), max(5, min(K, 20)), mine) if ws == 1 else None

    res = None
    if rank == 0:
        peak, peak_kind = _peak_hbm()
        kern_avg_ms = statistics.mean(f16["kern_ms"])
        # algorithmic bytes per pose-eval, counted for 16-bit storage with
        # brick scales as the logical work of the path: per view and sample the
        # 8-corner gather of the forward pass and again of the adjoint (4 B a
        # corner), the 8 B target and a 4 B brick scale.  The kernel fuses the
        # adjoint into the forward pass and reads each 32 B entry once, so it
        # moves fewer bytes (min_bytes: 32 B of spectrum + target; traffic: ncu's DRAM bytes)
        samples = 2 * CANDIDATES * OUT_RES * OUT_RES
        alg_bytes = samples * (8 * 4 + 8 * 4 + 8 + 4)
        min_bytes = samples * (32 + 8)
        achieved = alg_bytes / (kern_avg_ms * 1e-3) / 1e9
        traffic, ncu = None, {}
        tf = REPO / "profiles" / "tc_sncc_moments_f16pair_128cube_64cand_traffic.txt"
        if tf.exists():
            for line in tf.read_text().splitlines():
                if ":" in line and not line.startswith("#"):
                    k, v = line.split(":", 1)
                    ncu[k.strip()] = float(v)
            traffic = ncu.get("dram_bytes_per_launch")
        cpu = _cpu_baseline_leg(vol, poses_np, f_ap, f_lat, results)
        single_value = 1.0 / (statistics.mean(t_single) / 1e3)
        res = {
            "metric": METRIC,
            "value": value,
            "unit": UNIT,
            "n_gpus": ws,
            "steps": K,
            "warmup": W,
            "ms_per_step": total_ms / K,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f32",
            "data": "synthetic",
            "config": {
                "workload": WORKLOAD,
                "volume": [VOL_N] * 3,
                "spectrum": [2 * VOL_N] * 3,
                "candidates_per_gpu": CANDIDATES,
                "views": 2,
                "out_res": OUT_RES,
                "spectrum_storage": "f16 with power-of-two scales; the moments kernel reads the x-pair copy (two "
                                    "16-byte entries of 4 complex (y, z) corners side by side per sample, "
                                    "scale per 16x16 (z, y) slab); f32 interpolation, positions and phases "
                                    "from fp64 per-row/column tables, fp64 reductions",
                "step": "CUDA-graph replay of two kernels: gather + NCC/pose moments for both views, then the "
                        "fp64 finalize, pose gradient and losses as its programmatic dependent launch; the "
                        "roofline's kernel time comes from a second capture with event nodes around the kernels",
                "l2": "flushed before every timed step (256 MiB write)",
                "parallelism": f"replicas x{ws}",
            },
            "precisions": {
                n: {"value": CANDIDATES * K / (sum(r["step_ms"]) / 1e3), "ms_per_step": statistics.mean(r["step_ms"]),
                    "ms_per_step_min_median_max": [min(r["step_ms"]), statistics.median(r["step_ms"]),
                                                   max(r["step_ms"])],
                    "kernel_ms": statistics.mean(r["kern_ms"]), **cpu["accuracy"][n]}
                for n, r in results.items()
            },
            "fp32_single_candidate_eager": {"value": single_value, "ms_per_step": statistics.mean(t_single)},
            "f16_batched_over_fp32_single": value / ws / single_value,
            "roofline": {
                "bound": "hbm",
                "kernel": "tc_sncc_moments_kernel<f16, grad> + its dependent tc_sncc_final_kernel (timed together; "
                          "both views, 64 candidates)",
                "achieved": achieved,
                "peak": peak,
                "unit": "GB/s",
                "frac": achieved / peak,
                "peak_source": "measured (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured" else
                "fallback 6.65 TB/s",
                "traffic": traffic,
                "ncu_capture": {"source": "profiles/tc_sncc_moments_f16pair_128cube_64cand.md (cold, serialised)",
                                "kernel_us": ncu.get("ncu_kernel_us"),
                                "dram_pct_of_peak": ncu.get("dram_pct_of_peak"),
                                "l2_bytes_per_launch": ncu.get("l2_bytes_per_launch"),
                                "l2_gbs": (ncu["l2_bytes_per_launch"] / ncu["ncu_kernel_us"] / 1e3
                                           if "l2_bytes_per_launch" in ncu and "ncu_kernel_us" in ncu else None),
                                "l2_pct_of_peak": ncu.get("l2_pct_of_peak")},
                "alg_bytes_per_launch": alg_bytes,
                "alg_bytes_note": "64 pose-evals x 2.49 MB: 2 views x 16384 samples x (8 corners x 4 B forward "
                                  "gather + 8 corners x 4 B adjoint gather + 8 B target + 4 B brick scale)",
                "min_bytes_per_launch": min_bytes,
                "achieved_min_bytes_gbs": min_bytes / (kern_avg_ms * 1e-3) / 1e9,
                "frac_min_bytes": min_bytes / (kern_avg_ms * 1e-3) / 1e9 / peak,
                "min_bytes_note": "what the fused kernel must read: 32 B of spectrum (two x-pair entries) + 8 B "
                                  "target per sample",
                "kernel_ms": kern_avg_ms,
                "kernel_launches_timed": len(f16["kern_ms"]),
            },
            "cpu_baseline": cpu["baseline"],
            "e2e": {"value": CANDIDATES * ws / (e2e_ms / 1e3), "unit": UNIT,
                    "h2d_bytes_per_step": int(h_poses.numel() * 4), "d2h_bytes_per_step": int(4 * 3 + h_grad.numel() * 4),
                    "api": "fvr.graphs.BiplanarSpectralNCCStep(host_io=True): pinned host poses in, host loss + grad "
                           "out; one graph replay: a copy kernel reads the pinned poses, the epilogue writes loss "
                           "[ap, lateral, sum] and grad into pinned host memory",
                    "grad_equals_device_step": e2e_grad_match,
                    "eager_api_value": CANDIDATES / (statistics.mean(t_eager) / 1e3),
                    "eager_api": "forward_spectral_ncc(ap) + forward_spectral_ncc(lateral) + backward()"},
            "autotuned_variants": {f"{k[0]}:{'/'.join(str(x) for x in k[1:])}": v[0]
                                   for k, v in autotune.report().items()},
            "gpu_launches": int(f16["kernels_per_step"] * K),
            "kernels_per_step": int(f16["kernels_per_step"]),
            "clocks": f16["clocks"],
            "pou_cone_beam": pou,
            "pou_cone_beam_8_blocks": pou8,
            "spectral_ncc_forward_one_view": fwd_only,
            "numpy_renderer": npl,
            "registration": reg,
            "volume256_spectrum512": large,
            "reference_gpu": ref_gpu,
        }
    if ws > 1:
        dist.barrier()
        del step16
        dist.destroy_process_group()
    return res


def _f16_from_f32(eng, vol, dev, torch):
    """Brick-scaled f16 stencil built from the full-precision spectrum (the bf16
    cast before this is lossy, so rebuild the engine's spectrum first)."""
    import fvr

    fresh = fvr.TorchDiffFVREngine(torch.from_numpy(vol), spacing=(1.0, 1.0, 1.0), pad_factor=2.0, device=dev)
    fresh.to_precision(torch.float16)
    eng._stencil, eng._pair, eng.f_vol_5d = fresh._stencil, fresh._pair, fresh.f_vol_5d


_POU_SECTIONS = ("pou_slice", "pou_warp", "pou_warp_bwd", "pou_slice_adjoint")


def _pou_kernel_times(torch, step, steps, flush):
    """Mean CUDA-event time (ms) of each PoU kernel section over ``steps``
    eager steps (events recorded on the launching stream around each kernel)."""
    from fvr import profiling

    timer = profiling.LaunchTimer(_POU_SECTIONS, capacity=4 * len(_POU_SECTIONS))
    acc = {k: [] for k in _POU_SECTIONS}
    for _ in range(steps):
        flush.add_(1)
        with timer:
            step()
        torch.cuda.synchronize()
        for k in _POU_SECTIONS:
            acc[k].extend(timer.durations_ms(k))
    return {k: statistics.mean(v) for k, v in acc.items() if v}


def _pou_kernel_rooflines(kern_ms, B, N, P, entry):
    """Per-kernel HBM rooflines of the PoU step: algorithmic bytes per launch
    over the kernel's event time.  Block-image kernels: the slice of a real
    block is Hermitian, so one stencil entry (``entry`` bytes) per pair of
    mirrored (block, pose) slice samples must be read, and each sample writes
    (forward) or reads (adjoint) one float of the block image.  On the
    separable pinhole lattice the adjoint section is one fused launch that
    also does the warp adjoint (it reads the forward image instead of an
    image gradient), so no pou_warp_bwd section appears.  The warp kernels
    are bound by issued instructions, not bytes: their times are listed
    only."""
    peak, peak_kind = _peak_hbm()
    samples = B * N * P * P
    out = {"peak": peak, "unit": "GB/s", "peak_source": "measured (MEASURED_PEAKS.json hbm_gbs)"
           if peak_kind == "measured" else "fallback 6.65 TB/s"}
    for name in ("pou_slice", "pou_slice_adjoint"):
        if name in kern_ms:
            alg = samples * (entry // 2 + 4)
            ach = alg / (kern_ms[name] * 1e-3) / 1e9
            out[name] = {"ms": kern_ms[name], "alg_bytes_per_launch": alg, "achieved": ach, "frac": ach / peak}
    for name in ("pou_warp", "pou_warp_bwd"):
        if name in kern_ms:
            out[name] = {"ms": kern_ms[name], "bound": "issue (instructions), see profiles"}
    return out


def _pou_leg(torch, dev, flush, warmup, steps):
    """Secondary line: the PoU-FVR cone-beam step (192^3 ellipsoid volume, 4x4x4
    blocks at 50 % overlap, block_res 64 -> P = 128; pinhole SDD 1020 / SAD 765
    mm, 256^2 detector at 0.8 mm; 64 candidate poses, forward + pose gradient
    through the reference API forward_pinhole(...).sum().backward())."""
    from fvr import synthetic
    from fvr.cone_beam_fvr import PerspectiveSlabFVR

    out = {}
    for name, dt in (("f32", torch.float32), ("bf16", torch.bfloat16), ("f16", torch.float16)):
        vol = synthetic.make_ellipsoid_volume(192, SEED)
        m = PerspectiveSlabFVR.from_volume(vol, vox_mm=1.0, grid_blocks=(4, 4, 4), block_res=64, overlap=0.5,
                                           dtype=dt, device=dev)
        f = 1020.0 / 0.8
        k_inv = torch.tensor([[1.0 / f, 0.0, -128.0 / f], [0.0, 1.0 / f, -128.0 / f], [0.0, 0.0, 1.0]], device=dev)
        lattice = m.make_pinhole_lattice(k_inv, 1020.0, 256, 256)
        mats = synthetic.make_pinhole_mats(CANDIDATES, SEED + 1, sad_mm=765.0, device=dev)

        def step():
            mm = mats.detach().requires_grad_(True)
            m.forward_pinhole(mm, lattice).sum().backward()
            return mm.grad

        for _ in range(warmup):
            step()
        t, _ = _time_steps(torch, step, steps, flush)
        ms = statistics.mean(t)
        value = CANDIDATES / (ms / 1e3)
        kern = _pou_kernel_times(torch, step, steps, flush)
        entry = 64 if name == "f32" else 32
        out[name] = {"value": value, "ms_per_step": ms, "blocks": int(m.B), "P": int(m.P),
                     "kernels": _pou_kernel_rooflines(kern, int(m.B), CANDIDATES, int(m.P), entry)}
        del m, lattice
        torch.cuda.empty_cache()
    out["unit"] = UNIT
    out["workload"] = ("PoU-FVR cone-beam: seeded 192^3 ellipsoid volume (1 mm), 4x4x4 blocks, 50% overlap, "
                       "block_res 64 (P = 128), SDD 1020 / SAD 765 mm, 256x256 detector at 0.8 mm, 64 poses, "
                       "forward + pose gradient (eager autograd through forward_pinhole)")
    out["l2"] = "flushed before every timed step (256 MiB write)"
    return out


def _sncc_forward_leg(torch, dev, flush, warmup, steps):
    """Secondary line in the configuration the reference publishes its
    TorchDiffFVREngine zero-IFFT spectral-NCC GPU timings for: 128^3 volume,
    pad 2 (256^3 spectrum), 16-bit spectrum, one view, 64 candidates,
    out_res 128 / 256 / 512, forward only through forward_spectral_ncc
    (eager, no grad), on the seeded ellipsoid volume."""
    import fvr
    from fvr import synthetic

    vol = synthetic.make_ellipsoid_volume(VOL_N, SEED)
    poses = torch.from_numpy(synthetic.make_poses(CANDIDATES, SEED + 1)).to(dev)
    tp = torch.from_numpy(synthetic.make_poses(1, SEED + 2)).to(dev)
    eng = fvr.TorchDiffFVREngine(torch.from_numpy(vol), spacing=(1.0, 1.0, 1.0), pad_factor=2.0, device=dev)
    targets = {}
    with torch.no_grad():
        for R in (128, 256, 512):
            targets[R] = eng.prepare_spectral_target(eng(tp, view="ap", out_res=R))
    out = {}
    for name, dt in (("bf16", torch.bfloat16), ("f16", torch.float16)):
        if name == "bf16":
            eng.to_precision(dt)
        else:
            eng = fvr.TorchDiffFVREngine(torch.from_numpy(vol), spacing=(1.0, 1.0, 1.0), pad_factor=2.0, device=dev)
            eng.to_precision(dt)
        res = {}
        for R, ft in targets.items():
            def fn():
                with torch.no_grad():
                    return eng.forward_spectral_ncc(poses, ft, view="ap")

            for _ in range(warmup):
                fn()
            t, _ = _time_steps(torch, fn, steps, flush)
            ms = statistics.mean(t)
            res[str(R)] = {"ms_per_call": ms, "poses_per_s": CANDIDATES / (ms / 1e3)}
        out[name] = res
    del eng
    torch.cuda.empty_cache()
    out["workload"] = ("TorchDiffFVREngine.forward_spectral_ncc, one view (AP), 64 candidates, seeded 128^3 "
                       "ellipsoid volume -> 256^3 spectrum, out_res 128 / 256 / 512, forward only, eager")
    out["l2"] = "flushed before every timed call (256 MiB write)"
    return out


def _pou_eight_block_leg(torch, dev, flush, warmup, steps):
    """Secondary line in the block configuration the reference publishes its
    PoU-FVR GPU timings for (2x2x2 blocks at block_res 64 -> P = 128, SDD
    1020 mm, 256^2 detector at 1.0 mm, 64 poses): forward only and forward +
    pose gradient, eager, on the seeded 192^3 ellipsoid volume (the
    reference's own numbers are on a CT volume and another GPU)."""
    from fvr import synthetic
    from fvr.cone_beam_fvr import PerspectiveSlabFVR

    out = {}
    for name, dt in (("f32", torch.float32), ("bf16", torch.bfloat16)):
        vol = synthetic.make_ellipsoid_volume(192, SEED)
        m = PerspectiveSlabFVR.from_volume(vol, vox_mm=1.0, grid_blocks=(2, 2, 2), block_res=64, overlap=0.5,
                                           dtype=dt, device=dev)
        f = 1020.0 / 1.0
        k_inv = torch.tensor([[1.0 / f, 0.0, -128.0 / f], [0.0, 1.0 / f, -128.0 / f], [0.0, 0.0, 1.0]], device=dev)
        lattice = m.make_pinhole_lattice(k_inv, 1020.0, 256, 256)
        mats = synthetic.make_pinhole_mats(CANDIDATES, SEED + 1, sad_mm=765.0, device=dev)

        def fwd():
            with torch.no_grad():
                return m.forward_pinhole(mats, lattice)

        def fwd_bwd():
            mm = mats.detach().requires_grad_(True)
            m.forward_pinhole(mm, lattice).sum().backward()
            return mm.grad

        res = {"blocks": int(m.B), "P": int(m.P)}
        for key, fn in (("forward", fwd), ("forward_backward", fwd_bwd)):
            for _ in range(warmup):
                fn()
            t, _ = _time_steps(torch, fn, steps, flush)
            ms = statistics.mean(t)
            res[key] = {"ms_per_step": ms, "pose_evals_per_s": CANDIDATES / (ms / 1e3)}
        out[name] = res
        del m, lattice
        torch.cuda.empty_cache()
    out["workload"] = ("PoU-FVR cone-beam: seeded 192^3 ellipsoid volume (1 mm), 2x2x2 blocks, 50% overlap, "
                       "block_res 64 (P = 128), SDD 1020 / SAD 765 mm, 256x256 detector at 1.0 mm, 64 poses; "
                       "forward (no grad) and forward + pose gradient, eager")
    out["l2"] = "flushed before every timed step (256 MiB write)"
    return out


def _large_volume_leg(torch, dev, flush, warmup, steps):
    """Secondary line: the large torch-convention case.  Seeded 256^3
    ellipsoid volume (spacing 0.8 x 0.8 x 1.5 mm: voxel-unit spectrum, spacing[0]
    in the phase as the reference uses it) -> 512^3 spectrum, R = 192, 256
    candidates x 2 views, loss + pose gradient as one graph replay per step,
    per storage precision.  Accuracy: against the float64 C oracle (the
    reference's CPU path restated) on the first 4 candidates, whose timing is
    this line's CPU baseline."""
    import fvr
    from fvr import synthetic
    from fvr.graphs import BiplanarSpectralNCCStep

    n, C, R, sp = 256, 256, 192, (0.8, 0.8, 1.5)
    vol = synthetic.make_ellipsoid_volume(n, SEED)
    poses_np = synthetic.make_poses(C, SEED + 1)
    poses = torch.from_numpy(poses_np).to(dev)
    tp = torch.from_numpy(synthetic.make_poses(1, SEED + 2)).to(dev)
    eng = fvr.TorchDiffFVREngine(torch.from_numpy(vol), spacing=sp, pad_factor=2.0, device=dev)
    with torch.no_grad():
        f_ap = eng.prepare_spectral_target(eng(tp, view="ap", out_res=R))
        f_lat = eng.prepare_spectral_target(eng(tp, view="lateral", out_res=R))
    sub = poses[:4].contiguous()
    ref = _large_volume_fp64(vol, poses_np[:4], {"ap": f_ap.cpu().numpy(), "lateral": f_lat.cpu().numpy()}, R, sp[0])

    def rel(a, b):
        return float(np.linalg.norm(a - b) / np.linalg.norm(b))

    out = {}
    for name, dt in (("f32", torch.float32), ("bf16", torch.bfloat16), ("f16", torch.float16)):
        if name == "bf16":
            eng.to_precision(dt)
        elif name == "f16":  # brick-scaled f16 from the full-precision spectrum, not from the bf16 cast
            fresh = fvr.TorchDiffFVREngine(torch.from_numpy(vol), spacing=sp, pad_factor=2.0, device=dev)
            fresh.to_precision(dt)
            eng._stencil, eng._pair, eng.f_vol_5d = fresh._stencil, fresh._pair, fresh.f_vol_5d
            del fresh
        step = BiplanarSpectralNCCStep(eng, f_ap, f_lat, C, warmup=warmup)
        step(poses)
        for _ in range(warmup):
            step._g.replay()
        st, _ = _time_steps(torch, step._g.replay, steps, flush)
        ms = statistics.mean(st)
        lsub, gsub = eng.spectral_ncc_value_and_grad(sub, (f_ap, f_lat), ("ap", "lateral"))
        img = {v: eng(sub, view=v, out_res=R).cpu().numpy() for v in ("ap", "lateral")}
        out[name] = {"value": C / (ms / 1e3), "ms_per_step": ms, "ms_per_step_min_median_max":
                     [min(st), statistics.median(st), max(st)],
                     "roofline": _sncc_step_roofline(name, C, R, ms),
                     "image_rel_l2_vs_fp64": max(rel(img[v], ref["img"][v]) for v in ("ap", "lateral")),
                     "grad_rel_l2_vs_fp64": rel(gsub.cpu().numpy()[:, :5], ref["grad"][:, :5]),
                     "loss_abs_err_vs_fp64": abs(float(lsub) - ref["loss"])}
        del step
    stencil_bytes = {"f32": 513 ** 3 * 64, "f16": 513 ** 3 * 32, "bf16": 513 ** 3 * 32}
    return {"unit": UNIT, "precisions": out, "stencil_bytes": stencil_bytes, "cpu_baseline": ref["baseline"],
            "workload": "seeded 256^3 ellipsoid volume -> 512^3 spectrum (f32 / brick-scaled f16 / bf16 stencils), "
                        "R = 192, 256 candidates x 2 views, loss + 6-DOF gradient per step (CUDA-graph replay, "
                        "L2 flushed before each step)",
            "error_reference": "float64 C oracle and float64 NumPy images on candidates 0-3 (both views): image "
                               "relative L2 (worst view), pose-gradient relative L2 (tz excluded: never read), "
                               "loss absolute error"}


def _large_volume_fp64(vol, poses4, fts, R, sp0):
    """Float64 reference for the large case on 4 candidates: images (NumPy
    restatement) and loss + gradient (C oracle, all host threads, timed: the
    line's CPU baseline sample)."""
    from oracle import c_oracle
    from oracle import torch_convention as tc

    spec = tc.spectrum(vol, 2.0)
    hp = tc.hp_filter(R, R, 4.0)
    ncores = os.cpu_count() or 1
    t0 = time.perf_counter()
    loss, grad = 0.0, np.zeros((poses4.shape[0], 6))
    for v in ("ap", "lateral"):
        lo, _, gr = c_oracle.sncc(spec, poses4, fts[v], v, hp, sp0, threads=ncores)
        loss += lo
        grad += gr
    cpu_s = time.perf_counter() - t0
    img = {v: tc.forward_image(spec, poses4, v, R, sp0) for v in ("ap", "lateral")}
    del spec
    return {"loss": loss, "grad": grad, "img": img,
            "baseline": {"value": poses4.shape[0] / cpu_s, "unit": UNIT, "cores": ncores, "kind": "port",
                         "sample": "4 candidates x 2 views, loss + gradient, float64 C/OpenMP oracle, one run"}}


def _sncc_step_roofline(storage, C, R, ms):
    """Bytes the batched spectral-NCC step must read, over the step's CUDA-event
    time: per view and sample the 8 corners once (8 B a corner in f32, 4 B in
    16-bit storage; the adjoint is fused into the same pass) and the 8 B
    target.  The scope table's logical count (the 8-corner gather again for
    the adjoint, and a 4 B brick scale for f16) is reported beside it."""
    peak, peak_kind = _peak_hbm()
    corner = 8 if storage == "f32" else 4
    alg = 2 * C * R * R * (8 * corner + 8)
    logical = 2 * C * R * R * (2 * 8 * corner + 8 + (4 if storage == "f16" else 0))
    achieved = alg / (ms * 1e-3) / 1e9
    return {"bound": "hbm", "alg_bytes_per_step": alg, "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak, "scope_table_bytes_per_step": logical,
            "scope_table_frac": logical / (ms * 1e-3) / 1e9 / peak,
            "peak_source": "measured (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured" else
            "fallback 6.65 TB/s", "timing": "whole step (graph replay)"}


def _reference_modules():
    """The unmodified reference package installed in baseline/_ref, imported
    under the package name ``fvr_reference`` (its modules import one another
    relatively; this package already owns the name ``fvr``).  Only the two
    modules on the rendering path are imported, so its DICOM reader's
    third-party dependencies are not needed.  None when it is not installed."""
    import importlib
    import types

    root = REPO / "baseline" / "_ref" / "fvr"
    if not (root / "torch_engine.py").exists():
        return None
    if "fvr_reference" not in sys.modules:
        pkg = types.ModuleType("fvr_reference")
        pkg.__path__ = [str(root)]
        sys.modules["fvr_reference"] = pkg
    return (importlib.import_module("fvr_reference.torch_engine"),
            importlib.import_module("fvr_reference.cone_beam_fvr"))


def _reference_gpu_leg(torch, dev, flush, warmup, steps, mine):
    """The reference's own GPU path (its Triton slice and warp kernels, cuFFT
    through torch.fft, eager autograd) on this B200, through its public API,
    on the same seeded workloads, L2 flush and timing as this build's lines:
    the batched spectral-NCC step (forward_spectral_ncc(ap) +
    forward_spectral_ncc(lateral) + backward, 64 candidates, f32 and bf16
    storage), the PoU cone-beam forward + gradient in the 4x4x4 and 2x2x2
    block configurations, and the forward-only spectral NCC at out_res 128 /
    256 / 512.  ``mine`` holds this build's numbers for the same workloads;
    each entry carries both and their ratio."""
    from fvr import synthetic

    mods = _reference_modules()
    if mods is None:
        return {"unavailable": "the reference is not installed in baseline/_ref"}
    te, cb = mods
    out = {"source": "baseline/_ref (pip install --no-deps of the reference checkout), imported as fvr_reference",
           "l2": "flushed before every timed step (256 MiB write)"}

    def timed(fn):
        for _ in range(warmup):
            fn()
        t, _ = _time_steps(torch, fn, steps, flush)
        return statistics.mean(t)

    vol = synthetic.make_ellipsoid_volume(VOL_N, SEED)
    poses = torch.from_numpy(synthetic.make_poses(CANDIDATES, SEED + 1)).to(dev)
    tp = torch.from_numpy(synthetic.make_poses(1, SEED + 2)).to(dev)
    eng = te.TorchDiffFVREngine(torch.from_numpy(vol), spacing=(1.0, 1.0, 1.0), pad_factor=2.0, device=dev,
                                use_triton=True)
    with torch.no_grad():
        f_ap = eng.prepare_spectral_target(eng(tp, view="ap", out_res=OUT_RES))
        f_lat = eng.prepare_spectral_target(eng(tp, view="lateral", out_res=OUT_RES))
        fts = {R: eng.prepare_spectral_target(eng(tp, view="ap", out_res=R)) for R in (128, 256, 512)}

    def sncc_step():
        pp = poses.detach().requires_grad_(True)
        (eng.forward_spectral_ncc(pp, f_ap, view="ap") + eng.forward_spectral_ncc(pp, f_lat, view="lateral")).backward()

    screening = {}
    for name, dt in (("f32", torch.float32), ("bf16", torch.bfloat16)):
        if name == "bf16":
            eng.to_precision(dt)
        ms = timed(sncc_step)
        screening[name] = {"ms_per_step": ms, "pose_evals_per_s": CANDIDATES / (ms / 1e3)}
    screening["workload"] = WORKLOAD
    screening["api"] = "forward_spectral_ncc(ap) + forward_spectral_ncc(lateral) + backward(), eager, use_triton=True"
    for k, v in mine["screening"].items():
        screening[f"this_build_{k}"] = v
        screening[f"ratio_{k}_over_reference_bf16"] = v / screening["bf16"]["pose_evals_per_s"]
    out["screening"] = screening

    fwd = {}
    for R, ft in fts.items():
        def fn():
            with torch.no_grad():
                return eng.forward_spectral_ncc(poses, ft, view="ap")

        ms = timed(fn)
        entry = {"ms_per_call": ms, "poses_per_s": CANDIDATES / (ms / 1e3)}
        got = mine.get("forward_one_view", {}).get(str(R))
        if got is not None:
            entry["this_build_ms_per_call"] = got
            entry["ratio_time_reference_over_this_build"] = ms / got
        fwd[str(R)] = entry
    fwd["storage"] = "bf16 (reference to_precision); this build: bf16 stencil"
    out["spectral_ncc_forward_one_view"] = fwd
    del eng, fts, f_ap, f_lat
    torch.cuda.empty_cache()

    pou = {}
    for label, grid, pitch in (("grid4_P128_det0.8mm", 4, 0.8), ("grid2_P128_det1.0mm", 2, 1.0)):
        pv = synthetic.make_ellipsoid_volume(192, SEED)
        f = 1020.0 / pitch
        k_inv = torch.tensor([[1.0 / f, 0.0, -128.0 / f], [0.0, 1.0 / f, -128.0 / f], [0.0, 0.0, 1.0]], device=dev)
        mats = synthetic.make_pinhole_mats(CANDIDATES, SEED + 1, sad_mm=765.0, device=dev)
        res = {}
        for name, dt in (("f32", torch.float32), ("bf16", torch.bfloat16)):
            m = cb.PerspectiveSlabFVR.from_volume(pv, vox_mm=1.0, grid_blocks=(grid,) * 3, block_res=64, overlap=0.5,
                                                  dtype=dt).to(dev)
            lattice = m.make_pinhole_lattice(k_inv, 1020.0, 256, 256)

            def step():
                mm = mats.detach().requires_grad_(True)
                m.forward_pinhole(mm, lattice).sum().backward()

            ms = timed(step)
            res[name] = {"ms_per_step": ms, "pose_evals_per_s": CANDIDATES / (ms / 1e3), "blocks": int(m.B)}
            got = mine.get("pou", {}).get(label, {}).get(name)
            if got is not None:
                res[name]["this_build_ms_per_step"] = got
                res[name]["ratio_time_reference_over_this_build"] = ms / got
            del m, lattice
            torch.cuda.empty_cache()
        pou[label] = res
    pou["workload"] = ("forward_pinhole(mats).sum().backward(), 64 poses, seeded 192^3 volume, block_res 64 at 50% "
                       "overlap (P = 128), SDD 1020 / SAD 765 mm, 256^2 detector")
    out["pou_cone_beam"] = pou
    return out


REG_VOLUMES = ((128, 128, 128), (192, 192, 192), (160, 256, 256))  # (Z, Y, X) voxels at 1 mm
REG_INITS = 4


def _registration_leg(torch, dev, iters=200, n_cand=CANDIDATES):
    """Secondary line: multi-start biplanar registration on three seeded
    ellipsoid volumes (128^3, 192^3, 256 x 256 x 160 at 1 mm), PoU-FVR 4x4x4
    blocks at block_res 64 (P = 128, bf16 spectra), pinhole SDD 1020 / SAD
    765 mm, 256^2 detector at 1.0 mm, AP and lateral views; per volume four
    seeded ground-truth poses (inits), each registered from 64 candidates
    with 200 Adam iterations.  All 12 registrations (768 candidates) advance
    together: one CUDA-graph replay per Adam iteration renders every volume's
    candidates in both views, forms the losses against each init's
    references and takes the Adam step."""
    from fvr import synthetic
    from fvr.cone_beam_fvr import PerspectiveSlabFVR
    from fvr.registration import MultiVolumeRegistration, sample_multistart_theta, se3_exp

    H, f = 256, 1020.0 / 1.0
    k_inv = torch.tensor([[1.0 / f, 0.0, -0.5 * H / f], [0.0, 1.0 / f, -0.5 * H / f], [0.0, 0.0, 1.0]], device=dev)
    initA = synthetic.make_pinhole_mats(1, 0, sad_mm=765.0, rot_deg=0.0, trans_mm=0.0, device=dev)
    ry90 = torch.tensor([[0.0, 0.0, 1.0, 0.0], [0.0, 1.0, 0.0, 0.0], [-1.0, 0.0, 0.0, 0.0], [0.0, 0.0, 0.0, 1.0]],
                        device=dev)
    initB = ry90 @ initA
    problems, gts, blocks = [], [], []
    for shape in REG_VOLUMES:
        vol = synthetic.make_ellipsoid_volume(max(shape), SEED, shape=shape)
        model = PerspectiveSlabFVR.from_volume(vol, vox_mm=1.0, grid_blocks=(4, 4, 4), block_res=64, overlap=0.5,
                                               dtype=torch.bfloat16, device=dev)
        lattice = model.make_pinhole_lattice(k_inv, 1020.0, H, H)
        # references: rendered from f32 spectra (not the bf16 ones being registered) with seeded
        # Gaussian noise of 2 % of each image's maximum added
        ref_model = PerspectiveSlabFVR.from_volume(vol, vox_mm=1.0, grid_blocks=(4, 4, 4), block_res=64,
                                                   overlap=0.5, dtype=torch.float32, device=dev)
        gen = torch.Generator(device=dev)
        gen.manual_seed(SEED + 9)
        refsA, refsB, thetas, vgt = [], [], [], []
        for i in range(REG_INITS):
            rng = np.random.default_rng(SEED + 7 + 100 * i)
            theta_gt = torch.tensor(np.concatenate([np.radians(rng.uniform(-10, 10, 3)), rng.uniform(-12, 12, 3)])[None],
                                    dtype=torch.float32, device=dev)
            with torch.no_grad():
                dT = se3_exp(theta_gt)
                for refs, init in ((refsA, initA), (refsB, initB)):
                    img = ref_model.forward_pinhole(dT @ init, lattice)
                    refs.append(img + 0.02 * img.amax() * torch.randn(img.shape, generator=gen, device=dev))
            thetas.append(sample_multistart_theta(n_cand, dev, SEED + 8 + 100 * i))
            vgt.append(theta_gt)
        del ref_model
        problems.append((model, lattice, initA, initB, torch.cat(refsA), torch.cat(refsB), torch.cat(thetas)))
        gts.append(vgt)
        blocks.append(int(model.B))
    reg = MultiVolumeRegistration(problems, steps=iters)
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    reg.run(iters)
    best = reg.evaluate()
    b.record()
    b.synchronize()
    total_ms = a.elapsed_time(b)
    g = torch.linspace(-48.0, 48.0, 3, device=dev)
    pts = torch.stack(torch.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3)

    def mtre(T):
        return float((pts @ T[:3, :3].T + T[:3, 3] - pts).norm(dim=1).mean())

    out = {"iterations": iters, "candidates_per_init": n_cand, "inits_per_volume": REG_INITS,
           "candidates_total": reg.total, "wall_ms_total": total_ms, "ms_per_iteration": total_ms / iters,
           "volumes": []}
    with torch.no_grad():
        for shape, nb, vgt, vbest in zip(REG_VOLUMES, blocks, gts, best):
            res = {"shape_zyx": list(shape), "blocks": nb, "best_loss": [], "mtre_mm": [], "rot_err_deg": [],
                   "init_mtre_mm": []}
            for theta_gt, (loss, th) in zip(vgt, vbest):
                rel = se3_exp(th[None]) @ torch.linalg.inv(se3_exp(theta_gt))
                res["best_loss"].append(loss)
                res["mtre_mm"].append(mtre(rel[0]))
                res["rot_err_deg"].append(float(torch.rad2deg(torch.arccos(torch.clamp(
                    (torch.trace(rel[0, :3, :3]) - 1) / 2, -1, 1)))))
                res["init_mtre_mm"].append(mtre(torch.linalg.inv(se3_exp(theta_gt))[0]))
            out["volumes"].append(res)
    del reg, problems
    torch.cuda.empty_cache()
    out["workload"] = ("multi-start biplanar registration: seeded ellipsoid volumes 128^3, 192^3, 256x256x160 "
                       "(Z 160), PoU-FVR 4x4x4 blocks @ block_res 64 (bf16), SDD 1020 / SAD 765 mm, 256^2 at "
                       "1.0 mm, AP + lateral; 4 seeded ground-truth poses per volume (rot U(+-10 deg), trans "
                       "U(+-12 mm)) whose references are rendered from f32 spectra with 2% Gaussian noise, each "
                       "from 64 candidates (rot U(+-12 deg), trans U(+-15 mm)), 200 Adam "
                       "iterations for all 12 registrations at once, each iteration one CUDA-graph replay "
                       "(render every volume's candidates in both views, 0.75 edge NCC + 0.25 NCC loss, adjoint, "
                       "Adam); mTRE of each init's best candidate on a 3x3x3 fiducial grid (+-48 mm)")
    out["timing"] = "CUDA events around the 200 replays and the final evaluation of all 12 registrations"
    return out


def _numpy_leg(torch, dev, warmup, steps, with_cpu):
    """Secondary line: the NumPy-convention renderer (96^3 ellipsoid volume,
    pad 2 -> 192^3 complex128 spectrum) through the reference API
    SpectralGradientEngine.compute_biplanar_loss_and_gradients (AP + lateral
    spectral NCC, closed-form translation and central-difference rotation
    gradient: 14 slices of 192^2), numpy targets in, (loss, grad) out."""
    from fvr import synthetic
    from fvr.diff_fvr import DifferentiableFourierVolumeRenderer
    from fvr.gradients import SpectralGradientEngine

    vol = synthetic.make_ellipsoid_volume(96, SEED).astype(np.float64)
    pose = synthetic.make_poses(1, SEED + 1)[0].astype(np.float64)
    tpose = synthetic.make_poses(1, SEED + 2)[0].astype(np.float64)
    ren = DifferentiableFourierVolumeRenderer(vol, pad_factor=2.0, device=dev)
    eng = SpectralGradientEngine(ren)
    t_ap = ren.extract_frequency_slice(*tpose[:3], tpose[3], tpose[5], view="ap")
    t_lat = ren.extract_frequency_slice(*tpose[:3], tpose[4], tpose[5], view="lateral")
    for _ in range(warmup):
        eng.compute_biplanar_loss_and_gradients(pose, t_ap, t_lat)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(steps):
        loss, grad = eng.compute_biplanar_loss_and_gradients(pose, t_ap, t_lat)
    torch.cuda.synchronize()
    ms = (time.perf_counter() - t0) * 1e3 / steps
    out = {"value": 1e3 / ms, "unit": "pose-evals/s", "ms_per_call": ms,
           "timing": "host wall clock around the API call (numpy in, numpy out, synchronised)",
           "workload": "NumPy-convention renderer: seeded 96^3 ellipsoid volume -> 192^3 complex128 spectrum, "
                       "AP + lateral spectral NCC at one pose with the 6-DOF gradient "
                       "(compute_biplanar_loss_and_gradients, 14 slices of 192^2), fp64"}
    if with_cpu:
        from oracle import numpy_convention as nc

        f3d = nc.spectrum(vol, 2.0)
        ta = nc.extract_frequency_slice(f3d, *tpose[:3], tpose[3], tpose[5], view="ap")
        tl = nc.extract_frequency_slice(f3d, *tpose[:3], tpose[4], tpose[5], view="lateral")
        t0 = time.perf_counter()
        ref_loss, ref_grad = nc.biplanar_loss_and_gradients(f3d, pose, ta, tl)
        cpu_s = time.perf_counter() - t0
        out["cpu_baseline"] = {"value": 1.0 / cpu_s, "unit": "pose-evals/s", "cores": 1, "kind": "port",
                               "sample": "one call of the float64 NumPy oracle (oracle/numpy_convention.py)"}
        out["loss_abs_err_vs_oracle"] = abs(float(loss) - ref_loss)
        out["grad_max_abs_err_vs_oracle"] = float(np.max(np.abs(np.asarray(grad) - ref_grad)))
    return out


def _cpu_baseline_leg(vol, poses_np, f_ap, f_lat, results):
    """The reference's CPU path on this host (float64 C/OpenMP oracle), timed on
    one full step; the same FP64 run is the accuracy reference of every GPU
    precision."""
    from oracle import c_oracle
    from oracle import torch_convention as tc

    spec = tc.spectrum(vol, 2.0)
    hp = tc.hp_filter(OUT_RES, OUT_RES, 4.0)
    fts = {"ap": f_ap.cpu().numpy(), "lateral": f_lat.cpu().numpy()}
    ncores = os.cpu_count() or 1
    ref_grad = np.zeros((CANDIDATES, 6))
    ref_loss = 0.0
    t0 = time.perf_counter()
    reps = 0
    while True:
        ref_grad[:] = 0.0
        ref_loss = 0.0
        for view in ("ap", "lateral"):
            lo, _, gr = c_oracle.sncc(spec, poses_np, fts[view], view, hp, 1.0, threads=ncores)
            ref_grad += gr
            ref_loss += lo
        reps += 1
        if time.perf_counter() - t0 > 5.0 or reps >= 10:
            break
    cpu_s = (time.perf_counter() - t0) / reps

    def rel(a, b):
        return float(np.linalg.norm(a - b) / np.linalg.norm(b))

    sub = poses_np[:4]
    ref_img = {v: tc.forward_image(spec, sub, v, OUT_RES, 1.0) for v in ("ap", "lateral")}
    acc = {}
    for n, r in results.items():
        acc[n] = {"grad_rel_l2_vs_fp64": rel(r["grad"], ref_grad), "loss_abs_err": abs(r["loss"] - ref_loss),
                  "image_rel_l2_vs_fp64": max(rel(r["img"][v], ref_img[v]) for v in ("ap", "lateral"))}
    return {
        "baseline": {"value": CANDIDATES / cpu_s, "unit": UNIT, "cores": ncores, "kind": "port",
                     "sample": "one full step (64 candidates x 2 views, loss + gradient) of the float64 C/OpenMP "
                               f"oracle, mean of {reps} runs"},
        "accuracy": acc,
    }


def run_reference(args):
    """The reference's CPU path for this workload: the float64 C/OpenMP oracle
    restatement of TorchDiffFVREngine.forward_spectral_ncc + backward (the
    reference is Python/PyTorch and does not travel), timed on all host cores."""
    ws, rank, _ = _dist()
    if rank != 0:
        return None
    from fvr import synthetic
    from oracle import c_oracle
    from oracle import torch_convention as tc

    vol = synthetic.make_ellipsoid_volume(VOL_N, SEED)
    poses = synthetic.make_poses(CANDIDATES, SEED + 1)
    tpose = synthetic.make_poses(1, SEED + 2)
    spec = tc.spectrum(vol, 2.0)
    hp = tc.hp_filter(OUT_RES, OUT_RES, 4.0)
    fts = {v: tc.prepare_spectral_target(tc.forward_image(spec, tpose, v, OUT_RES, 1.0)) for v in ("ap", "lateral")}
    ncores = os.cpu_count() or 1

    def step():
        for v in ("ap", "lateral"):
            c_oracle.sncc(spec, poses, fts[v], v, hp, 1.0, threads=ncores)

    for _ in range(args.warmup):
        step()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        step()
    dt = time.perf_counter() - t0
    value = CANDIDATES * args.steps / dt
    torch_cpu = _reference_torch_cpu_sample(vol, poses, tpose, ncores)
    return {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": dt / args.steps * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic", "impl": "reference",
        "config": {"workload": WORKLOAD, "parallelism": "host cores"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": ncores, "kind": "port",
                         "sample": "every step is one full workload step (64 candidates x 2 views, loss + gradient)"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "reference_pytorch_cpu": torch_cpu,
    }


def _reference_torch_cpu_sample(vol, poses_np, tpose_np, ncores):
    """The reference's own PyTorch-CPU implementation (baseline/_ref,
    TorchDiffFVREngine with use_triton=False: grid_sample gather, torch.fft,
    autograd) on the same workload step, timed over 3 steps after one warm-up
    step, all host threads: reported beside the float64 C port, which is the
    line's value."""
    import torch

    mods = _reference_modules()
    if mods is None:
        return {"unavailable": "the reference is not installed in baseline/_ref"}
    te = mods[0]
    torch.set_num_threads(ncores)
    eng = te.TorchDiffFVREngine(torch.from_numpy(vol), spacing=(1.0, 1.0, 1.0), pad_factor=2.0, device="cpu",
                                use_triton=False)
    tp = torch.from_numpy(tpose_np)
    with torch.no_grad():
        f_ap = eng.prepare_spectral_target(eng(tp, view="ap", out_res=OUT_RES))
        f_lat = eng.prepare_spectral_target(eng(tp, view="lateral", out_res=OUT_RES))
    poses = torch.from_numpy(poses_np)

    def step():
        pp = poses.detach().requires_grad_(True)
        (eng.forward_spectral_ncc(pp, f_ap, view="ap") + eng.forward_spectral_ncc(pp, f_lat, view="lateral")).backward()

    step()
    t0 = time.perf_counter()
    for _ in range(3):
        step()
    dt = (time.perf_counter() - t0) / 3
    return {"value": CANDIDATES / dt, "unit": UNIT, "cores": ncores, "ms_per_step": dt * 1e3,
            "sample": "3 full workload steps (64 candidates x 2 views, loss + gradient) after 1 warm-up step",
            "api": "baseline/_ref TorchDiffFVREngine(use_triton=False, device='cpu'): forward_spectral_ncc(ap) + "
                   "forward_spectral_ncc(lateral) + backward()"}


PRECISION_NAMES = ("f32", "bf16", "f16")


def run_profile_case(args, torch):
    """One small hot-path case for a profiler: builds the workload, lets the
    autotuner settle, then runs ``--steps`` steps inside an NVTX range named
    ``fvr_profile`` and prints the mean step time (CUDA events).

    ``sncc``: the batched spectral-NCC graph step (``--volume``^3 ellipsoid
    volume, ``--candidates`` poses x AP + lateral, ``--out-res``^2) in the
    ``--precision`` storage.  ``pou``: the PoU-FVR forward + pose gradient
    (``--volume``^3, ``--grid``^3 blocks at ``--block-res``, 50 % overlap,
    SDD 1020 / SAD 765 mm, ``--det``^2 at 0.8 mm, ``--candidates`` poses)."""
    from fvr import synthetic

    dt = {"f32": torch.float32, "bf16": torch.bfloat16, "f16": torch.float16}[args.precision]
    dev = torch.device("cuda", 0)
    vol = synthetic.make_ellipsoid_volume(args.volume, SEED)
    if args.profile_case == "sncc":
        from fvr.graphs import BiplanarSpectralNCCStep
        from fvr.torch_engine import TorchDiffFVREngine

        poses = torch.from_numpy(synthetic.make_poses(args.candidates, SEED + 1)).to(dev)
        tp = torch.from_numpy(synthetic.make_poses(1, SEED + 2)).to(dev)
        eng = TorchDiffFVREngine(torch.from_numpy(vol), device=dev)
        with torch.no_grad():
            fa = eng.prepare_spectral_target(eng(tp, view="ap", out_res=args.out_res))
            fl = eng.prepare_spectral_target(eng(tp, view="lateral", out_res=args.out_res))
        eng.to_precision(dt)
        st = BiplanarSpectralNCCStep(eng, fa, fl, args.candidates, graph=False)

        def step():
            st(poses)
    else:
        from fvr.cone_beam_fvr import PerspectiveSlabFVR

        g = args.grid
        m = PerspectiveSlabFVR.from_volume(vol, vox_mm=1.0, grid_blocks=(g, g, g), block_res=args.block_res,
                                           overlap=0.5, dtype=dt, device=dev)
        H = args.det
        f = 1020.0 / 0.8
        k_inv = torch.tensor([[1.0 / f, 0.0, -0.5 * H / f], [0.0, 1.0 / f, -0.5 * H / f], [0.0, 0.0, 1.0]],
                             device=dev)
        lattice = m.make_pinhole_lattice(k_inv, 1020.0, H, H)
        mats = synthetic.make_pinhole_mats(args.candidates, SEED + 1, sad_mm=765.0, device=dev)

        def step():
            mm = mats.detach().requires_grad_(True)
            m.forward_pinhole(mm, lattice).sum().backward()

    # backward on this thread, so the NVTX range also covers the adjoint kernels
    torch.autograd.set_multithreading_enabled(False)
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.nvtx.range_push("fvr_profile")
    a.record()
    for _ in range(args.steps):
        step()
    b.record()
    torch.cuda.nvtx.range_pop()
    torch.cuda.synchronize()
    return {"profile_case": args.profile_case, "precision": args.precision,
            "ms_per_step": a.elapsed_time(b) / args.steps}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--profile-case", choices=["sncc", "pou"], default=None,
                    help="run one small case for a profiler instead of the benchmark")
    ap.add_argument("--precision", choices=PRECISION_NAMES, default="f16")
    ap.add_argument("--volume", type=int, default=128)
    ap.add_argument("--candidates", type=int, default=64)
    ap.add_argument("--out-res", type=int, default=128)
    ap.add_argument("--grid", type=int, default=4)
    ap.add_argument("--block-res", type=int, default=64)
    ap.add_argument("--det", type=int, default=256)
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)
    if args.profile_case is not None:
        import torch

        print(json.dumps(run_profile_case(args, torch)), flush=True)
        return
    if args.impl == "reference":
        res = run_reference(args)
    else:
        import torch

        res = run_b200(args, torch)
    if res is not None:
        print(json.dumps(res), flush=True)


if __name__ == "__main__":
    main()
