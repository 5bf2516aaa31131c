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


def _peak_hbm():
    p = REPO / "MEASURED_PEAKS.json"
    try:
        v = float(json.loads(p.read_text())["hbm_gbs"])
        return v, "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.idx = gpu_index
        self.proc = None
        self.path = Path(os.environ.get("TMPDIR", "/tmp")) / f"fvr_clocks_{os.getpid()}.csv"

    def start(self):
        try:
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.idx}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.fh,
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.fh.close()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.path.read_text().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        try:
            self.path.unlink()
        except Exception:
            pass
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def _setup(torch, dev):
    from oracle import torch_convention as tc  # seeded inputs only (generator), not timed
    import fvr
    from fvr import _runtime as RT

    vol = tc.make_ellipsoid_volume(VOL_N, SEED)
    poses = tc.make_poses(CANDIDATES, SEED + 1)
    tpose = tc.make_poses(1, SEED + 2)
    eng = fvr.TorchDiffFVREngine(torch.from_numpy(vol), spacing=(1.0, 1.0, 1.0), pad_factor=2.0, device=dev)
    with torch.no_grad():
        t_ap = eng(torch.from_numpy(tpose).to(dev), view="ap", out_res=OUT_RES)
        t_lat = eng(torch.from_numpy(tpose).to(dev), view="lateral", out_res=OUT_RES)
    f_ap = eng.prepare_spectral_target(t_ap)
    f_lat = eng.prepare_spectral_target(t_lat)
    return vol, poses, eng, f_ap, f_lat, (t_ap, t_lat), tc, RT


def _time_steps(torch, fn, steps, flush, stream=None):
    """Per-step device time with CUDA events; L2 flushed (256 MiB write) before each step."""
    times = []
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    for k in range(steps):
        flush.add_(1)
        a, b = ev[k]
        a.record()
        fn()
        b.record()
    torch.cuda.synchronize()
    for a, b in ev:
        times.append(a.elapsed_time(b))
    return times


def run_b200(args, torch):
    import torch.distributed as dist
    from fvr import _lib as L
    from fvr import profiling
    from fvr.graphs import BiplanarSpectralNCCStep

    ws, rank, local = _dist()
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    if ws > 1:
        import datetime

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=dev)
    vol, poses_np, eng, f_ap, f_lat, targets, tc, RT = _setup(torch, dev)
    flush = torch.zeros(64 * 1024 * 1024, dtype=torch.float32, device=dev)  # 256 MiB > 126 MB L2
    poses = torch.from_numpy(poses_np).to(dev)
    K, W = args.steps, args.warmup

    # --- FP32 single-candidate eager path (the plain baseline of the target) -----------
    def eager_step(e, p):
        pp = p.detach().requires_grad_(True)
        loss = e.forward_spectral_ncc(pp, f_ap, view="ap") + e.forward_spectral_ncc(pp, f_lat, view="lateral")
        loss.backward()
        return loss, pp.grad

    p1 = poses[:1].clone()
    for _ in range(W):
        eager_step(eng, p1)
    t_single = _time_steps(torch, lambda: eager_step(eng, p1), K, flush)

    # --- FP32 batched, graph-captured ---------------------------------------------------------
    step32 = BiplanarSpectralNCCStep(eng, f_ap, f_lat, CANDIDATES, warmup=W)
    loss32, grad32 = step32(poses)
    grad32 = grad32.clone()
    t32 = _time_steps(torch, step32._g.replay, K, flush)
    sub = poses_np[:4]
    img32 = {v: eng(torch.from_numpy(sub).to(dev), view=v, out_res=OUT_RES).cpu().numpy() for v in ("ap", "lateral")}
    del step32

    # --- BF16 batched, graph-captured (headline) ----------------------------------------------
    eng.to_precision(torch.bfloat16)
    timer = profiling.LaunchTimer(["tc_sncc_moments"], capacity=4)
    step16 = BiplanarSpectralNCCStep(eng, f_ap, f_lat, CANDIDATES, warmup=W, capture_context=timer)
    kernels_per_step = step16._g.kernels_per_replay
    loss16, grad16 = step16(poses)
    grad16 = grad16.clone()
    img16 = {v: eng(torch.from_numpy(sub).to(dev), view=v, out_res=OUT_RES).cpu().numpy() for v in ("ap", "lateral")}
    for _ in range(W):
        step16._g.replay()
    clocks = ClockSampler(local)
    clocks.start()
    if ws > 1:
        dist.barrier()
    torch.cuda.synchronize()
    step_ms, kern_ms = [], []
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(K)]
    for k in range(K):
        flush.add_(1)
        a, b = ev[k]
        a.record()
        step16._g.replay()
        b.record()
        b.synchronize()
        step_ms.append(a.elapsed_time(b))
        kern_ms.extend(timer.durations_ms("tc_sncc_moments"))
    torch.cuda.synchronize()
    if ws > 1:
        dist.barrier()
    clk = clocks.stop()
    total_ms = float(sum(step_ms))
    if ws > 1:
        t = torch.tensor([total_ms], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
    ms_per_step = total_ms / K
    value = ws * CANDIDATES * K / (total_ms / 1e3)

    # --- e2e through the public step API with host buffers ---------------------------------
    h_poses = torch.from_numpy(poses_np).pin_memory()
    h_loss = torch.empty((), dtype=torch.float32).pin_memory()
    h_grad = torch.empty((CANDIDATES, 6), dtype=torch.float32).pin_memory()

    def e2e_step():
        loss, grad = step16(h_poses.to(dev, non_blocking=True))
        h_loss.copy_(loss, non_blocking=True)
        h_grad.copy_(grad, non_blocking=True)

    for _ in range(W):
        e2e_step()
    t_e2e = _time_steps(torch, e2e_step, K, flush)
    e2e_ms = statistics.mean(t_e2e)

    # eager public API (no graph), host buffers, for reference
    def e2e_eager():
        lo, gr = eager_step(eng, h_poses.to(dev, non_blocking=True))
        h_loss.copy_(lo.detach(), non_blocking=True)
        h_grad.copy_(gr, non_blocking=True)

    for _ in range(W):
        e2e_eager()
    t_eager = _time_steps(torch, e2e_eager, K, flush)

    res = None
    if rank == 0:
        # --- accuracy vs the FP64 oracle -------------------------------------------------
        from oracle import c_oracle

        spec = tc.spectrum(vol, 2.0)
        hp = tc.hp_filter(OUT_RES, OUT_RES, 4.0)
        ref_grad = np.zeros((CANDIDATES, 6))
        ref_loss = 0.0
        for view, ft in (("ap", f_ap), ("lateral", f_lat)):
            lo, _, gr = c_oracle.sncc(spec, poses_np, ft.cpu().numpy(), view, hp, 1.0)
            ref_grad += gr
            ref_loss += lo

        def rel(a, b):
            return float(np.linalg.norm(a - b) / np.linalg.norm(b))

        img_err = {}
        for name, imgs in (("f32", img32), ("bf16", img16)):
            img_err[name] = max(rel(imgs[v], tc.forward_image(spec, sub, v, OUT_RES, 1.0)) for v in ("ap", "lateral"))
        acc = {
            "bf16": {"grad_rel_l2": rel(grad16.cpu().numpy(), ref_grad), "loss_abs": abs(float(loss16) - ref_loss),
                     "image_rel_l2": img_err["bf16"]},
            "f32": {"grad_rel_l2": rel(grad32.cpu().numpy(), ref_grad), "loss_abs": abs(float(loss32) - ref_loss),
                    "image_rel_l2": img_err["f32"]},
            "oracle": "float64 C/NumPy oracle, all 64 candidates (gradient) / 4 candidates (image)",
        }

        # --- roofline of the dominant kernel --------------------------------------------
        peak, peak_kind = _peak_hbm()
        kern_avg_ms = statistics.mean(kern_ms) if kern_ms else float("nan")
        bytes_per_sample = 32 + 8  # bf16 stencil entry (8 complex corners) + complex64 target sample
        alg_bytes = CANDIDATES * OUT_RES * OUT_RES * bytes_per_sample
        achieved = alg_bytes / (kern_avg_ms * 1e-3) / 1e9
        traffic = None
        tf = REPO / "profiles" / "tc_sncc_moments_cfg2_traffic.txt"
        if tf.exists():
            for line in tf.read_text().splitlines():
                if line.startswith("dram_bytes_per_launch:"):
                    traffic = float(line.split(":", 1)[1])

        # --- CPU baseline: the C oracle on this host, one full step ------------------------
        ncores = os.cpu_count() or 1
        t0 = time.perf_counter()
        reps = 0
        while True:
            for view, ft in (("ap", f_ap), ("lateral", f_lat)):
                c_oracle.sncc(spec, poses_np, ft.cpu().numpy(), view, hp, 1.0, threads=ncores)
            reps += 1
            if time.perf_counter() - t0 > 5.0 or reps >= 10:
                break
        cpu_s = (time.perf_counter() - t0) / reps
        cpu_value = CANDIDATES / cpu_s

        single_value = 1.0 / (statistics.mean(t_single) / 1e3)
        res = {
            "metric": METRIC,
            "value": value,
            "unit": UNIT,
            "n_gpus": ws,
            "steps": K,
            "warmup": W,
            "ms_per_step": ms_per_step,
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
                "spectrum_storage": "bf16 stencil (8 corners per 32-byte entry), f32 interpolation/accumulation",
                "step": "CUDA-graph replay of forward_spectral_ncc(AP) + forward_spectral_ncc(lateral) + backward",
                "l2": "flushed before every timed step (256 MiB write)",
                "parallelism": f"replicas x{ws}",
            },
            "fp32": {"value": CANDIDATES * K / (sum(t32) / 1e3), "ms_per_step": statistics.mean(t32)},
            "fp32_single_candidate_eager": {"value": single_value, "ms_per_step": statistics.mean(t_single)},
            "bf16_batched_over_fp32_single": value / ws / single_value,
            "accuracy_vs_fp64": acc,
            "roofline": {
                "bound": "hbm",
                "kernel": "tc_sncc_moments_kernel<bf16, grad>",
                "achieved": achieved,
                "peak": peak,
                "unit": "GB/s",
                "frac": achieved / peak,
                "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured" else
                "fallback 6.65 TB/s",
                "traffic": traffic,
                "alg_bytes_per_launch": alg_bytes,
                "alg_bytes_note": "64 candidates x 16384 samples x (32 B bf16 stencil entry + 8 B target)",
                "kernel_ms": kern_avg_ms,
                "kernel_launches_timed": len(kern_ms),
            },
            "cpu_baseline": {"value": cpu_value, "unit": UNIT, "cores": ncores, "kind": "port",
                             "sample": "one full step (64 candidates x 2 views, loss + gradient) of the float64 "
                                       f"C/OpenMP oracle, mean of {reps} runs"},
            "e2e": {"value": CANDIDATES * ws / (e2e_ms / 1e3), "unit": UNIT, "h2d_bytes_per_step": int(h_poses.numel() * 4),
                    "d2h_bytes_per_step": int(4 + h_grad.numel() * 4),
                    "api": "fvr.graphs.BiplanarSpectralNCCStep (pinned host poses in, loss + grad out)",
                    "eager_api_value": CANDIDATES / (statistics.mean(t_eager) / 1e3)},
            "gpu_launches": int(kernels_per_step * K),
            "kernels_per_step": int(kernels_per_step),
            "clocks": clk,
        }
    if ws > 1:
        dist.barrier()
        del step16
        dist.destroy_process_group()
    return res


def run_reference(args):
    """The reference's CPU path for this workload: the float64 C/OpenMP oracle
    restatement of TorchDiffFVREngine.forward_spectral_ncc + backward (the
    reference is Python/PyTorch and does not travel), timed on all host cores."""
    ws, rank, _ = _dist()
    if rank != 0:
        return None
    from oracle import c_oracle
    from oracle import torch_convention as tc

    vol = tc.make_ellipsoid_volume(VOL_N, SEED)
    poses = tc.make_poses(CANDIDATES, SEED + 1)
    tpose = tc.make_poses(1, SEED + 2)
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
    return {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": dt / args.steps * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic", "impl": "reference",
        "config": {"workload": WORKLOAD, "parallelism": "host cores"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": ncores, "kind": "port",
                         "sample": "every step is one full workload step (64 candidates x 2 views, loss + gradient)"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)
    if args.impl == "reference":
        res = run_reference(args)
    else:
        import torch

        res = run_b200(args, torch)
    if res is not None:
        print(json.dumps(res), flush=True)


if __name__ == "__main__":
    main()
