"""Micro-benchmark of one hot path on a seeded synthetic workload.

    python -m fvr.kernel_bench sncc  [--precision f16|bf16|f32] [--volume 128] [--candidates 64] [--out-res 128]
    python -m fvr.kernel_bench pou   [--precision f32|bf16] [--volume 192] [--grid 4] [--block-res 64]
                                     [--candidates 64] [--det 256]
    python -m fvr.kernel_bench gather [--precision f16|bf16] [--volume 128] [--candidates 64] [--out-res 128]

``gather`` times fvr_bench_gather32 over exactly the stencil entries one
spectral-NCC launch of the ``sncc`` workload reads, in its sweep order, with
and without an L2 flush before each launch: the memory system's ceiling for
that gather with no arithmetic around it.

Builds the workload, lets the autotuner settle, then runs ``--launches``
steps inside an NVTX range named ``fvr_profile`` (so a profiler can select
exactly those launches with ``--nvtx --nvtx-include fvr_profile/``) and prints
the mean step time measured with CUDA events.
"""
from __future__ import annotations

import argparse
import json

import torch

from . import synthetic

PRECISION = {"f32": torch.float32, "bf16": torch.bfloat16, "f16": torch.float16}


def _sncc(args):
    from .graphs import BiplanarSpectralNCCStep
    from .torch_engine import TorchDiffFVREngine

    dev = torch.device("cuda", 0)
    vol = synthetic.make_ellipsoid_volume(args.volume, 0)
    poses = torch.from_numpy(synthetic.make_poses(args.candidates, 1)).to(dev)
    tp = torch.from_numpy(synthetic.make_poses(1, 2)).to(dev)
    eng = TorchDiffFVREngine(torch.from_numpy(vol), device=dev)
    with torch.no_grad():
        fa = eng.prepare_spectral_target(eng(tp, view="ap", out_res=args.out_res))
        fl = eng.prepare_spectral_target(eng(tp, view="lateral", out_res=args.out_res))
    eng.to_precision(PRECISION[args.precision])
    step = BiplanarSpectralNCCStep(eng, fa, fl, args.candidates, graph=False)
    for _ in range(3):
        step(poses)
    return lambda: step(poses)


def _pou(args):
    from .cone_beam_fvr import PerspectiveSlabFVR

    dev = torch.device("cuda", 0)
    vol = synthetic.make_ellipsoid_volume(args.volume, 0)
    g = args.grid
    fvr = PerspectiveSlabFVR.from_volume(vol, vox_mm=1.0, grid_blocks=(g, g, g), block_res=args.block_res,
                                         overlap=0.5, dtype=PRECISION[args.precision], device=dev)
    H = args.det
    f = 1020.0 / 0.8
    k_inv = torch.tensor([[1.0 / f, 0.0, -0.5 * H / f], [0.0, 1.0 / f, -0.5 * H / f], [0.0, 0.0, 1.0]],
                         device=dev)
    lattice = fvr.make_pinhole_lattice(k_inv, 1020.0, H, H)
    mats = synthetic.make_pinhole_mats(args.candidates, 1, sad_mm=765.0, device=dev)

    def step():
        m = mats.detach().requires_grad_(True)
        fvr.forward_pinhole(m, lattice).sum().backward()

    for _ in range(3):
        step()
    return step


def _gather(args):
    from . import profiling
    from .torch_engine import TorchDiffFVREngine

    dev = torch.device("cuda", 0)
    vol = synthetic.make_ellipsoid_volume(args.volume, 0)
    poses = torch.from_numpy(synthetic.make_poses(args.candidates, 1)).to(dev)
    eng = TorchDiffFVREngine(torch.from_numpy(vol), device=dev)
    eng.to_precision(PRECISION[args.precision])
    cells = profiling.sncc_cell_sequence(eng, poses, ("ap", "lateral"), args.out_res)
    flush = torch.zeros(64 * 1024 * 1024, dtype=torch.float32, device=dev)
    cold = profiling.gather_ceiling_ms(eng, cells, flush=flush, reps=9)
    warm = profiling.gather_ceiling_ms(eng, cells, reps=9)
    n = int(cells.numel())
    print(json.dumps({"path": "gather", "precision": args.precision, "entries": n,
                      "unique_entries": int(torch.unique(cells).numel()),
                      "cold_ms": cold, "warm_ms": warm, "cold_gbs_of_entries": n * 32 / cold / 1e6,
                      "warm_gbs_of_entries": n * 32 / warm / 1e6}))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("path", choices=["sncc", "pou", "gather"])
    ap.add_argument("--precision", default="f16")
    ap.add_argument("--volume", type=int, default=128)
    ap.add_argument("--candidates", type=int, default=64)
    ap.add_argument("--out-res", type=int, default=128)
    ap.add_argument("--grid", type=int, default=4)
    ap.add_argument("--block-res", type=int, default=64)
    ap.add_argument("--det", type=int, default=256)
    ap.add_argument("--launches", type=int, default=3)
    args = ap.parse_args()
    # backward on this thread, so the NVTX range below also covers the adjoint kernels
    torch.autograd.set_multithreading_enabled(False)
    if args.path == "gather":
        _gather(args)
        return
    step = _sncc(args) if args.path == "sncc" else _pou(args)
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.nvtx.range_push("fvr_profile")
    a.record()
    for _ in range(args.launches):
        step()
    b.record()
    torch.cuda.nvtx.range_pop()
    torch.cuda.synchronize()
    print(json.dumps({"path": args.path, "precision": args.precision, "ms_per_step": a.elapsed_time(b) / args.launches}))


if __name__ == "__main__":
    main()
