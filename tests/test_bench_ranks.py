"""bench.py's multi-rank plumbing on CPU: the slowest rank's time through a
world_size-2 gloo group, and the reference arm's non-zero ranks exiting
without work (no GPU needed)."""
import os
import subprocess
import sys
from pathlib import Path

import torch
import torch.distributed as dist
import torch.multiprocessing as mp

REPO = Path(__file__).resolve().parents[1]


def _rank_main(rank, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, str(REPO))
    import bench

    dist.init_process_group("gloo", rank=rank, world_size=2)
    try:
        got = bench._max_over_ranks(torch, dist, 2, torch.device("cpu"), 10.0 + 5.0 * rank)
        out[rank] = got
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_gloo():
    port = 29500 + os.getpid() % 2000
    with mp.Manager() as m:
        out = m.dict()
        mp.start_processes(_rank_main, args=(port, out), nprocs=2, start_method="spawn", join=True)
        assert dict(out) == {0: 15.0, 1: 15.0}


def test_max_over_ranks_single_rank_is_local():
    sys.path.insert(0, str(REPO))
    import bench

    assert bench._max_over_ranks(torch, None, 1, torch.device("cpu"), 3.5) == 3.5


def test_reference_arm_other_ranks_exit_without_work():
    env = dict(os.environ, WORLD_SIZE="2", RANK="1", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, str(REPO / "bench.py"), "--impl", "reference", "--gpus", "2", "--steps", "1",
                        "--warmup", "1"], cwd=REPO, env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    assert r.stdout.strip() == ""


def test_scope_table_byte_counts():
    """The bench's logical byte counts reproduce the per-pose-eval figures of
    the spectral-NCC step: 4.46 MB (f32) and 2.36 MB (bf16) at out_res 128
    with 2 views, with the bytes that step must read (8 corners once + the
    8 B target per sample) beside them.  The PoU block-image kernels count
    one stencil entry per mirrored pair of slice samples plus one image float
    per sample."""
    sys.path.insert(0, str(REPO))
    import bench

    rl = {s: bench._sncc_step_roofline(s, 1, 128, 1.0) for s in ("f32", "bf16", "f16")}
    per_eval = {s: r["scope_table_bytes_per_step"] for s, r in rl.items()}
    assert rl["f32"]["alg_bytes_per_step"] == 2 * 128 * 128 * 72
    assert rl["bf16"]["alg_bytes_per_step"] == rl["f16"]["alg_bytes_per_step"] == 2 * 128 * 128 * 40
    assert abs(per_eval["f32"] / 1e6 - 4.46) < 0.01
    assert abs(per_eval["bf16"] / 1e6 - 2.36) < 0.01
    assert abs(per_eval["f16"] / 1e6 - 2.49) < 0.01  # + 4 B brick scale per sample
    pou = bench._pou_kernel_rooflines({"pou_slice": 1.0, "pou_slice_adjoint": 1.0}, 52, 64, 128, 64)
    for k in ("pou_slice", "pou_slice_adjoint"):  # one 64 B entry per mirrored sample pair + one image float
        assert pou[k]["alg_bytes_per_launch"] == 52 * 64 * 128 * 128 * (32 + 4)
