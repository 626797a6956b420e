"""Multi-rank host logic on CPU: two gloo ranks shard a screen, each solves its
block (the CPU oracle stands in for the rank's GPU here), the field is
gathered, and step times reduce to their maximum. No GPU involved."""
import os
import socket

import numpy as np
import pytest

import cases
from xrt_rs import parallel, synth


def test_shard_range_partitions_exactly():
    for n in (0, 1, 7, 256, 1001):
        for world in (1, 2, 3, 8):
            spans = [parallel.shard_range(n, r, world) for r in range(world)]
            assert spans[0][0] == 0 and spans[-1][1] == n
            assert all(a <= b for a, b in spans)
            assert all(spans[i][1] == spans[i + 1][0] for i in range(world - 1))
            sizes = [b - a for a, b in spans]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        parallel.shard_range(10, 2, 2)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, result_dir):
    import datetime
    import sys

    import torch.distributed as dist

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path[:0] = [root, os.path.join(root, "xrt-rs_b200"), os.path.join(root, "tests")]
    from oracle import oracle as orc
    from xrt_rs import parallel as par
    from xrt_rs import synth as syn

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    rays, screen = syn.config0(seed=3)
    rays = {k: v[:1500] for k, v in rays.items()}
    keys = ("x", "y", "z", "nx", "ny", "nz", "nl", "es_re", "es_im", "ep_re", "ep_im", "energy")

    def compute(r, s):
        return orc.kahan_f64([r[k] for k in keys], [s["x"], s["y"], s["z"]], threads=1)

    full = par.solve_sharded(rays, screen, compute=compute)
    worst = par.max_over_ranks(10.0 + rank)
    np.savez(os.path.join(result_dir, f"rank{rank}.npz"), *full, worst=worst)
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_shard_and_gather(tmp_path, oracle):
    import torch.multiprocessing as mp

    world = 2
    mp.start_processes(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world,
                       join=True, start_method="spawn")
    rays, screen = synth.config0(seed=3)
    rays = {k: v[:1500] for k, v in rays.items()}
    ref = oracle.kahan_f64(*cases.as_lists(rays, screen))
    for rank in range(world):
        got = np.load(tmp_path / f"rank{rank}.npz")
        for c in range(4):
            assert np.array_equal(got[f"arr_{c}"], ref[c])
        assert float(got["worst"]) == 11.0


def _rank_device_gather(rank, world, port, result_dir):
    import datetime
    import sys

    import torch
    import torch.distributed as dist

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path[:0] = [root, os.path.join(root, "xrt-rs_b200"), os.path.join(root, "tests")]
    from oracle import oracle as orc
    from xrt_rs import parallel as par
    from xrt_rs import synth as syn

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    rays, screen = syn.config0(seed=4)
    rays = {k: v[:800] for k, v in rays.items()}
    keys = ("x", "y", "z", "nx", "ny", "nz", "nl", "es_re", "es_im", "ep_re", "ep_im", "energy")
    # The screen-sharded bench step: this rank's block of the screen as
    # views of the full columns, its field into block tensors, one gather.
    m = len(screen["x"])
    a, b = par.shard_range(m, rank, world)
    full_pix = [torch.from_numpy(screen[k]) for k in "xyz"]
    block = [t[a:b] for t in full_pix]
    local = orc.kahan_f64([rays[k] for k in keys], [t.numpy() for t in block], threads=1)
    local_t = [torch.from_numpy(np.ascontiguousarray(c)) for c in local]
    out = [torch.full((m,), float("nan"), dtype=torch.float64) for _ in range(4)]
    par.gather_field_device(local_t, m, out=out)
    np.savez(os.path.join(result_dir, f"dev{rank}.npz"), *[t.numpy() for t in out])
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_device_gather_of_screen_blocks(tmp_path, oracle, world):
    """gather_field_device (the all-gather of the strong-scaling bench step)
    with gloo ranks on CPU tensors: every rank ends with the full field, equal
    bit for bit to the unsharded solve, for even and uneven blocks."""
    import torch.multiprocessing as mp

    mp.start_processes(_rank_device_gather, args=(world, _free_port(), str(tmp_path)),
                       nprocs=world, join=True, start_method="spawn")
    rays, screen = synth.config0(seed=4)
    rays = {k: v[:800] for k, v in rays.items()}
    ref = oracle.kahan_f64(*cases.as_lists(rays, screen))
    for rank in range(world):
        got = np.load(tmp_path / f"dev{rank}.npz")
        for c in range(4):
            assert np.array_equal(got[f"arr_{c}"], ref[c])
