"""Screen-sharded solve over NCCL on the real device path.

`xrt_rs.parallel.solve_sharded` with the NCCL backend, one rank on one GPU:
the rank solves its (whole) block through libxk.so and the all-gather runs on
device tensors. The result must equal the unsharded call bit for bit. More
ranks need more GPUs (ranks whose collectives wait on one another are never
put on one GPU); the multi-rank host logic is covered with gloo ranks on the
CPU in test_parallel.py. The run is a child process so that its process group
does not outlive the test.
"""
import os
import socket
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

SCRIPT = r"""
import datetime, sys
import numpy as np
import torch, torch.distributed as dist
sys.path.insert(0, "xrt-rs_b200"); sys.path.insert(0, "tests")
import cases, xrt_rs
from xrt_rs import parallel
torch.cuda.set_device(0)
dist.init_process_group("nccl", rank=0, world_size=1, timeout=datetime.timedelta(seconds=60),
                        device_id=torch.device("cuda", 0))
ctx = xrt_rs.GpuContext.new(0)
ok = True
for path in ("f32pr", "f64"):
    rays, pix = cases.random_case(4000, 1000, seed=9)
    rl, pl = cases.as_lists(rays, pix)
    ref = xrt_rs.diffraction_integral(rl, pl, path=path, ctx=ctx)
    got = parallel.solve_sharded(dict(zip(xrt_rs.RAY_FIELDS, rl)), dict(zip("xyz", pl)),
                                 path=path, ctx=ctx)
    ok = ok and all(np.array_equal(a, b) for a, b in zip(ref, got))
    t = parallel.max_over_ranks(1.5)
    ok = ok and t == 1.5
ctx.close()
dist.destroy_process_group()
print("SHARDED_OK" if ok else "SHARDED_MISMATCH")
"""


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_solve_sharded_nccl_one_rank():
    env = dict(os.environ, MASTER_ADDR="127.0.0.1", MASTER_PORT=str(_free_port()),
               RANK="0", WORLD_SIZE="1", LOCAL_RANK="0", NCCL_NVLS_ENABLE="0")
    r = subprocess.run([sys.executable, "-c", SCRIPT], cwd=ROOT, env=env, capture_output=True,
                       text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-3000:]
    assert "SHARDED_OK" in r.stdout, r.stdout[-2000:] + r.stderr[-2000:]
