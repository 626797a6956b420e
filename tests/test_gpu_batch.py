"""Batched solves (xk_batch_*): one plan, one persistent launch per kernel
variant over every solve's items, replayed from a CUDA graph.

Each solve's result must equal the single-solve API's result bitwise (the
cross-item reduction is in a fixed order, independent of which warp ran
which item), match the oracle within the path's tolerance, and repeat
exactly on graph replay.

These solves reach k*|p - r| ~ 1e12 rad (25 keV, 10 m), where FP64's own
rounding of the phase leaves the FP64 formula ~1e-4 away from its exact
value, so the FP32 phase-reduced results are checked against the oracle with
an extended-precision phase (oracle.kahan_ld); FP64-path results against the
FP64 oracle, operation for operation.
"""
import numpy as np
import pytest

import cases
import xrt_rs
from xrt_rs import synth

pytestmark = pytest.mark.gpu

PR_TOL = 1e-4
F64_TOL = 1e-10


def uneven_solves(seed=0, count=10):
    solves = synth.config3(seed=seed, count=count, ray_range=(300, 30000), pix_range=(17, 4000))
    out = [(r, p) for r, p, _ in solves]
    poly = cases.polychromatic()                    # routed to FP64 (mixed energies)
    out.insert(3, poly)
    out.insert(5, (cases.rays_from([]), cases.pixels_from([0.0, 0.1], 0.0, 1000.0)))  # no rays
    out.append(cases.random_case(1500, 333, seed=7, general_normals=True))
    return out


def test_batch_equals_single_solves_and_oracle(ctx, oracle):
    solves = uneven_solves()
    batch = xrt_rs.Batch(solves, path="f32pr", ctx=ctx)
    outs = batch.run()
    assert batch.stats["graph"] == 1
    assert batch.stats["routed_f64"] >= 2
    for i, ((rays, pix), got) in enumerate(zip(solves, outs)):
        alone = xrt_rs.diffraction_integral(*cases.as_lists(rays, pix), path="f32pr", ctx=ctx)
        for a, b in zip(got, alone):
            assert np.array_equal(a, b), f"solve {i} differs alone vs in the batch"
        plan = batch.plan(i)
        f64 = plan["path"] == xrt_rs.XK_PATH_F64
        ref = (oracle.kahan_f64 if f64 else oracle.kahan_ld)(*cases.as_lists(rays, pix))
        if np.linalg.norm(np.concatenate(cases.field_c(ref))) == 0:
            assert all(np.all(o == 0) for o in got)
            continue
        assert cases.rel_l2(got, ref) < (F64_TOL if f64 else PR_TOL), (i, plan)


def test_graph_replay_is_exact(ctx):
    solves = uneven_solves(seed=1, count=6)
    batch = xrt_rs.Batch(solves, path="f32pr", ctx=ctx)
    first = [tuple(a.copy() for a in o) for o in batch.run()]
    second = batch.run()
    for a, b in zip(first, second):
        for x, y in zip(a, b):
            assert np.array_equal(x, y)
    nograph = xrt_rs.Batch(solves, path="f32pr", ctx=ctx, graph=False)
    third = nograph.run()
    assert nograph.stats["graph"] == 0
    for a, b in zip(first, third):
        for x, y in zip(a, b):
            assert np.array_equal(x, y)


def test_batch_f64_path(ctx, oracle):
    solves = uneven_solves(seed=2, count=4)
    batch = xrt_rs.Batch(solves, path="f64", ctx=ctx)
    outs = batch.run()
    assert batch.stats["routed_f64"] == len(solves)
    for (rays, pix), got in zip(solves, outs):
        ref = oracle.kahan_f64(*cases.as_lists(rays, pix))
        if np.linalg.norm(np.concatenate(cases.field_c(ref))) == 0:
            continue
        assert cases.rel_l2(got, ref) < F64_TOL
