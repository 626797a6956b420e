"""Continuous-batching server (xk_server_*).

Requests of different sizes are submitted from the test thread while others
run; each result must match the oracle, and a request's result must be the
same — bitwise — whether it ran alone or in a mix, because its items add
into its own slots in a fixed order whichever epoch or warp runs them.
Failures are made on the host: a request larger than the HBM budget, an
injected allocation failure, an unknown ray-set handle, a wait that times
out, a shutdown with requests still queued. None of them faults the GPU.
"""
import numpy as np
import pytest

import cases
import xrt_rs
from xrt_rs import XkError, _lib, synth
from xrt_rs.serve import Server

pytestmark = pytest.mark.gpu

PR_TOL = 1e-4
F64_TOL = 1e-10


def small_requests(seed, count):
    return [(r, p) for r, p, _ in synth.config3(seed=seed, count=count, ray_range=(500, 20000),
                                                 pix_range=(64, 3000))]


def test_results_match_oracle_and_are_mix_independent(ctx, oracle):
    reqs = small_requests(seed=11, count=8)
    srv = Server(ctx, epoch_pairs=5e8)
    # Alone: one request at a time.
    alone = []
    for rays, pix in reqs:
        t = srv.submit(pix, rays=rays)
        alone.append(tuple(a.copy() for a in srv.wait(t)))
    # In the mix: everything in flight together, submitted back to back.
    tickets = [srv.submit(pix, rays=rays) for rays, pix in reqs]
    mixed = [srv.wait(t) for t in tickets]
    st = srv.stats()
    assert st["completed"] == 2 * len(reqs) and st["failed"] == 0
    for i, ((rays, pix), a, b) in enumerate(zip(reqs, alone, mixed)):
        for x, y in zip(a, b):
            assert np.array_equal(x, y), f"request {i} differs alone vs in the mix"
        exact = oracle.kahan_ld(*cases.as_lists(rays, pix))
        assert cases.rel_l2(b, exact) < PR_TOL, i
    srv.close()


@pytest.mark.parametrize("policy", [0, 1])
def test_results_do_not_depend_on_the_policy(ctx, policy):
    """Both epoch-sharing policies (aged shortest-remaining-first, equal
    share) give every request the same field, bit for bit, as a request served
    alone: the policy decides only when a request's work items run."""
    reqs = small_requests(seed=12, count=6)
    ref_srv = Server(ctx, epoch_pairs=5e8, policy=1)
    alone = []
    for rays, pix in reqs:
        alone.append(tuple(a.copy() for a in ref_srv.wait(ref_srv.submit(pix, rays=rays))))
    ref_srv.close()
    srv = Server(ctx, epoch_pairs=3e8, policy=policy, aging_ms=50.0)
    tickets = [srv.submit(pix, rays=rays) for rays, pix in reqs]
    for i, (t, a) in enumerate(zip(tickets, alone)):
        b = srv.wait(t)
        for x, y in zip(a, b):
            assert np.array_equal(x, y), f"request {i} differs under policy {policy}"
    srv.close()


def test_unknown_policy_is_rejected(ctx):
    with pytest.raises(XkError) as ei:
        Server(ctx, policy=7)
    assert ei.value.code == _lib.XK_ERR_INVALID


def test_requests_overlap_on_the_device(ctx):
    """A request submitted while a large one runs completes before it: the
    small one joins the running epochs instead of waiting behind the queue."""
    big_rays, big_pix, _ = synth.config2_cell(10_000.0, 1000.0, seed=3, n_rays=1 << 18, grid=256)
    small_rays, small_pix = cases.random_case(2000, 500, seed=2)
    srv = Server(ctx, epoch_pairs=2e9)
    t_big = srv.submit(big_pix, rays=big_rays)
    t_small = srv.submit(small_pix, rays=small_rays)
    srv.wait(t_small)
    small = srv.last_stats
    srv.wait(t_big)
    big = srv.last_stats
    assert small["total_ms"] < big["total_ms"]
    assert big["epochs"] > 1
    srv.close()


def test_resident_ray_set_serves_several_screens(ctx, oracle):
    rays, _ = synth.config0(seed=4)
    srv = Server(ctx)
    h = srv.upload_rays(rays)
    screens = [synth.line_screen(300, 0.5, 1000.0), synth.grid_screen(20, 20, 0.3, 800.0),
               synth.line_screen(77, 0.2, 1500.0)]
    tickets = [srv.submit(pix, rayset=h) for pix in screens]
    for t, pix in zip(tickets, screens):
        out = srv.wait(t)
        ref = oracle.kahan_ld(*cases.as_lists(rays, pix))
        assert cases.rel_l2(out, ref) < PR_TOL
    assert srv.stats()["resident_ray_bytes"] > 0
    srv.release_rays(h)
    with pytest.raises(xrt_rs.XkError) as ei:
        srv.submit(screens[0], rayset=h)
    assert ei.value.code == xrt_rs._lib.XK_ERR_NOT_FOUND
    srv.close()


@pytest.mark.parametrize("amplitudes", [True, False])
def test_ray_set_from_a_beam(ctx, amplitudes):
    """xk_server_upload_beam builds the set on the device from the beam's
    columns; requests on it equal requests carrying the same rays from the
    host (beam_to_diffraction_rays, bit-exact) bit for bit."""
    beam, nrm, good = cases.beam_case(6000, seed=8, amplitudes=amplitudes)
    rays = xrt_rs.beam_to_diffraction_rays(beam, nrm, good, ctx=ctx)
    screens = [synth.grid_screen(17, 13, 0.3, 2000.0), synth.line_screen(101, 0.4, 2500.0)]
    for scr in screens:
        scr["y"], scr["z"] = scr["z"].copy(), scr["y"].copy()  # the beam runs along +y
    srv = Server(ctx)
    before = srv.stats()["resident_ray_bytes"]
    h = srv.upload_beam(beam, nrm, good)
    assert srv.stats()["resident_ray_bytes"] - before == 96 * len(good)
    for scr in screens:
        a = srv.wait(srv.submit(scr, rayset=h))
        b = srv.wait(srv.submit(scr, rays=rays))
        for x, y in zip(a, b):
            assert np.array_equal(x, y)
        assert np.linalg.norm(a[0]) > 0
    srv.release_rays(h)
    assert srv.stats()["resident_ray_bytes"] == before
    with pytest.raises(xrt_rs.XkError) as ei:
        srv.upload_beam(beam, nrm, np.array([0, len(beam["x"])], dtype=np.uint64))
    assert ei.value.code == xrt_rs._lib.XK_ERR_INVALID
    srv.close()


def test_budget_queues_and_rejects(ctx, oracle):
    reqs = small_requests(seed=12, count=5)
    one = max(len(r["x"]) for r, _ in reqs)
    # A budget that holds about one request at a time: the rest queue.
    srv = Server(ctx, hbm_budget_bytes=3e7 + 400.0 * one)
    tickets = [srv.submit(pix, rays=rays) for rays, pix in reqs]
    queued = 0
    for t, (rays, pix) in zip(tickets, reqs):
        out = srv.wait(t)
        queued += srv.last_stats["queue_ms"] > 0.5
        assert cases.rel_l2(out, oracle.kahan_ld(*cases.as_lists(rays, pix))) < PR_TOL
    # Larger than the whole budget: rejected, the server keeps serving.
    big_rays, big_pix = cases.random_case(200_000, 4000, seed=1)
    t = srv.submit(big_pix, rays=big_rays)
    with pytest.raises(xrt_rs.XkError) as ei:
        srv.wait(t)
    assert ei.value.code == xrt_rs._lib.XK_ERR_BUDGET
    rays, pix = reqs[0]
    assert cases.rel_l2(srv.wait(srv.submit(pix, rays=rays)),
                        oracle.kahan_ld(*cases.as_lists(rays, pix))) < PR_TOL
    srv.close()


def test_injected_allocation_failures_fail_only_their_request(ctx, oracle):
    reqs = small_requests(seed=13, count=6)
    srv = Server(ctx, inject_alloc_failure_every=3)
    tickets = [srv.submit(pix, rays=rays) for rays, pix in reqs]
    failed = 0
    for t, (rays, pix) in zip(tickets, reqs):
        try:
            out = srv.wait(t)
        except xrt_rs.XkError as e:
            assert e.code == xrt_rs._lib.XK_ERR_OOM
            failed += 1
            continue
        assert cases.rel_l2(out, oracle.kahan_ld(*cases.as_lists(rays, pix))) < PR_TOL
    assert failed == 2
    srv.close()


def test_f64_requests_through_the_server(ctx, oracle, tmp_path):
    rays, pix = cases.random_case(1500, 200, seed=8)
    log = tmp_path / "requests.jsonl"
    srv = Server(ctx, log=str(log))
    out = srv.wait(srv.submit(pix, rays=rays, path="f64"))
    assert srv.last_stats["path"] == xrt_rs.XK_PATH_F64
    assert cases.rel_l2(out, oracle.kahan_f64(*cases.as_lists(rays, pix))) < F64_TOL
    srv.close()
    import json
    rec = [json.loads(line) for line in log.read_text().splitlines()]
    assert len(rec) == 1 and rec[0]["pairs"] == 1500 * 200 and rec[0]["rc"] == 0
    assert {"queue_ms", "total_ms", "queue_depth", "admitted_bytes"} <= set(rec[0])


def test_wait_timeout_and_shutdown_with_queued_requests(ctx):
    big_rays, big_pix, _ = synth.config2_cell(10_000.0, 1000.0, seed=5, n_rays=1 << 18, grid=256)
    srv = Server(ctx, max_active=1)
    t1 = srv.submit(big_pix, rays=big_rays)
    with pytest.raises(xrt_rs.XkError) as ei:
        srv.wait(t1, timeout_ms=0.0)
    assert ei.value.code == xrt_rs._lib.XK_ERR_TIMEOUT
    for _ in range(4):
        srv.submit(big_pix, rays=big_rays)
    srv.close()  # cancels what was not admitted, finishes the rest, returns
