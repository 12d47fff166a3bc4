"""The continuous-batching server: each result is the same alone and in a mix, admission follows
the HBM budget, and requests that cannot fit are refused before any work."""
import time

import numpy as np
import pytest

from fastwarp_b200 import CudaBackend, FastwarpError, SynRecipe
from fastwarp_b200._native import FW_ERR_CANCELLED
from fastwarp_b200.phantoms import blob_pair
from fastwarp_b200.serve import Server

pytestmark = pytest.mark.gpu


def small_recipe():
    return SynRecipe(gradient_step=0.25, update_field_variance=3.0, cc_radius=2,
                     iterations=[6, 4], shrink_factors=[2, 1], smoothing_sigmas=[1.0, 0.0],
                     convergence_threshold=-1.0)


@pytest.fixture(scope="module")
def pairs():
    return [blob_pair(40, seed=101), blob_pair(48, seed=202), blob_pair(32, seed=303)]


def test_each_result_is_the_same_alone_and_in_the_mix(pairs):
    r = small_recipe()
    alone = []
    with Server(0, slots=1) as s:
        for g, f, m in pairs:
            res = s.wait(s.submit(r, g, [f], g, [m]))
            assert res["status"] == 0, res["error"]
            alone.append(res)
    with Server(0, slots=4) as s:
        tickets = []
        for rep in range(3):
            for i, (g, f, m) in enumerate(pairs):
                tickets.append((i, s.submit(r, g, [f], g, [m], tag=10 * rep + i)))
        for i, t in tickets:
            res = s.wait(t)
            assert res["status"] == 0, res["error"]
            assert np.array_equal(res["warp"], alone[i]["warp"])
            assert np.array_equal(res["inverse_warp"], alone[i]["inverse_warp"])
            assert res["final_energy"] == alone[i]["final_energy"]
            assert res["iterations"] == 10
        st = s.stats()
        assert st["completed"] == 9 and st["failed"] == 0


def test_admission_keeps_the_reserved_memory_within_the_budget(pairs):
    r = small_recipe()
    g, f, m = pairs[1]
    with Server(0, slots=4) as probe:
        one = probe.estimate(r, g, [f], g, [m])
    budget = int(1.5 * one)  # room for one request at a time
    with Server(0, budget_bytes=budget, slots=4) as s:
        ts = [s.submit(r, g, [f], g, [m]) for _ in range(4)]
        outs = [s.wait(t) for t in ts]
        st = s.stats()
    assert all(o["status"] == 0 for o in outs)
    assert st["peak_reserved_bytes"] <= budget
    # one at a time: each started after the previous finished
    starts = sorted(o["queued_s"] for o in outs)
    assert starts[-1] > 0.0


def test_a_request_larger_than_the_budget_is_refused(pairs):
    r = small_recipe()
    g, f, m = pairs[0]
    with Server(0, budget_bytes=1 << 20, slots=2) as s:
        with pytest.raises(FastwarpError, match="budget"):
            s.submit(r, g, [f], g, [m])


def test_device_resident_images_and_fields(pairs):
    r = small_recipe()
    g, f, m = pairs[2]
    with CudaBackend(0) as b:
        fi, mi = b.upload_image(g, f), b.upload_image(g, m)
        with Server(0, slots=2) as s:
            host = s.wait(s.submit(r, g, [f], g, [m]))
            s.mark()
            dev = s.wait(s.submit(r, g, [fi], g, [mi], keep_on_device=True))
            assert dev["status"] == 0, dev["error"]
            assert dev["warp_dev"] and dev["device_end_ms"] > dev["device_start_ms"] >= 0.0
            assert dev["final_energy"] == host["final_energy"]
            Server.free_device_fields(dev)


def test_a_mixed_stream_of_masked_mattes_and_two_channel_requests(pairs, backend):
    """Ragged shapes and request kinds in flight together (masks, a Mattes channel, two
    channels): every served result equals the same registration run directly."""
    from fastwarp_b200 import run_syn
    from fastwarp_b200.backend import make_grid
    (g1, f1, m1), (g2, f2, m2), (g3, f3, m3) = pairs
    base = small_recipe()
    masked = (g1, np.where(np.indices(f1.shape)[0] > 4, 1.0, 0.0))
    mattes = SynRecipe(gradient_step=0.1, update_field_variance=3.0, cc_radius=2, iterations=[4, 3],
                       shrink_factors=[2, 1], smoothing_sigmas=[1.0, 0.0],
                       convergence_threshold=-1.0, channel_metrics=["mattes"], mi_bins=24)
    two = SynRecipe(gradient_step=0.25, update_field_variance=3.0, cc_radius=2, iterations=[3],
                    shrink_factors=[1], smoothing_sigmas=[0.0], convergence_threshold=-1.0,
                    channel_weights=[0.5, 0.5])
    mg = make_grid((30, 30, 30), (1.4, 1.4, 1.4), (-1.0, -2.0, 0.5))
    mmask = np.ones((30, 30, 30))
    mmask[20:] = 0.0
    jobs = [
        dict(recipe=base, g=g1, f=[f1], m=[m1], fixed_mask=masked),
        dict(recipe=mattes, g=g2, f=[f2], m=[m2]),
        dict(recipe=two, g=g3, f=[f3, 1 - f3], m=[m3, 1 - m3], moving_mask=(mg, mmask)),
        dict(recipe=base, g=g2, f=[f2], m=[m2], moving_mask=(mg, mmask)),
    ]
    direct = []
    for j in jobs:
        direct.append(run_syn(backend, j["recipe"], j["g"], j["f"], j["g"], j["m"],
                              fixed_mask=j.get("fixed_mask"), moving_mask=j.get("moving_mask")))
    with Server(0, slots=3) as s:
        ts = [s.submit(j["recipe"], j["g"], j["f"], j["g"], j["m"],
                       fixed_mask=j.get("fixed_mask"), moving_mask=j.get("moving_mask"))
              for j in jobs]
        served = [s.wait(t) for t in ts]
    for d, r in zip(direct, served):
        assert r["status"] == 0, r["error"]
        assert np.array_equal(r["warp"], d.warp)
        assert np.array_equal(r["inverse_warp"], d.inverse_warp)


def long_recipe(iterations=20000):
    """One level of many iterations at 96^3 (several seconds), to be cancelled while it runs."""
    return SynRecipe(gradient_step=0.25, update_field_variance=3.0, cc_radius=2,
                     iterations=[iterations], shrink_factors=[1], smoothing_sigmas=[0.0],
                     convergence_threshold=-1.0)


def test_a_cancel_stops_a_running_request_inside_its_level_graph(pairs):
    """A host-injected cancel (SynOptions::cancel, syn.rs:80-85) of a running request in a
    3-slot server: the record kernel of its level graph reads the slot's flag once per iteration,
    so the request ends FW_ERR_CANCELLED long before its 20000 iterations; the two requests
    running beside it are bit-identical to the same requests served alone, and the slot serves
    the next request normally (the flag is cleared with the cancelled request)."""
    r = small_recipe()
    (g1, f1, m1), (g2, f2, m2), _ = pairs
    g, f, m = blob_pair(96, seed=7)
    with Server(0, slots=1) as s:
        alone = [s.wait(s.submit(r, g1, [f1], g1, [m1])), s.wait(s.submit(r, g2, [f2], g2, [m2]))]
    with Server(0, slots=3) as s:
        tl = s.submit(long_recipe(), g, [f], g, [m])
        t1 = s.submit(r, g1, [f1], g1, [m1])
        t2 = s.submit(r, g2, [f2], g2, [m2])
        time.sleep(0.4)
        t0 = time.perf_counter()
        s.cancel(tl)
        cancelled = s.wait(tl)
        waited = time.perf_counter() - t0
        others = [s.wait(t1), s.wait(t2)]
        after = s.wait(s.submit(r, g1, [f1], g1, [m1]))
        st = s.stats()
    assert cancelled["status"] == FW_ERR_CANCELLED and "cancelled" in cancelled["error"]
    # 20000 iterations would take seconds; the cancel lands within an iteration or two
    assert waited < 0.5, waited
    assert cancelled["run_s"] < 2.0, cancelled["run_s"]
    for got, want in zip(others + [after], alone + [alone[0]]):
        assert got["status"] == 0, got["error"]
        assert np.array_equal(got["warp"], want["warp"])
        assert np.array_equal(got["inverse_warp"], want["inverse_warp"])
        assert got["final_energy"] == want["final_energy"]
    assert st["failed"] == 1 and st["completed"] == 3


def test_a_cancelled_queued_request_never_runs(pairs):
    r = small_recipe()
    g1, f1, m1 = pairs[0]
    g, f, m = blob_pair(96, seed=7)
    with Server(0, slots=1) as s:
        tl = s.submit(long_recipe(), g, [f], g, [m])
        tq = s.submit(r, g1, [f1], g1, [m1])
        s.cancel(tq)
        q = s.wait(tq, timeout=5.0)
        s.cancel(tl)
        lres = s.wait(tl)
        nxt = s.wait(s.submit(r, g1, [f1], g1, [m1]))
        with pytest.raises(FastwarpError, match="unknown or already taken"):
            s.cancel(tq)
    assert q["status"] == FW_ERR_CANCELLED and q["run_s"] == 0.0
    assert lres["status"] == FW_ERR_CANCELLED
    assert nxt["status"] == 0 and nxt["iterations"] == 10


def test_the_context_cancel_flag_fails_a_run_until_cleared(pairs, backend):
    from fastwarp_b200 import run_syn
    g, f, m = pairs[2]
    r = small_recipe()
    backend.request_cancel(True)
    try:
        with pytest.raises(FastwarpError, match="cancelled") as e:
            run_syn(backend, r, g, [f], g, [m])
        assert e.value.code == FW_ERR_CANCELLED
    finally:
        backend.request_cancel(False)
    res = run_syn(backend, r, g, [f], g, [m])
    assert len(res.iterations) == 10


def test_each_result_is_the_same_alone_and_in_an_open_loop_stream(backend):
    """Config 5's form in miniature: requests of the three kinds (single-channel SyN, affine-only
    Mattes MI fit, two-channel SyN) on their own grids, generated on the device, arrive by a
    seeded Poisson process while earlier ones run, through a 3-slot server under an HBM budget.
    Every SyN result is bit-identical, and every affine fit identical, to the same request served
    alone."""
    import threading

    from fastwarp_b200 import linear_transform
    from fastwarp_b200.backend import linear_recipe
    from fastwarp_b200.phantoms import stream_requests
    reqs = stream_requests(backend, 7, mix=(0.4, 0.3, 0.3), dims=(36, 48),
                           template_shape=(44, 48, 40), seed=5151)
    assert {q["kind"] for q in reqs} == {"syn", "affine", "syn2"}
    syn = {"syn": small_recipe(),
           "syn2": SynRecipe(gradient_step=0.25, update_field_variance=3.0, cc_radius=2,
                             iterations=[4, 3], shrink_factors=[2, 1], smoothing_sigmas=[1.0, 0.0],
                             convergence_threshold=-1.0, channel_weights=[0.5, 0.5])}
    lr = linear_recipe(iterations=(8, 6), shrink_factors=(2, 1), smoothing_sigmas=(1.0, 0.0))

    def submit(s, q):
        if q["kind"] == "affine":
            g = q["grid"]
            c = tuple(g.origin[a] + 0.5 * (g.size[a] - 1) * g.spacing[a] for a in range(3))
            start = linear_transform("affine", list(np.eye(3).ravel()) + [0.0] * 3, center=c)
            return s.submit_linear(lr, g, q["fixed"][0], g, q["moving"][0], start)
        return s.submit(syn[q["kind"]], q["grid"], q["fixed"], q["grid"], q["moving"],
                        q["initial"])

    def wait(s, q, t):
        o = s.wait_linear(t) if q["kind"] == "affine" else s.wait(t)
        assert o["status"] == 0, o["error"]
        return o

    with Server(0, slots=1) as s:
        alone = [wait(s, q, submit(s, q)) for q in reqs]
    rng = np.random.default_rng(77)
    gaps = rng.exponential(0.02, size=len(reqs))
    with Server(0, budget_bytes=40 << 30, slots=3) as s:
        tickets = [None] * len(reqs)

        def feeder():
            for i, q in enumerate(reqs):
                time.sleep(gaps[i])
                tickets[i] = submit(s, q)
        th = threading.Thread(target=feeder)
        th.start()
        streamed = []
        for i, q in enumerate(reqs):
            while tickets[i] is None:
                time.sleep(0.001)
            streamed.append(wait(s, q, tickets[i]))
        th.join()
        st = s.stats()
    assert st["completed"] == len(reqs) and st["failed"] == 0
    for q, a, b in zip(reqs, alone, streamed):
        if q["kind"] == "affine":
            assert a["parameters"] == b["parameters"]
        else:
            assert np.array_equal(a["warp"], b["warp"])
            assert np.array_equal(a["inverse_warp"], b["inverse_warp"])
            assert a["final_energy"] == b["final_energy"]
