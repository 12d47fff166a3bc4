"""Linear-stage requests in the server (the reference's affine-only registrations): they share the
slots, queue and HBM budget with SyN requests, and their results are bit-identical to the same
stage run alone (every evaluation is deterministic and no state is shared between requests)."""
import numpy as np
import pytest

from fastwarp_b200 import FastwarpError, SynRecipe, linear_transform
from fastwarp_b200.backend import linear_recipe, run_linear_stage
from fastwarp_b200.phantoms import blob_pair
from fastwarp_b200.serve import Server

pytestmark = pytest.mark.gpu


def test_linear_and_syn_requests_run_together_and_match_the_stage_alone(backend):
    g, fixed, moving = blob_pair(40, seed=91)
    center = tuple((s - 1) * sp / 2.0 for s, sp in zip(g.size, g.spacing))
    r = linear_recipe(iterations=(10, 6), shrink_factors=(2, 1), smoothing_sigmas=(1.0, 0.0))
    starts = {"euler": [0.0] * 6, "affine": list(np.eye(3).ravel()) + [0.0] * 3}
    alone = {}
    for kind, start in starts.items():
        t, _ = run_linear_stage(backend, r, backend.upload_image(g, fixed),
                                backend.upload_image(g, moving),
                                linear_transform(kind, start, center=center))
        alone[kind] = list(t.parameters[:len(start)])
    syn = SynRecipe(gradient_step=0.25, update_field_variance=3.0, cc_radius=2, iterations=[4, 3],
                    shrink_factors=[2, 1], smoothing_sigmas=[1.0, 0.0], convergence_threshold=-1.0)
    fi, mi = backend.upload_image(g, fixed), backend.upload_image(g, moving)
    with Server(0, slots=3) as s:
        tickets = {}
        for kind, start in starts.items():
            tickets[kind] = s.submit_linear(r, g, fixed, g, moving,
                                            linear_transform(kind, start, center=center), tag=1)
        tickets["device"] = s.submit_linear(r, g, fi, g, mi,
                                            linear_transform("euler", starts["euler"],
                                                             center=center), tag=2)
        ts = s.submit(syn, g, [fixed], g, [moving], tag=3)
        with pytest.raises(FastwarpError, match="is a SyN request"):
            s.wait_linear(ts)
        with pytest.raises(FastwarpError, match="is a linear-stage request"):
            s.wait(tickets["euler"])
        out = {k: s.wait_linear(t) for k, t in tickets.items()}
        res = s.wait(ts)
        stats = s.stats()
    for k in ("euler", "affine"):
        assert out[k]["status"] == 0 and out[k]["parameters"] == alone[k], k
        assert [lv["skipped"] for lv in out[k]["levels"]] == [False, False]
    assert out["device"]["parameters"] == alone["euler"]
    assert res["status"] == 0 and res["iterations"] == 7
    assert stats["completed"] == 4 and stats["failed"] == 0


def test_a_failing_linear_request_reports_its_error(backend):
    g, _, moving = blob_pair(24, seed=3)
    flat = np.full(tuple(g.size)[::-1], 0.5, np.float32)
    r = linear_recipe(iterations=(5,), shrink_factors=(1,), smoothing_sigmas=(0.0,))
    with Server(0, slots=1) as s:
        t = s.submit_linear(r, g, flat, g, moving,
                            linear_transform("euler", [0.0] * 6, center=(11.5, 11.5, 11.5)))
        out = s.wait_linear(t)
        assert out["status"] != 0 and "too few usable samples" in out["error"]
        assert s.stats()["failed"] == 1
