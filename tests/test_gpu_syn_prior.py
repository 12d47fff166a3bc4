"""A later SyN stage (run_syn_from, syn.rs:620-660, 761-774, 803-820, 971-977) on the device
against the oracle: the moving images and mask go through the earlier stages' collapsed field on
every iteration, and the result is collapsed with it.

Both engines start the second stage from the same prior (the oracle's first-stage fields), so
the comparison has the bars of the first-stage tests: 1e-5 relative on the first iteration's
energy, 1e-4 on the last, 0.05 mm RMS on both collapsed fields.
"""
import numpy as np
import pytest

import oracle as O
from fastwarp_b200 import (FastwarpError, SynRecipe, make_affine, run_syn, run_syn_device,
                           run_syn_from)
from fastwarp_b200.phantoms import blob_pair

pytestmark = pytest.mark.gpu


def ogrid(g):
    return O.make_grid(tuple(g.size), tuple(g.spacing), tuple(g.origin),
                       np.array(g.direction[:]).reshape(3, 3))


def oaffine(a):
    return O.make_affine(np.array(a.matrix[:]).reshape(3, 3), tuple(a.offset[:]))


RECIPE = dict(gradient_step=0.25, update_field_variance=3.0, cc_radius=2, iterations=[6, 5],
              shrink_factors=[2, 1], smoothing_sigmas=[1.0, 0.0], convergence_threshold=-1.0)


def orecipe():
    return O.syn_recipe(0.25, 3.0, 0.0, 2, (6, 5), (2, 1), (1.0, 0.0), False, -1.0, 10, (1.0,))


def rms(a, b):
    return float(np.sqrt(((np.asarray(a, np.float64) - b) ** 2).sum(-1).mean()))


@pytest.fixture(scope="module")
def stage1():
    g, fixed, moving = blob_pair(40, seed=515)
    initial = make_affine(np.array([[1.01, 0.02, 0.0], [-0.015, 0.99, 0.01], [0.0, 0.0, 1.0]]),
                          (0.6, -0.4, 0.3))
    w, iw, recs, last = O.syn_run(orecipe(), ogrid(g), [fixed], ogrid(g), [moving],
                                  oaffine(initial))
    return g, fixed, moving, initial, w, iw, recs, last


def test_a_second_stage_from_a_prior_matches_the_oracle(backend, stage1):
    g, fixed, moving, initial, w, iw, recs1, last = stage1
    res = run_syn_from(backend, SynRecipe(**RECIPE), g, [fixed], g, [moving], initial, w, iw)
    ow, oiw, orecs, _ = O.syn_run(orecipe(), ogrid(g), [fixed], ogrid(g), [moving],
                                  oaffine(initial), prior=(last, w, iw))
    assert len(res.iterations) == len(orecs) == 11
    e0, o0 = res.iterations[0]["energy"], orecs[0].energy
    assert abs(e0 - o0) <= 1e-5 * abs(o0), (e0, o0)
    assert abs(res.iterations[-1]["energy"] - orecs[-1].energy) <= 1e-4 * abs(orecs[-1].energy)
    assert rms(res.warp, ow) <= 0.05 and rms(res.inverse_warp, oiw) <= 0.05
    # the prior matters: the second stage starts better aligned than the first did
    assert o0 < recs1[0].energy
    assert rms(res.warp, w) > 0.01


def test_a_second_stage_with_a_moving_mask_matches_the_oracle(backend, stage1):
    g, fixed, moving, initial, w, iw, _, last = stage1
    n = tuple(g.size)
    z, y, x = np.meshgrid(*[np.arange(s, dtype=float) for s in n[::-1]], indexing="ij")
    mask = (((x - 20) / 15) ** 2 + ((y - 20) / 17) ** 2 + ((z - 20) / 16) ** 2 < 1.0)
    mask = mask.astype(np.float32)
    res = run_syn_from(backend, SynRecipe(**RECIPE), g, [fixed], g, [moving], initial, w, iw,
                       moving_mask=(g, mask))
    ow, oiw, orecs, _ = O.syn_run(orecipe(), ogrid(g), [fixed], ogrid(g), [moving],
                                  oaffine(initial),
                                  masks=dict(moving_grid=ogrid(g), moving=mask),
                                  prior=(last, w, iw))
    assert abs(res.iterations[0]["energy"] - orecs[0].energy) <= 1e-5 * abs(orecs[0].energy)
    assert abs(res.iterations[-1]["energy"] - orecs[-1].energy) <= 1e-4 * abs(orecs[-1].energy)
    assert rms(res.warp, ow) <= 0.05 and rms(res.inverse_warp, oiw) <= 0.05


def test_a_zero_prior_gives_the_first_stage_result(backend, stage1):
    g, fixed, moving, initial, _, _, _, last = stage1
    zero = np.zeros(O.grid_shape(last) + (3,))
    a = run_syn(backend, SynRecipe(**RECIPE), g, [fixed], g, [moving], initial)
    b = run_syn_from(backend, SynRecipe(**RECIPE), g, [fixed], g, [moving], initial, zero, zero)
    assert rms(a.warp, b.warp) <= 1e-4 and rms(a.inverse_warp, b.inverse_warp) <= 1e-4
    assert abs(a.iterations[-1]["energy"] - b.iterations[-1]["energy"]) <= \
        1e-6 * abs(a.iterations[-1]["energy"])


def test_a_prior_off_the_last_level_grid_is_refused(backend, stage1):
    g, fixed, moving, initial, w, iw, _, _ = stage1
    r = SynRecipe(**{**RECIPE, "shrink_factors": [4, 2]})  # last level 20^3, the prior is 40^3
    prior = (backend.upload_field(g, w), backend.upload_field(g, iw))
    fi, mi = backend.upload_image(g, fixed), backend.upload_image(g, moving)
    with pytest.raises(FastwarpError, match="not on the grid of this stage's last level"):
        run_syn_device(backend, r, [fi], [mi], initial, prior=prior)
