"""The batching form (config 4's shape): subjects of their own grids registered to one template
in lockstep by fw_batch_syn_run, against each subject registered alone (fw_syn_run_device).

Every batched kernel runs the single kernel's tile body and reduces each subject in the single
kernel's tile order; the autotuner picks tile depths and persistent grids, so a subject's fields
can differ from its run alone only where a reduction grouped by another tile shape rounds
differently. The bar is the north star's full-registration bar: 0.05 mm RMS on both fields and
1e-4 relative final CC; the tests also report the largest field difference, which is normally 0.
"""
import os

import numpy as np
import pytest

from fastwarp_b200 import SynRecipe, run_syn_batch, run_syn_device
from fastwarp_b200._native import FW_ERR_NOT_FINITE
from fastwarp_b200.phantoms import batch_subjects

pytestmark = pytest.mark.gpu


def recipe(**kw):
    base = dict(gradient_step=0.1, update_field_variance=3.0, total_field_variance=0.0,
                cc_radius=2, iterations=[8, 6], shrink_factors=[2, 1],
                smoothing_sigmas=[1.0, 0.0], convergence_threshold=-1.0,
                convergence_window=10, channel_weights=[0.5, 0.5])
    base.update(kw)
    return SynRecipe(**base)


def compare(backend, r, fixed, subjects, batch):
    worst = 0.0
    for (moving, initial), got in zip(subjects, batch.subjects):
        w, iw, recs = run_syn_device(backend, r, fixed, moving, initial)
        ww, wiw = backend.download_field(w), backend.download_field(iw)
        assert len(got.iterations) == len(recs)
        rms = np.sqrt(((got.warp - ww) ** 2).sum(-1).mean())
        rms_i = np.sqrt(((got.inverse_warp - wiw) ** 2).sum(-1).mean())
        assert rms <= 0.05 and rms_i <= 0.05, (rms, rms_i)
        e, e0 = got.iterations[-1]["energy"], recs[-1]["energy"]
        assert abs(e - e0) <= 1e-4 * abs(e0), (e, e0)
        worst = max(worst, float(np.abs(got.warp - ww).max()), float(np.abs(got.inverse_warp - wiw).max()))
    return worst


def test_a_ragged_two_channel_batch_matches_each_subject_alone(backend):
    """Five subjects of their own grids (36-52 voxels per axis), two channels, two levels."""
    g, fixed, subjects = batch_subjects(backend, 5, template_shape=(44, 48, 40), dims=(36, 52),
                                        seed=4101)
    assert len({tuple(m[0].grid.size) for m, _ in subjects}) > 1  # ragged sources
    r = recipe()
    batch = run_syn_batch(backend, r, fixed, subjects)
    assert batch.statuses == [0] * 5
    worst = compare(backend, r, fixed, subjects, batch)
    print(f"largest field difference batch vs alone: {worst:.3e} mm; tuning {batch.tuning}")
    for t in batch.tuning:
        assert t["warp_zchunk"] >= 1 and t["cc_blocks_per_sm"] >= 1 and t["level"] >= 0
    # a second batch of the same shape takes the tuned shapes from the cache
    again = run_syn_batch(backend, r, fixed, subjects)
    assert all(t["from_cache"] == 1 for t in again.tuning)
    for a, b in zip(batch.subjects, again.subjects):
        assert np.array_equal(a.warp, b.warp) and np.array_equal(a.inverse_warp, b.inverse_warp)


def test_subjects_that_converge_early_leave_the_work_list(backend):
    """The window monitor stops each subject on its own (1e-3 over 4 iterations stops most of them
    within a few iterations, at different iterations); the others go on in the same graph, and
    each subject still matches its run alone (the same monitor on the same energies)."""
    g, fixed, subjects = batch_subjects(backend, 4, template_shape=(40, 44, 36), dims=(34, 46),
                                        seed=4202)
    r = recipe(iterations=[30], shrink_factors=[1], smoothing_sigmas=[0.0],
               convergence_threshold=1e-3, convergence_window=4, channel_weights=[1.0])
    one = [(m[:1], a) for m, a in subjects]
    batch = run_syn_batch(backend, r, fixed[:1], one)
    counts = [len(s.iterations) for s in batch.subjects]
    print(f"iterations per subject: {counts}")
    assert min(counts) < 30
    compare(backend, r, fixed[:1], one, batch)


def test_a_failing_subject_leaves_the_others_untouched(backend):
    """A subject whose moving image is not finite fails on its own (FW_ERR_NOT_FINITE, no fields);
    the other subjects of the batch give their results alone."""
    g, fixed, subjects = batch_subjects(backend, 3, template_shape=(36, 40, 32), dims=(30, 40),
                                        seed=4303)
    bad_img = subjects[1][0][0]
    data = bad_img.download()
    data[data.shape[0] // 2] = np.nan
    bad = backend.upload_image(bad_img.grid, data)
    one = [(m[:1], a) for m, a in subjects]
    one[1] = ([bad], subjects[1][1])
    r = recipe(iterations=[5], shrink_factors=[1], smoothing_sigmas=[0.0], channel_weights=[1.0])
    batch = run_syn_batch(backend, r, fixed[:1], one)
    assert batch.statuses[1] == FW_ERR_NOT_FINITE and batch.subjects[1] is None
    assert batch.statuses[0] == 0 and batch.statuses[2] == 0
    compare(backend, r, fixed[:1], [one[0], one[2]],
            type(batch)([batch.subjects[0], batch.subjects[2]], [0, 0], [], [], 0))


def test_the_default_tile_shapes_without_the_autotuner(backend):
    """FASTWARP_BATCH_TUNE=0 runs the default shapes (no timing); results keep the same bar."""
    g, fixed, subjects = batch_subjects(backend, 3, template_shape=(36, 36, 36), dims=(32, 40),
                                        seed=4404)
    r = recipe(iterations=[4, 3])
    os.environ["FASTWARP_BATCH_TUNE"] = "0"
    try:
        batch = run_syn_batch(backend, r, fixed, subjects)
    finally:
        del os.environ["FASTWARP_BATCH_TUNE"]
    assert all(t["tune_ms"] == 0.0 for t in batch.tuning)
    compare(backend, r, fixed, subjects, batch)


def test_batch_recipe_limits_are_refused(backend):
    from fastwarp_b200 import FastwarpError
    g, fixed, subjects = batch_subjects(backend, 1, template_shape=(24, 24, 24), dims=(20, 24),
                                        seed=4505)
    with pytest.raises(FastwarpError, match="CC channels only"):
        run_syn_batch(backend, recipe(channel_metrics=["cc", "mattes"]), fixed, subjects)
    with pytest.raises(FastwarpError, match="total-field smoothing"):
        run_syn_batch(backend, recipe(total_field_variance=0.5), fixed, subjects)
