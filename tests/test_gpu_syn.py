"""The SyN step and the whole SyN stage on the GPU against the f64 oracle.

Bars: a single SyN step matches to 1e-5 relative on the CC value and 1e-4 voxel on both update
fields; a full registration matches to 0.05 mm RMS displacement and 1e-4 relative final CC.
The oracle runs the same seeded 64^3 blob pair (config 1: CC radius 2, gradient step 0.25,
update variance 3, total variance 0, 30 iterations, convergence threshold -1 so that both
engines run every iteration, as crates/fastwarp-gpu/tests/syn_parity.rs:244-260 pins it).
"""
import numpy as np
import pytest

import oracle as O
from fastwarp_b200 import SynRecipe, run_syn, syn_step
from fastwarp_b200.phantoms import blob_pair

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def pair():
    return blob_pair(64)


def config1(iterations=30):
    return SynRecipe(gradient_step=0.25, update_field_variance=3.0, total_field_variance=0.0,
                     cc_radius=2, iterations=[iterations], shrink_factors=[1],
                     smoothing_sigmas=[0.0], convergence_threshold=-1.0, convergence_window=10,
                     channel_weights=[1.0])


def oracle_recipe(r: SynRecipe):
    return O.syn_recipe(r.gradient_step, r.update_field_variance, r.total_field_variance,
                        r.cc_radius, r.iterations, r.shrink_factors, r.smoothing_sigmas,
                        r.sigma_units_mm, r.convergence_threshold, r.convergence_window,
                        r.channel_weights, metrics=r.channel_metrics or None,
                        mi_bins=r.mi_bins)


def ogrid(g):
    return O.make_grid(tuple(g.size), tuple(g.spacing), tuple(g.origin),
                       np.array(g.direction[:]).reshape(3, 3))


def test_one_syn_step_from_zero_matches(backend, pair):
    g, fixed, moving = pair
    r = config1(1)
    og = ogrid(g)
    fi = backend.upload_image(g, fixed)
    mi = backend.upload_image(g, moving)
    state = {k: backend.zero_field(g) for k in ("f2m", "f2m_inv", "m2m", "m2m_inv")}
    rec, fu, mu = syn_step(backend, r, [fi], [mi], None, state)
    ostate = {k: np.zeros((64, 64, 64, 3)) for k in ("f2m", "f2m_inv", "m2m", "m2m_inv")}
    orec, ofu, omu = O.syn_step(oracle_recipe(r), og, og, [fixed], og, [moving], None, ostate)
    assert abs(rec["energy"] - orec.energy) <= 1e-5 * abs(orec.energy)
    assert np.abs(fu - ofu).max() <= 1e-4
    assert np.abs(mu - omu).max() <= 1e-4
    for k in state:
        assert np.abs(backend.download_field(state[k]) - ostate[k]).max() <= 1e-4
    assert [s[0] for s in rec["inversions"]] == [s.iterations for s in orec.inversions]


def test_a_syn_step_from_a_deformed_state_matches(backend, pair):
    """The oracle runs five iterations; both engines then take the sixth from that state."""
    g, fixed, moving = pair
    r = config1(1)
    og = ogrid(g)
    ostate = {k: np.zeros((64, 64, 64, 3)) for k in ("f2m", "f2m_inv", "m2m", "m2m_inv")}
    for _ in range(5):
        O.syn_step(oracle_recipe(r), og, og, [fixed], og, [moving], None, ostate)
    fi = backend.upload_image(g, fixed)
    mi = backend.upload_image(g, moving)
    state = {k: backend.upload_field(g, v) for k, v in ostate.items()}
    rec, fu, mu = syn_step(backend, r, [fi], [mi], None, state)
    orec, ofu, omu = O.syn_step(oracle_recipe(r), og, og, [fixed], og, [moving], None, ostate)
    assert abs(rec["energy"] - orec.energy) <= 1e-5 * abs(orec.energy)
    assert np.abs(fu - ofu).max() <= 1e-4
    assert np.abs(mu - omu).max() <= 1e-4


def test_full_registration_matches_the_oracle(backend, pair):
    g, fixed, moving = pair
    r = config1(30)
    og = ogrid(g)
    res = run_syn(backend, r, g, [fixed], g, [moving])
    ow, oinv, orecs, _ = O.syn_run(oracle_recipe(r), og, [fixed], og, [moving])
    assert len(res.iterations) == len(orecs) == 30
    rms = np.sqrt(((res.warp.astype(np.float64) - ow) ** 2).sum(-1).mean())
    rms_inv = np.sqrt(((res.inverse_warp.astype(np.float64) - oinv) ** 2).sum(-1).mean())
    assert rms <= 0.05 and rms_inv <= 0.05, (rms, rms_inv)
    e, oe = res.iterations[-1]["energy"], orecs[-1].energy
    assert abs(e - oe) <= 1e-4 * abs(oe)
    assert res.iterations[-1]["energy"] < res.iterations[0]["energy"]


def test_multilevel_registration_with_pyramid_smoothing_matches(backend):
    g, fixed, moving = blob_pair(48, seed=77)
    r = SynRecipe(gradient_step=0.25, update_field_variance=3.0, cc_radius=2,
                  iterations=[8, 6], shrink_factors=[2, 1], smoothing_sigmas=[1.0, 0.0],
                  convergence_threshold=-1.0)
    og = ogrid(g)
    res = run_syn(backend, r, g, [fixed], g, [moving])
    ow, oinv, orecs, _ = O.syn_run(oracle_recipe(r), og, [fixed], og, [moving])
    assert len(res.iterations) == len(orecs) == 14
    rms = np.sqrt(((res.warp.astype(np.float64) - ow) ** 2).sum(-1).mean())
    assert rms <= 0.05, rms
    assert abs(res.iterations[-1]["energy"] - orecs[-1].energy) <= 1e-4 * abs(orecs[-1].energy)


def test_two_channel_registration_matches(backend):
    g, fixed, moving = blob_pair(40, seed=91)
    r = SynRecipe(gradient_step=0.25, update_field_variance=3.0, cc_radius=2, iterations=[6],
                  shrink_factors=[1], smoothing_sigmas=[0.0], convergence_threshold=-1.0,
                  channel_weights=[0.5, 0.5])
    f2, m2 = 1.0 - fixed, 1.0 - moving  # inverted contrast (T2-like)
    og = ogrid(g)
    res = run_syn(backend, r, g, [fixed, f2], g, [moving, m2])
    ow, _, orecs, _ = O.syn_run(oracle_recipe(r), og, [fixed, f2], og, [moving, m2])
    rms = np.sqrt(((res.warp.astype(np.float64) - ow) ** 2).sum(-1).mean())
    assert rms <= 0.05, rms
    assert abs(res.iterations[-1]["energy"] - orecs[-1].energy) <= 1e-4 * abs(orecs[-1].energy)


def test_the_op_by_op_loop_over_the_backend_matches_the_graph_driver(backend):
    """The reference's loop shape (syn.rs:776-986: one synchronous Backend op at a time) on this
    engine gives the graph-captured driver's result."""
    from fastwarp_b200.syn import run_syn_ops
    g, fixed, moving = blob_pair(40, seed=55)
    r = SynRecipe(gradient_step=0.25, update_field_variance=3.0, cc_radius=2,
                  iterations=[5, 4], shrink_factors=[2, 1], smoothing_sigmas=[1.0, 0.0],
                  convergence_threshold=-1.0)
    res = run_syn(backend, r, g, [fixed], g, [moving])
    w, iw, recs = run_syn_ops(backend, r, g, [fixed], g, [moving])
    assert len(recs) == len(res.iterations) == 9
    assert np.sqrt(((w - res.warp) ** 2).sum(-1).mean()) <= 1e-3
    assert np.sqrt(((iw - res.inverse_warp) ** 2).sum(-1).mean()) <= 1e-3
    assert abs(recs[-1]["energy"] - res.iterations[-1]["energy"]) <= 1e-5 * abs(recs[-1]["energy"])
    og = ogrid(g)
    ow, _, orecs, _ = O.syn_run(oracle_recipe(r), og, [fixed], og, [moving])
    assert np.sqrt(((w - ow) ** 2).sum(-1).mean()) <= 0.05


def test_convergence_monitor_stops_the_level_on_the_device(backend, pair):
    g, fixed, moving = pair
    r = config1(60)
    r.convergence_threshold = 1e-3  # loose: the monitor stops the level early
    og = ogrid(g)
    res = run_syn(backend, r, g, [fixed], g, [moving])
    ow, _, orecs, _ = O.syn_run(oracle_recipe(r), og, [fixed], og, [moving])
    assert len(res.iterations) == len(orecs) < 60


def test_direct_launch_mode_gives_the_graph_result(backend, monkeypatch):
    """FASTWARP_SYN_GRAPHS=0 launches the same kernels straight onto the stream with the loops on
    the host (the profiling mode); it must give the graph driver's result bit for bit."""
    g, fixed, moving = blob_pair(40, seed=56)
    r = SynRecipe(gradient_step=0.25, update_field_variance=3.0, cc_radius=2,
                  iterations=[5, 4], shrink_factors=[2, 1], smoothing_sigmas=[1.0, 0.0],
                  convergence_threshold=1e-3, convergence_window=3)
    res = run_syn(backend, r, g, [fixed], g, [moving])
    monkeypatch.setenv("FASTWARP_SYN_GRAPHS", "0")
    direct = run_syn(backend, r, g, [fixed], g, [moving])
    assert len(direct.iterations) == len(res.iterations)
    assert np.array_equal(direct.warp, res.warp)
    assert np.array_equal(direct.inverse_warp, res.inverse_warp)
    assert direct.iterations[-1]["energy"] == res.iterations[-1]["energy"]


# ---- masks (syn.rs:496-580): the fixed mask through F^-1 times the moving mask through
# affine(M^-1), nearest voxel, every iteration; the CC pairs take only those voxels ------------

def masks_for(n):
    """A fixed mask on the fixed grid (a ball left out, value 2: any non-zero is inside) and a
    moving mask on its own coarser, shifted grid (a slab left out)."""
    from fastwarp_b200.backend import make_grid
    z, y, x = np.meshgrid(*[np.arange(n, dtype=float)] * 3, indexing="ij")
    fm = np.where((x - 0.3 * n) ** 2 + (y - 0.6 * n) ** 2 + (z - 0.5 * n) ** 2 < (0.18 * n) ** 2,
                  0.0, 2.0)
    m_n = (n * 2) // 3 + 3
    mgrid = make_grid((m_n, m_n, m_n), (1.5, 1.5, 1.5), (-1.2, -0.9, -1.05))
    mz = np.arange(m_n) * 1.5 - 1.05
    mm = np.ones((m_n, m_n, m_n))
    mm[(mz > 0.65 * n) & (mz < 0.8 * n), :, :] = 0.0
    return fm, mgrid, mm


def test_one_masked_syn_step_matches(backend, pair):
    g, fixed, moving = pair
    r = config1(1)
    og = ogrid(g)
    fm, mgrid, mm = masks_for(64)
    fi, mi = backend.upload_image(g, fixed), backend.upload_image(g, moving)
    fmi, mmi = backend.upload_image(g, fm), backend.upload_image(mgrid, mm)
    state = {k: backend.zero_field(g) for k in ("f2m", "f2m_inv", "m2m", "m2m_inv")}
    rec, fu, mu = syn_step(backend, r, [fi], [mi], None, state, fixed_mask=fmi, moving_mask=mmi)
    ostate = {k: np.zeros((64, 64, 64, 3)) for k in ("f2m", "f2m_inv", "m2m", "m2m_inv")}
    orec, ofu, omu = O.syn_step(oracle_recipe(r), og, og, [fixed], og, [moving], None, ostate,
                                masks=dict(fixed_grid=og, fixed=fm, moving_grid=ogrid(mgrid),
                                           moving=mm))
    assert abs(rec["energy"] - orec.energy) <= 1e-5 * abs(orec.energy)
    assert np.abs(fu - ofu).max() <= 1e-4
    assert np.abs(mu - omu).max() <= 1e-4
    # the mask changed the step: the unmasked oracle step differs
    ustate = {k: np.zeros((64, 64, 64, 3)) for k in ("f2m", "f2m_inv", "m2m", "m2m_inv")}
    urec, ufu, _ = O.syn_step(oracle_recipe(r), og, og, [fixed], og, [moving], None, ustate)
    assert abs(urec.energy - orec.energy) > 1e-4


def test_masked_registration_matches_the_oracle(backend):
    g, fixed, moving = blob_pair(48, seed=78)
    r = SynRecipe(gradient_step=0.25, update_field_variance=3.0, cc_radius=2,
                  iterations=[8, 6], shrink_factors=[2, 1], smoothing_sigmas=[1.0, 0.0],
                  convergence_threshold=-1.0)
    fm, mgrid, mm = masks_for(48)
    og = ogrid(g)
    res = run_syn(backend, r, g, [fixed], g, [moving], fixed_mask=(g, fm),
                  moving_mask=(mgrid, mm))
    ow, oinv, orecs, _ = O.syn_run(oracle_recipe(r), og, [fixed], og, [moving],
                                   masks=dict(fixed_grid=og, fixed=fm, moving_grid=ogrid(mgrid),
                                              moving=mm))
    assert len(res.iterations) == len(orecs) == 14
    rms = np.sqrt(((res.warp.astype(np.float64) - ow) ** 2).sum(-1).mean())
    rms_inv = np.sqrt(((res.inverse_warp.astype(np.float64) - oinv) ** 2).sum(-1).mean())
    assert rms <= 0.05 and rms_inv <= 0.05, (rms, rms_inv)
    assert abs(res.iterations[-1]["energy"] - orecs[-1].energy) <= 1e-4 * abs(orecs[-1].energy)


def test_masks_of_ones_give_the_unmasked_run_bit_for_bit(backend):
    """syn.rs:1239: masks of ones leave a run unchanged."""
    g, fixed, moving = blob_pair(40, seed=57)
    r = SynRecipe(gradient_step=0.25, update_field_variance=3.0, cc_radius=2,
                  iterations=[4, 3], shrink_factors=[2, 1], smoothing_sigmas=[1.0, 0.0],
                  convergence_threshold=-1.0)
    res = run_syn(backend, r, g, [fixed], g, [moving])
    ones = np.ones((40, 40, 40))
    masked = run_syn(backend, r, g, [fixed], g, [moving], fixed_mask=(g, ones),
                     moving_mask=(g, ones))
    assert np.array_equal(res.warp, masked.warp)
    assert np.array_equal(res.inverse_warp, masked.inverse_warp)
    assert [i["energy"] for i in res.iterations] == [i["energy"] for i in masked.iterations]


def test_an_all_zero_mask_is_refused(backend):
    """recipe.rs:239-246."""
    from fastwarp_b200 import _native as N
    g, fixed, moving = blob_pair(24, seed=58)
    r = config1(2)
    with pytest.raises(N.FastwarpError, match="moving mask has no voxel inside"):
        run_syn(backend, r, g, [fixed], g, [moving], moving_mask=(g, np.zeros((24, 24, 24))))


# ---- Mattes channels (SynMetric::Mattes, syn.rs:301-335): the dense MI pair drives the side ----
# updates. Bars: one step matches to 1e-5 relative on the energy and 5e-4 of the largest update
# component (the MI derivative tolerance, parity.rs:45-48); a run to 0.05 mm RMS and 1e-4
# relative final energy.

def mattes(iterations=1, **kw):
    base = dict(gradient_step=0.1, update_field_variance=3.0, cc_radius=2,
                iterations=[iterations], shrink_factors=[1], smoothing_sigmas=[0.0],
                convergence_threshold=-1.0, channel_metrics=["mattes"], mi_bins=32)
    base.update(kw)
    return SynRecipe(**base)


def test_one_mattes_syn_step_matches(backend, pair):
    g, fixed, moving = pair
    r = mattes()
    og = ogrid(g)
    fi, mi = backend.upload_image(g, fixed), backend.upload_image(g, moving)
    state = {k: backend.zero_field(g) for k in ("f2m", "f2m_inv", "m2m", "m2m_inv")}
    rec, fu, mu = syn_step(backend, r, [fi], [mi], None, state)
    ostate = {k: np.zeros((64, 64, 64, 3)) for k in ("f2m", "f2m_inv", "m2m", "m2m_inv")}
    orec, ofu, omu = O.syn_step(oracle_recipe(r), og, og, [fixed], og, [moving], None, ostate)
    assert abs(rec["energy"] - orec.energy) <= 1e-5 * abs(orec.energy)
    assert abs(rec["energy_weighted"] - orec.energy_weighted) <= 1e-5 * abs(orec.energy_weighted)
    assert np.abs(fu - ofu).max() <= 5e-4 * np.abs(ofu).max()
    assert np.abs(mu - omu).max() <= 5e-4 * np.abs(omu).max()


def test_mattes_registration_matches_the_oracle(backend):
    g, fixed, moving = blob_pair(40, seed=61)
    r = mattes(iterations=5, shrink_factors=[2, 1], smoothing_sigmas=[1.0, 0.0])
    r.iterations = [5, 4]
    og = ogrid(g)
    res = run_syn(backend, r, g, [fixed], g, [moving])
    ow, oinv, orecs, _ = O.syn_run(oracle_recipe(r), og, [fixed], og, [moving])
    assert len(res.iterations) == len(orecs) == 9
    rms = np.sqrt(((res.warp.astype(np.float64) - ow) ** 2).sum(-1).mean())
    assert rms <= 0.05, rms
    assert abs(res.iterations[-1]["energy"] - orecs[-1].energy) <= 1e-4 * abs(orecs[-1].energy)


def test_a_cc_and_a_mattes_channel_with_masks_match_the_oracle(backend):
    g, fixed, moving = blob_pair(40, seed=62)
    r = mattes(iterations=4, channel_weights=[0.5, 0.5], channel_metrics=["cc", "mattes"])
    fm, mgrid, mm = masks_for(40)
    f2, m2 = 1.0 - fixed, 1.0 - moving
    og = ogrid(g)
    res = run_syn(backend, r, g, [fixed, f2], g, [moving, m2], fixed_mask=(g, fm),
                  moving_mask=(mgrid, mm))
    ow, _, orecs, _ = O.syn_run(oracle_recipe(r), og, [fixed, f2], og, [moving, m2],
                                masks=dict(fixed_grid=og, fixed=fm, moving_grid=ogrid(mgrid),
                                           moving=mm))
    rms = np.sqrt(((res.warp.astype(np.float64) - ow) ** 2).sum(-1).mean())
    assert rms <= 0.05, rms
    for a, b in zip(res.iterations, orecs):
        assert abs(a["energy"] - b.energy) <= 1e-4 * abs(b.energy)
        assert abs(a["energy_weighted"] - b.energy_weighted) <= 1e-4 * abs(b.energy_weighted)


def test_mattes_recipe_errors(backend):
    from fastwarp_b200 import _native as N
    g, fixed, moving = blob_pair(16, seed=63)
    with pytest.raises(N.FastwarpError, match="at least five histogram bins"):
        run_syn(backend, mattes(mi_bins=4), g, [fixed], g, [moving])
    flat = np.full_like(fixed, 0.5)
    with pytest.raises(N.FastwarpError, match="the fixed image is constant"):
        run_syn(backend, mattes(), g, [flat], g, [moving])


def test_the_op_by_op_loop_with_a_mattes_channel_matches_the_graph_driver(backend):
    from fastwarp_b200.syn import run_syn_ops
    g, fixed, moving = blob_pair(32, seed=64)
    r = mattes(iterations=3, channel_weights=[0.6, 0.4], channel_metrics=["mattes", "cc"])
    f2, m2 = 1.0 - fixed, 1.0 - moving
    res = run_syn(backend, r, g, [fixed, f2], g, [moving, m2])
    w, iw, recs = run_syn_ops(backend, r, g, [fixed, f2], g, [moving, m2])
    assert len(recs) == len(res.iterations) == 3
    assert np.sqrt(((w - res.warp) ** 2).sum(-1).mean()) <= 1e-3
    assert abs(recs[-1]["energy"] - res.iterations[-1]["energy"]) <= 1e-5 * abs(recs[-1]["energy"])
