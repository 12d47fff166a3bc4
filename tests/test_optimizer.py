"""The linear-stage optimiser (optimizer.rs:142-435): the library's host implementation against
the reference's own optimiser tests (optimizer.rs:437-600) and against the oracle's independent
restatement, on a quadratic metric given as a Python callback (no GPU needed: the optimiser is
host code over whatever metric it is handed)."""
import numpy as np
import pytest

import oracle as O
from fastwarp_b200 import linear_transform
from fastwarp_b200.backend import cg_settings_ants, optimize_level


def cube_corners(half):
    return [[x, y, z] for x in (-half, half) for y in (-half, half) for z in (-half, half)]


def quadratic(target, weights=(1.0,) * 6):
    def value(t):
        p = list(t.parameters[:6])
        return sum(w * (a - b) ** 2 for w, a, b in zip(weights, p, target))

    def value_and_derivative(t):
        p = list(t.parameters[:6])
        d = [-2.0 * w * (a - b) for w, a, b in zip(weights, p, target)]
        return value(t), d
    return value, value_and_derivative


def rigid():
    return linear_transform("euler", [0.0] * 6, center=(0.0, 0.0, 0.0))


def test_rigid_scales_are_squared_corner_shifts_per_unit_parameter():
    from fastwarp_b200 import _native as N
    import ctypes as C
    corners = (C.c_double * 24)(*np.ravel(cube_corners(50.0)))
    out = (C.c_double * 12)()
    t = rigid()
    assert N.lib().fw_linear_estimate_scales(corners, C.byref(t), C.c_double(0.01), out) == 0
    for s in out[3:6]:
        assert abs(s - 1.0) < 1e-9
    want = np.hypot(50.0, 50.0) ** 2
    for s in out[:3]:
        assert abs(s - want) / want < 1e-3


def test_affine_scales_follow_the_corner_distance_from_the_centre():
    from fastwarp_b200 import _native as N
    import ctypes as C
    corners = (C.c_double * 24)(*np.ravel(cube_corners(40.0)))
    out = (C.c_double * 12)()
    t = linear_transform("affine", list(np.eye(3).ravel()) + [0.0, 0.0, 0.0],
                         center=(0.0, 0.0, 0.0))
    assert N.lib().fw_linear_estimate_scales(corners, C.byref(t), C.c_double(0.01), out) == 0
    for s in out[:9]:
        assert abs(s - 40.0 ** 2) < 1e-6
    for s in out[9:12]:
        assert abs(s - 1.0) < 1e-9


def test_step_scale_is_the_corner_shift_of_the_step():
    from fastwarp_b200 import _native as N
    import ctypes as C
    corners = (C.c_double * 24)(*np.ravel(cube_corners(50.0)))
    t = rigid()
    step = (C.c_double * 12)(0.0, 0.0, 0.0, 3.0, 4.0, 0.0)
    out = C.c_double()
    assert N.lib().fw_linear_estimate_step_scale(corners, C.byref(t), step, C.c_double(0.01),
                                                 C.byref(out)) == 0
    assert abs(out.value - 5.0) < 1e-9
    zero = (C.c_double * 12)()
    N.lib().fw_linear_estimate_step_scale(corners, C.byref(t), zero, C.c_double(0.01),
                                          C.byref(out))
    assert out.value == 0.0


def test_conjugate_gradient_with_line_search_minimises_a_quadratic():
    value, vd = quadratic([0.0, 0.0, 0.0, 3.0, -2.0, 1.0])
    t, trace = optimize_level(value, vd, cube_corners(20.0), rigid(),
                              cg_settings_ants(0.1, 200, 1e-12, 10))
    p = list(t.parameters[:6])
    assert abs(p[3] - 3.0) < 0.05 and abs(p[4] + 2.0) < 0.05 and abs(p[5] - 1.0) < 0.05, p
    assert trace["best_value"] < 0.01
    assert trace["line_search_evaluations"] > 0
    assert trace["initial_learning_rate"] > 0.0


def test_the_monitor_stops_a_converged_level_and_zero_iterations_return_the_start():
    value, vd = quadratic([0.0] * 6)
    _, trace = optimize_level(value, vd, cube_corners(20.0), rigid(),
                              cg_settings_ants(0.1, 500, 1e-6, 10))
    assert trace["converged"] and trace["iterations"] < 500
    assert len(trace["values"]) == trace["iterations"]
    assert trace["converged_value"] is not None
    t, trace = optimize_level(value, vd, cube_corners(20.0), rigid(),
                              cg_settings_ants(0.1, 0, 1e-6, 10))
    assert trace["iterations"] == 0 and list(t.parameters[:6]) == [0.0] * 6


@pytest.mark.parametrize("kind", ["euler", "affine"])
def test_the_library_optimiser_retraces_the_oracle_restatement(kind):
    """Both are f64 restatements of optimizer.rs: on one metric they take the same steps."""
    target = [0.05, -0.03, 0.02, 3.0, -2.0, 1.0]
    if kind == "euler":
        t0 = rigid()
        ot0 = O.linear_transform("euler", [0.0] * 6, center=(0.0, 0.0, 0.0))
        n = 6
    else:
        ident = list(np.eye(3).ravel()) + [0.0, 0.0, 0.0]
        t0 = linear_transform("affine", ident, center=(1.0, -2.0, 0.5))
        ot0 = O.linear_transform("affine", ident, center=(1.0, -2.0, 0.5))
        target = ident[:6] + [0.1, 0.0, 1.0, 2.0, -1.0, 0.5]
        n = 12
    w = [1.0 + 0.3 * i for i in range(n)]

    def value(t):
        return sum(wi * (t.parameters[i] - target[i]) ** 2 for i, wi in enumerate(w))

    def vd(t):
        return value(t), [-2.0 * wi * (t.parameters[i] - target[i]) for i, wi in enumerate(w)]

    corners = cube_corners(30.0)
    t, trace = optimize_level(value, vd, corners, t0, cg_settings_ants(0.1, 60, 1e-9, 10))
    ot, otrace = O.cg_optimize_level(value, vd, corners, ot0, O.cg_settings_ants(0.1, 60, 1e-9, 10))
    assert trace["values"] == otrace["values"]
    assert trace["iterations"] == otrace["iterations"]
    assert trace["line_search_evaluations"] == otrace["line_search_evaluations"]
    assert list(t.parameters[:n]) == list(ot.parameters[:n])
