"""limit_flow in the CPU oracle (reference src/TimeAdvanceFunc.cuh:117-230,
limits src/DParameter.cu:333-357): unphysical interior nodes (NaN, or
density / velocity / pressure outside their limits) take the average of the
good nodes of their 3x3x3 neighbourhood, or their own values clamped to the
limits when no neighbour is good; T follows from the state equation and cv
from the new state.  Good and bad are judged on the state before the call."""
import numpy as np
import pytest

import cases
import pyoracle

R_AIR = 8314.462618 / 28.9647


def _tube():
    case = cases.sod(24, 9, scheme=52)
    oz = pyoracle.OracleZone(case)
    oz.initialize()
    return case, oz


def _limits(case):
    # as the reference derives them from the freestream (rho_inf = 1, p_inf = 1, v_ref)
    v = case.param["v_ref"]
    return [1e-6, -1000 * v, -1000 * v, -1000 * v, 1e-6], [1e3, 1000 * v, 1000 * v, 1000 * v, 1e3]


def _view(case, oz, key="bv"):
    g = case.ngg
    a = oz[key]
    return a.reshape(a.shape[0], case.mz + 2 * g, case.my + 2 * g, case.mx + 2 * g)


def test_isolated_bad_node_takes_its_good_neighbours_mean():
    case, oz = _tube()
    ll, ul = _limits(case)
    g = case.ngg
    B = _view(case, oz)
    before = B.copy()
    i, j = 5, 4
    B[4, g, g + j, g + i] = np.nan       # a NaN pressure
    B[0, g, g + 2, g + 15] = -1.0        # a negative density elsewhere
    assert oz.limit_flow(ll, ul) == 2
    nb = before[:5, g, g + j - 1:g + j + 2, g + i - 1:g + i + 2].reshape(5, -1)
    good = np.ones(nb.shape[1], bool)
    good[4] = False                      # the node itself (3x3 in 2-D: the centre is entry 4)
    want = nb[:, good].mean(axis=1)
    got = B[:5, g, g + j, g + i]
    assert np.allclose(got, want, rtol=1e-15, atol=1e-300)
    assert np.isclose(B[5, g, g + j, g + i], got[4] / (got[0] * R_AIR), rtol=1e-15)
    C = _view(case, oz, "cv")
    assert np.isclose(C[0, g, g + j, g + i], got[0], rtol=1e-15)
    # every other interior node is untouched
    mask = np.ones(B.shape[1:], bool)
    mask[g, g + j, g + i] = mask[g, g + 2, g + 15] = False
    assert np.array_equal(B[:5][:, mask], before[:5][:, mask])


def test_neighbouring_bad_nodes_use_only_the_good_ones():
    """Two adjacent bad nodes: each averages the good nodes around it and
    never the other bad node (judged before the call)."""
    case, oz = _tube()
    ll, ul = _limits(case)
    g = case.ngg
    B = _view(case, oz)
    before = B.copy()
    B[0, g, g + 4, g + 8] = np.nan
    B[0, g, g + 4, g + 9] = 2e3          # above the density limit
    assert oz.limit_flow(ll, ul) == 2
    for i in (8, 9):
        keep = np.ones(9, bool)
        keep[4] = False
        keep[5 if i == 8 else 3] = False  # the other bad node
        assert np.allclose(B[:5, g, g + 4, g + i], before[:5, g, g + 3:g + 6, g + i - 1:g + i + 2]
                           .reshape(5, -1)[:, keep].mean(axis=1), rtol=1e-15, atol=1e-300)


def test_all_bad_neighbourhood_is_clamped():
    case, oz = _tube()
    ll, ul = _limits(case)
    g = case.ngg
    B = _view(case, oz)
    B[4, g, g + 1:g + 4, g + 9:g + 12] = 5e3   # a 3x3 patch above the pressure limit
    n = oz.limit_flow(ll, ul)
    assert n == 9
    assert B[4, g, g + 2, g + 10] == ul[4]     # the centre has no good neighbour: clamped
    assert B[4, g, g + 1, g + 9] < ul[4]       # a corner of the patch has good neighbours: averaged


def test_physical_state_is_left_alone():
    case, oz = _tube()
    ll, ul = _limits(case)
    before = oz["bv"].copy(), oz["cv"].copy()
    assert oz.limit_flow(ll, ul) == 0
    assert np.array_equal(oz["bv"], before[0]) and np.array_equal(oz["cv"], before[1])


def test_setup_reader_takes_limit_flow_and_its_bounds(tmp_path):
    """limit_flow and the bounds the reference derives from its reference
    state (src/DParameter.cu:333-349): rho 1e-6..1e3 rho_inf, velocity
    +-1000 v_inf (the speed of sound when |v_inf| < 1), p 1e-6..1e3 p_inf."""
    import ctypes

    import corefl_b200

    setup = tmp_path / "setup.txt"
    setup.write_text("bool limit_flow = 1\nstring reference_state = free\n"
                     "struct free {\n  string type = inflow\n  int label = 5\n  real density = 1.2\n"
                     "  real velocity = 0.5\n  real pressure = 1e5\n}\n")
    p = corefl_b200.cfk_param()
    err = ctypes.create_string_buffer(256)
    assert corefl_b200.lib().cfk_param_from_setup(str(setup).encode(), ctypes.byref(p), err, 256) == 0
    assert p.limit_flow == 1
    T = 1e5 * 28.9647 / (1.2 * 8314.462618)
    c = (1.4 * 8314.462618 / 28.9647 * T) ** 0.5
    assert list(p.limit_ll) == pytest.approx([1.2e-6, -1000 * c, -1000 * c, -1000 * c, 0.1], rel=1e-15)
    assert list(p.limit_ul) == pytest.approx([1.2e3, 1000 * c, 1000 * c, 1000 * c, 1e8], rel=1e-15)
    setup.write_text("int hardCodedMech = 1\n")
    rc = corefl_b200.lib().cfk_param_from_setup(str(setup).encode(), ctypes.byref(p), err, 256)
    assert rc != 0 and b"hardCodedMech" in err.value


def test_oracle_rk3_step_applies_limit_flow():
    """With limit_flow set, the oracle's stage loop repairs a density spike
    above the bound in every stage: after one step no interior density
    exceeds it, while the same step without limit_flow leaves it there."""
    base = cases.sod(48, 7, scheme=52)
    v = base.param["v_ref"]
    ll, ul = [1e-6, -1000 * v, -1000 * v, -1000 * v, 1e-6], [2.0, 1000 * v, 1000 * v, 1000 * v, 1e3]
    bv = base.bv.copy()
    g = base.ngg
    B = bv.reshape(6, base.mz + 2 * g, base.my + 2 * g, base.mx + 2 * g)
    B[0, g, g + 3, g + 10] = 4.0
    B[5] = B[4] / (B[0] * R_AIR)
    out = {}
    for on in (0, 1):
        case = base.__class__(**{**base.__dict__, "bv": bv.copy(),
                                 "param": dict(base.param, limit_flow=on, limit_ll=ll, limit_ul=ul)})
        oz = pyoracle.OracleZone(case)
        oz.initialize()
        oz.step()
        out[on] = case.interior(oz["bv"][0]).max()
    assert out[1] <= 2.0 < out[0]
