"""Parity of the chemistry kernels against the CPU oracle: the Wu-splitting
reaction step (point implicit and explicit, both schedules) and the explicit
finite-rate source, on seeded batches of H2/air reactors (Li-2004,
9 species / 19 reactions; PREMIX H2/O2/Ar, 9 species / 18 reactions).

Bar: per step from identical inputs, max |gpu - oracle| / max |oracle| of
every conserved-variable plane <= 1e-12; substep counts identical; the
work-queue schedule bit-identical to one thread per node.
"""
import numpy as np
import pytest

import cases
import mechanism
import pyoracle
from gpuzone import GpuZone, rel_err

pytestmark = pytest.mark.gpu


def _pair(case):
    oz = pyoracle.OracleZone(case)
    oz.call("orc_compute_cv_from_bv")
    gz = GpuZone(case)
    gz.ctx.cv_from_bv()
    gz.torch.cuda.synchronize()
    return oz, gz


def _nsub_tensor(gz):
    import torch
    return torch.zeros(gz.case.N, dtype=torch.int32, device="cuda:0")


@pytest.mark.parametrize("schedule", [0, 1])
@pytest.mark.parametrize("mech_name", ["li2004", "premix_h2_ar"])
def test_wu_reaction_point_implicit_per_step(schedule, mech_name):
    mech = mechanism.load(mech_name)
    if mech_name == "li2004":
        case = cases.reactor_batch(mech, 512, seed=7)
    else:  # stoichiometric H2/O2 diluted 70 % Ar
        X = np.zeros(mech.n_spec)
        X[mech.index("H2")], X[mech.index("O2")], X[mech.index("AR")] = 0.2, 0.1, 0.7
        T = np.linspace(1100.0, 1900.0, 300)
        case = cases.reactor(mech, T, 30000.0, X)
    oz, gz = _pair(case)
    nsub = _nsub_tensor(gz)
    dt = 1e-7
    for s in range(6):
        gz.load_from(oz, keys=("cv", "bv", "sv", "reaction_timeScale"))
        ns_o = oz.reaction_step(dt, want_nsub=True)
        gz.ctx.wu_reaction_step(dt, schedule=schedule, nsub_ptr=nsub.data_ptr())
        gz.ctx.sync()
        assert np.array_equal(nsub.cpu().numpy(), ns_o), f"substep counts differ at step {s}"
        e = rel_err(gz.get("cv"), oz["cv"])
        assert e <= 1e-12, f"step {s}: conserved-variable relative difference {e:.3e}"
        assert rel_err(gz.get("bv")[[0, 4, 5]], oz["bv"][[0, 4, 5]], momentum=()) <= 1e-12
        assert rel_err(gz.get("reaction_timeScale")[None], oz["reaction_timeScale"][None], momentum=()) <= 1e-12


def test_wu_reaction_explicit_per_step():
    mech = mechanism.load("li2004")
    case = cases.reactor_batch(mech, 256, seed=3)
    case.param["chem_advance_method"] = 0
    oz, gz = _pair(case)
    for s in range(4):
        gz.load_from(oz, keys=("cv", "bv", "sv", "reaction_timeScale"))
        oz.reaction_step(2e-8)
        gz.ctx.wu_reaction_step(2e-8, schedule=0)
        gz.ctx.sync()
        assert rel_err(gz.get("cv"), oz["cv"]) <= 1e-12


def test_work_queue_is_bit_identical_to_plain_schedule():
    mech = mechanism.load("li2004")
    case = cases.reactor_batch(mech, 4096, seed=11)
    a = GpuZone(case)
    b = GpuZone(case)
    for z in (a, b):
        z.ctx.cv_from_bv()
    na, nb = _nsub_tensor(a), _nsub_tensor(b)
    for _ in range(8):
        a.ctx.wu_reaction_step(1e-7, schedule=0, nsub_ptr=na.data_ptr())
        b.ctx.wu_reaction_step(1e-7, schedule=1, nsub_ptr=nb.data_ptr())
    a.ctx.sync()
    b.ctx.sync()
    assert np.array_equal(a.get("cv"), b.get("cv"))
    assert np.array_equal(na.cpu().numpy(), nb.cpu().numpy())
    assert na.cpu().numpy().max() > na.cpu().numpy().min()  # uneven work really occurred


def test_finite_rate_chemistry_source():
    mech = mechanism.load("li2004")
    case = cases.reactor_batch(mech, 300, seed=5)
    oz, gz = _pair(case)
    # advance a little so that radicals exist
    for _ in range(3):
        oz.reaction_step(1e-7)
    gz.load_from(oz, keys=("cv", "bv", "sv", "reaction_timeScale"))
    oz["dq"][:] = 0
    gz.t["dq"].zero_()
    oz.call("orc_finite_rate_chemistry")
    gz.ctx.finite_rate_chemistry()
    gz.ctx.sync()
    assert rel_err(gz.get("dq")[5:], oz["dq"][5:], momentum=()) <= 1e-12
    assert rel_err(gz.get("reaction_timeScale")[None], oz["reaction_timeScale"][None], momentum=()) <= 1e-12


def test_ignition_of_the_reference_reactor_case():
    """The reference's constant-volume example (1000 K, 2 atm, Li-2004) on the
    GPU: the final equilibrium matches the reference's golden trajectory and
    the ignition time (T = 1500 K) matches the oracle's (same integrator)."""
    import os
    golden = np.load(os.path.join(os.path.dirname(__file__), "golden", "reactor_li2004.npz"))
    mech = mechanism.load("li2004")
    X = np.zeros(9)
    X[mech.index("H2")], X[mech.index("O2")], X[mech.index("N2")] = 0.295775, 0.147887, 0.556338
    case = cases.reactor(mech, [1000.0], 202650.0, X)
    gz = GpuZone(case)
    gz.ctx.cv_from_bv()
    dt, t, Ts = 2e-7, 0.0, []
    while t < 1.2e-3 - 1e-12:
        gz.ctx.wu_reaction_step(dt, schedule=1)
        t += dt
        Ts.append(float(gz.t["bv"][5, 0].item()))
    Ts = np.array(Ts)
    ts = dt * np.arange(1, len(Ts) + 1)
    assert Ts[-1] == pytest.approx(golden["T"][-1], rel=1e-5)
    t_ign = np.interp(1500.0, Ts, ts)
    assert t_ign == pytest.approx(8.88e-4, rel=0.01)
