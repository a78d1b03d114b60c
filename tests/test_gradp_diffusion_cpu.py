"""The pressure-gradient term of the mixture diffusion flux
(gradPInDiffusionFlux; reference src/ViscousScheme.cu:495-520 for the
collocated schemes, :742-766, 931-955, 1115-1139 for the second-order one)
in the CPU oracle.

On a block of uniform composition the mass-fraction gradients vanish, so
without the term the species rows of the viscous flux difference are exactly
zero and with it they are driven by grad p alone: nonzero, and summing to
zero over the species (the correction velocity keeps the diffusion fluxes
mass-conserving) to round-off; species heavier and lighter than the mixture
are driven in opposite directions."""
import numpy as np
import pytest

import cases
import mechanism
import pyoracle


def _uniform_composition_case(order):
    mech = mechanism.load("li2004")
    base = cases.mix_wave(mech, 11, ny=9, nz=7, scheme=52, viscous=True, viscous_order=order)
    sv = np.repeat(base.sv.mean(axis=1, keepdims=True), base.sv.shape[1], axis=1)
    rng = np.random.default_rng(3)
    bv = base.bv.copy()
    bv[4] = bv[4] * (1 + 0.05 * rng.standard_normal(bv.shape[1]))
    R = cases.R_U * (sv / mech.mw[:, None]).sum(axis=0)
    bv[0] = bv[4] / (bv[5] * R)
    return base.__class__(**{**base.__dict__, "sv": sv, "bv": bv}), mech


def _species_rows(case, gradp):
    c = case.__class__(**{**case.__dict__, "param": {**case.param, "gradPInDiffusionFlux": gradp}})
    oz = pyoracle.OracleZone(c)
    oz.initialize()
    oz["dq"][:] = 0
    oz.call("orc_compute_viscous_flux")
    return oz["dq"][5:5 + c.mech.n_spec].copy()


@pytest.mark.parametrize("order", [2, 8])
def test_gradp_term_alone_drives_uniform_composition(order):
    case, mech = _uniform_composition_case(order)
    off = _species_rows(case, 0)
    on = _species_rows(case, 1)
    assert np.all(off == 0.0)
    scale = np.abs(on).max()
    assert scale > 0
    present = np.abs(case.sv[:, 0]) > 0
    assert np.all(np.abs(on[present]).max(axis=1) > 1e-6 * scale)
    assert np.abs(on.sum(axis=0)).max() <= 1e-12 * scale


def test_gradp_sign_follows_molecular_weight():
    """The term's driving force is (W/W_k - 1) Y_k grad(p)/p, whose sign
    is set by whether species k is heavier or lighter than the mixture: at
    the node where the term acts most strongly the flux differences of the
    heavier species share one sign and those of the lighter species the
    other (for this composition the correction velocity, a common shift,
    does not reverse any of them)."""
    case, mech = _uniform_composition_case(2)
    on = _species_rows(case, 1)
    y = case.sv[:, 0]
    W = 1.0 / np.sum(y / mech.mw)
    heavy = [l for l in range(mech.n_spec) if y[l] > 0 and mech.mw[l] > W]
    light = [l for l in range(mech.n_spec) if y[l] > 0 and mech.mw[l] < W]
    assert heavy and light
    node = np.argmax(np.abs(on).sum(axis=0))
    s_heavy = np.sign(on[heavy, node])
    s_light = np.sign(on[light, node])
    assert np.all(s_heavy == s_heavy[0]) and np.all(s_light == -s_heavy[0])
