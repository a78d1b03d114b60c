"""The collocated viscous schemes in the CPU oracle: 8th order (viscous_order =
8, reference src/ViscousScheme.cu:41-70, 129-612) and its 4th-order variant
(viscous_order = 4, which the reference does not have).

Pins: (1) on a Cartesian block with physical (outflow) faces and a velocity
that is cubic across the block, every node -- including the four next to each
wall, where the reference switches to one-sided and reduced stencils exact for
polynomials of degree 4 -- gets the exact shear term J mu u''(y); (2) on a
periodic block a sine shear converges at 8th order (error ratio ~ 2^8 per
grid halving) and is far below the 2nd-order scheme's error."""
import numpy as np

import cases
import pyoracle

R_U, MW_AIR = 8314.462618, 28.9647


def _set_shear(case, yphys, u):
    """rho = 1, p uniform (so T and Sutherland mu are uniform), u = u(y)."""
    bv = case.bv
    bv[0] = 1.0
    bv[1] = u(yphys)
    bv[2] = 0.0
    bv[3] = 0.0
    bv[4] = 1.0
    bv[5] = 1.0 * MW_AIR / (1.0 * R_U)


def _viscous_dq(case):
    oz = pyoracle.OracleZone(case)
    oz.initialize()
    oz["dq"][:] = 0
    oz.call("orc_compute_viscous_flux")
    return oz


import pytest


@pytest.mark.parametrize("order", [8, 4])
def test_one_sided_boundary_stencils_exact_for_cubic_shear(order):
    c = cases.sod(24, 12, scheme=4, viscous_order=order)
    g = c.ngg
    # physical y of every padded node: sod puts node j at y = 0.01 j
    jj = np.broadcast_to(np.arange(-g, c.my + g)[None, :, None], c.shape()).reshape(-1)
    yphys = 0.01 * jj
    a, b, cc, d = 0.3, 2.0, -40.0, 900.0
    _set_shear(c, yphys, lambda y: a + b * y + cc * y ** 2 + d * y ** 3)
    oz = _viscous_dq(c)
    mu = c.interior(oz["mul"])
    jac = c.interior(oz["jac"])
    y = c.interior(yphys.reshape(1, -1))[0]
    expect = jac * mu * (2 * cc + 6 * d * y)
    got = oz["dq"][1].reshape(c.mz, c.my, c.mx)
    assert np.abs(got - expect).max() <= 1e-9 * np.abs(expect).max()
    # no x momentum flux differences in y-only shear for the other rows
    assert np.abs(oz["dq"][2]).max() <= 1e-9 * np.abs(expect).max()


def _periodic_sine_error(n, order):
    c = cases.sine_wave(n=n, ny=n, nz=9, scheme=72, viscous=True, amp=0.0, viscous_order=order)
    g = c.ngg
    jj = np.broadcast_to(np.arange(-g, c.my + g)[None, :, None], c.shape()).reshape(-1)
    # node-based periodicity: nodes 0 and n-1 coincide; eta = j / (n - 1)
    L = np.abs(c.metric[4]).max() ** -1 * (n - 1)  # dy/deta = 1 / eta_y
    eta = jj / (n - 1)
    _set_shear(c, eta, lambda e: 0.1 * np.sin(2 * np.pi * e))
    oz = _viscous_dq(c)
    mu = c.interior(oz["mul"])
    jac = c.interior(oz["jac"])
    e = c.interior(eta.reshape(1, -1))[0]
    expect = jac * mu * (-(2 * np.pi / L) ** 2 * 0.1 * np.sin(2 * np.pi * e))
    got = oz["dq"][1].reshape(c.mz, c.my, c.mx)
    return np.abs(got - expect).max() / np.abs(expect).max()


def test_periodic_sine_shear_converges_at_eighth_order():
    e17, e33 = _periodic_sine_error(17, 8), _periodic_sine_error(33, 8)
    assert e33 < 1e-6
    assert e17 / e33 > 150  # 2^8 = 256
    assert _periodic_sine_error(33, 2) > 100 * e33


def test_periodic_sine_shear_converges_at_fourth_order():
    """viscous_order = 4 (not in the reference): the same collocated scheme
    with 4th-order central differences converges at 4th order."""
    e17, e33 = _periodic_sine_error(17, 4), _periodic_sine_error(33, 4)
    assert 12 < e17 / e33 < 20  # 2^4 = 16
    assert e33 < _periodic_sine_error(33, 2) / 5
