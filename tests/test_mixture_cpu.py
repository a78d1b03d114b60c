"""The oracle's mixture flow path (WENO5 characteristic with species, NASA-7
thermo, temperature Newton iteration) against an exact Riemann solution:
a shock tube of pure argon, whose NASA-7 cp is exactly 2.5 R (gamma = 5/3),
so the exact solution of the gamma-law Riemann problem applies."""
import math

import numpy as np
import pytest

import cases
import mechanism
import pyoracle


def exact_riemann(gamma, left, right, x, x0, t):
    """Exact solution of the 1-D Riemann problem for a gamma-law gas: Newton
    iteration on the star pressure with the shock / rarefaction pressure
    functions and sampling of the wave pattern (Toro, Riemann Solvers and
    Numerical Methods for Fluid Dynamics, ch. 4).  States are (rho, u, p);
    returns rho, u, p at the positions x at time t."""
    rl, ul, pl = left
    rr, ur, pr = right
    cl, cr = math.sqrt(gamma * pl / rl), math.sqrt(gamma * pr / rr)
    g1, g2 = (gamma - 1) / (2 * gamma), (gamma + 1) / (2 * gamma)

    def f(p, rk, pk, ck):
        if p > pk:
            A, B = 2 / ((gamma + 1) * rk), (gamma - 1) / (gamma + 1) * pk
            return (p - pk) * math.sqrt(A / (p + B)), math.sqrt(A / (B + p)) * (1 - (p - pk) / (2 * (B + p)))
        return 2 * ck / (gamma - 1) * ((p / pk) ** g1 - 1), (p / pk) ** (-g2) / (rk * ck)

    p = 0.5 * (pl + pr)
    for _ in range(100):
        fl, dl = f(p, rl, pl, cl)
        fr, dr = f(p, rr, pr, cr)
        dp = (fl + fr + ur - ul) / (dl + dr)
        p = max(p - dp, 1e-12)
        if abs(dp) < 1e-14 * p:
            break
    fl, _ = f(p, rl, pl, cl)
    fr, _ = f(p, rr, pr, cr)
    us = 0.5 * (ul + ur) + 0.5 * (fr - fl)
    out = np.zeros((3, x.size))
    for n, xx in enumerate(x):
        s = (xx - x0) / t
        if s <= us:  # left of the contact
            if p > pl:
                sl = ul - cl * math.sqrt(g2 * p / pl + g1)
                if s < sl:
                    out[:, n] = (rl, ul, pl)
                else:
                    r = rl * ((p / pl + (gamma - 1) / (gamma + 1)) / ((gamma - 1) / (gamma + 1) * p / pl + 1))
                    out[:, n] = (r, us, p)
            else:
                shl, cml = ul - cl, cl * (p / pl) ** g1
                stl = us - cml
                if s < shl:
                    out[:, n] = (rl, ul, pl)
                elif s > stl:
                    out[:, n] = (rl * (p / pl) ** (1 / gamma), us, p)
                else:
                    u = 2 / (gamma + 1) * (cl + (gamma - 1) / 2 * ul + s)
                    c = 2 / (gamma + 1) * (cl + (gamma - 1) / 2 * (ul - s))
                    r = rl * (c / cl) ** (2 / (gamma - 1))
                    out[:, n] = (r, u, pl * (c / cl) ** (2 * gamma / (gamma - 1)))
        else:  # right of the contact
            if p > pr:
                sr = ur + cr * math.sqrt(g2 * p / pr + g1)
                if s > sr:
                    out[:, n] = (rr, ur, pr)
                else:
                    r = rr * ((p / pr + (gamma - 1) / (gamma + 1)) / ((gamma - 1) / (gamma + 1) * p / pr + 1))
                    out[:, n] = (r, us, p)
            else:
                shr, cmr = ur + cr, cr * (p / pr) ** g1
                stR = us + cmr
                if s > shr:
                    out[:, n] = (rr, ur, pr)
                elif s < stR:
                    out[:, n] = (rr * (p / pr) ** (1 / gamma), us, p)
                else:
                    u = 2 / (gamma + 1) * (-cr + (gamma - 1) / 2 * ur + s)
                    c = 2 / (gamma + 1) * (cr - (gamma - 1) / 2 * (ur - s))
                    r = rr * (c / cr) ** (2 / (gamma - 1))
                    out[:, n] = (r, u, pr * (c / cr) ** (2 * gamma / (gamma - 1)))
    return out


def test_exact_riemann_reproduces_sod_golden():
    import os
    golden = np.load(os.path.join(os.path.dirname(__file__), "golden", "sod_exact.npz"))
    xs = np.linspace(0.02, 0.98, 97)
    ex = exact_riemann(1.4, (1.0, 0.0, 1.0), (0.125, 0.0, 0.1), xs, 0.5, 0.2)
    for slot, key in ((0, "rho"), (1, "u"), (2, "p")):
        ref = np.interp(xs, golden["x"], golden[key])
        assert np.median(np.abs(ex[slot] - ref)) < 1e-3, key


def test_oracle_argon_tube_against_exact_solution():
    mech = mechanism.load("premix_h2_ar")
    k = mech.index("AR")
    assert np.allclose(mech.low[k, :5], [2.5, 0, 0, 0, 0]) and np.allclose(mech.high[k, :5], [2.5, 0, 0, 0, 0])
    left = dict(rho=1.0, p=1.0e5, Y={"AR": 1.0})
    right = dict(rho=0.125, p=1.0e4, Y={"AR": 1.0})
    c = cases.mix_tube(mech, 400, 7, scheme=52, left=left, right=right, length=1.0)
    z = pyoracle.OracleZone(c)
    z.initialize()
    t, t_end = 0.0, 5e-4
    while t < t_end - 1e-12:
        t += z.step()
    xs = np.linspace(0.0, 1.0, 400)
    ex = exact_riemann(5.0 / 3.0, (1.0, 0.0, 1.0e5), (0.125, 0.0, 1.0e4), xs, 0.5, t)
    bv = z["bv"]
    scale = (1.0, math.sqrt(5.0 / 3.0 * 1.0e5), 1.0e5)
    for n, slot in enumerate((0, 1, 4)):
        got = c.interior(bv[slot])[0, 3]
        err = np.abs(got - ex[n]).mean() / scale[n]
        assert err < 4e-3, (slot, err)
    # the species stay pure argon and gamma is 5/3 everywhere
    assert np.allclose(c.interior(z["sv"][k])[0], 1.0, atol=1e-12)
    assert np.allclose(c.interior(z["gamma"])[0], 5.0 / 3.0, rtol=1e-12)


@pytest.mark.parametrize("scheme", [2, 3, 4])
def test_oracle_pv_schemes_argon_tube_against_exact_solution(scheme):
    """Roe, AUSM+ and HLLC in their mixture form (reference
    src/InviscidScheme.cu:171-765, mixture branches) on the argon tube: the
    side energies and gamma from NASA-7 thermo reproduce the exact
    gamma = 5/3 Riemann solution."""
    mech = mechanism.load("premix_h2_ar")
    left = dict(rho=1.0, p=1.0e5, Y={"AR": 1.0})
    right = dict(rho=0.125, p=1.0e4, Y={"AR": 1.0})
    c = cases.mix_tube(mech, 400, 7, scheme=scheme, left=left, right=right, length=1.0, reconstruction=2)
    z = pyoracle.OracleZone(c)
    z.initialize()
    t, t_end = 0.0, 5e-4
    while t < t_end - 1e-12:
        t += z.step()
    xs = np.linspace(0.0, 1.0, 400)
    ex = exact_riemann(5.0 / 3.0, (1.0, 0.0, 1.0e5), (0.125, 0.0, 1.0e4), xs, 0.5, t)
    bv = z["bv"]
    scale = (1.0, math.sqrt(5.0 / 3.0 * 1.0e5), 1.0e5)
    for n, slot in enumerate((0, 1, 4)):
        got = c.interior(bv[slot])[0, 3]
        err = np.abs(got - ex[n]).mean() / scale[n]
        assert err < 6e-3, (slot, err)


@pytest.mark.parametrize("scheme", [2, 3, 4])
def test_oracle_pv_species_fluxes_sum_to_mass_flux(scheme):
    """With first-order reconstruction the face mass fractions sum to one, so
    the species fluxes of every scheme sum to the mass flux (for Roe the
    species waves cancel: sum_k (d(rho Y_k) - Y~_k d rho) = 0)."""
    mech = mechanism.load("li2004")
    c = cases.perturbed(cases.mix_wave(mech, 11, ny=9, nz=7, scheme=scheme, viscous=False, reconstruction=1),
                        seed=3, amp=2e-2)
    z = pyoracle.OracleZone(c)
    z.initialize()
    z.call("orc_compute_inviscid_flux")
    ns = mech.n_spec
    for key in ("fFlux", "gFlux", "hFlux"):
        f = z[key]
        mass = f[0]
        spec = f[5:5 + ns].sum(axis=0)
        nz_ = np.abs(mass) > 0
        assert nz_.any()
        assert np.abs(spec[nz_] - mass[nz_]).max() <= 1e-11 * np.abs(mass).max(), key
