"""CPU tests of the chemistry: mechanism tables, the oracle's kinetics and
point-implicit reactor against the reference's golden ignition data and
against an independent stiff integration."""
import os

import numpy as np
import pytest

import cases
import mechanism
import pyoracle

HERE = os.path.dirname(os.path.abspath(__file__))


def test_bundled_mechanisms_have_the_reference_sizes():
    li = mechanism.load("li2004")
    assert li.n_spec == 9 and li.n_reac == 19  # 21 listed, two DUPLICATE pairs merged
    assert li.species == ["H2", "H", "O2", "O", "OH", "HO2", "H2O2", "H2O", "N2"]
    assert sorted(set(li.reac_type.tolist())) == [1, 3, 4, 6]
    assert (li.reac_type == 3).sum() == 2 and (li.reac_type == 6).sum() == 2
    r = int(np.where(li.reac_type == 6)[0][0])  # H + O2 (+M) = HO2 (+M)
    assert li.troe_alpha[r] == 0.8 and li.third_body_coeff[r, li.index("H2O")] == 11.0
    assert li.Ea[0] == pytest.approx(1.66e4 / 1.98720425864083)
    pm = mechanism.load("premix_h2_ar")
    assert pm.n_spec == 9 and pm.n_reac == 18 and "AR" in pm.species
    # element balance of every reaction
    for m in (li, pm):
        for r in range(m.n_reac):
            assert np.array_equal((m.stoi_f[r] @ m.elem_comp), (m.stoi_b[r] @ m.elem_comp))


def _reactor_run(dt, t_end, stop_T=None):
    m = mechanism.load("li2004")
    X = np.zeros(9)
    X[m.index("H2")], X[m.index("O2")], X[m.index("N2")] = 0.295775, 0.147887, 0.556338
    c = cases.reactor(m, 1000.0, 202650.0, X)
    z = pyoracle.OracleZone(c)
    z.call("orc_compute_cv_from_bv")
    t, ts, Ts = 0.0, [], []
    while t < t_end - 1e-12:
        z.reaction_step(dt)
        t += dt
        ts.append(t)
        Ts.append(z["bv"][5][0])
        if stop_T is not None and Ts[-1] > stop_T:
            break
    return m, z, np.array(ts), np.array(Ts)


def test_oracle_reactor_equilibrium_matches_reference_golden():
    """The reference's 0-D H2/air example ends at equilibrium: the oracle's
    point-implicit reactor reaches the golden final temperature, pressure and
    composition.  (The golden ignition time, 4.23e-4 s, comes from a
    mechanism file the reference does not ship; see the next test.)"""
    golden = np.load(os.path.join(HERE, "golden", "reactor_li2004.npz"))
    m, z, ts, Ts = _reactor_run(2e-7, 1.2e-3)
    assert Ts[-1] == pytest.approx(golden["T"][-1], rel=1e-6)
    assert z["bv"][4][0] == pytest.approx(golden["p"][-1], rel=1e-6)
    Y = z["sv"][:9, 0]
    X = (Y / m.mw) / (Y / m.mw).sum()
    assert np.allclose(X, golden["X"][-1], atol=2e-6)


def test_oracle_ignition_agrees_with_independent_stiff_integration():
    """Constant-volume ignition of the same case integrated independently:
    kinetics restated in numpy (mole-based rates, Kc from the NASA-7
    Gibbs energies) and scipy's BDF at rtol 1e-9.  The oracle's
    point-implicit Wu substeps give the same ignition time to 0.5 %."""
    from scipy.integrate import solve_ivp

    m = mechanism.load("li2004")
    Ru = 8.314462618
    W = m.mw * 1e-3

    def nasa(T):
        a = np.where((T < m.t_mid)[:, None], m.low, m.high)
        cp = a[:, 0] + a[:, 1] * T + a[:, 2] * T**2 + a[:, 3] * T**3 + a[:, 4] * T**4
        h = a[:, 0] + a[:, 1] / 2 * T + a[:, 2] / 3 * T**2 + a[:, 3] / 4 * T**3 + a[:, 4] / 5 * T**4 + a[:, 5] / T
        s = a[:, 0] * np.log(T) + a[:, 1] * T + a[:, 2] / 2 * T**2 + a[:, 3] / 3 * T**3 + a[:, 4] / 4 * T**4 + a[:, 6]
        return cp, h, s

    def wdot(T, C):
        Cc = C * 1e-6
        _, h, s = nasa(T)
        g = h - s
        w = np.zeros(m.n_spec)
        for r in range(m.n_reac):
            k = m.A[r] * T ** m.b[r] * np.exp(-m.Ea[r] / T)
            t = m.reac_type[r]
            if t == 3:
                k += m.A2[r] * T ** m.b2[r] * np.exp(-m.Ea2[r] / T)
            M = (m.third_body_coeff[r] * Cc).sum()
            if t == 4:
                k *= M
            if t >= 5:
                Pr = m.A2[r] * T ** m.b2[r] * np.exp(-m.Ea2[r] / T) * M / k
                F = 1.0
                if t >= 6:
                    al = m.troe_alpha[r]
                    Fc = (1 - al) * np.exp(-T / m.troe_t3[r]) + al * np.exp(-T / m.troe_t1[r])
                    cq, n = -0.4 - 0.67 * np.log10(Fc), 0.75 - 1.27 * np.log10(Fc)
                    f1 = (np.log10(Pr) + cq) / (n - 0.14 * (np.log10(Pr) + cq))
                    F = 10 ** (np.log10(Fc) / (1 + f1 * f1))
                k = k * Pr / (1 + Pr) * F
            nu = m.stoi_b[r] - m.stoi_f[r]
            Kc = np.exp(-(nu * g).sum()) * (101325 / (Ru * T) * 1e-6) ** nu.sum()
            w += nu * (k * np.prod(Cc ** m.stoi_f[r]) - k / Kc * np.prod(Cc ** m.stoi_b[r]))
        return w * 1e6

    X = np.zeros(9)
    X[m.index("H2")], X[m.index("O2")], X[m.index("N2")] = 0.295775, 0.147887, 0.556338
    Y0 = X * W / (X * W).sum()
    rho = 202650.0 * (X * W).sum() / (Ru * 1000.0)

    def rhs(t, y):
        T, Y = y[-1], y[:-1]
        wd = wdot(T, rho * Y / W)
        cp, h, _ = nasa(T)
        cv = ((cp - 1) * Ru / W * Y).sum()
        return np.concatenate([wd * W / rho, [-((h - 1) * Ru * T * wd).sum() / (rho * cv)]])

    ev = lambda t, y: y[-1] - 1500.0
    ev.terminal = True
    sol = solve_ivp(rhs, (0, 1.2e-3), np.concatenate([Y0, [1000.0]]), method="BDF", rtol=1e-9, atol=1e-14,
                    events=ev)
    t_bdf = sol.t_events[0][0]
    _, _, ts, Ts = _reactor_run(2e-7, 1.2e-3, stop_T=1600.0)
    t_orc = np.interp(1500.0, Ts, ts)
    assert t_orc == pytest.approx(t_bdf, rel=5e-3)
