"""The chemistry surrogate inside the reacting flow step.

A reflected-shock ignition case (cases.reflected_shock_tube: stoichiometric
H2-O2 with 70 % Ar, the PREMIX mechanism, frozen Rankine-Hugoniot states of
the incident and reflected shocks, WENO5 + mixture-averaged viscous fluxes,
adiabatic no-slip end and side walls) runs under Wu's splitting twice from the
same state: with the plain point-implicit reaction sub-step, recording one
training row per node per step from the reaction sub-step with its frozen
transport term (cfk_wu_splitting_step_record), and, after the network is
trained on those rows, with the gated surrogate sub-step
(cfk_wu_splitting_step_surrogate).  The default gate keeps a node on the
plain integrator when its plain step would take fewer than 50 substeps; at
this flow's CFL step (~7e-8 s) that leaves 17 % of the node-steps to the
network.  The run is made with that threshold at 10 substeps: over three
training seeds it put 40 % of the node-steps on the network with the
ignition delay unchanged, where with the rule off (71-74 % on the network)
the ignition delay moved by 0.6-3 %.  Bar: ignition delay (the time the
domain's peak temperature has risen by 400 K) and peak temperature within
1 % of the plain run's; at least 30 % of the node-steps on the network."""
import numpy as np
import pytest

import cases
import corefl_b200 as cf
import mechanism
import surrogate as sg
from gpuzone import GpuZone

pytestmark = pytest.mark.gpu

MACH, NX, NY, LENGTH, HEIGHT = 2.6, 128, 16, 0.02, 0.004
STEPS = 600
MIN_SUBSTEPS = 10.0  # the gate's few-substeps threshold for this flow


def _case():
    return cases.reflected_shock_tube(mechanism.load("premix_h2_ar"), NX, NY, length=LENGTH, height=HEIGHT,
                                      mach=MACH)


def _peak_trace(gz, steps, step_fn):
    """Physical time and the domain's peak temperature after every step."""
    torch = gz.torch
    t, peak, now = [], torch.empty(steps, dtype=torch.float64, device="cuda:0"), 0.0
    case = gz.case
    g = case.ngg
    T = gz.t["bv"][5].view(case.mz + 2 * g, case.my + 2 * g, case.mx + 2 * g)[g:g + case.mz, g:g + case.my,
                                                                              g:g + case.mx]
    stats = []
    for s in range(steps):
        dt, st = step_fn(s)
        now += dt
        t.append(now)
        peak[s] = T.max()
        if st:
            stats.append(st)
    return np.array(t), peak.cpu().numpy(), stats


IGN_RISE = 400.0  # K above the domain's peak temperature after the first step


def _ignition(t, peak):
    """Ignition delay of the domain: the time at which its peak temperature
    first exceeds the value after the first step by IGN_RISE, interpolated
    linearly between the two steps around the crossing.  Also returned: the
    peak temperature, the largest single-step rise and the time of that rise
    (a reported figure only: when two steps rise almost equally, a small
    change flips the argmax between them)."""
    rise = np.diff(np.concatenate([[peak[0]], peak]))
    kr = int(np.argmax(rise))
    t_rise = 0.5 * (t[kr] + (t[kr - 1] if kr else 0.0))
    thr = peak[0] + IGN_RISE
    above = np.nonzero(peak > thr)[0]
    if above.size == 0:
        return np.inf, peak.max(), rise.max(), t_rise
    k = int(above[0])
    t0, p0 = (t[k - 1], peak[k - 1]) if k else (0.0, peak[0])
    return t0 + (thr - p0) / (peak[k] - p0) * (t[k] - t0), peak.max(), rise.max(), t_rise


def test_surrogate_flow_ignition_matches_plain():
    torch = pytest.importorskip("torch")
    case = _case()
    mech = case.mech
    plain = GpuZone(case)
    plain.initialize()
    plain.ctx.surrogate_init(7, mech.element_mass_fractions())
    n = case.N
    X = torch.empty((STEPS * n, cf.SG_NIN), dtype=torch.float32, device="cuda:0")
    G = torch.empty((STEPS * n, cf.SG_NOUT), dtype=torch.float32, device="cuda:0")

    def rec(s):
        return plain.ctx.wu_splitting_step_record(X[s * n].data_ptr(), G[s * n].data_ptr()), None

    t_p, pk_p, _ = _peak_trace(plain, STEPS, rec)
    tau_p, peak_p, rise_p, trise_p = _ignition(t_p, pk_p)
    assert peak_p > pk_p[0] + 1000.0 and tau_p < 0.9 * t_p[-1], "the plain run must ignite inside the window"

    losses = sg.fit(plain.ctx, X, G, epochs=300, batch=8192)
    weights, norm = plain.ctx.surrogate_get_params()
    model = GpuZone(case)
    model.initialize()
    model.ctx.surrogate_init(7, mech.element_mass_fractions())
    model.ctx.surrogate_set_params(weights, norm)
    gate = model.ctx.surrogate_default_gate(min_substeps=MIN_SUBSTEPS)

    def surr(s):
        return model.ctx.wu_splitting_step_surrogate(gate, s, want_stats=(s % 20 == 19))

    t_s, pk_s, stats = _peak_trace(model, STEPS, surr)
    tau_s, peak_s, _, trise_s = _ignition(t_s, pk_s)
    on_net = sum(st["surrogate"] for st in stats) / sum(st["cells"] for st in stats)
    reasons = {k: sum(st[k] for st in stats) for k in stats[0] if k.startswith("fallback_") or k.startswith("judge")}
    print("fallback reasons over the window:", reasons)
    e_tau, e_pk = abs(tau_s - tau_p) / tau_p, abs(peak_s - peak_p) / peak_p
    print(f"loss {losses[0]:.3e} -> {losses[-1]:.3e}; tau_ign plain {tau_p:.4e} s, surrogate {tau_s:.4e} s "
          f"(err {e_tau:.2e}); T_peak plain {peak_p:.1f} K, surrogate {peak_s:.1f} K (err {e_pk:.2e}); "
          f"on network {on_net:.3f}; time of the largest rise plain {trise_p:.4e} s, surrogate {trise_s:.4e} s")
    assert e_tau <= 1e-2
    assert e_pk <= 1e-2
    assert on_net >= 0.3
