"""The MLP chemistry surrogate on the GPU.

* forward and backward tcgen05 kernels against the FP64 restatement
  (oracle/mlp.py): bf16-rounded variant to 1e-2, plain FP64 to 3e-2 (forward)
  and 5e-2 (gradients), relative;
* training on trajectories recorded from the plain integrator lowers the loss;
* the gated step: nodes sent to the plain integrator (gate or judge) are
  bit-identical to the plain step; surrogate nodes conserve element mass,
  total mass and energy;
* what the trained network gains: on unseen reactors, ignition delay and
  peak temperature within 1 % of the plain integrator's over full
  trajectories, and the step throughput on a burnt state mix.
"""
import numpy as np
import pytest

import cases
import mechanism
import mlp
import surrogate as sg
from gpuzone import GpuZone

pytestmark = pytest.mark.gpu


def _hot_batch(m, n, seed):
    """H2/air reactors that ignite and burn out within 80 microseconds:
    T ~ U[1250, 1700] K, p log-uniform in [1, 10] atm, phi ~ U[0.5, 2]."""
    rng = np.random.default_rng(seed)
    T = rng.uniform(1250.0, 1700.0, n)
    p = 101325.0 * np.exp(rng.uniform(0.0, np.log(10.0), n))
    phi = rng.uniform(0.5, 2.0, n)
    X = np.zeros((n, m.n_spec))
    X[:, m.index("H2")], X[:, m.index("O2")], X[:, m.index("N2")] = 2 * phi, 1.0, 3.76
    X /= X.sum(axis=1, keepdims=True)
    return cases.reactor(m, T, p, X)


def _zone(n=512, seed=7, mech_name="li2004", hot=False):
    m = mechanism.load(mech_name)
    gz = GpuZone(_hot_batch(m, n, seed) if hot else cases.reactor_batch(m, n, seed=seed))
    gz.ctx.cv_from_bv()
    gz.ctx.surrogate_init(1234, m.element_mass_fractions())
    return m, gz


def _identity_norm(lo=-10.0, hi=10.0):
    nm = np.zeros(81, np.float32)  # out_scale 0: no asinh transform
    nm[12:24] = 1.0
    nm[35:46] = 1.0
    nm[46:58] = lo
    nm[58:70] = hi
    return nm


def _random_biases(w, seed):
    rng = np.random.default_rng(seed)
    b = mlp.unpack(w)
    b[0][:, 15] = rng.normal(0, 0.2, 128)
    b[1][:, 128] = rng.normal(0, 0.2, 128)
    b[2][:, 128] = rng.normal(0, 0.2, 128)
    b[3][:11, 128] = rng.normal(0, 0.2, 11)
    return mlp.pack(b)


def test_forward_matches_fp64_network():
    _, gz = _zone()
    torch = gz.torch
    w = _random_biases(mlp.init_weights(seed=2), 3)
    gz.ctx.surrogate_set_params(weights=w, norm=_identity_norm())
    rng = np.random.default_rng(0)
    n = 1000  # not a multiple of the 128-row tile
    X = rng.normal(size=(n, 12)).astype(np.float32)
    Xd = torch.from_numpy(X).to("cuda:0")
    Yd = torch.zeros((n, 16), dtype=torch.float32, device="cuda:0")
    gz.ctx.surrogate_forward(Xd.data_ptr(), n, Yd.data_ptr())
    y = Yd.cpu().numpy().astype(np.float64)[:, :11]
    wf = gz.ctx.surrogate_get_params()[0].astype(np.float64)
    yb = mlp.forward(wf, X.astype(np.float64), bf16_round=True)[0][:, :11]
    y64 = mlp.forward(wf, X.astype(np.float64))[0][:, :11]
    scale = np.abs(y64).max()
    assert np.abs(y - yb).max() / scale <= 1e-2
    assert np.abs(y - y64).max() / scale <= 3e-2


def test_gradients_match_fp64_backward():
    _, gz = _zone()
    torch = gz.torch
    w = _random_biases(mlp.init_weights(seed=4), 5)
    gz.ctx.surrogate_set_params(weights=w, norm=_identity_norm())
    rng = np.random.default_rng(1)
    n = 777
    X = rng.normal(size=(n, 12)).astype(np.float32)
    T = rng.normal(size=(n, 11)).astype(np.float32)
    g = torch.zeros(mlp.NPARAM, dtype=torch.float32, device="cuda:0")
    Xd, Td = torch.from_numpy(X).to("cuda:0"), torch.from_numpy(T).to("cuda:0")  # kept alive across the call
    loss = gz.ctx.surrogate_gradients(Xd.data_ptr(), Td.data_ptr(), n, g.data_ptr())
    g = g.cpu().numpy().astype(np.float64)
    wf = gz.ctx.surrogate_get_params()[0].astype(np.float64)
    lb, gb = mlp.loss_and_grad(wf, X.astype(np.float64), T.astype(np.float64), bf16_round=True)
    l64, g64 = mlp.loss_and_grad(wf, X.astype(np.float64), T.astype(np.float64))
    assert loss == pytest.approx(l64, rel=1e-2)
    for b in range(4):
        sl = slice(mlp.OFF[b], mlp.OFF[b] + mlp.SHAPES[b][0] * mlp.SHAPES[b][1])
        nb = np.linalg.norm(g64[sl])
        assert np.linalg.norm(g[sl] - gb[sl]) / nb <= 1e-2, f"block {b} vs bf16-rounded FP64"
        assert np.linalg.norm(g[sl] - g64[sl]) / nb <= 5e-2, f"block {b} vs FP64"


N_TRAIN, STEPS = 4096, 800


@pytest.fixture(scope="module")
def trained():
    """A network trained on 800 plain steps (80 microseconds: induction,
    ignition and burnout) of 1024 seeded reactors."""
    m, gz = _zone(n=N_TRAIN, seed=101, hot=True)
    X, G = sg.record_trajectories(gz.ctx, N_TRAIN, STEPS, 1e-7, gz.torch)
    losses = sg.fit(gz.ctx, X, G, epochs=200, batch=8192, lr0=2e-3, lr1=1e-5, seed=3)
    w, nm = gz.ctx.surrogate_get_params()
    return {"weights": w, "norm": nm, "losses": losses, "X": X[:N_TRAIN].cpu().numpy()}


def test_recorded_features_and_training_loss(trained):
    # first recorded rows are the initial states of the seeded batch
    m = mechanism.load("li2004")
    case = _hot_batch(m, N_TRAIN, 101)
    f = mlp.raw_features(case.bv[5, :N_TRAIN], case.bv[4, :N_TRAIN], case.sv[:9, :N_TRAIN].T, 1e-7)
    assert np.allclose(trained["X"], f, rtol=2e-7, atol=2e-6)
    losses = trained["losses"]
    assert np.all(np.isfinite(losses))
    assert losses[-1] < 0.4 * losses[0]


def test_all_fallback_equals_plain_integrator(trained):
    _, a = _zone(n=700, seed=3)
    _, b = _zone(n=700, seed=3)
    a.ctx.surrogate_set_params(trained["weights"], trained["norm"])
    gate = a.ctx.surrogate_default_gate(dT_max=-1.0, judge_stride=0)
    for s in range(3):
        st = a.ctx.surrogate_reaction_step(1e-7, gate, s, want_stats=True)
        b.ctx.wu_reaction_step(1e-7, schedule=1)
        assert st["cells"] == 700 and st["surrogate"] == 0
    a.ctx.sync()
    b.ctx.sync()
    for k in ("cv", "bv", "sv", "reaction_timeScale"):
        assert np.array_equal(a.get(k), b.get(k)), k


def test_judged_nodes_take_the_plain_result(trained):
    _, a = _zone(n=600, seed=4)
    _, b = _zone(n=600, seed=4)
    a.ctx.surrogate_set_params(trained["weights"], trained["norm"])
    gate = a.ctx.surrogate_default_gate(ood_margin=1e30, dT_max=1e30, dT_consistency=1e30, judge_stride=1,
                                        judge_tol_T=1e30, judge_tol_bc=1e30, min_substeps=0.0)
    st = a.ctx.surrogate_reaction_step(1e-7, gate, 0, want_stats=True)
    b.ctx.wu_reaction_step(1e-7, schedule=1)
    assert st["judged"] + st["fallback_newton"] == 600 and st["surrogate"] == 0
    assert st["judge_failed"] == 0 and st["judge_max_dT"] >= 0
    for k in ("cv", "bv", "sv"):
        assert np.array_equal(a.get(k), b.get(k)), k


def test_surrogate_nodes_conserve_elements_mass_and_energy(trained):
    m, gz = _zone(n=1500, seed=5)
    gz.ctx.surrogate_set_params(trained["weights"], trained["norm"])
    mu = m.element_mass_fractions()
    cv0, sv0 = gz.get("cv"), gz.get("sv")
    gate = gz.ctx.surrogate_default_gate(ood_margin=1e30, dT_max=1e30, dT_consistency=1e30, judge_stride=0,
                                         min_substeps=0.0)
    st = gz.ctx.surrogate_reaction_step(1e-7, gate, 0, want_stats=True)
    assert st["surrogate"] > 0.9 * 1500
    cv1, sv1, bv1 = gz.get("cv"), gz.get("sv"), gz.get("bv")
    assert np.array_equal(cv1[0], cv0[0]) and np.array_equal(cv1[4], cv0[4])  # density, total energy
    assert np.abs(sv1[:9].sum(axis=0) - 1.0).max() <= 1e-14
    Z0, Z1 = mu @ sv0[:9], mu @ sv1[:9]
    assert np.abs(Z1 - Z0).max() <= 1e-10
    assert np.allclose(cv1[5:14], cv1[0] * sv1[:9], rtol=1e-14, atol=0)
    R = 8314.462618 * (sv1[:9] / m.mw[:, None]).sum(axis=0)
    assert np.allclose(bv1[4], bv1[0] * R * bv1[5], rtol=1e-12)


def _trajectories(gz, steps, dt, fn):
    """Temperature after each step (device copies), and the stats returned."""
    torch = gz.torch
    T = torch.empty((steps, gz.case.N), dtype=torch.float64, device="cuda:0")
    stats = []
    for s in range(steps):
        st = fn(s)
        if st:
            stats.append(st)
        T[s].copy_(gz.t["bv"][5])
    return T.cpu().numpy(), stats


def test_trained_surrogate_accuracy_against_plain(trained):
    """Unseen reactors, 600 steps of 1e-7 s from the unburnt state: the gated
    surrogate step (default gate, judge every 64th node) against the plain
    FP64 work-queue step.  Induction and ignition stay on the plain
    integrator (cost and dT gates); the network takes burnt nodes.  Bar:
    ignition delay (time of max dT/dt) and peak temperature within 1 %."""
    n, steps, dt = 1024, 600, 1e-7
    _, a = _zone(n=n, seed=202, hot=True)
    _, b = _zone(n=n, seed=202, hot=True)
    a.ctx.surrogate_set_params(trained["weights"], trained["norm"])
    gate = a.ctx.surrogate_default_gate()
    T0 = a.get("bv")[5].copy()
    Ta, stats = _trajectories(a, steps, dt, lambda s: a.ctx.surrogate_reaction_step(dt, gate, s,
                                                                                      want_stats=(s % 50 == 49)))
    Tb, _ = _trajectories(b, steps, dt, lambda s: b.ctx.wu_reaction_step(dt, schedule=1))
    tau_a, pk_a, _ = sg.ignition_metrics(dt, T0, Ta)
    tau_b, pk_b, rise_b = sg.ignition_metrics(dt, T0, Tb)
    ign = (rise_b > 20.0) & (tau_b < (steps - 50) * dt)
    e_tau = (np.abs(tau_a[ign] - tau_b[ign]) / tau_b[ign]).max()
    e_pk = (np.abs(pk_a - pk_b) / pk_b).max()
    on_net = sum(st["surrogate"] for st in stats) / sum(st["cells"] for st in stats)
    print(f"ignited {ign.mean():.2f}, on network {on_net:.3f}, tau_ign err {e_tau:.2e}, T_peak err {e_pk:.2e}, "
          f"max |dT| {np.abs(Ta - Tb).max():.1f} K")
    assert ign.mean() > 0.5
    assert e_tau <= 1e-2
    assert e_pk <= 1e-2
    assert on_net >= 0.5


def test_trained_surrogate_throughput_on_burnt_mix(trained):
    """131072 unseen reactors advanced 400 steps by the surrogate path to a
    mostly burnt state; from that same state, 3 plain work-queue steps
    against 3 gated surrogate steps (judge on).  The network replaces the
    burnt nodes' hundreds of point-implicit substeps.  The surrogate step
    still integrates the judged and reverted burnt nodes with the plain
    integrator, whose serial substep chain (~1800 substeps) bounds the step
    time from below whatever the node count, while the plain step grows with
    the node count: at this size the bar is 1.7x (measured 1.9x; the benchmark measures
    2^20 nodes)."""
    torch = pytest.importorskip("torch")
    n, dt = 131072, 1e-7
    _, gz = _zone(n=n, seed=303, hot=True)
    gz.ctx.surrogate_set_params(trained["weights"], trained["norm"])
    adv = gz.ctx.surrogate_default_gate(judge_stride=0)
    for s in range(400):
        gz.ctx.surrogate_reaction_step(dt, adv, s)
    gz.ctx.sync()
    keys = ("cv", "bv", "sv", "reaction_timeScale")
    saved = {k: gz.t[k].clone() for k in keys}
    gate = gz.ctx.surrogate_default_gate()
    ms = {}
    for mode in ("plain", "surrogate"):
        for k in keys:
            gz.t[k].copy_(saved[k])
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for s in range(3):
            if mode == "plain":
                gz.ctx.wu_reaction_step(dt, schedule=1)
            else:
                gz.ctx.surrogate_reaction_step(dt, gate, 400 + s)
        e1.record()
        torch.cuda.synchronize()
        ms[mode] = e0.elapsed_time(e1)
    print(f"plain {ms['plain']:.1f} ms, surrogate {ms['surrogate']:.1f} ms, "
          f"speed-up {ms['plain'] / ms['surrogate']:.2f}x")
    assert ms["plain"] / ms["surrogate"] >= 1.7
