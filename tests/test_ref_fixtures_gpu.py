"""The CUDA library against the reference's own recorded runs (see
test_ref_fixtures_cpu.py for the runs and the bar): every step of each run
replayed from the same inputs through the C ABI."""
import pytest

import reffix

pytestmark = pytest.mark.gpu

TOL = 1e-12


@pytest.mark.parametrize("name", reffix.names())
def test_library_replays_reference_run(name):
    reports = reffix.replay(reffix.GpuReplay(name))
    for r in reports:
        print(f"{name} step {r.step}: dt {r.dt_rel:.2e}, cv normwise {r.cv_norm:.2e}, pointwise {r.cv_point:.2e}",
              r.extra)
    for r in reports:
        assert r.dt_rel <= 1e-13, f"step {r.step}: time step differs by {r.dt_rel:.3e}"
        assert r.cv_norm <= TOL, f"step {r.step}: normwise {r.cv_norm:.3e}"
        assert r.cv_point <= TOL, f"step {r.step}: pointwise {r.cv_point:.3e}"
