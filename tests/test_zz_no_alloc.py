"""The allocation-free local time step (cfk_local_time_step_static).

Some callers cannot allocate device memory (a memory policy that forbids
allocation after start-up, a framework that owns all device memory, a
time-critical loop in which a cudaMalloc would synchronise the device).  This entry point gives them the CFL step without a
context: its scratch is a file-scope device array.  The tests call it through
the C ABI twice in a row — on two different zones, so that scratch left over
from the first call cannot leak into the second — and check both results
against the context entry point and against the CPU oracle's local and global
time step, with the tolerance of the other time-step tests (1e-14 relative).
The device buffers here belong to the caller (torch); the entry point itself
allocates nothing, which the free-memory check after its first call on the
device shows.
"""
import ctypes

import numpy as np
import pytest

import cases
import corefl_b200 as cfk
import pyoracle
from gpuzone import GpuZone

pytestmark = pytest.mark.gpu


def _zone_struct(gz):
    c = gz.case
    z = cfk.cfk_zone(c.mx, c.my, c.mz, c.ngg)
    for k, v in gz.t.items():
        setattr(z, k, v.data_ptr())
    return z


def _static_dt(gz, dt_dev):
    err = ctypes.create_string_buffer(256)
    z = _zone_struct(gz)
    rc = cfk.lib().cfk_local_time_step_static(ctypes.byref(gz.ctx.cparam), ctypes.byref(z),
                                              ctypes.c_void_p(dt_dev.data_ptr()), None, err, 256)
    assert rc == 0, err.value.decode()
    gz.torch.cuda.synchronize()
    return float(dt_dev.item())


def test_static_local_time_step_matches_context_entry_point_twice():
    import torch

    big = GpuZone(cases.perturbed(cases.sine_wave(n=33, scheme=72, viscous=True), seed=11))
    small = GpuZone(cases.perturbed(cases.sod(64, 7, scheme=52), seed=12))
    dt_dev = torch.zeros(1, dtype=torch.float64, device="cuda:0")
    for gz in (big, small):  # two calls in a row, the second on a smaller zone
        gz.initialize()
        dt_ref = gz.ctx.local_time_step()
        dt_local_ref = gz.get("dt_local").copy()
        gz.t["dt_local"].zero_()
        dt = _static_dt(gz, dt_dev)
        assert dt == pytest.approx(dt_ref, rel=1e-14)
        assert np.allclose(gz.get("dt_local"), dt_local_ref, rtol=1e-14, atol=0)


def test_static_local_time_step_matches_oracle_twice_and_allocates_nothing():
    """Both calls against the oracle's orc_local_time_step/orc_global_time_step
    from the same state; device free memory is unchanged by calls after the
    first (which may load the library's module and look up the scratch
    address), and the caller's current device is the same afterwards."""
    import torch

    dt_dev = torch.zeros(1, dtype=torch.float64, device="cuda:0")
    zones = []
    for case in (cases.perturbed(cases.sine_wave(n=29, scheme=72, viscous=True), seed=13),
                 cases.perturbed(cases.sod(96, 7, scheme=52), seed=14)):
        oz = pyoracle.OracleZone(case)
        oz.initialize()
        gz = GpuZone(case)
        gz.load_from(oz, keys=("cv", "bv", "mul"))
        oz.call("orc_local_time_step")
        dt_o = oz.L.orc_global_time_step(ctypes.byref(oz.z))
        zones.append((gz, oz, dt_o))
    _static_dt(zones[0][0], dt_dev)  # first call on this device: module load and address lookup
    torch.cuda.synchronize()
    dev_before = torch.cuda.current_device()
    free_before = torch.cuda.mem_get_info()[0]
    for gz, oz, dt_o in zones:
        gz.t["dt_local"].zero_()
        dt = _static_dt(gz, dt_dev)
        assert dt == pytest.approx(dt_o, rel=1e-14)
        assert np.allclose(gz.get("dt_local"), oz["dt_local"], rtol=1e-14, atol=0)
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free_before
    assert torch.cuda.current_device() == dev_before


def test_static_local_time_step_rejects_oversized_zone():
    """More first-pass CTAs than scratch slots: a clear error, nothing launched."""
    import torch

    case = cases.sod(64, 7, scheme=52)
    p = cfk.make_param(case.param, case.faces)
    z = cfk.cfk_zone(1024, 1024, 1024, 3)  # 4 * 1024 * 1024 row segments > 262144
    dt_dev = torch.zeros(1, dtype=torch.float64, device="cuda:0")
    err = ctypes.create_string_buffer(256)
    rc = cfk.lib().cfk_local_time_step_static(ctypes.byref(p), ctypes.byref(z), ctypes.c_void_p(dt_dev.data_ptr()),
                                              None, err, 256)
    assert rc == -1
    assert b"too large" in err.value
