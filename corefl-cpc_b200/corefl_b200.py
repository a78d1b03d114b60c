"""ctypes binding of libcorefl_b200.so (the C ABI declared in include/corefl_b200.h).

The library is the product: every compute call goes to its sm_100a kernels.
There is no fallback — if the shared library is missing or no CUDA device is
present, loading or creating a context fails with an exception.
"""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libcorefl_b200.so")


class cfk_face(ctypes.Structure):
    _fields_ = [("face", ctypes.c_int), ("direction", ctypes.c_int), ("label", ctypes.c_int)]


class cfk_wall(ctypes.Structure):
    _fields_ = [("thermal_type", ctypes.c_int), ("catalytic_type", ctypes.c_int), ("temperature", ctypes.c_double),
                ("yk", ctypes.c_double * 9)]


_I3 = ctypes.c_int * 3


class cfk_inner_face(ctypes.Structure):
    _fields_ = [("range_start", _I3), ("range_end", _I3), ("face", ctypes.c_int), ("direction", ctypes.c_int),
                ("target_start", _I3), ("target_end", _I3), ("target_block", ctypes.c_int),
                ("target_face", ctypes.c_int), ("target_direction", ctypes.c_int), ("src_tar", _I3),
                ("loop_dir", _I3), ("target_loop_dir", _I3), ("n_point", _I3)]


class cfk_plt_block(ctypes.Structure):
    _fields_ = [("mx", ctypes.c_int), ("my", ctypes.c_int), ("mz", ctypes.c_int), ("ngg", ctypes.c_int)] + [
        (n, ctypes.c_void_p) for n in ("x", "y", "z", "bv", "sv", "ov")]


class cfk_plt_target(ctypes.Structure):
    _fields_ = [("mx", ctypes.c_int), ("my", ctypes.c_int), ("mz", ctypes.c_int), ("ngg", ctypes.c_int),
                ("bv", ctypes.c_void_p), ("sv", ctypes.c_void_p)]


class cfk_inflow(ctypes.Structure):
    _fields_ = [("subsonic", ctypes.c_int)] + [(n, ctypes.c_double) for n in (
        "density", "u", "v", "w", "pressure", "temperature", "mw")] + [("sv", ctypes.c_double * 9)] + [
        ("inflow_type", ctypes.c_int)] + [(n, ctypes.c_double) for n in (
            "density_lower", "u_lower", "v_lower", "w_lower", "p_lower", "t_lower")] + [
        ("sv_lower", ctypes.c_double * 9), ("delta_omega", ctypes.c_double), ("fluctuation_type", ctypes.c_int),
        ("fluctuation_intensity", ctypes.c_double), ("seed", ctypes.c_ulonglong)]


class cfk_outflow(ctypes.Structure):
    _fields_ = [("back_pressure_on", ctypes.c_int), ("back_pressure", ctypes.c_double)]


class cfk_param(ctypes.Structure):
    _fields_ = [
        ("dim", ctypes.c_int), ("n_var", ctypes.c_int), ("n_spec", ctypes.c_int), ("n_scalar", ctypes.c_int),
        ("n_reac", ctypes.c_int), ("inviscid_scheme", ctypes.c_int), ("reconstruction", ctypes.c_int),
        ("limiter", ctypes.c_int), ("viscous_order", ctypes.c_int), ("positive_preserving", ctypes.c_int),
        ("gradPInDiffusionFlux", ctypes.c_int), ("fixed_dt", ctypes.c_int), ("chem_advance_method", ctypes.c_int),
        ("n_face", ctypes.c_int), ("faces", cfk_face * 6),
        ("entropy_fix_factor", ctypes.c_double), ("Pr", ctypes.c_double), ("Sc", ctypes.c_double),
        ("cfl", ctypes.c_double), ("dt", ctypes.c_double), ("weno_eps_scale", ctypes.c_double),
        ("v_ref", ctypes.c_double), ("rho_ref", ctypes.c_double), ("sensor_threshold", ctypes.c_double),
        ("device", ctypes.c_int), ("shock_sensor", ctypes.c_int), ("sensor_eps", ctypes.c_double),
        ("wall", cfk_wall), ("inflow", cfk_inflow), ("outflow", cfk_outflow),
        ("limit_flow", ctypes.c_int), ("limit_ll", ctypes.c_double * 5), ("limit_ul", ctypes.c_double * 5),
    ]


_DP = ctypes.POINTER(ctypes.c_double)

MAX_SPEC, MAX_REAC = 9, 24
TILE_VARIANTS = 3  # CFK_TILE_VARIANTS


class cfk_mechanism(ctypes.Structure):
    _fields_ = [
        ("n_spec", ctypes.c_int), ("n_reac", ctypes.c_int), ("mw", ctypes.c_double * MAX_SPEC),
        ("t_low", ctypes.c_double * MAX_SPEC), ("t_mid", ctypes.c_double * MAX_SPEC),
        ("t_high", ctypes.c_double * MAX_SPEC), ("low", (ctypes.c_double * 7) * MAX_SPEC),
        ("high", (ctypes.c_double * 7) * MAX_SPEC), ("geometry", ctypes.c_int * MAX_SPEC),
        ("LJ_potent_inv", ctypes.c_double * MAX_SPEC), ("vis_coeff", ctypes.c_double * MAX_SPEC),
        ("ZRotF298", ctypes.c_double * MAX_SPEC),
        ("WjDivWi_to_One4th", (ctypes.c_double * MAX_SPEC) * MAX_SPEC),
        ("sqrt_WiDivWjPl1Mul8", (ctypes.c_double * MAX_SPEC) * MAX_SPEC),
        ("binary_diffusivity_coeff", (ctypes.c_double * MAX_SPEC) * MAX_SPEC),
        ("kb_over_eps_jk", (ctypes.c_double * MAX_SPEC) * MAX_SPEC),
        ("reac_type", ctypes.c_int * MAX_REAC), ("rev_type", ctypes.c_int * MAX_REAC),
        ("order", ctypes.c_int * MAX_REAC),
        ("stoi_f", (ctypes.c_int * MAX_SPEC) * MAX_REAC), ("stoi_b", (ctypes.c_int * MAX_SPEC) * MAX_REAC),
        ("A", ctypes.c_double * MAX_REAC), ("b", ctypes.c_double * MAX_REAC), ("Ea", ctypes.c_double * MAX_REAC),
        ("A2", ctypes.c_double * MAX_REAC), ("b2", ctypes.c_double * MAX_REAC), ("Ea2", ctypes.c_double * MAX_REAC),
        ("third_body_coeff", (ctypes.c_double * MAX_SPEC) * MAX_REAC),
        ("troe_alpha", ctypes.c_double * MAX_REAC), ("troe_t3", ctypes.c_double * MAX_REAC),
        ("troe_t1", ctypes.c_double * MAX_REAC), ("troe_t2", ctypes.c_double * MAX_REAC),
    ]


def make_mechanism(m) -> cfk_mechanism:
    """cfk_mechanism from a mechanism.Mechanism table."""
    o = cfk_mechanism()
    o.n_spec, o.n_reac = m.n_spec, m.n_reac

    def f1(name, vals, src=None):
        arr = getattr(o, name)
        for i, v in enumerate(vals):
            arr[i] = v

    def f2(name, vals):
        arr = getattr(o, name)
        for i in range(vals.shape[0]):
            for j in range(vals.shape[1]):
                arr[i][j] = vals[i, j]

    for k in ("mw", "t_low", "t_mid", "t_high", "LJ_potent_inv", "vis_coeff", "ZRotF298"):
        f1(k, getattr(m, k))
    f1("geometry", [int(v) for v in m.geometry])
    f2("low", m.low)
    f2("high", m.high)
    for k in ("WjDivWi_to_One4th", "sqrt_WiDivWjPl1Mul8", "binary_diffusivity_coeff", "kb_over_eps_jk"):
        f2(k, getattr(m, k))
    f1("reac_type", m.reac_type)
    f1("rev_type", m.rev_type)
    f1("order", m.order)
    f2("stoi_f", m.stoi_f)
    f2("stoi_b", m.stoi_b)
    for k in ("A", "b", "Ea", "A2", "b2", "Ea2", "troe_alpha", "troe_t3", "troe_t1", "troe_t2"):
        f1(k, getattr(m, k))
    f2("third_body_coeff", m.third_body_coeff)
    return o


class cfk_zone(ctypes.Structure):
    _fields_ = [("mx", ctypes.c_int), ("my", ctypes.c_int), ("mz", ctypes.c_int), ("ngg", ctypes.c_int)] + [
        (n, ctypes.c_void_p) for n in ("jac", "metric", "cv", "bv", "sv", "qn", "mul", "mach", "acoustic_speed",
                                       "gamma", "thermal_conductivity", "rho_D", "reaction_timeScale", "dq",
                                       "dt_local", "Cn", "shock_sensor", "y")
    ]


ZONE_FIELDS = [f for f, _ in cfk_zone._fields_[4:]]

_FP = ctypes.POINTER(ctypes.c_float)
SG_NPARAM, SG_NNORM, SG_NIN, SG_NOUT = 41216, 81, 12, 11


class cfk_surrogate_gate(ctypes.Structure):
    _fields_ = [("ood_margin", ctypes.c_double), ("dT_max", ctypes.c_double), ("dT_consistency", ctypes.c_double),
                ("judge_tol_T", ctypes.c_double), ("judge_tol_bc", ctypes.c_double),
                ("min_substeps", ctypes.c_double), ("judge_stride", ctypes.c_int), ("revert_steps", ctypes.c_int)]


class cfk_surrogate_stats(ctypes.Structure):
    _fields_ = [(n, ctypes.c_longlong) for n in ("cells", "surrogate", "fallback_ood", "fallback_ignition",
                                                 "fallback_consistency", "fallback_revert", "fallback_newton",
                                                 "fallback_cheap", "judged", "judge_failed")] + \
               [(n, ctypes.c_double) for n in ("judge_max_dT", "judge_mean_dT", "judge_max_dbc")]

_lib = None


def lib() -> ctypes.CDLL:
    """Load the library once; raise if it is absent (no fallback path exists)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `make -C corefl-cpc_b200` "
                               "(or __graft_entry__.build()); there is no CPU fallback")
        L = ctypes.CDLL(LIB_PATH)
        vp, i, d = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
        sigs = {
            "cfk_create": (i, [ctypes.POINTER(cfk_param), ctypes.POINTER(vp)]),
            "cfk_destroy": (i, [vp]),
            "cfk_last_error": (ctypes.c_char_p, [vp]),
            "cfk_param_from_setup": (i, [ctypes.c_char_p, ctypes.POINTER(cfk_param), ctypes.c_char_p, ctypes.c_size_t]),
            "cfk_bind_zone": (i, [vp, ctypes.POINTER(cfk_zone)]),
            "cfk_alloc_zone": (i, [vp, i, i, i, ctypes.POINTER(cfk_zone)]),
            "cfk_compute_viscous_flux": (i, [vp, vp]),
            "cfk_compute_inviscid_flux": (i, [vp, vp]),
            "cfk_compute_shock_sensor": (i, [vp, vp]),
            "cfk_autotune_tiles": (i, [vp, i, ctypes.POINTER(d), ctypes.POINTER(i), vp]),
            "cfk_set_tile_variants": (i, [vp, ctypes.POINTER(i)]),
            "cfk_viscous_variant": (i, [vp, i, ctypes.POINTER(i), _DP]),
            "cfk_update_cv_and_bv_rk": (i, [vp, d, i, vp]),
            "cfk_update_physical_properties": (i, [vp, vp]),
            "cfk_limit_flow": (i, [vp, ctypes.POINTER(ctypes.c_longlong), vp]),
            "cfk_compute_cv_from_bv": (i, [vp, vp]),
            "cfk_apply_boundary_conditions": (i, [vp, vp]),
            "cfk_eliminate_k_gradient": (i, [vp, vp]),
            "cfk_halo_size": (i, [vp, i, ctypes.POINTER(ctypes.c_longlong)]),
            "cfk_halo_pack": (i, [vp, i, i, vp, vp]),
            "cfk_halo_assign": (i, [vp, i, i, vp, vp]),
            "cfk_write_flowfield": (i, [ctypes.c_char_p, ctypes.POINTER(cfk_plt_block), i, i,
                                        ctypes.POINTER(ctypes.c_char_p), i, i, d, ctypes.c_char_p, ctypes.c_size_t]),
            "cfk_read_flowfield": (i, [ctypes.c_char_p, ctypes.POINTER(cfk_plt_target), i,
                                       ctypes.POINTER(ctypes.c_char_p), i, _DP, ctypes.c_char_p, ctypes.c_size_t]),
            "cfk_register_inner_face": (i, [i, i, vp, vp, i, ctypes.POINTER(cfk_inner_face)]),
            "cfk_inner_communication": (i, [vp, vp, ctypes.POINTER(cfk_inner_face), vp]),
            "cfk_read_inner_interface": (i, [ctypes.c_char_p, i, i, i, ctypes.POINTER(cfk_inner_face), i,
                                             ctypes.POINTER(i), ctypes.c_char_p, ctypes.c_size_t]),
            "cfk_local_time_step": (i, [vp, _DP, vp]),
            "cfk_rk3_step": (i, [vp, _DP, vp]),
            "cfk_rk3_step_graph": (i, [vp, _DP, vp]),
            "cfk_wu_splitting_step": (i, [vp, i, _DP, vp]),
            "cfk_wu_splitting_step_record": (i, [vp, i, vp, vp, _DP, vp]),
            "cfk_wu_splitting_step_surrogate": (i, [vp, ctypes.POINTER(cfk_surrogate_gate), i,
                                                    ctypes.POINTER(cfk_surrogate_stats), _DP, vp]),
            "cfk_memcpy_h2d": (i, [vp, vp, vp, ctypes.c_size_t, vp]),
            "cfk_memcpy_d2h": (i, [vp, vp, vp, ctypes.c_size_t, vp]),
            "cfk_memcpy_d2d": (i, [vp, vp, vp, ctypes.c_size_t, vp]),
            "cfk_stream_sync": (i, [vp, vp]),
            "cfk_host_alloc": (i, [ctypes.c_size_t, ctypes.POINTER(vp)]),
            "cfk_host_free": (i, [vp]),
            "cfk_kernel_launches": (ctypes.c_longlong, [vp]),
            "cfk_set_profiling": (i, [vp, i]),
            "cfk_profile_read": (i, [vp, _DP, ctypes.POINTER(ctypes.c_longlong)]),
            "cfk_measure_fp64_peak": (i, [_DP]),
            "cfk_local_time_step_static": (i, [ctypes.POINTER(cfk_param), ctypes.POINTER(cfk_zone), vp, vp,
                                               ctypes.c_char_p, ctypes.c_size_t]),
            "cfk_set_mechanism": (i, [vp, ctypes.POINTER(cfk_mechanism)]),
            "cfk_finite_rate_chemistry": (i, [vp, vp]),
            "cfk_wu_reaction_step": (i, [vp, d, i, vp, vp]),
            "cfk_surrogate_init": (i, [vp, ctypes.c_ulonglong, i, _DP]),
            "cfk_surrogate_record": (i, [vp, i, d, vp, vp, vp]),
            "cfk_surrogate_fit_normalization": (i, [vp, vp, vp, ctypes.c_longlong]),
            "cfk_surrogate_train": (i, [vp, vp, vp, ctypes.c_longlong, i, i, d, d, ctypes.c_ulonglong, _DP]),
            "cfk_surrogate_gradients": (i, [vp, vp, vp, ctypes.c_longlong, vp, _DP]),
            "cfk_surrogate_forward": (i, [vp, vp, ctypes.c_longlong, vp]),
            "cfk_surrogate_get_params": (i, [vp, _FP, _FP]),
            "cfk_surrogate_set_params": (i, [vp, _FP, _FP]),
            "cfk_surrogate_default_gate": (i, [ctypes.POINTER(cfk_surrogate_gate)]),
            "cfk_surrogate_reaction_step": (i, [vp, d, ctypes.POINTER(cfk_surrogate_gate), i,
                                                ctypes.POINTER(cfk_surrogate_stats), vp]),
        }
        for name, (res, args) in sigs.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def register_inner_face(dim, ngg, src, tar, target_block) -> cfk_inner_face:
    """cfk_register_inner_face: an inner face from the two records of the
    mesh's inner-interface file (1-based, sign-coded ranges)."""
    f = cfk_inner_face()
    rc = lib().cfk_register_inner_face(dim, ngg, (ctypes.c_int * 6)(*src), (ctypes.c_int * 6)(*tar), target_block,
                                       ctypes.byref(f))
    if rc != 0:
        raise CfkError(f"cfk_register_inner_face({src}, {tar}) failed ({rc})")
    return f


def _host_ptr(a):
    import numpy as np

    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"], "float64 C-contiguous host arrays"
    return a.ctypes.data


def write_flowfield(path, blocks, names, ngg_output=0, n_scalar=0, n_other=0, solution_time=0.0):
    """cfk_write_flowfield.  blocks: dicts with mx, my, mz, ngg and host
    float64 arrays x, y, z (padded), bv (6 planes), sv, ov."""
    arr = (cfk_plt_block * len(blocks))()
    for n, b in enumerate(blocks):
        arr[n] = cfk_plt_block(b["mx"], b["my"], b["mz"], b["ngg"],
                               *[_host_ptr(b.get(k)) for k in ("x", "y", "z", "bv", "sv", "ov")])
    cn = (ctypes.c_char_p * len(names))(*[x.encode() for x in names])
    err = ctypes.create_string_buffer(256)
    rc = lib().cfk_write_flowfield(str(path).encode(), arr, len(blocks), ngg_output, cn, n_scalar, n_other,
                                   solution_time, err, 256)
    if rc != 0:
        raise CfkError(f"cfk_write_flowfield: {rc}: {err.value.decode()}")


def read_flowfield(path, targets, species=()):
    """cfk_read_flowfield into host arrays.  targets: dicts with mx, my, mz,
    ngg and float64 arrays bv (6 planes) and sv; returns the solution time."""
    arr = (cfk_plt_target * len(targets))()
    for n, b in enumerate(targets):
        arr[n] = cfk_plt_target(b["mx"], b["my"], b["mz"], b["ngg"], _host_ptr(b.get("bv")), _host_ptr(b.get("sv")))
    sp = (ctypes.c_char_p * max(1, len(species)))(*[x.encode() for x in species])
    t = ctypes.c_double()
    err = ctypes.create_string_buffer(256)
    rc = lib().cfk_read_flowfield(str(path).encode(), arr, len(targets), sp, len(species), ctypes.byref(t), err, 256)
    if rc != 0:
        raise CfkError(f"cfk_read_flowfield: {rc}: {err.value.decode()}")
    return t.value


def read_inner_interface(path, dim, ngg, n_block, max_faces=64):
    """cfk_read_inner_interface: the registered inner faces of every block,
    as a list per block."""
    faces = (cfk_inner_face * max_faces)()
    counts = (ctypes.c_int * n_block)()
    err = ctypes.create_string_buffer(256)
    rc = lib().cfk_read_inner_interface(str(path).encode(), dim, ngg, n_block, faces, max_faces, counts, err, 256)
    if rc != 0:
        raise CfkError(f"cfk_read_inner_interface: {rc}: {err.value.decode()}")
    out, n = [], 0
    for b in range(n_block):
        out.append([faces[n + q] for q in range(counts[b])])
        n += counts[b]
    return out


def make_param(p: dict, faces) -> cfk_param:
    cp = cfk_param()
    for k, v in p.items():
        if k == "wall_yk":
            for l, y in enumerate(v):
                cp.wall.yk[l] = y
        elif k == "inflow_type":
            cp.inflow.inflow_type = v
        elif k in ("inflow_sv", "inflow_sv_lower"):
            arr = getattr(cp.inflow, k[7:])
            for l, y in enumerate(v):
                arr[l] = y
        elif k.startswith("wall_"):
            setattr(cp.wall, k[5:], v)
        elif k.startswith("inflow_"):
            setattr(cp.inflow, k[7:], v)
        elif k.startswith("outflow_"):
            setattr(cp.outflow, k[8:], v)
        elif k in ("limit_ll", "limit_ul"):
            setattr(cp, k, (ctypes.c_double * 5)(*v))
        elif k in dict(cfk_param._fields_):
            setattr(cp, k, v)
    cp.n_face = len(faces)
    for n, (f, dr, lab) in enumerate(faces):
        cp.faces[n] = cfk_face(f, dr, lab)
    return cp


class CfkError(RuntimeError):
    pass


class Context:
    """One solver context: settings, a bound zone, and the per-stage calls."""

    def __init__(self, param: dict, faces):
        self.L = lib()
        self.cparam = make_param(param, faces)
        h = ctypes.c_void_p()
        rc = self.L.cfk_create(ctypes.byref(self.cparam), ctypes.byref(h))
        if rc != 0:
            raise CfkError(f"cfk_create failed with status {rc}")
        self.h = h

    def _ck(self, rc, what):
        if rc != 0:
            raise CfkError(f"{what}: status {rc}: {self.L.cfk_last_error(self.h).decode()}")

    def close(self):
        if self.h:
            self.L.cfk_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def bind(self, mx, my, mz, ngg, ptrs: dict):
        z = cfk_zone(mx, my, mz, ngg)
        for k, v in ptrs.items():
            setattr(z, k, v)
        self._ck(self.L.cfk_bind_zone(self.h, ctypes.byref(z)), "cfk_bind_zone")

    def alloc_zone(self, mx, my, mz) -> cfk_zone:
        z = cfk_zone()
        self._ck(self.L.cfk_alloc_zone(self.h, mx, my, mz, ctypes.byref(z)), "cfk_alloc_zone")
        return z

    def set_mechanism(self, mech):
        self._mech = make_mechanism(mech)
        self._ck(self.L.cfk_set_mechanism(self.h, ctypes.byref(self._mech)), "cfk_set_mechanism")

    def finite_rate_chemistry(self, stream=None):
        self._ck(self.L.cfk_finite_rate_chemistry(self.h, stream), "finite_rate_chemistry")

    def wu_reaction_step(self, dt, schedule=0, nsub_ptr=None, stream=None):
        self._ck(self.L.cfk_wu_reaction_step(self.h, dt, schedule, nsub_ptr, stream), "wu_reaction_step")

    # ---- MLP chemistry surrogate (device pointers are plain ints) --------
    def surrogate_init(self, seed, elem_mu):
        import numpy as np
        mu = np.ascontiguousarray(elem_mu, dtype=np.float64)
        self._ck(self.L.cfk_surrogate_init(self.h, seed, mu.shape[0], mu.ctypes.data_as(_DP)), "surrogate_init")

    def surrogate_record(self, phase, dt, X=None, G=None, stream=None):
        self._ck(self.L.cfk_surrogate_record(self.h, phase, dt, X, G, stream), "surrogate_record")

    def surrogate_fit_normalization(self, X, G, n):
        self._ck(self.L.cfk_surrogate_fit_normalization(self.h, X, G, n), "surrogate_fit_normalization")

    def surrogate_train(self, X, G, n, epochs, batch, lr0, lr1, seed=0):
        losses = (ctypes.c_double * epochs)()
        self._ck(self.L.cfk_surrogate_train(self.h, X, G, n, epochs, batch, lr0, lr1, seed, losses), "surrogate_train")
        return list(losses)

    def surrogate_gradients(self, X, G, n, grad_out) -> float:
        loss = ctypes.c_double()
        self._ck(self.L.cfk_surrogate_gradients(self.h, X, G, n, grad_out, ctypes.byref(loss)), "surrogate_gradients")
        return loss.value

    def surrogate_forward(self, X, n, Y):
        self._ck(self.L.cfk_surrogate_forward(self.h, X, n, Y), "surrogate_forward")

    def surrogate_get_params(self):
        import numpy as np
        w = np.zeros(SG_NPARAM, np.float32)
        nm = np.zeros(SG_NNORM, np.float32)
        self._ck(self.L.cfk_surrogate_get_params(self.h, w.ctypes.data_as(_FP), nm.ctypes.data_as(_FP)),
                 "surrogate_get_params")
        return w, nm

    def surrogate_set_params(self, weights=None, norm=None):
        import numpy as np
        w = None if weights is None else np.ascontiguousarray(weights, dtype=np.float32)
        nm = None if norm is None else np.ascontiguousarray(norm, dtype=np.float32)
        self._ck(self.L.cfk_surrogate_set_params(self.h, None if w is None else w.ctypes.data_as(_FP),
                                                 None if nm is None else nm.ctypes.data_as(_FP)),
                 "surrogate_set_params")

    @staticmethod
    def surrogate_default_gate(**over) -> cfk_surrogate_gate:
        g = cfk_surrogate_gate()
        lib().cfk_surrogate_default_gate(ctypes.byref(g))
        for k, v in over.items():
            setattr(g, k, v)
        return g

    def surrogate_reaction_step(self, dt, gate, step_index=0, want_stats=False, stream=None):
        st = cfk_surrogate_stats() if want_stats else None
        self._ck(self.L.cfk_surrogate_reaction_step(self.h, dt, ctypes.byref(gate), step_index,
                                                    ctypes.byref(st) if st is not None else None, stream),
                 "surrogate_reaction_step")
        if st is None:
            return None
        return {n: getattr(st, n) for n, _ in cfk_surrogate_stats._fields_}

    def viscous(self, stream=None):
        self._ck(self.L.cfk_compute_viscous_flux(self.h, stream), "viscous")

    def inviscid(self, stream=None):
        self._ck(self.L.cfk_compute_inviscid_flux(self.h, stream), "inviscid")

    def shock_sensor(self, stream=None):
        self._ck(self.L.cfk_compute_shock_sensor(self.h, stream), "shock sensor")

    def autotune_tiles(self, reps=5, stream=None):
        """Time each tile variant of every WENO sweep and keep the fastest;
        returns (choice[3], ms[3][TILE_VARIANTS])."""
        ms = (ctypes.c_double * (3 * TILE_VARIANTS))()
        ch = (ctypes.c_int * 3)()
        self._ck(self.L.cfk_autotune_tiles(self.h, reps, ms, ch, stream), "autotune_tiles")
        return list(ch), [list(ms[d * TILE_VARIANTS:(d + 1) * TILE_VARIANTS]) for d in range(3)]

    def viscous_variant(self, set_to=None):
        """The fused air viscous kernel's form (0 staged, 1 ring, 2 ring with
        the L2 prefetch of the metric two planes ahead) and the last
        autotune's per-launch times; set_to selects a form."""
        v = ctypes.c_int(set_to if set_to is not None else 0)
        ms = (ctypes.c_double * 3)()
        self._ck(self.L.cfk_viscous_variant(self.h, 1 if set_to is not None else 0, ctypes.byref(v), ms),
                 "viscous_variant")
        return v.value, list(ms)

    def set_tile_variants(self, var):
        v = (ctypes.c_int * 3)(*var)
        self._ck(self.L.cfk_set_tile_variants(self.h, v), "set_tile_variants")

    def update_rk(self, dt, rk, stream=None):
        self._ck(self.L.cfk_update_cv_and_bv_rk(self.h, dt, rk, stream), "update")

    def limit_flow(self, stream=None) -> int:
        """cfk_limit_flow: repairs the out-of-bounds nodes; returns their number."""
        n = ctypes.c_longlong()
        self._ck(self.L.cfk_limit_flow(self.h, ctypes.byref(n), stream), "limit_flow")
        return n.value

    def properties(self, stream=None):
        self._ck(self.L.cfk_update_physical_properties(self.h, stream), "properties")

    def cv_from_bv(self, stream=None):
        self._ck(self.L.cfk_compute_cv_from_bv(self.h, stream), "cv_from_bv")

    def eliminate_k_gradient(self, stream=None):
        self._ck(self.L.cfk_eliminate_k_gradient(self.h, stream), "eliminate_k_gradient")

    def halo_size(self, face) -> int:
        """cfk_halo_size: doubles in the halo buffer of a block face on axis `face`."""
        n = ctypes.c_longlong()
        self._ck(self.L.cfk_halo_size(self.h, face, ctypes.byref(n)), "halo_size")
        return n.value

    def halo_pack(self, face, direction, buf_ptr, stream=None):
        self._ck(self.L.cfk_halo_pack(self.h, face, direction, buf_ptr, stream), "halo_pack")

    def halo_assign(self, face, direction, buf_ptr, stream=None):
        self._ck(self.L.cfk_halo_assign(self.h, face, direction, buf_ptr, stream), "halo_assign")

    def inner_communication(self, target: "Context", face: cfk_inner_face, stream=None):
        self._ck(self.L.cfk_inner_communication(self.h, target.h, ctypes.byref(face), stream), "inner_communication")

    def boundary_conditions(self, stream=None):
        self._ck(self.L.cfk_apply_boundary_conditions(self.h, stream), "bc")

    def local_time_step(self, stream=None) -> float:
        dt = ctypes.c_double()
        self._ck(self.L.cfk_local_time_step(self.h, ctypes.byref(dt), stream), "local_time_step")
        return dt.value

    def rk3_step(self, stream=None, graph=False, want_dt=True) -> float:
        dt = ctypes.c_double(0.0)
        fn = self.L.cfk_rk3_step_graph if graph else self.L.cfk_rk3_step
        self._ck(fn(self.h, ctypes.byref(dt) if want_dt else None, stream), "rk3_step")
        return dt.value

    def wu_splitting_step(self, schedule=1, stream=None) -> float:
        dt = ctypes.c_double(0.0)
        self._ck(self.L.cfk_wu_splitting_step(self.h, schedule, ctypes.byref(dt), stream), "wu_splitting_step")
        return dt.value

    def wu_splitting_step_record(self, X_ptr, G_ptr, schedule=1, stream=None) -> float:
        """cfk_wu_splitting_step_record: a plain Wu step that also writes one
        training row per node into the device float arrays at X_ptr, G_ptr."""
        dt = ctypes.c_double(0.0)
        self._ck(self.L.cfk_wu_splitting_step_record(self.h, schedule, X_ptr, G_ptr, ctypes.byref(dt), stream),
                 "wu_splitting_step_record")
        return dt.value

    def wu_splitting_step_surrogate(self, gate, step_index=0, want_stats=False, stream=None):
        """cfk_wu_splitting_step_surrogate: returns (dt, stats or None)."""
        dt = ctypes.c_double(0.0)
        st = cfk_surrogate_stats() if want_stats else None
        self._ck(self.L.cfk_wu_splitting_step_surrogate(self.h, ctypes.byref(gate), step_index,
                                                        ctypes.byref(st) if st is not None else None,
                                                        ctypes.byref(dt), stream), "wu_splitting_step_surrogate")
        stats = {n: getattr(st, n) for n, _ in cfk_surrogate_stats._fields_} if st is not None else None
        return dt.value, stats

    def sync(self, stream=None):
        self._ck(self.L.cfk_stream_sync(self.h, stream), "sync")

    def h2d(self, dst, src, nbytes, stream=None):
        self._ck(self.L.cfk_memcpy_h2d(self.h, dst, src, nbytes, stream), "h2d")

    def d2h(self, dst, src, nbytes, stream=None):
        self._ck(self.L.cfk_memcpy_d2h(self.h, dst, src, nbytes, stream), "d2h")

    def d2d(self, dst, src, nbytes, stream=None):
        self._ck(self.L.cfk_memcpy_d2d(self.h, dst, src, nbytes, stream), "d2d")

    @property
    def kernel_launches(self) -> int:
        return int(self.L.cfk_kernel_launches(self.h))

    def set_profiling(self, on: bool):
        self._ck(self.L.cfk_set_profiling(self.h, 1 if on else 0), "set_profiling")

    def profile_read(self) -> dict:
        ms = (ctypes.c_double * NPHASE)()
        kn = (ctypes.c_longlong * NPHASE)()
        self._ck(self.L.cfk_profile_read(self.h, ms, kn), "profile_read")
        return {name: (ms[k], kn[k]) for k, name in enumerate(PHASES)}


PHASES = ("inviscid", "viscous", "update", "bc", "properties", "dt", "reaction")
NPHASE = len(PHASES)


def measure_fp64_peak() -> float:
    t = ctypes.c_double()
    rc = lib().cfk_measure_fp64_peak(ctypes.byref(t))
    if rc != 0:
        raise CfkError(f"cfk_measure_fp64_peak failed with status {rc}")
    return t.value
