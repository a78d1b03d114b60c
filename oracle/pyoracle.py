"""ctypes binding of the CPU oracle (oracle/liboracle.so).

TEST INFRASTRUCTURE ONLY: the tests, the smoke check and the benchmark's CPU
baseline use it as the checker.  The product (corefl-cpc_b200/) never
imports it.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "liboracle.so")

_DP = ctypes.POINTER(ctypes.c_double)


class orc_face(ctypes.Structure):
    _fields_ = [("face", ctypes.c_int), ("direction", ctypes.c_int), ("label", ctypes.c_int)]


class orc_zone(ctypes.Structure):
    _fields_ = [("mx", ctypes.c_int), ("my", ctypes.c_int), ("mz", ctypes.c_int), ("ngg", ctypes.c_int)] + [
        (n, _DP) for n in ("cv", "bv", "sv", "qn", "metric", "jac", "mul", "mach", "fFlux", "gFlux", "hFlux",
                           "acoustic_speed", "gamma", "thermal_conductivity", "rho_D", "reaction_timeScale", "dq",
                           "dt_local", "Cn", "vis_flux", "shock_sensor")
    ] + [("dt_step", ctypes.c_double), ("y", _DP), ("inflow_draws", ctypes.c_ulonglong)]


class orc_param(ctypes.Structure):
    _fields_ = [
        ("dim", ctypes.c_int), ("n_var", ctypes.c_int), ("n_spec", ctypes.c_int), ("n_scalar", ctypes.c_int),
        ("n_reac", ctypes.c_int), ("inviscid_scheme", ctypes.c_int), ("reconstruction", ctypes.c_int),
        ("limiter", ctypes.c_int), ("viscous_order", ctypes.c_int), ("positive_preserving", ctypes.c_int),
        ("gradPInDiffusionFlux", ctypes.c_int), ("entropy_fix_factor", ctypes.c_double), ("Pr", ctypes.c_double),
        ("Sc", ctypes.c_double), ("cfl", ctypes.c_double), ("dt", ctypes.c_double), ("fixed_dt", ctypes.c_int),
        ("weno_eps_scale", ctypes.c_double), ("v_ref", ctypes.c_double), ("rho_ref", ctypes.c_double),
        ("sensor_threshold", ctypes.c_double), ("chem_advance_method", ctypes.c_int), ("n_face", ctypes.c_int),
        ("faces", orc_face * 6), ("mech", ctypes.c_void_p), ("shock_sensor", ctypes.c_int),
        ("sensor_eps", ctypes.c_double), ("wall_thermal_type", ctypes.c_int), ("wall_catalytic_type", ctypes.c_int),
        ("wall_temperature", ctypes.c_double), ("wall_yk", ctypes.c_double * 20),
        ("inflow_subsonic", ctypes.c_int), ("inflow_density", ctypes.c_double), ("inflow_u", ctypes.c_double),
        ("inflow_v", ctypes.c_double), ("inflow_w", ctypes.c_double), ("inflow_pressure", ctypes.c_double),
        ("inflow_temperature", ctypes.c_double), ("inflow_mw", ctypes.c_double), ("inflow_sv", ctypes.c_double * 20),
        ("inflow_type", ctypes.c_int), ("inflow_density_lower", ctypes.c_double), ("inflow_u_lower", ctypes.c_double),
        ("inflow_v_lower", ctypes.c_double), ("inflow_w_lower", ctypes.c_double), ("inflow_p_lower", ctypes.c_double),
        ("inflow_t_lower", ctypes.c_double), ("inflow_sv_lower", ctypes.c_double * 20),
        ("inflow_delta_omega", ctypes.c_double), ("inflow_fluctuation_type", ctypes.c_int),
        ("inflow_fluctuation_intensity", ctypes.c_double), ("inflow_seed", ctypes.c_ulonglong),
        ("outflow_back_pressure_on", ctypes.c_int), ("outflow_back_pressure", ctypes.c_double),
        ("limit_flow", ctypes.c_int), ("limit_ll", ctypes.c_double * 5), ("limit_ul", ctypes.c_double * 5),
    ]


MAXS, MAXR = 20, 64


class orc_mech(ctypes.Structure):
    _fields_ = [
        ("n_spec", ctypes.c_int), ("n_reac", ctypes.c_int),
        ("mw", ctypes.c_double * MAXS), ("imw", ctypes.c_double * MAXS), ("gas_const", ctypes.c_double * MAXS),
        ("t_low", ctypes.c_double * MAXS), ("t_mid", ctypes.c_double * MAXS), ("t_high", ctypes.c_double * MAXS),
        ("low_coeff", (ctypes.c_double * 7) * MAXS), ("high_coeff", (ctypes.c_double * 7) * MAXS),
        ("geometry", ctypes.c_double * MAXS), ("LJ_potent_inv", ctypes.c_double * MAXS),
        ("vis_coeff", ctypes.c_double * MAXS),
        ("WjDivWi_to_One4th", (ctypes.c_double * MAXS) * MAXS),
        ("sqrt_WiDivWjPl1Mul8", (ctypes.c_double * MAXS) * MAXS),
        ("binary_diffusivity_coeff", (ctypes.c_double * MAXS) * MAXS),
        ("kb_over_eps_jk", (ctypes.c_double * MAXS) * MAXS),
        ("ZRotF298", ctypes.c_double * MAXS),
        ("reac_type", ctypes.c_int * MAXR), ("rev_type", ctypes.c_int * MAXR),
        ("stoi_f", (ctypes.c_int * MAXS) * MAXR), ("stoi_b", (ctypes.c_int * MAXS) * MAXR),
        ("reac_order", ctypes.c_int * MAXR),
        ("A", ctypes.c_double * MAXR), ("b", ctypes.c_double * MAXR), ("Ea", ctypes.c_double * MAXR),
        ("A2", ctypes.c_double * MAXR), ("b2", ctypes.c_double * MAXR), ("Ea2", ctypes.c_double * MAXR),
        ("third_body_coeff", (ctypes.c_double * MAXS) * MAXR),
        ("troe_alpha", ctypes.c_double * MAXR), ("troe_t3", ctypes.c_double * MAXR),
        ("troe_t1", ctypes.c_double * MAXR), ("troe_t2", ctypes.c_double * MAXR),
    ]


def make_mech(m) -> orc_mech:
    """orc_mech tables from a mechanism.Mechanism (gas constants R_u/W as the
    reference's DParameter builds them, src/DParameter.cu:72-83)."""
    R_U = 8314.462618
    o = orc_mech()
    ns, nr = m.n_spec, m.n_reac
    o.n_spec, o.n_reac = ns, nr

    def fill1(name, vals):
        arr = getattr(o, name)
        for i, v in enumerate(vals):
            arr[i] = v

    def fill2(name, vals):
        arr = getattr(o, name)
        for i in range(vals.shape[0]):
            for j in range(vals.shape[1]):
                arr[i][j] = vals[i, j]

    fill1("mw", m.mw)
    fill1("imw", [1.0 / w for w in m.mw])
    fill1("gas_const", [R_U / w for w in m.mw])
    for k in ("t_low", "t_mid", "t_high", "geometry", "LJ_potent_inv", "vis_coeff", "ZRotF298"):
        fill1(k, getattr(m, k))
    fill2("low_coeff", m.low)
    fill2("high_coeff", m.high)
    for k in ("WjDivWi_to_One4th", "sqrt_WiDivWjPl1Mul8", "binary_diffusivity_coeff", "kb_over_eps_jk"):
        fill2(k, getattr(m, k))
    fill1("reac_type", m.reac_type)
    fill1("rev_type", m.rev_type)
    fill1("reac_order", m.order)
    fill2("stoi_f", m.stoi_f)
    fill2("stoi_b", m.stoi_b)
    for k in ("A", "b", "Ea", "A2", "b2", "Ea2", "troe_alpha", "troe_t3", "troe_t1", "troe_t2"):
        fill1(k, getattr(m, k))
    fill2("third_body_coeff", m.third_body_coeff)
    return o


_lib = None


_I3 = ctypes.c_int * 3


class orc_inner_face(ctypes.Structure):
    _fields_ = [("range_start", _I3), ("range_end", _I3), ("face", ctypes.c_int), ("direction", ctypes.c_int),
                ("target_start", _I3), ("target_end", _I3), ("target_block", ctypes.c_int),
                ("target_face", ctypes.c_int), ("target_direction", ctypes.c_int), ("src_tar", _I3),
                ("loop_dir", _I3), ("target_loop_dir", _I3), ("n_point", _I3)]


def register_inner_face(dim, ngg, src, tar, target_block) -> orc_inner_face:
    """InnerFace registration from the two records of an inner-interface file
    (1-based, sign-coded {x1, x2, y1, y2, z1, z2}; target_block 1-based)."""
    f = orc_inner_face()
    rc = lib().orc_register_inner_face(dim, ngg, (ctypes.c_int * 6)(*src), (ctypes.c_int * 6)(*tar), target_block,
                                       ctypes.byref(f))
    if rc != 0:
        raise ValueError(f"cannot register inner face {src} -> {tar}")
    return f


def use_native_build() -> bool:
    """Switch this process to the oracle built with -march=native for the
    host it runs on (the timed CPU baseline); must precede the first lib().
    Returns False, keeping the portable build, when the compiler fails."""
    global LIB_PATH
    if _lib is not None:
        raise RuntimeError("the oracle library is already loaded")
    r = subprocess.run(["make", "-C", _HERE, "native"], capture_output=True)
    if r.returncode != 0:
        return False
    LIB_PATH = os.path.join(_HERE, "_native", "liboracle.so")
    return True


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            subprocess.run(["make", "-C", _HERE], check=True, capture_output=True)
        L = ctypes.CDLL(LIB_PATH)
        zp, pp = ctypes.POINTER(orc_zone), ctypes.POINTER(orc_param)
        for name in ("orc_compute_cv_from_bv", "orc_update_physical_properties", "orc_local_time_step",
                     "orc_compute_inviscid_flux", "orc_compute_viscous_flux", "orc_apply_boundary_conditions",
                     "orc_eliminate_k_gradient", "orc_compute_shock_sensor"):
            getattr(L, name).argtypes = [zp, pp]
            getattr(L, name).restype = None
        L.orc_update_cv_and_bv_rk.argtypes = [zp, pp, ctypes.c_double, ctypes.c_int]
        L.orc_update_cv_and_bv_rk.restype = None
        L.orc_rk3_step.argtypes = [zp, pp, ctypes.c_double]
        L.orc_rk3_step.restype = ctypes.c_double
        L.orc_wu_splitting_step.argtypes = [zp, pp, ctypes.c_double]
        L.orc_wu_splitting_step.restype = ctypes.c_double
        L.orc_update_cv_and_bv_rk_wu.argtypes = [zp, pp, ctypes.c_double, ctypes.c_int]
        L.orc_update_cv_and_bv_rk_wu.restype = None
        L.orc_local_time_step_without_reaction.argtypes = [zp, pp]
        L.orc_local_time_step_without_reaction.restype = None
        L.orc_global_time_step.argtypes = [zp]
        L.orc_global_time_step.restype = ctypes.c_double
        L.orc_weno5.argtypes = [_DP, _DP, ctypes.c_double, ctypes.c_int]
        L.orc_weno5.restype = ctypes.c_double
        L.orc_weno7.argtypes = [_DP, _DP, ctypes.c_double, ctypes.c_int]
        L.orc_weno7.restype = ctypes.c_double
        L.orc_sutherland.argtypes = [ctypes.c_double]
        L.orc_sutherland.restype = ctypes.c_double
        L.orc_num_threads.restype = ctypes.c_int
        L.orc_wu_reaction_step.argtypes = [zp, pp, ctypes.c_double, ctypes.c_void_p]
        L.orc_wu_reaction_step.restype = None
        L.orc_finite_rate_chemistry.argtypes = [zp, pp]
        L.orc_finite_rate_chemistry.restype = None
        L.orc_register_inner_face.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                                              ctypes.c_int, ctypes.POINTER(orc_inner_face)]
        L.orc_register_inner_face.restype = ctypes.c_int
        L.orc_inner_communication.argtypes = [zp, zp, pp, ctypes.POINTER(orc_inner_face)]
        L.orc_inner_communication.restype = None
        L.orc_limit_flow.argtypes = [zp, pp, ctypes.c_void_p, ctypes.c_void_p]
        L.orc_limit_flow.restype = ctypes.c_int
        L.orc_halo_size.argtypes = [zp, pp, ctypes.c_int]
        L.orc_halo_size.restype = ctypes.c_long
        L.orc_halo_pack.argtypes = [zp, pp, ctypes.c_int, ctypes.c_int, ctypes.c_void_p]
        L.orc_halo_pack.restype = None
        L.orc_halo_assign.argtypes = [zp, pp, ctypes.c_int, ctypes.c_int, ctypes.c_void_p]
        L.orc_halo_assign.restype = None
        L.orc_noise_uniform.argtypes = [ctypes.c_ulonglong] * 4
        L.orc_noise_uniform.restype = ctypes.c_double
        _lib = L
    return _lib


def _ptr(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_DP)


class OracleZone:
    """Host arrays of one block in the reference layout, owned by numpy."""

    def __init__(self, case):
        c = case
        g = c.ngg
        nv = c.param["n_var"]
        ns = max(c.param["n_spec"], 1)
        nsc = max(c.param["n_scalar"], 1)
        P, N = c.P, c.N
        P1 = (c.mx + 2) * (c.my + 2) * (c.mz + 2)
        self.case = c
        self.arrays = {
            "cv": np.zeros((nv, P)), "bv": c.bv.copy(), "sv": np.zeros((nsc, P)), "qn": np.zeros((nv, P)),
            "metric": np.ascontiguousarray(c.metric), "jac": np.ascontiguousarray(c.jac), "mul": np.zeros(P),
            "mach": np.zeros(P), "fFlux": np.zeros((nv, P)), "gFlux": np.zeros((nv, P)), "hFlux": np.zeros((nv, P)),
            "acoustic_speed": np.zeros(P), "gamma": np.zeros(P), "thermal_conductivity": np.zeros(P),
            "rho_D": np.zeros((ns, P)), "reaction_timeScale": np.zeros(P), "dq": np.zeros((nv, N)),
            "dt_local": np.zeros(N), "Cn": np.zeros((nv, N)), "vis_flux": np.zeros((nv - 1, P1)),
            "shock_sensor": np.zeros(P),
        }
        if c.sv.shape[0]:
            self.arrays["sv"][: c.sv.shape[0]] = c.sv
        if getattr(c, "y", None) is not None:
            self.arrays["y"] = np.ascontiguousarray(c.y, dtype=np.float64)
        self.z = orc_zone(c.mx, c.my, c.mz, g)
        for k, a in self.arrays.items():
            setattr(self.z, k, _ptr(a))
        self.p = orc_param()
        for k, v in c.param.items():
            if k in ("wall_yk", "inflow_sv", "inflow_sv_lower", "limit_ll", "limit_ul"):
                arr = getattr(self.p, k)
                for l, y in enumerate(v):
                    arr[l] = y
            elif k in dict(orc_param._fields_):
                setattr(self.p, k, v)
        self.p.n_face = len(c.faces)
        for n, (f, d, lab) in enumerate(c.faces):
            self.p.faces[n] = orc_face(f, d, lab)
        self.mech = make_mech(c.mech) if getattr(c, "mech", None) is not None else None
        self.p.mech = ctypes.cast(ctypes.pointer(self.mech), ctypes.c_void_p) if self.mech is not None else None
        self.L = lib()

    def __getitem__(self, k):
        return self.arrays[k]

    def initialize(self):
        """Start of a run: properties, BCs (+ 2-D k-ghost copy), properties
        (reference src/Driver.cu:126-211), then cv from bv over the padded
        block (reference src/RK.cuh:37-46)."""
        zr, pr = ctypes.byref(self.z), ctypes.byref(self.p)
        self.L.orc_update_physical_properties(zr, pr)
        self.L.orc_apply_boundary_conditions(zr, pr)
        if self.case.mz == 1:
            self.L.orc_eliminate_k_gradient(zr, pr)
        self.L.orc_update_physical_properties(zr, pr)
        self.L.orc_compute_cv_from_bv(zr, pr)

    def step(self) -> float:
        return self.L.orc_rk3_step(ctypes.byref(self.z), ctypes.byref(self.p), self.p.dt)

    def wu_splitting_step(self) -> float:
        return self.L.orc_wu_splitting_step(ctypes.byref(self.z), ctypes.byref(self.p), self.p.dt)

    def reaction_step(self, dt: float, want_nsub: bool = False):
        """Wu-splitting reaction step over the zone (point implicit when
        chem_advance_method == 1); optionally returns the substeps per node."""
        ns = np.zeros(self.case.N, dtype=np.int32) if want_nsub else None
        self.L.orc_wu_reaction_step(ctypes.byref(self.z), ctypes.byref(self.p), dt,
                                    ns.ctypes.data if want_nsub else None)
        return ns

    def inner_communication(self, target: "OracleZone", face: orc_inner_face):
        self.L.orc_inner_communication(ctypes.byref(self.z), ctypes.byref(target.z), ctypes.byref(self.p),
                                       ctypes.byref(face))

    def limit_flow(self, ll, ul) -> int:
        """orc_limit_flow with the limits ll, ul of (rho, u, v, w, p)."""
        lo = np.ascontiguousarray(ll, dtype=np.float64)
        hi = np.ascontiguousarray(ul, dtype=np.float64)
        return self.L.orc_limit_flow(ctypes.byref(self.z), ctypes.byref(self.p), lo.ctypes.data, hi.ctypes.data)

    def halo_pack(self, face, direction) -> np.ndarray:
        """orc_halo_pack: the face's packed halo (float64 numpy array)."""
        buf = np.empty(self.L.orc_halo_size(ctypes.byref(self.z), ctypes.byref(self.p), face))
        self.L.orc_halo_pack(ctypes.byref(self.z), ctypes.byref(self.p), face, direction, buf.ctypes.data)
        return buf

    def halo_assign(self, face, direction, buf: np.ndarray):
        buf = np.ascontiguousarray(buf, dtype=np.float64)
        self.L.orc_halo_assign(ctypes.byref(self.z), ctypes.byref(self.p), face, direction, buf.ctypes.data)

    def call(self, name, *args):
        return getattr(self.L, name)(ctypes.byref(self.z), ctypes.byref(self.p), *args)
