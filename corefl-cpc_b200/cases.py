"""Input builders for the workloads of this library (host side, numpy).

Each builder returns a :class:`Case`: ghost-padded node coordinates, the
Jacobian and the nine metric terms in the reference's VectorField3D layout
(reference src/gxl_lib/Array.cuh:246-322), the initial basic variables
(rho, u, v, w, p, T) and the settings of the run.

Grid metrics follow Block::compute_jac_metric (reference
src/Mesh.cpp:244-533): second-order central differences of the coordinates,
J = det(d(x,y,z)/d(xi,eta,zeta)) and grad(xi) etc. from the cofactors, on the
reference's ghost grid (src/Mesh.cpp:1014-1080): face ghosts are point
reflections through the boundary node, with z(k) = z(0) + k for 2-D blocks,
and edge and corner ghosts stay 0, so the metrics of the ghost nodes next to
them are the reference's own.
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

R_U = 8314.462618
MW_AIR = 28.9647
GAMMA_AIR = 1.4
R_AIR = R_U / MW_AIR


@dataclasses.dataclass
class Case:
    name: str
    mx: int
    my: int
    mz: int
    ngg: int
    metric: np.ndarray  # (9, P)
    jac: np.ndarray  # (P,)
    bv: np.ndarray  # (6, P)
    sv: np.ndarray  # (n_scalar, P)
    param: dict
    faces: list  # [(face, direction, label)]
    x: np.ndarray | None = None  # (P,) node x, for checks against exact solutions
    mech: object = None  # mechanism.Mechanism for the mixture model
    xyz: tuple | None = None  # interior node coordinates (x, y, z), each [k, j, i]
    y: np.ndarray | None = None  # (P,) padded node y (DZone::y), for the mixing-layer inflow

    @property
    def P(self) -> int:
        g = self.ngg
        return (self.mx + 2 * g) * (self.my + 2 * g) * (self.mz + 2 * g)

    @property
    def N(self) -> int:
        return self.mx * self.my * self.mz

    def shape(self, g: int | None = None):
        g = self.ngg if g is None else g
        return (self.mz + 2 * g, self.my + 2 * g, self.mx + 2 * g)

    def interior(self, a: np.ndarray) -> np.ndarray:
        """View of the interior nodes of a padded plane, indexed [k, j, i]."""
        g = self.ngg
        return a.reshape(self.shape())[g:g + self.mz, g:g + self.my, g:g + self.mx]


def ghost_grid(x: np.ndarray, y: np.ndarray, z: np.ndarray, ngg: int):
    """Coordinate arrays [k, j, i] with ngg + 1 ghost layers, filled as the
    reference's Mesh::init_ghost_grid does (reference src/Mesh.cpp:1014-1162):
    face ghosts (outside the block across one face) are point reflections
    through the boundary node, x(-q) = 2 x(0) - x(q); for 2-D blocks the
    k-ghosts copy the node with z(k) = z(0) + k; then edges and corners by the
    parallelogram rule in three passes — the (i, j) edges of the k-planes of
    the block, the (i, k) edges of its j-planes, and the (j, k) edges and the
    corners for every i — e.g. x(-i, -j, k) = x(-i, 0, k) + x(0, -j, k) - x(0, 0, k)."""
    e = ngg + 1
    mz, my, mx = x.shape
    two_d = mz == 1
    out = []
    for n, c in enumerate((x, y, z)):
        a = np.zeros((mz + 2 * e, my + 2 * e, mx + 2 * e))
        I, J, K = slice(e, e + mx), slice(e, e + my), slice(e, e + mz)
        a[K, J, I] = c
        for q in range(1, e + 1):
            a[K, J, e - q] = 2 * c[:, :, 0] - c[:, :, q]
            a[K, J, e + mx - 1 + q] = 2 * c[:, :, mx - 1] - c[:, :, mx - 1 - q]
            a[K, e - q, I] = 2 * c[:, 0, :] - c[:, q, :]
            a[K, e + my - 1 + q, I] = 2 * c[:, my - 1, :] - c[:, my - 1 - q, :]
            if two_d:
                a[e - q, J, I] = c[0] + (-q) if n == 2 else c[0]
                a[e + q, J, I] = c[0] + q if n == 2 else c[0]
            else:
                a[e - q, J, I] = 2 * c[0] - c[q]
                a[e + mz - 1 + q, J, I] = 2 * c[mz - 1] - c[mz - 1 - q]
        lo = lambda m, q: e - q  # noqa: E731  index of node -q
        hi = lambda m, q: e + m - 1 + q  # noqa: E731  index of node m - 1 + q
        i0, i1, j0, j1, k0, k1 = e, e + mx - 1, e, e + my - 1, e, e + mz - 1
        # pass 1: (i, j) edges for k in [0, mz)
        for qi in range(1, e + 1):
            for qj in range(1, e + 1):
                for (ii, iref), (jj, jref) in (((lo(mx, qi), i0), (lo(my, qj), j0)),
                                               ((hi(mx, qi), i1), (hi(my, qj), j1)),
                                               ((lo(mx, qi), i0), (hi(my, qj), j1)),
                                               ((hi(mx, qi), i1), (lo(my, qj), j0))):
                    a[K, jj, ii] = a[K, jref, ii] + a[K, jj, iref] - a[K, jref, iref]
        # pass 2: (i, k) edges for j in [0, my)
        for qi in range(1, e + 1):
            for qk in range(1, e + 1):
                for (ii, iref), (kk, kref) in (((lo(mx, qi), i0), (lo(mz, qk), k0)),
                                               ((hi(mx, qi), i1), (hi(mz, qk), k1)),
                                               ((lo(mx, qi), i0), (hi(mz, qk), k1)),
                                               ((hi(mx, qi), i1), (lo(mz, qk), k0))):
                    a[kk, J, ii] = a[kref, J, ii] + a[kk, J, iref] - a[kref, J, iref]
        # pass 3: (j, k) edges and corners for every i
        for qj in range(1, e + 1):
            for qk in range(1, e + 1):
                for (jj, jref), (kk, kref) in (((lo(my, qj), j0), (lo(mz, qk), k0)),
                                               ((hi(my, qj), j1), (hi(mz, qk), k1)),
                                               ((lo(my, qj), j0), (hi(mz, qk), k1)),
                                               ((hi(my, qj), j1), (lo(mz, qk), k0))):
                    a[kk, jj, :] = a[kk, jref, :] + a[kref, jj, :] - a[kref, jref, :]
        out.append(a)
    return out


def _jac_metric_formula(X, Y, Z):
    """J and the nine metric terms at every node of the (n-2)-shaped inner
    part of coordinate arrays [k, j, i], in the reference's arithmetic order
    (reference src/Mesh.cpp:250-298)."""
    def d(a, axis):
        sl_p = [slice(1, -1)] * 3
        sl_m = [slice(1, -1)] * 3
        sl_p[axis] = slice(2, None)
        sl_m[axis] = slice(0, -2)
        return (a[tuple(sl_p)] - a[tuple(sl_m)]) * 0.5

    # derivative w.r.t. (xi, eta, zeta) = array axes (2, 1, 0)
    dxd1, dyd1, dzd1 = d(X, 2), d(Y, 2), d(Z, 2)
    dxd2, dyd2, dzd2 = d(X, 1), d(Y, 1), d(Z, 1)
    dxd3, dyd3, dzd3 = d(X, 0), d(Y, 0), d(Z, 0)
    with np.errstate(divide="ignore", invalid="ignore"):
        jac = (dxd1 * dyd2 * dzd3 + dxd2 * dyd3 * dzd1 + dxd3 * dyd1 * dzd2 - dxd1 * dyd3 * dzd2 -
               dxd2 * dyd1 * dzd3 - dxd3 * dyd2 * dzd1)
        m = np.empty((9,) + jac.shape)
        m[0] = (dyd2 * dzd3 - dyd3 * dzd2) / jac
        m[1] = (dxd3 * dzd2 - dxd2 * dzd3) / jac
        m[2] = (dxd2 * dyd3 - dxd3 * dyd2) / jac
        m[3] = (dyd3 * dzd1 - dyd1 * dzd3) / jac
        m[4] = (dxd1 * dzd3 - dxd3 * dzd1) / jac
        m[5] = (dxd3 * dyd1 - dxd1 * dyd3) / jac
        m[6] = (dyd1 * dzd2 - dyd2 * dzd1) / jac
        m[7] = (dxd2 * dzd1 - dxd1 * dzd2) / jac
        m[8] = (dxd1 * dyd2 - dxd2 * dyd1) / jac
    return jac, m


def metrics(x: np.ndarray, y: np.ndarray, z: np.ndarray, ngg: int):
    """Jacobian and metric on the padded grid from interior node coordinates
    indexed [k, j, i], as the reference's Block::compute_jac_metric leaves
    them (reference src/Mesh.cpp:244-533) on the ghost grid of ghost_grid():
    the central-difference formula at every padded node, then, in the
    reference's sweep order (the k-ghost planes of the face interior outwards
    from k = 0 and from k = mz - 1, the j-ghost planes with edges, the i-ghost
    planes with edges and corners), a node whose Jacobian is not positive
    takes the metric and Jacobian of its neighbour one plane inwards.  A
    non-positive Jacobian inside the block is an error (the reference stops).
    Returns (jac (P,), metric (9, P), xg (P,) the padded x coordinates)."""
    mz, my, mx = x.shape
    two_d = mz == 1
    X, Y, Z = ghost_grid(x, y, z, ngg)
    jac_f, met_f = _jac_metric_formula(X, Y, Z)  # shape (mz + 2 ngg, my + 2 ngg, mx + 2 ngg)
    g = ngg
    jac = np.zeros_like(jac_f)
    met = np.zeros_like(met_f)

    def put(sel_k, sel_j, sel_i):
        jac[sel_k, sel_j, sel_i] = jac_f[sel_k, sel_j, sel_i]
        met[:, sel_k, sel_j, sel_i] = met_f[:, sel_k, sel_j, sel_i]

    def fix(axis, p, q, sel_a, sel_b):
        """Plane p along `axis` over the ranges sel_a, sel_b of the other two
        axes (in k, j, i order); non-positive Jacobians take plane q's values."""
        idx = [None, None, None]
        others = [a for a in (0, 1, 2) if a != axis]
        idx[axis] = p
        idx[others[0]], idx[others[1]] = sel_a, sel_b
        src = list(idx)
        src[axis] = q
        t = tuple(idx)
        put(*t)
        bad = ~(jac[t] > 0)
        if bad.any():
            jac[t] = np.where(bad, jac[tuple(src)], jac[t])
            met[(slice(None),) + t] = np.where(bad[None], met[(slice(None),) + tuple(src)], met[(slice(None),) + t])

    ii = slice(g + 1, g + mx - 1)
    jj = slice(g + 1, g + my - 1)
    # block 0: i in [1, mx-1), j in [1, my-1), k in [1, mz-1) (k = 0 for 2-D)
    kk = slice(g, g + 1) if two_d else slice(g + 1, g + mz - 1)
    put(kk, jj, ii)
    if np.any(~(jac[kk, jj, ii] > 0)):
        raise ValueError("non-positive Jacobian in the generated grid")
    all_k = slice(0, mz + 2 * g)
    all_j = slice(0, my + 2 * g)
    for k in range(0, -g - 1, -1):  # block 1: k = 0 .. -ngg
        fix(0, g + k, g + k + 1, jj, ii)
    for k in range(mz - 1, mz + g):  # block 2: k = mz-1 .. mz+ngg-1
        fix(0, g + k, g + k - 1, jj, ii)
    for j in range(0, -g - 1, -1):  # block 3: j = 0 .. -ngg, all k
        fix(1, g + j, g + j + 1, all_k, ii)
    for j in range(my - 1, my + g):  # block 4
        fix(1, g + j, g + j - 1, all_k, ii)
    for i in range(0, -g - 1, -1):  # block 5: i = 0 .. -ngg, all j, k
        fix(2, g + i, g + i + 1, all_k, all_j)
    for i in range(mx - 1, mx + g):  # block 6
        fix(2, g + i, g + i - 1, all_k, all_j)
    xg = X[1:-1, 1:-1, 1:-1]
    return jac.reshape(-1).copy(), met.reshape(9, -1).copy(), xg.reshape(-1).copy()


def _air_param(**kw) -> dict:
    p = dict(dim=3, n_var=5, n_spec=0, n_scalar=0, n_reac=0, inviscid_scheme=72, reconstruction=2, limiter=0,
             viscous_order=0, positive_preserving=0, gradPInDiffusionFlux=0, fixed_dt=0, chem_advance_method=0,
             entropy_fix_factor=0.125, Pr=0.72, Sc=0.5, cfl=0.5, dt=0.0, weno_eps_scale=1.0, v_ref=1.0, rho_ref=1.0,
             sensor_threshold=0.0, shock_sensor=0, sensor_eps=-1.0)
    p.update(kw)
    return p


def ghost_layers(scheme: int, viscous_order: int = 0) -> int:
    """Ghost layers of an inviscid scheme (reference src/Parameter.cpp:196-252),
    at least 4 with the 8th-order viscous scheme (:296-300) and 2 with the
    4th-order one."""
    g = 2
    if scheme in (71, 72):
        g = 4
    elif scheme in (51, 52):
        g = 3
    return max(g, 4) if viscous_order == 8 else g


def _reference_scale(rho: float, u: float, p: float) -> tuple[float, float]:
    """rho_ref and v_ref of the reference state (reference src/BoundCond.cpp:274-283):
    v_ref = |u|, or the speed of sound when |u| < 1."""
    t = p * MW_AIR / (rho * R_U)
    c = math.sqrt(GAMMA_AIR * R_U / MW_AIR * t)
    v = abs(u) if abs(u) >= 1 else c
    return rho, v


def sod(nx: int = 400, ny: int = 7, scheme: int = 52, cfl: float = 0.5, reconstruction: int = 2,
        viscous_order: int = 0) -> Case:
    """Sod shock tube on x in [0,1] as an nx-by-ny 2-D block (the reference
    runs 1-D problems with 7 nodes in y), outflow on all four faces,
    left (1,0,1) / right (0.125,0,0.1) split at x = 0.5 (the right state is
    applied to x in [0.5, 1.5] inclusive, reference src/Field.cu:290).
    scheme: 52/72 WENO5/7 characteristic, 1 LF, 2 Roe, 3 AUSM+, 4 HLLC with
    `reconstruction` 1 first order, 2 MUSCL, 3 NND2; viscous_order 2 or 8
    adds the viscous flux (Sutherland viscosity)."""
    ngg = ghost_layers(scheme, viscous_order)
    xs = np.linspace(0.0, 1.0, nx)
    ys = np.arange(ny) * 0.01
    x = np.broadcast_to(xs[None, None, :], (1, ny, nx)).copy()
    y = np.broadcast_to(ys[None, :, None], (1, ny, nx)).copy()
    z = np.zeros_like(x)
    jac, metric, xg = metrics(x, y, z, ngg)
    P = jac.size
    bv = np.zeros((6, P))
    right = (xg >= 0.5) & (xg <= 1.5)
    rho = np.where(right, 0.125, 1.0)
    p = np.where(right, 0.1, 1.0)
    bv[0] = rho
    bv[4] = p
    bv[5] = p * MW_AIR / (rho * R_U)
    rho_ref, v_ref = _reference_scale(1.0, 0.0, 1.0)
    param = _air_param(dim=2, inviscid_scheme=scheme, reconstruction=reconstruction, cfl=cfl,
                       weno_eps_scale=(rho_ref * v_ref) ** 2, v_ref=v_ref, rho_ref=rho_ref,
                       viscous_order=viscous_order)
    faces = [(0, -1, 6), (0, 1, 6), (1, -1, 6), (1, 1, 6)]
    return Case("sod", nx, ny, 1, ngg, metric, jac, bv, np.zeros((0, P)), param, faces, x=xg, xyz=(x, y, z))


def sine_wave(n: int = 257, scheme: int = 72, viscous: bool = True, amp: float = 0.05, reynolds: float = 1000.0,
              dt: float | None = None, cfl: float = 0.5, ny: int | None = None, nz: int | None = None,
              reconstruction: int = 2, viscous_order: int = 2) -> Case:
    """3-D viscous single-species wave on a curvilinear periodic block:
    x = xi + amp*sin(2 pi eta) sin(2 pi zeta), y = eta, z = zeta on [0,1]^3
    with n nodes per direction (node-based periodicity: node 0 and node n-1
    coincide, so n = 257 gives 256 unique points), rho = 1 + 0.01 sin(2 pi x),
    u = 1, v = w = 0, p = 1/gamma.  The solver is dimensional with
    Sutherland's law, so the length is scaled by L = Re * mu(T) / (rho U)
    to give rho U L / mu = Re.  dt: fixed step; None means CFL-controlled."""
    ny = n if ny is None else ny
    nz = n if nz is None else nz
    vo = viscous_order if viscous else 0
    ngg = ghost_layers(scheme, vo)
    p0 = 1.0 / GAMMA_AIR
    T0 = p0 * MW_AIR / (1.0 * R_U)
    mu0 = 1.7894e-5 * (T0 / 288.16) ** 1.5 * (288.16 + 110) / (T0 + 110)
    L = reynolds * mu0 / (1.0 * 1.0) if viscous else 1.0
    xi = np.linspace(0.0, 1.0, n)
    eta = np.linspace(0.0, 1.0, ny)
    zeta = np.linspace(0.0, 1.0, nz)
    Z3, Y3, X3 = np.meshgrid(zeta, eta, xi, indexing="ij")
    x = (X3 + amp * np.sin(2 * np.pi * Y3) * np.sin(2 * np.pi * Z3)) * L
    y = Y3 * L
    z = Z3 * L
    jac, metric, xg = metrics(x, y, z, ngg)
    P = jac.size
    bv = np.zeros((6, P))
    xr = xg / L
    bv[0] = 1.0 + 0.01 * np.sin(2 * np.pi * xr)
    bv[1] = 1.0
    bv[4] = p0
    bv[5] = p0 * MW_AIR / (bv[0] * R_U)
    rho_ref, v_ref = _reference_scale(1.0, 1.0, p0)
    param = _air_param(dim=3, inviscid_scheme=scheme, reconstruction=reconstruction,
                       viscous_order=vo, cfl=cfl,
                       weno_eps_scale=(rho_ref * v_ref) ** 2, v_ref=v_ref, rho_ref=rho_ref,
                       fixed_dt=1 if dt is not None else 0, dt=dt or 0.0)
    faces = [(0, -1, 8), (0, 1, 8), (1, -1, 8), (1, 1, 8), (2, -1, 8), (2, 1, 8)]
    return Case("sine_wave", n, ny, nz, ngg, metric, jac, bv, np.zeros((0, P)), param, faces, x=xg,
                xyz=(x, y, z))


def perturbed(case: Case, seed: int = 0, amp: float = 1e-3) -> Case:
    """Copy of `case` with a seeded relative perturbation of rho, u, v, w, p so
    that parity tests exercise every characteristic field."""
    rng = np.random.default_rng(seed)
    bv = case.bv.copy()
    for l in range(5):
        scale = np.abs(bv[l]).max() if np.abs(bv[l]).max() > 0 else 1.0
        bv[l] = bv[l] + amp * scale * rng.standard_normal(bv[l].shape)
    bv[0] = np.abs(bv[0])
    bv[4] = np.abs(bv[4])
    bv[5] = bv[4] / (bv[0] * _gas_constant(case))
    return dataclasses.replace(case, bv=bv)


def with_walls(case: Case, thermal_type: int = 0, temperature: float | None = None, catalytic_type: int = 0,
               yk=None, faces=((1, -1), (1, 1))) -> Case:
    """Copy of `case` whose listed (face, direction) boundaries are no-slip
    walls (label 2): thermal_type 0 isothermal at `temperature` (default 0.95
    of the mean temperature of the initial field), 1 adiabatic; for mixtures
    catalytic_type 1 holds the wall at mass fractions `yk`."""
    walls = set(faces)
    new_faces = [(f, d, 2 if (f, d) in walls else lab) for f, d, lab in case.faces]
    for f, d in walls:
        if not any((f, d) == (a, b) for a, b, _ in case.faces):
            new_faces.append((f, d, 2))
    param = dict(case.param)
    if temperature is None:
        temperature = 0.95 * float(np.mean(case.bv[5]))
    param.update(wall_thermal_type=thermal_type, wall_temperature=temperature, wall_catalytic_type=catalytic_type)
    if yk is not None:
        param["wall_yk"] = list(yk)
    return dataclasses.replace(case, param=param, faces=new_faces, name=case.name + "_walls")


def with_inflow(case: Case, rho: float, u: float, p: float, v: float = 0.0, w: float = 0.0, Y=None,
                subsonic: int = 0, faces=((0, -1),)) -> Case:
    """Copy of `case` whose listed (face, direction) boundaries are constant
    inflows (label 5) of density rho, velocity (u, v, w), pressure p and, for
    mixtures, mass fractions Y (array in mechanism order); the temperature
    and mean molecular weight follow from the state equation.  subsonic = the
    reference's inflow_sub."""
    marks = set(faces)
    new_faces = [(f, d, 5 if (f, d) in marks else lab) for f, d, lab in case.faces]
    for f, d in marks:
        if not any((f, d) == (a, b) for a, b, _ in case.faces):
            new_faces.append((f, d, 5))
    if case.mech is None:
        mw, sv = MW_AIR, []
    else:
        Y = np.asarray(Y, dtype=float)
        mw, sv = 1.0 / float(np.sum(Y / case.mech.mw)), list(Y)
    param = dict(case.param)
    param.update(inflow_subsonic=subsonic, inflow_density=rho, inflow_u=u, inflow_v=v, inflow_w=w, inflow_pressure=p,
                 inflow_temperature=p * mw / (rho * R_U), inflow_mw=mw, inflow_sv=sv)
    return dataclasses.replace(case, param=param, faces=new_faces, name=case.name + "_inflow")


def with_back_pressure(case: Case, p_back: float) -> Case:
    """Copy of `case` whose outflow faces hold the back pressure p_back
    where the flow leaving them is subsonic (the reference's
    if_backPressure / backPressure)."""
    param = dict(case.param)
    param.update(outflow_back_pressure_on=1, outflow_back_pressure=p_back)
    return dataclasses.replace(case, param=param, name=case.name + "_pback")


def split(case: Case, h: int, axis: int = 0, periodic: bool | None = None):
    """Two blocks cut from `case` across `axis` (0 i, 1 j, 2 k), sharing the
    node plane at index h: A holds nodes 0..h, B nodes h..m-1 along that
    axis.  Every padded array is sliced from the whole block's, so both
    blocks carry exactly its metrics and state.  Returns (A, B, links) where
    links lists the inner faces as the mesh's inner-interface records:
    (block, src, tar, target_block), block 0-based, ranges and target_block
    1-based as the reference's inner%4d.txt holds them (in 3-D the lower
    tangential axis is the marked one).  The cut is an inner face; if the
    case's faces across `axis` are periodic (periodic None: read from
    case.faces), A's min face and B's max face become an inner face too,
    else they keep the case's labels."""
    g = case.ngg
    m = [case.mx, case.my, case.mz]
    if axis == 2 and case.mz == 1:
        raise ValueError("a 2-D block cannot be cut along k")
    if periodic is None:
        periodic = any(f == axis and lab == 8 for f, _, lab in case.faces)
    shape = lambda a: a.reshape(a.shape[:-1] + (case.mz + 2 * g, case.my + 2 * g, case.mx + 2 * g))
    pos = -1 - axis  # position of the axis in the padded (k, j, i) shape

    def cut(a, lo, hi):
        if a is None:
            return None
        b = shape(a)
        sl = [slice(None)] * b.ndim
        sl[pos] = slice(lo, hi + 2 * g + 1)
        b = b[tuple(sl)]
        return np.ascontiguousarray(b.reshape(a.shape[:-1] + (b.shape[-3] * b.shape[-2] * b.shape[-1],)))

    def block(lo, hi, keep):
        faces = [fc for fc in case.faces if fc[0] != axis or (not periodic and (fc[0], fc[1]) == keep)]
        ext = dict(zip(("mx", "my", "mz"), m))
        ext["mx my mz".split()[axis]] = hi - lo + 1
        return dataclasses.replace(case, name=f"{case.name}_{'ijk'[axis]}{lo}-{hi}", **ext,
                                   metric=cut(case.metric, lo, hi), jac=cut(case.jac, lo, hi), bv=cut(case.bv, lo, hi),
                                   sv=cut(case.sv, lo, hi), faces=faces, x=cut(case.x, lo, hi))

    A = block(0, h, (axis, -1))
    B = block(h, m[axis] - 1, (axis, 1))
    two_d = case.mz == 1

    def rng(v):
        r = [0] * 6
        tang = [a for a in range(3 if not two_d else 2) if a != axis]
        for a in range(3):
            if a == axis:
                r[2 * a] = r[2 * a + 1] = v
            elif two_d or a != tang[0]:
                r[2 * a], r[2 * a + 1] = 1, m[a]
            else:
                r[2 * a], r[2 * a + 1] = -1, -m[a]
        return r

    na, nb = h + 1, m[axis] - h
    links = [(0, rng(na), rng(1), 2), (1, rng(1), rng(na), 1)]
    if periodic:
        links += [(0, rng(1), rng(nb), 2), (1, rng(nb), rng(1), 1)]
    return A, B, links


def split_i(case: Case, h: int, periodic_i: bool | None = None):
    """split() across i (kept for the existing callers)."""
    return split(case, h, 0, periodic_i)


def _gas_constant(case: Case) -> np.ndarray:
    """Specific gas constant per padded node: air, or R_u sum Y_k / W_k."""
    if case.mech is None:
        return np.full(case.P, R_AIR)
    return R_U * (case.sv[:case.mech.n_spec] / case.mech.mw[:, None]).sum(axis=0)


def _mix_param(mech, **kw) -> dict:
    ns = mech.n_spec
    p = _air_param(n_spec=ns, n_scalar=ns, n_var=5 + ns, n_reac=mech.n_reac, chem_advance_method=1)
    p.update(kw)
    return p


def mole_to_mass(mech, X: np.ndarray) -> np.ndarray:
    """Mole fractions -> mass fractions with the mechanism's weights (last axis)."""
    W = mech.mw
    num = X * W
    return num / num.sum(axis=-1, keepdims=True)


def reactor(mech, T, p, X, ngg: int = 0) -> Case:
    """Batch of independent constant-volume 0-D reactors (one per node of an
    n x 1 x 1 block, zero ghosts by default): rest state, temperature T [K],
    pressure p [Pa], mole fractions X (n x ns).  Metric and Jacobian are those
    of a unit cell; Cn = 0 so the Wu reaction step is a pure 0-D integration."""
    T = np.atleast_1d(np.asarray(T, dtype=np.float64))
    p = np.broadcast_to(np.asarray(p, dtype=np.float64), T.shape).copy()
    X = np.atleast_2d(np.asarray(X, dtype=np.float64))
    X = np.broadcast_to(X, (T.size, mech.n_spec)).copy()
    n = T.size
    Y = mole_to_mass(mech, X)
    W = 1.0 / (Y / mech.mw).sum(axis=1)
    rho = p * W / (R_U * T)
    P = (n + 2 * ngg) * (1 + 2 * ngg) * (1 + 2 * ngg)
    shape = (1 + 2 * ngg, 1 + 2 * ngg, n + 2 * ngg)

    def pad(a):
        out = np.empty(shape)
        out[...] = np.pad(a[None, None, :], ((ngg, ngg), (ngg, ngg), (ngg, ngg)), mode="edge")
        return out.reshape(-1)

    bv = np.zeros((6, P))
    bv[0] = pad(rho)
    bv[4] = pad(p)
    bv[5] = pad(T)
    sv = np.stack([pad(Y[:, l]) for l in range(mech.n_spec)])
    metric = np.zeros((9, P))
    metric[0] = metric[4] = metric[8] = 1.0
    jac = np.ones(P)
    param = _mix_param(mech, dim=2 if True else 3, inviscid_scheme=0, cfl=0.5)
    return Case("reactor", n, 1, 1, ngg, metric, jac, bv, sv, param, [], mech=mech)


def reactor_batch(mech, n: int, seed: int = 0) -> Case:
    """Seeded batch of H2/air reactors: T ~ U[1000, 1600] K, p log-uniform in
    [1, 10] atm, equivalence ratio ~ U[0.5, 2], H2 : O2 : N2 = 2 phi : 1 : 3.76."""
    rng = np.random.default_rng(seed)
    T = rng.uniform(1000.0, 1600.0, n)
    p = 101325.0 * np.exp(rng.uniform(0.0, np.log(10.0), n))
    phi = rng.uniform(0.5, 2.0, n)
    X = np.zeros((n, mech.n_spec))
    X[:, mech.index("H2")] = 2 * phi
    X[:, mech.index("O2")] = 1.0
    X[:, mech.index("N2")] = 3.76
    X /= X.sum(axis=1, keepdims=True)
    return reactor(mech, T, p, X)


def without_reactions(mech):
    """Copy of a mechanism with its reaction list emptied (non-reacting
    mixture flow: species, thermo and transport only)."""
    d = {f.name: getattr(mech, f.name) for f in dataclasses.fields(mech)}
    for name, v in d.items():
        if isinstance(v, np.ndarray) and v.ndim >= 1 and v.shape[0] == mech.n_reac and name not in (
                "mw", "t_low", "t_mid", "t_high", "low", "high", "geometry", "LJ_potent_inv", "vis_coeff",
                "ZRotF298", "WjDivWi_to_One4th", "sqrt_WiDivWjPl1Mul8", "binary_diffusivity_coeff",
                "kb_over_eps_jk", "elem_comp") and mech.n_reac != mech.n_spec:
            d[name] = v[:0]
    return type(mech)(**d)


def _mix_reference(rho, u, p, gamma_est=1.4):
    """rho_ref and v_ref of a mixture reference state: v_ref = |u|, or an
    estimate of the sound speed when |u| < 1 (reference src/BoundCond.cpp:274-283
    uses the mixture's own sound speed; only the WENO epsilon depends on it)."""
    v = abs(u) if abs(u) >= 1 else math.sqrt(gamma_est * p / rho)
    return rho, v


def mix_tube(mech, nx: int = 200, ny: int = 7, scheme: int = 52, reacting: bool = False, left=None, right=None,
             length: float = 0.1, reconstruction: int = 2, viscous_order: int = 0) -> Case:
    """Shock tube of a mixture as an nx-by-ny 2-D block on x in [0, length],
    outflow on all faces, split at the middle.  States are dicts with
    rho [kg/m^3], p [Pa] and Y (mass fractions by species name).  Default:
    the high-pressure state of the reference's reactive shock-tube example
    (rho 0.18075, p 35594, H2/O2/Ar 0.0128/0.1014/0.8859 by mass) on the
    left, its low-pressure one (rho 0.072, p 7173) with 20 % O2 / 80 % Ar on
    the right: a shock, a contact carrying a composition jump and an
    expansion.  `reacting` keeps the mechanism's reactions."""
    m = mech if reacting else without_reactions(mech)
    if left is None:
        left = dict(rho=0.18075, p=35594.0, Y={"H2": 0.012772428, "O2": 0.101362139, "AR": 0.885865433})
    if right is None:
        right = dict(rho=0.072, p=7173.0, Y={"O2": 0.2, "AR": 0.8})
    ngg = ghost_layers(scheme, viscous_order)
    xs = np.linspace(0.0, length, nx)
    ys = np.arange(ny) * length / 100.0
    x = np.broadcast_to(xs[None, None, :], (1, ny, nx)).copy()
    y = np.broadcast_to(ys[None, :, None], (1, ny, nx)).copy()
    z = np.zeros_like(x)
    jac, metric, xg = metrics(x, y, z, ngg)
    P = jac.size
    ns = m.n_spec
    yl, yr = np.zeros(ns), np.zeros(ns)
    for k, v in left["Y"].items():
        yl[m.index(k)] = v
    for k, v in right["Y"].items():
        yr[m.index(k)] = v
    rside = xg > 0.5 * length
    sv = np.where(rside[None, :], yr[:, None], yl[:, None])
    bv = np.zeros((6, P))
    bv[0] = np.where(rside, right["rho"], left["rho"])
    bv[4] = np.where(rside, right["p"], left["p"])
    Rm = R_U * (sv / m.mw[:, None]).sum(axis=0)
    bv[5] = bv[4] / (bv[0] * Rm)
    rho_ref, v_ref = _mix_reference(left["rho"], 0.0, left["p"])
    param = _mix_param(m, dim=2, inviscid_scheme=scheme, reconstruction=reconstruction, cfl=0.5,
                       weno_eps_scale=(rho_ref * v_ref) ** 2, v_ref=v_ref, rho_ref=rho_ref, n_reac=m.n_reac,
                       viscous_order=viscous_order)
    faces = [(0, -1, 6), (0, 1, 6), (1, -1, 6), (1, 1, 6)]
    return Case("mix_tube", nx, ny, 1, ngg, metric, jac, bv, sv, param, faces, x=xg, mech=m, xyz=(x, y, z))


def mix_wave(mech, n: int = 17, scheme: int = 72, viscous: bool = True, ny: int | None = None,
             nz: int | None = None, length: float = 2e-3, reacting: bool = False, T0: float = 600.0,
             dt: float | None = None, reconstruction: int = 2, viscous_order: int = 2) -> Case:
    """Curvilinear periodic 3-D block of a non-uniform H2/N2 - air mixture:
    x = xi + 0.05 sin(2 pi eta) sin(2 pi zeta) on [0, length]^3 (node-based
    periodicity), mixture fraction Z = 0.5 + 0.4 sin(2 pi x / length) between
    a fuel stream (H2 : N2 = 1 : 1 by mole) and air, T = T0 + 50 sin(2 pi y),
    p = 1 atm, u = 50 m/s: viscous stress, heat conduction and
    mixture-averaged species diffusion are all active."""
    m = mech if reacting else without_reactions(mech)
    ny = n if ny is None else ny
    nz = n if nz is None else nz
    vo = viscous_order if viscous else 0
    ngg = ghost_layers(scheme, vo)
    xi, eta, zeta = np.linspace(0, 1, n), np.linspace(0, 1, ny), np.linspace(0, 1, nz)
    Z3, Y3, X3 = np.meshgrid(zeta, eta, xi, indexing="ij")
    x = (X3 + 0.05 * np.sin(2 * np.pi * Y3) * np.sin(2 * np.pi * Z3)) * length
    jac, metric, xg = metrics(x, Y3 * length, Z3 * length, ngg)
    P = jac.size
    ns = m.n_spec
    Xf, Xa = np.zeros(ns), np.zeros(ns)
    Xf[m.index("H2")], Xf[m.index("N2")] = 0.5, 0.5
    Xa[m.index("O2")], Xa[m.index("N2")] = 0.21, 0.79
    Yf, Ya = mole_to_mass(m, Xf), mole_to_mass(m, Xa)
    Zm = 0.5 + 0.4 * np.sin(2 * np.pi * xg / length)
    sv = Zm[None, :] * Yf[:, None] + (1 - Zm[None, :]) * Ya[:, None]
    # ghost nodes take the same analytic fields (periodic block)
    Rm = R_U * (sv / m.mw[:, None]).sum(axis=0)
    shape = (nz + 2 * ngg, ny + 2 * ngg, n + 2 * ngg)
    jj = np.broadcast_to(np.arange(-ngg, ny + ngg)[None, :, None], shape).reshape(-1)
    T = T0 + 50.0 * np.sin(2 * np.pi * jj / (ny - 1))
    bv = np.zeros((6, P))
    bv[4] = 101325.0
    bv[5] = T
    bv[0] = bv[4] / (Rm * T)
    bv[1] = 50.0
    rho_ref, v_ref = _mix_reference(float(bv[0].mean()), 50.0, 101325.0)
    param = _mix_param(m, dim=3, inviscid_scheme=scheme, reconstruction=reconstruction,
                       viscous_order=vo, cfl=0.5,
                       weno_eps_scale=(rho_ref * v_ref) ** 2, v_ref=v_ref, rho_ref=rho_ref, n_reac=m.n_reac,
                       fixed_dt=1 if dt is not None else 0, dt=dt or 0.0)
    faces = [(0, -1, 8), (0, 1, 8), (1, -1, 8), (1, 1, 8), (2, -1, 8), (2, 1, 8)]
    return Case("mix_wave", n, ny, nz, ngg, metric, jac, bv, sv, param, faces, x=xg, mech=m,
                xyz=(x, Y3 * length, Z3 * length))


def mixture_enthalpy(mech, T: float, Y: np.ndarray) -> float:
    """Specific enthalpy (J/kg) of a mixture from the NASA-7 polynomials,
    h_k = R_u/W_k T (a0 + a1 T/2 + a2 T^2/3 + a3 T^3/4 + a4 T^4/5 + a5/T)."""
    h = 0.0
    for k in range(mech.n_spec):
        a = mech.low[k] if T < mech.t_mid[k] else mech.high[k]
        hk = T * (a[0] + T * (a[1] / 2 + T * (a[2] / 3 + T * (a[3] / 4 + T * a[4] / 5)))) + a[5]
        h += Y[k] * R_U / mech.mw[k] * hk
    return h


def mixture_cp(mech, T: float, Y: np.ndarray) -> float:
    cp = 0.0
    for k in range(mech.n_spec):
        a = mech.low[k] if T < mech.t_mid[k] else mech.high[k]
        cp += Y[k] * R_U / mech.mw[k] * (a[0] + T * (a[1] + T * (a[2] + T * (a[3] + T * a[4]))))
    return cp


def reflected_shock_states(mech, Y: np.ndarray, T1: float, p1: float, mach: float):
    """Frozen-chemistry Rankine-Hugoniot states of a shock of Mach `mach`
    (against the frozen sound speed) running into gas at rest (T1, p1, Y) and
    of its reflection from a closed end: returns dicts for state 2 (behind the
    incident shock, lab velocity u towards the end wall) and state 5 (behind
    the reflected shock, at rest), each with rho, u, p, T, and the reflected
    shock's speed."""
    from scipy.optimize import fsolve

    R = R_U * float(np.sum(Y / mech.mw))
    cp1 = mixture_cp(mech, T1, Y)
    c1 = math.sqrt(cp1 / (cp1 - R) * R * T1)
    rho1 = p1 / (R * T1)
    W = mach * c1
    h1 = mixture_enthalpy(mech, T1, Y)

    def incident(x):
        T2, r = x  # r = rho2 / rho1
        w2 = W / r
        p2 = rho1 * r * R * T2
        return [(p1 + rho1 * W * W - p2 - rho1 * r * w2 * w2) / p1,
                (h1 + 0.5 * W * W - mixture_enthalpy(mech, T2, Y) - 0.5 * w2 * w2) / h1 if h1 else 0.0]

    T2, r2 = fsolve(incident, [2.0 * T1, 3.0], xtol=1e-12)
    rho2, u2 = rho1 * r2, W * (1 - 1 / r2)
    p2 = rho2 * R * T2
    h2 = mixture_enthalpy(mech, T2, Y)

    def reflected(x):
        T5, r, Wr = x  # r = rho5 / rho2
        wa, wb = u2 + Wr, Wr
        p5 = rho2 * r * R * T5
        return [(rho2 * wa - rho2 * r * wb) / (rho2 * u2),
                (p2 + rho2 * wa * wa - p5 - rho2 * r * wb * wb) / p2,
                (h2 + 0.5 * wa * wa - mixture_enthalpy(mech, T5, Y) - 0.5 * wb * wb) / abs(h2)]

    T5, r5, Wr = fsolve(reflected, [1.7 * T2, 2.5, 0.5 * u2], xtol=1e-12)
    rho5 = rho2 * r5
    return (dict(rho=rho2, u=u2, p=rho2 * R * T2, T=T2), dict(rho=rho5, u=0.0, p=rho5 * R * T5, T=T5),
            dict(incident_speed=W, reflected_speed=Wr, c1=c1))


def reflected_shock_tube(mech, nx: int = 2048, ny: int = 512, length: float = 0.1, height: float = 0.025,
                         stretch: float = 1.02, mach: float = 2.2, T1: float = 300.0, p1: float = 0.1 * 101325.0,
                         x_shock: float | None = None, scheme: int = 52, viscous_order: int = 2,
                         ny_keep: int | None = None) -> Case:
    """Reflected-shock ignition: stoichiometric H2-O2 diluted by 70 % Ar (2 : 1 : 7
    by mole) at (T1, p1), hit by an incident shock of Mach `mach`, as the gas
    just after the shock has reflected from the closed end x = length: state 5
    (at rest, hot) for x >= x_shock, state 2 (towards the wall) elsewhere,
    from frozen Rankine-Hugoniot jumps (reflected_shock_states).  2-D block of
    nx x ny nodes, uniform in x, stretched in y from the no-slip wall y = 0 by
    the ratio `stretch` per cell; faces: x = 0 outflow, x = length adiabatic
    no-slip wall (the end wall), y = 0 adiabatic no-slip wall, y = height
    symmetry.  WENO5 characteristic (52) with mixture-averaged viscous fluxes;
    the mechanism's reactions are kept.  ny_keep: only the first ny_keep rows of
    that grid (a wall strip with the same spacing, hence the same CFL step)."""
    X = np.zeros(mech.n_spec)
    X[mech.index("H2")], X[mech.index("O2")], X[mech.index("AR")] = 2.0, 1.0, 7.0
    Y = mole_to_mass(mech, X / X.sum())
    s2, s5, _ = reflected_shock_states(mech, Y, T1, p1, mach)
    ngg = ghost_layers(scheme, viscous_order)
    xs = np.linspace(0.0, length, nx)
    widths = stretch ** np.arange(ny - 1)
    ys = np.concatenate([[0.0], np.cumsum(widths)]) * (height / widths.sum())
    if ny_keep is not None:  # the wall strip of the same grid: its first ny_keep rows
        ys = ys[:ny_keep]
        ny = ny_keep
    x = np.broadcast_to(xs[None, None, :], (1, ny, nx)).copy()
    y = np.broadcast_to(ys[None, :, None], (1, ny, nx)).copy()
    z = np.zeros_like(x)
    jac, metric, xg = metrics(x, y, z, ngg)
    P = jac.size
    x_shock = 0.9 * length if x_shock is None else x_shock
    hot = xg >= x_shock
    bv = np.zeros((6, P))
    for l, key in ((0, "rho"), (1, "u"), (4, "p"), (5, "T")):
        bv[l] = np.where(hot, s5[key], s2[key])
    sv = np.repeat(Y[:, None], P, axis=1)
    rho_ref, v_ref = s2["rho"], abs(s2["u"])
    param = _mix_param(mech, dim=2, inviscid_scheme=scheme, reconstruction=2, cfl=0.5, viscous_order=viscous_order,
                       weno_eps_scale=(rho_ref * v_ref) ** 2, v_ref=v_ref, rho_ref=rho_ref, n_reac=mech.n_reac,
                       wall_thermal_type=1, wall_temperature=s5["T"], wall_catalytic_type=0)
    faces = [(0, -1, 6), (0, 1, 2), (1, -1, 2), (1, 1, 3)]
    return Case("reflected_shock_tube", nx, ny, 1, ngg, metric, jac, bv, sv, param, faces, x=xg, mech=mech,
                xyz=(x, y, z))


def mixing_layer_streams(mech, upper: dict, lower: dict, ma_c: float, velocity_ratio: float,
                         upper_faster: bool = True):
    """The two streams of a mixing layer from the convective Mach number and
    the velocity ratio, as get_mixing_layer_info computes them (reference
    src/MixingLayer.cu:9-119, mixture branch): each stream's density and
    frozen sound speed from (T, p, Y); u_slow = Ma_c (c_upper + c_lower) /
    (r - 1), u_fast = r u_slow for r > 1 (u_fast = Ma_c (c_upper + c_lower) /
    (1 - r), u_slow = r u_fast otherwise), the faster stream above y = 0 when
    upper_faster.  Streams are dicts with T [K], p [Pa] and Y (mass fractions
    by species name); returns dicts with rho, u, p, T and the Y vector."""
    out = []
    for st in (upper, lower):
        Y = np.zeros(mech.n_spec)
        for k, v in st["Y"].items():
            Y[mech.index(k)] = v
        imw = float(np.sum(Y / mech.mw))
        cp = mixture_cp(mech, st["T"], Y)
        R = R_U * imw
        gamma = cp / (cp - R)
        out.append(dict(rho=st["p"] / (R * st["T"]), c=math.sqrt(gamma * R * st["T"]), p=st["p"], T=st["T"], Y=Y))
    up, lo = out
    if velocity_ratio > 1:
        u_slow = ma_c * (up["c"] + lo["c"]) / (velocity_ratio - 1)
        u_fast = velocity_ratio * u_slow
    else:
        u_fast = ma_c * (up["c"] + lo["c"]) / (1 - velocity_ratio)
        u_slow = u_fast * velocity_ratio
    ma_up, ma_lo = (u_fast / up["c"], u_slow / lo["c"]) if upper_faster else (u_slow / up["c"], u_fast / lo["c"])
    up["u"], lo["u"] = ma_up * up["c"], ma_lo * lo["c"]
    return up, lo


def mixing_layer(mech, nx: int = 512, ny: int = 256, nz: int = 128, length: float = 0.05, height: float = 0.025,
                 span: float = 0.0125, delta_omega: float = 5e-4, ma_c: float = 0.2, velocity_ratio: float = 1.5,
                 T0: float = 600.0, p0: float = 101325.0, fluctuation: float = 0.01, seed: int = 2026,
                 cluster: float = 3.0, scheme: int = 72, viscous_order: int = 2, reacting: bool = True,
                 window: tuple | None = None) -> Case:
    """Spatially developing H2/air mixing layer: air above y = 0 (the faster
    stream) and H2/N2 (1 : 1 by mole) below, both at T0 and p0, with the
    velocity ratio and convective Mach number of mixing_layer_streams; the
    initial field is the reference's tanh profile u(y) = (u1 + u2)/2 +
    (u1 - u2)/2 tanh(2 y / delta_omega) with every other variable from the
    stream on its side (reference src/Initialize.cu, initialize_mixing_layer).
    Curvilinear block of nx x ny x nz nodes on [0, length] x [-height/2,
    height/2] x [0, span], clustered towards y = 0 by y = (height/2) sinh(c
    eta) / sinh(c) (eta in [-1, 1]).  Faces: x = 0 the mixing-layer inflow
    with white noise of relative intensity `fluctuation` on u, v, w (seeded),
    x = length and both y faces outflow, z periodic.  WENO7 characteristic
    with mixture-averaged viscous fluxes; `reacting` keeps the reactions.
    window (wx, wy, wz): a piece of that grid (same spacing, so the same CFL
    step): the first wx nodes in x, the middle wy rows, the first wz in z."""
    m = mech if reacting else without_reactions(mech)
    X_fuel = np.zeros(m.n_spec)
    X_fuel[m.index("H2")], X_fuel[m.index("N2")] = 0.5, 0.5
    X_air = np.zeros(m.n_spec)
    X_air[m.index("O2")], X_air[m.index("N2")] = 0.21, 0.79
    Yf, Ya = mole_to_mass(m, X_fuel), mole_to_mass(m, X_air)
    names = m.species
    up, lo = mixing_layer_streams(m, dict(T=T0, p=p0, Y={names[l]: Ya[l] for l in range(m.n_spec) if Ya[l] > 0}),
                                  dict(T=T0, p=p0, Y={names[l]: Yf[l] for l in range(m.n_spec) if Yf[l] > 0}),
                                  ma_c, velocity_ratio)
    ngg = ghost_layers(scheme, viscous_order)
    xs = np.linspace(0.0, length, nx)
    eta = np.linspace(-1.0, 1.0, ny)
    ys = 0.5 * height * np.sinh(cluster * eta) / np.sinh(cluster)
    zs = np.linspace(0.0, span, nz)
    if window is not None:  # a piece of the same grid: the first wx x nodes, the middle wy rows, the first wz
        wx, wy, wz = window
        xs, zs = xs[:wx], zs[:wz]
        j0 = (ny - wy) // 2
        ys = ys[j0:j0 + wy]
        nx, ny, nz = wx, wy, wz
    Z3, Y3, X3 = np.meshgrid(zs, ys, xs, indexing="ij")
    x, y, z = X3.copy(), Y3.copy(), Z3.copy()
    jac, metric, xg = metrics(x, y, z, ngg)
    _, Yg, _ = ghost_grid(x, y, z, ngg)
    yg = Yg[1:-1, 1:-1, 1:-1].reshape(-1).copy()
    P = jac.size
    above = yg >= 0
    bv = np.zeros((6, P))
    bv[1] = 0.5 * (up["u"] + lo["u"]) + 0.5 * (up["u"] - lo["u"]) * np.tanh(2 * yg / delta_omega)
    for l, key in ((0, "rho"), (4, "p"), (5, "T")):
        bv[l] = np.where(above, up[key], lo[key])
    sv = np.where(above[None, :], up["Y"][:, None], lo["Y"][:, None])
    rho_ref, v_ref = _mix_reference(up["rho"], up["u"], up["p"])
    param = _mix_param(m, dim=3, inviscid_scheme=scheme, reconstruction=2, cfl=0.5, viscous_order=viscous_order,
                       weno_eps_scale=(rho_ref * v_ref) ** 2, v_ref=v_ref, rho_ref=rho_ref, n_reac=m.n_reac,
                       inflow_type=2, inflow_density=up["rho"], inflow_u=up["u"], inflow_v=0.0, inflow_w=0.0,
                       inflow_pressure=up["p"], inflow_temperature=up["T"],
                       inflow_mw=1.0 / float(np.sum(up["Y"] / m.mw)), inflow_sv=list(up["Y"]),
                       inflow_density_lower=lo["rho"], inflow_u_lower=lo["u"], inflow_v_lower=0.0,
                       inflow_w_lower=0.0, inflow_p_lower=lo["p"], inflow_t_lower=lo["T"],
                       inflow_sv_lower=list(lo["Y"]), inflow_delta_omega=delta_omega,
                       inflow_fluctuation_type=1 if fluctuation > 0 else 0, inflow_fluctuation_intensity=fluctuation,
                       inflow_seed=seed)
    faces = [(0, -1, 5), (0, 1, 6), (1, -1, 6), (1, 1, 6), (2, -1, 8), (2, 1, 8)]
    return Case("mixing_layer", nx, ny, nz, ngg, metric, jac, bv, sv, param, faces, x=xg, mech=m, xyz=(x, y, z),
                y=yg)
