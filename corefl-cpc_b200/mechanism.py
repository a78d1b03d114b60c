"""Chemkin mechanism, NASA-7 thermo and transport data -> the species and
reaction tables of the solver (host-side set-up, numpy).

Follows the reference's readers: species/elements and molecular weights
(reference src/ChemData.cpp:14-62, 400-426, atomic weights src/Element.cpp),
NASA-7 two-range polynomials in fixed columns (src/ChemData.cpp:330-520),
transport records and the derived mixture-averaged tables
(src/ChemData.cpp:740-866), reactions with third bodies, LOW/TROE fall-off,
REV and merged DUPLICATE pairs, Ea divided by R_c (src/ChemData.cpp:869-1177).

Reaction type codes (as the reference's `label`): 0 irreversible, 1
elementary, 3 merged duplicate (second Arrhenius in A2/b2/Ea2), 4 third
body, 5 Lindemann fall-off, 6 Troe (3 parameters), 7 Troe (4 parameters).
"""
from __future__ import annotations

import dataclasses
import math
import os
import re

import numpy as np

R_U = 8314.462618
R_C = 1.98720425864083
BOLTZMANN = 1.380649e-23
ATOMIC_WEIGHT = {"H": 1.008, "O": 15.999, "N": 14.007, "C": 12.011, "AR": 39.95, "HE": 4.002602}

MECH_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "mech")


@dataclasses.dataclass
class Mechanism:
    species: list
    elements: list
    mw: np.ndarray
    elem_comp: np.ndarray  # (ns, n_elem)
    t_low: np.ndarray
    t_mid: np.ndarray
    t_high: np.ndarray
    low: np.ndarray  # (ns, 7)
    high: np.ndarray  # (ns, 7)
    geometry: np.ndarray
    LJ_potent_inv: np.ndarray
    vis_coeff: np.ndarray
    ZRotF298: np.ndarray
    WjDivWi_to_One4th: np.ndarray
    sqrt_WiDivWjPl1Mul8: np.ndarray
    binary_diffusivity_coeff: np.ndarray
    kb_over_eps_jk: np.ndarray
    reac_type: np.ndarray
    rev_type: np.ndarray
    stoi_f: np.ndarray  # (nr, ns)
    stoi_b: np.ndarray
    order: np.ndarray
    A: np.ndarray
    b: np.ndarray
    Ea: np.ndarray
    A2: np.ndarray
    b2: np.ndarray
    Ea2: np.ndarray
    third_body_coeff: np.ndarray  # (nr, ns)
    troe_alpha: np.ndarray
    troe_t3: np.ndarray
    troe_t1: np.ndarray
    troe_t2: np.ndarray

    @property
    def n_spec(self):
        return len(self.species)

    @property
    def n_reac(self):
        return len(self.reac_type)

    def index(self, name):
        return self.species.index(name.upper())

    def element_mass_fractions(self) -> np.ndarray:
        """mu[e, k] = a_ek W_e / W_k: mass of element e per mass of species k,
        so that Z_e = mu @ Y are the element mass fractions (each column sums
        to 1).  Elements present in no species are dropped."""
        W_e = np.array([ATOMIC_WEIGHT[el] for el in self.elements])
        mu = (self.elem_comp * W_e[None, :]).T / self.mw[None, :]
        return mu[self.elem_comp.sum(axis=0) > 0]

    def save(self, path):
        d = {f.name: getattr(self, f.name) for f in dataclasses.fields(self)}
        d["species"] = np.array(self.species)
        d["elements"] = np.array(self.elements)
        np.savez_compressed(path, **d)

    @staticmethod
    def load(path) -> "Mechanism":
        z = np.load(path)
        kw = {f.name: z[f.name] for f in dataclasses.fields(Mechanism)}
        kw["species"] = [str(s) for s in z["species"]]
        kw["elements"] = [str(s) for s in z["elements"]]
        return Mechanism(**kw)


def load(name: str) -> Mechanism:
    """A bundled mechanism table: 'li2004' (9 species / 19 reactions, N2) or
    'premix_h2_ar' (9 species / 18 reactions, Ar)."""
    return Mechanism.load(os.path.join(MECH_DIR, name + ".npz"))


def _lines(path):
    with open(path, encoding="latin-1") as f:
        return f.read().splitlines()


def _strip_comment(s):
    i = s.find("!")
    return s if i < 0 else s[:i]


def parse(mech_path: str, therm_path: str, tran_path: str) -> Mechanism:
    lines = _lines(mech_path)
    # ---- elements and species
    text = "\n".join(_strip_comment(l) for l in lines).upper()
    m = re.search(r"\bELEM(?:ENTS)?\b(.*?)\bEND\b", text, re.S)
    elements = m.group(1).split()
    m = re.search(r"\bSPEC(?:IES)?\b(.*?)\bEND\b", text, re.S)
    species = m.group(1).split()
    ns = len(species)
    sidx = {s: i for i, s in enumerate(species)}

    # ---- thermo (two ranges, fixed columns)
    th = _lines(therm_path)
    t_low = np.zeros(ns); t_mid = np.zeros(ns); t_high = np.zeros(ns)
    low = np.zeros((ns, 7)); high = np.zeros((ns, 7))
    elem_comp = np.zeros((ns, len(elements)), dtype=np.int64)
    got = set()
    k = 0
    default_mid = 1000.0
    while k < len(th):
        line = th[k]
        up = line.upper()
        if up.startswith("THERMO"):
            if k + 1 < len(th):
                parts = th[k + 1].split()
                if len(parts) >= 3:
                    default_mid = float(parts[1])
            k += 2
            continue
        if not line.strip() or line.lstrip().startswith("!") or up.split()[0] in ("END",):
            k += 1
            continue
        name = up[:18].split()[0] if up[:18].split() else ""
        if name in sidx and name not in got and k + 3 < len(th):
            i = sidx[name]
            t_low[i] = float(line[45:55])
            t_high[i] = float(line[55:65])
            mid = line[65:75].strip()
            t_mid[i] = float(mid) if mid else default_mid
            for e in range(4):
                comp = line[24 + 5 * e: 29 + 5 * e].strip()
                if not comp or comp.startswith("0"):
                    break
                el = comp[:2].strip().upper()
                cnt = int(float(comp[2:].strip() or 0))
                if el in elements:
                    elem_comp[i, elements.index(el)] = cnt
            l2, l3, l4 = th[k + 1], th[k + 2], th[k + 3]
            f = lambda s, c: float(s[15 * c: 15 * c + 15])
            high[i] = [f(l2, 0), f(l2, 1), f(l2, 2), f(l2, 3), f(l2, 4), f(l3, 0), f(l3, 1)]
            low[i] = [f(l3, 2), f(l3, 3), f(l3, 4), f(l4, 0), f(l4, 1), f(l4, 2), f(l4, 3)]
            got.add(name)
            k += 4
            continue
        k += 1
    missing = set(species) - got
    if missing:
        raise ValueError(f"no thermo data for {sorted(missing)}")
    mw = np.array([sum(ATOMIC_WEIGHT[el] * elem_comp[i, e] for e, el in enumerate(elements)) for i in range(ns)])

    # ---- transport
    geometry = np.zeros(ns); eps_kb = np.zeros(ns); sigma = np.zeros(ns); mu = np.zeros(ns)
    alpha = np.zeros(ns); zrot = np.zeros(ns)
    got = set()
    for line in _lines(tran_path):
        up = _strip_comment(line).upper().split()
        if not up or up[0] not in sidx or up[0] in got:
            continue
        i = sidx[up[0]]
        geometry[i], eps_kb[i], sigma[i], mu[i], alpha[i], zrot[i] = [float(v) for v in up[1:7]]
        got.add(up[0])
    missing = set(species) - got
    if missing:
        raise ValueError(f"no transport data for {sorted(missing)}")
    pi = math.pi
    LJ_potent_inv = 1.0 / eps_kb
    vis_coeff = 2.6693e-6 * np.sqrt(mw) / (sigma * sigma)
    TRedInv = eps_kb / 298
    F298 = 1 + 0.5 * pi * pi * pi * np.sqrt(TRedInv) + (2 + 0.25 * pi * pi) * TRedInv + math.sqrt(pi * pi * pi) * \
        np.sqrt(TRedInv * TRedInv * TRedInv)
    ZRotF298 = zrot * F298
    WjDivWi = np.array([[(mw[j] / mw[i]) ** 0.25 for j in range(ns)] for i in range(ns)])
    sqrtW = np.array([[1.0 / math.sqrt(8 * (1 + mw[i] / mw[j])) for j in range(ns)] for i in range(ns)])

    conv = 1e-18 * math.sqrt(1e-7) * (1e8 ** 1.5) / math.sqrt(BOLTZMANN)

    def red_dipole(i):
        return 0.0 if mu[i] == 0 else conv * mu[i] / math.sqrt(eps_kb[i] * sigma[i] ** 3)

    bdc = np.zeros((ns, ns)); kbe = np.zeros((ns, ns))
    for j in range(ns):
        Wjj = mw[j] * 0.5
        bdc[j, j] = 0.0188324 / (math.sqrt(Wjj) * sigma[j] * sigma[j])
        kbe[j, j] = 1.0 / eps_kb[j]
        for k2 in range(j + 1, ns):
            Wjk = mw[j] * mw[k2] / (mw[j] + mw[k2])
            xi = 1.0
            if (mu[j] != 0) != (mu[k2] != 0):
                p_, n_ = (j, k2) if mu[j] != 0 else (k2, j)
                alpha_n_star = alpha[n_] / sigma[n_] ** 3
                mu_p_star = red_dipole(p_)
                xi = 1.0 + 0.25 * alpha_n_star * mu_p_star * mu_p_star * math.sqrt(eps_kb[p_] / eps_kb[n_])
            sig = 0.5 * (sigma[j] + sigma[k2]) * xi ** (-1.0 / 6.0)
            bdc[j, k2] = bdc[k2, j] = 0.0188324 / (math.sqrt(Wjk) * sig * sig)
            ejk = xi * xi * math.sqrt(eps_kb[j] * eps_kb[k2])
            kbe[j, k2] = kbe[k2, j] = 1.0 / ejk

    # ---- reactions
    m = re.search(r"\bREAC(?:TIONS)?\b[^\n]*\n(.*?)\n\s*END\b", "\n".join(lines).upper(), re.S)
    body = m.group(1).splitlines() if m else []
    R = []  # dicts

    def new_reac():
        return dict(type=1, rev=0, sf=np.zeros(ns, np.int64), sb=np.zeros(ns, np.int64), order=0, A=0.0, b=0.0,
                    Ea=0.0, A2=0.0, b2=0.0, Ea2=0.0, tb=np.ones(ns), ta=0.0, t3=0.0, t1=0.0, t2=0.0, dup=False)

    def parse_side(s, stoich, sign, r):
        for tok in s.split("+"):
            tok = tok.strip()
            if not tok:
                continue
            c = 1
            if tok[0].isdigit():
                c = int(tok[0])
                tok = tok[1:]
            stoich[sidx[tok]] += c
            r["order"] += sign * c

    cur = None
    for raw in body:
        line = _strip_comment(raw).strip()
        if not line:
            continue
        if "=" in line:
            toks = line.split()
            eq = "".join(toks[:-3])
            r = new_reac()
            r["A"], r["b"], r["Ea"] = float(toks[-3]), float(toks[-2]), float(toks[-1]) / R_C
            if "(+M)" in eq:
                r["type"] = 5
                eq = eq.replace("(+M)", "")
            elif "+M" in eq:
                r["type"] = 4
                eq = eq.replace("+M", "")
            if "<=>" in eq:
                lhs, rhs = eq.split("<=>")
            elif "=>" in eq:
                lhs, rhs = eq.split("=>")
                r["type"] = 0
            else:
                lhs, rhs = eq.split("=")
            parse_side(lhs, r["sf"], -1, r)
            parse_side(rhs, r["sb"], +1, r)
            R.append(r)
            cur = r
            continue
        up = line.replace("/", " ").split()
        key = up[0]
        if key in ("DUPLICATE", "DUP"):
            cur["dup"] = True
            cur["type"] = 3
        elif key == "REV":
            cur["A2"], cur["b2"], cur["Ea2"] = float(up[1]), float(up[2]), float(up[3]) / R_C
            cur["rev"] = 1
        elif key == "LOW":
            cur["A2"], cur["b2"], cur["Ea2"] = float(up[1]), float(up[2]), float(up[3]) / R_C
        elif key == "TROE":
            cur["type"] = 6
            cur["ta"], cur["t3"], cur["t1"] = float(up[1]), float(up[2]), float(up[3])
            if len(up) > 4:
                cur["t2"] = float(up[4])
                cur["type"] = 7
        else:
            for q in range(0, len(up) - 1, 2):
                if up[q] in sidx:
                    cur["tb"][sidx[up[q]]] = float(up[q + 1])
    # merge DUPLICATE pairs: the second's Arrhenius goes to A2/b2/Ea2 of the first
    merged = []
    open_dups = []
    for r in R:
        if r["dup"]:
            partner = next((d for d in open_dups if np.array_equal(d["sf"], r["sf"]) and np.array_equal(d["sb"], r["sb"])),
                           None)
            if partner is not None:
                partner["A2"], partner["b2"], partner["Ea2"] = r["A"], r["b"], r["Ea"]
                open_dups.remove(partner)
                continue
            open_dups.append(r)
        merged.append(r)
    nr = len(merged)
    g = lambda k, dt=float: np.array([r[k] for r in merged], dtype=dt)
    return Mechanism(
        species=species, elements=elements, mw=mw, elem_comp=elem_comp, t_low=t_low, t_mid=t_mid, t_high=t_high,
        low=low, high=high, geometry=geometry, LJ_potent_inv=LJ_potent_inv, vis_coeff=vis_coeff, ZRotF298=ZRotF298,
        WjDivWi_to_One4th=WjDivWi, sqrt_WiDivWjPl1Mul8=sqrtW, binary_diffusivity_coeff=bdc, kb_over_eps_jk=kbe,
        reac_type=g("type", np.int64), rev_type=g("rev", np.int64),
        stoi_f=np.array([r["sf"] for r in merged]).reshape(nr, ns), stoi_b=np.array([r["sb"] for r in merged]).reshape(nr, ns),
        order=g("order", np.int64), A=g("A"), b=g("b"), Ea=g("Ea"), A2=g("A2"), b2=g("b2"), Ea2=g("Ea2"),
        third_body_coeff=np.array([r["tb"] for r in merged]).reshape(nr, ns), troe_alpha=g("ta"), troe_t3=g("t3"),
        troe_t1=g("t1"), troe_t2=g("t2"))
