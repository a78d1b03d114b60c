"""Regenerates the golden fixtures in this folder from the reference's own
example data.  Usage: python make_golden.py <reference root>

sod_exact.npz  — exact Riemann solution of the Sod problem at t = 0.2
                 (reference example/sodShockTube/exact.dat: x, u, rho, p).
reactor_li2004.npz — constant-volume H2/air ignition trajectory of the
                 reference's 0-D reactor (Li-2004 species, 1000 K, 2 atm,
                 X = 0.295775 H2 / 0.147887 O2 / 0.556338 N2; reference
                 example/constantVolumeReactor/const_volume_reactor_output.dat):
                 t, T, p and mole fractions every 5000 reactor steps.
"""
import os
import sys

import numpy as np

REF = None  # the reference checkout, from the command line
HERE = os.path.dirname(os.path.abspath(__file__))


def sod_exact():
    path = os.path.join(REF, "example", "sodShockTube", "exact.dat")
    with open(path) as f:
        f.readline()  # variables="x","u","density","pressure"
        vals = np.array([float(v) for v in f.read().split()]).reshape(-1, 4)
    np.savez_compressed(os.path.join(HERE, "sod_exact.npz"), x=vals[:, 0], u=vals[:, 1], rho=vals[:, 2], p=vals[:, 3])
    print("sod_exact.npz:", vals.shape[0], "points")


def reactor():
    path = os.path.join(REF, "example", "constantVolumeReactor", "const_volume_reactor_output.dat")
    with open(path) as f:
        header = f.readline().strip()
        rows = [[float(v) for v in line.split(",")] for line in f if line.strip()]
    a = np.array(rows)
    names = [h.split("<sub>")[1].split("</sub>")[0] for h in header.split(",")[3:-1]]
    np.savez_compressed(os.path.join(HERE, "reactor_li2004.npz"), t=a[:, 0], T=a[:, 1], p=a[:, 2], X=a[:, 3:-1],
                        species=np.array(names))
    print("reactor_li2004.npz:", a.shape[0], "records", names)


if __name__ == "__main__":
    if len(sys.argv) != 2 or not os.path.isdir(sys.argv[1]):
        sys.exit("usage: python make_golden.py <reference root>")
    REF = sys.argv[1]
    sod_exact()
    reactor()
