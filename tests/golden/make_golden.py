"""Regenerates the golden fixtures in this folder from the reference's own
example data (run in a checkout that has the reference at REFERENCE_ROOT).

sod_exact.npz  — exact Riemann solution of the Sod problem at t = 0.2
                 (reference example/sodShockTube/exact.dat: x, u, rho, p).
"""
import os
import sys

import numpy as np

REF = os.environ.get("REFERENCE_ROOT", "/root/reference")
HERE = os.path.dirname(os.path.abspath(__file__))


def sod_exact():
    path = os.path.join(REF, "example", "sodShockTube", "exact.dat")
    with open(path) as f:
        f.readline()  # variables="x","u","density","pressure"
        vals = np.array([float(v) for v in f.read().split()]).reshape(-1, 4)
    np.savez_compressed(os.path.join(HERE, "sod_exact.npz"), x=vals[:, 0], u=vals[:, 1], rho=vals[:, 2], p=vals[:, 3])
    print("sod_exact.npz:", vals.shape[0], "points")


if __name__ == "__main__":
    if not os.path.isdir(REF):
        sys.exit(f"reference not found at {REF}")
    sod_exact()
