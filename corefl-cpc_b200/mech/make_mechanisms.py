"""Builds the bundled mechanism tables (*.npz in this folder) from the
Chemkin files that ship with the reference's examples.
Usage: python make_mechanisms.py <reference root>

li2004.npz        example/constantVolumeReactor/input/chemistry/2004-Li-IntJ.Chem.Kinet.inp
                  (+ therm.dat, tran.dat): 9 species, 19 reactions after the
                  two DUPLICATE pairs are merged, N2 as the bath gas.
premix_h2_ar.npz  example/reactiveShockTube/input/chemistry/H2_mech-PREMIX.inp
                  (+ therm.dat, tran.dat): 9 species with Ar, 18 reactions.
"""
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
import mechanism  # noqa: E402

SOURCES = {
    "li2004": ("constantVolumeReactor", "2004-Li-IntJ.Chem.Kinet.inp"),
    "premix_h2_ar": ("reactiveShockTube", "H2_mech-PREMIX.inp"),
}

if __name__ == "__main__":
    if len(sys.argv) != 2 or not os.path.isdir(sys.argv[1]):
        sys.exit("usage: python make_mechanisms.py <reference root>")
    REF = sys.argv[1]
    for name, (ex, mech) in SOURCES.items():
        d = os.path.join(REF, "example", ex, "input", "chemistry")
        m = mechanism.parse(os.path.join(d, mech), os.path.join(d, "therm.dat"), os.path.join(d, "tran.dat"))
        m.save(os.path.join(HERE, name + ".npz"))
        print(name, m.n_spec, "species", m.n_reac, "reactions", m.species)
