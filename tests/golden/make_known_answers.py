"""Writes tests/golden/known_answers.json: closed-form values of the reference's
force and energy expressions for single pairs, bonds, angles and wall
distances, plus the rock-salt Madelung constant for the Ewald sums.

These are computed here from the formulas as printed in the reference
(fluid_fluid.f90:99-116, intra_molec.f90:44-47, bending.f90:64-96,
fluid_wall.f90:96-121) with Python floats, independently of the oracle, and
serve as known-answer fixtures for it.  Run: python tests/golden/make_known_answers.py
"""
import json
import math
import os

import numpy as np

C16 = float(np.float32(2.0) ** (np.float32(1.0) / np.float32(6.0)))  # 2.**(1./6.) in REAL*4
CLAMP = float(np.float32(0.98))


def lj(r, eps=1.0, sig=1.0):
    rc2 = (C16 * sig) ** 2
    rd = (sig * sig / rc2) ** 3
    shift = rd * (rd - 1.0)
    s6 = (sig * sig / (r * r)) ** 3
    e = 4.0 * eps * ((s6 * s6 - s6) - shift)
    f = 4.0 * eps * (12.0 * s6 * s6 - 6.0 * s6) / r   # magnitude, repulsive > 0
    return e, f


def fene(r, k=30.0, R0=1.5):
    x = min(r * r / (R0 * R0), CLAMP)
    e = -0.5 * k * R0 * R0 * math.log(1.0 - x)
    f = -k * r / (1.0 - x)   # along the bond, attractive < 0
    return e, f


def wall(z, L, a=1.0, s=1.0):
    e = a * (s / z) ** 9 - a * (s / z) ** 3 + a * (s / (L - z)) ** 9 - a * (s / (L - z)) ** 3
    f = (9 * a * s ** 9 / z ** 10 - 3 * a * s ** 3 / z ** 4) - (9 * a * s ** 9 / (L - z) ** 10 - 3 * a * s ** 3 / (L - z) ** 4)
    return e, f


def main():
    out = {"lj": [], "fene": [], "bend": [], "wall": []}
    for r in (0.95, 1.0, 1.05, 1.1):
        e, f = lj(r)
        out["lj"].append({"r": r, "energy": e, "force": f})
    for r in (0.8, 0.97, 1.2, 1.49):
        e, f = fene(r)
        out["fene"].append({"r": r, "energy": e, "force": f})
    for theta_deg in (10.0, 45.0, 90.0, 150.0):
        th = math.radians(theta_deg)
        out["bend"].append({"theta": th, "k": 2.0, "energy": 0.5 * 2.0 * th * th})
    for z in (0.9, 1.2, 2.0, 5.0):
        e, f = wall(z, 20.0)
        out["wall"].append({"z": z, "L": 20.0, "energy": e, "force_z": f})
    # rock salt: E per ion pair = -M / a (a = nearest-neighbour distance), M below
    out["madelung_nacl"] = 1.747564594633182
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "known_answers.json")
    with open(path, "w") as fh:
        json.dump(out, fh, indent=1)
    print("wrote", path)


if __name__ == "__main__":
    main()
