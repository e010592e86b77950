"""Writes the reference-held fixtures that pin the oracle's energy terms.

The reference ships the output of one of its own runs (SYSTEM 4 of
control_simulation.h: one 102-bead chain, bulk periodic box 70 x 90 x 90,
SOLVENT 1, PARTICLE_4, BIN_TYPE 0, Langevin thermostat, dt = 2e-4,
10 + 10000 steps):
  conf_new  the restart file store_config(2) wrote at step 10000
            (md_main.f90:168-169: every n_safe = 100 steps; the run ends at
            10010, so the last write is step 10000), in the formats of
            store_config.f90:20-61;
  fort.60   every 10th step: i_time, V/N, V/N + KE/N, KE/N
            (verlet_velocities.f90:219-223, format i7,3g17.5), with
            V = v_wall_wall + v_fluid_wall + v_fluid_fluid + v_intra_molec
            (:187) and N = n_mon_tot = 102 (init_params.f90:478-480);
  fort.41   every 5th observed step: i_time, v_fluid_fluid, v_intra_molec,
            v_fluid_wall (observation.f90:304-307, format i7,3f15.5);
  mfa_output the inputs the run was made with (box, epsilon table, FENE
            constants, time step; the header of mfa_input echoed).

The potential energy of a configuration does not depend on the thermostat's
noise, so the oracle's v_fluid_fluid + v_intra_molec at conf_new's positions
must equal fort.60's V/N of step 10000 to its five printed digits and each
of fort.41's two terms at that step to the precision the 7-decimal positions
of conf_new allow, and 0.5 sum m v^2 / N of conf_new's velocities fort.60's
KE/N.

This script copies conf_new as it is (tests/golden/reference_conf_new) and
writes the fort.60 and fort.41 rows around step 10000 and the run's inputs,
read from mfa_output and system_input, to tests/golden/reference_system4.json.
Run: python tests/golden/make_reference_system4.py [reference dir]
"""
import json
import os
import shutil
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def main(ref):
    shutil.copyfile(os.path.join(ref, "conf_new"), os.path.join(HERE, "reference_conf_new"))
    rows = {}
    for ln in open(os.path.join(ref, "fort.60")):
        f = ln.split()
        if len(f) == 4 and 9950 <= int(f[0]) <= 10010:
            rows[f[0]] = {"v_per_n": float(f[1]), "e_per_n": float(f[2]), "t_per_n": float(f[3]),
                          "text": ln.rstrip("\n")}
    terms = {}
    for ln in open(os.path.join(ref, "fort.41")):
        f = ln.split()
        if len(f) == 4 and 9950 <= int(f[0]) <= 10010:
            terms[f[0]] = {"v_fluid_fluid": float(f[1]), "v_intra_molec": float(f[2]),
                           "v_fluid_wall": float(f[3]), "text": ln.rstrip("\n")}
    out = [ln.rstrip("\n") for ln in open(os.path.join(ref, "mfa_output"))]

    def value(label):
        """First number on the first mfa_output line that carries `label`."""
        for ln in out:
            if label in ln:
                return float(ln.split()[0])
        raise KeyError(label)

    eps, sigma, mass, friction = [], [], [], []
    k = 0
    while k < len(out):
        if out[k].strip().endswith("mass"):
            mass.append(float(out[k].split()[0]))
            eps.append([float(out[k + 1 + j].split()[0]) for j in range(4)])
            sigma.append(float(out[k + 5].split()[0]))
            friction.append(float(out[k + 6].split()[0]))
            k += 7
        else:
            k += 1
    box = None
    for ln in out:
        if "MD Box dimensions" in ln:
            box = [float(x) for x in ln.split()[:3]]
    nbins = None
    for ln in out:
        if "binning boxes" in ln:
            nbins = [int(x) for x in ln.split()[:3]]
    sysin = [ln for ln in open(os.path.join(ref, "system_input")) if not ln.lstrip().startswith("#")]
    first = sysin[0].split()
    fixture = {
        "source": "feindas/mfa shipped run outputs: conf_new, fort.60, mfa_output, system_input",
        "switches": {"SYSTEM": 4, "SYMMETRY": 1, "SOLVENT": 1, "PARTICLE_4": True, "BIN_TYPE": 0,
                     "THERMOSTAT": 1, "CHAIN_BC": 2, "RUN_2D": True, "BENDING": True, "EXT_FORCE": 1},
        "n_mon": int(first[0]), "n_chain": int(first[1]), "n_part": int(first[0]) * int(first[1]),
        "box": box, "n_bin": nbins,
        "mass": mass, "eps": eps, "sigma": sigma, "friction": friction,
        "dt": value("time step increment"), "temp": value("temperature"),
        "k_chain": value("effective spring constant within chain"),
        "r_chain": value("max. spacing between neighbored monomers"),
        "k_bend": value("Bending elastic constant"),
        "k_elastic": value("Force constant of the external elastic field"),
        "conf_step": 10000,
        "fort60": rows,
        "fort41": terms,
    }
    with open(os.path.join(HERE, "reference_system4.json"), "w") as fh:
        json.dump(fixture, fh, indent=1)
        fh.write("\n")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
