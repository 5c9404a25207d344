"""Builds the golden fixtures of the test suite from the reference checkout.

Run here (where the reference is mounted) after `make -C oracle ref`, which
compiles the reference's own vtk.c into oracle/_ref/vtk:

    python tests/golden/make_golden.py [reference checkout]

without an argument it reads the checkout the oracle's Makefile names (REF).

Outputs (all small, committed):
  configuration.dat, polymer.dat     the reference's input files (2 types)
  configuration_3types.dat           the reference's configuration.dat~ (3 types)
  density_240000_z3.dat              the first 3 z-slices of density_240000.dat
                                     (header rewritten to Nz=3)
  density_240000_z3.vtk              the reference vtk.c run on that file
  density_invariants.json            per density_<step>.dat: bead total,
                                     integrality of the counts, per-type mean
                                     phi and omega, and a few sample lines
  out_vtk_head.txt                   the first 20 lines of the reference out.vtk
"""
import json
import os
import shutil
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))


def density_stats(path):
    with open(path) as f:
        h1 = f.readline()
        h2 = f.readline()
        data = np.loadtxt(f)
    nx, ny, nz = [int(t.split("=")[1]) for t in h1.strip().split(",")]
    n_types = data.shape[1] // 2
    phi, omega = data[:, :n_types], data[:, n_types:]
    cells = nx * ny * nz
    return nx, ny, nz, n_types, cells, phi, omega, h1, h2


def main(ref):
    for name, dst in (("configuration.dat", "configuration.dat"), ("configuration.dat~", "configuration_3types.dat"),
                      ("polymer.dat", "polymer.dat")):
        shutil.copyfile(os.path.join(ref, name), os.path.join(HERE, dst))

    # small VTK known-answer case
    src = os.path.join(ref, "density_240000.dat")
    with open(src) as f:
        lines = f.readlines()
    nx, ny = 24, 24
    sub = os.path.join(HERE, "density_240000_z3.dat")
    with open(sub, "w") as f:
        f.write("Nx=24, Ny=24, Nz=3\n")
        f.write(lines[1])
        f.writelines(lines[2:2 + nx * ny * 3])
    vtk = os.path.join(ROOT, "oracle", "_ref", "vtk")
    if not os.path.exists(vtk):
        raise SystemExit("build the reference converter first: make -C oracle ref")
    cwd = os.getcwd()
    os.chdir(HERE)
    try:
        subprocess.run([vtk, "density_240000_z3.dat", "density_240000_z3.vtk"], check=True, stdout=subprocess.DEVNULL)
    finally:
        os.chdir(cwd)

    with open(os.path.join(ref, "out.vtk")) as f:
        head = [next(f) for _ in range(20)]
    with open(os.path.join(HERE, "out_vtk_head.txt"), "w") as f:
        f.writelines(head)

    inv = {}
    for name in sorted(os.listdir(ref)):
        if not (name.startswith("density_") and name.endswith(".dat")):
            continue
        nx, ny, nz, nt, cells, phi, omega, h1, h2 = density_stats(os.path.join(ref, name))
        # phi = count * n_cells / n_beads: recover counts with the bead total
        # that makes every entry an integer
        total = None
        for cand in (409600,):
            c = phi * cand / cells
            if np.max(np.abs(c - np.round(c))) < 1e-3:
                total = cand
        counts = np.round(phi * total / cells).astype(np.int64) if total else None
        inv[name] = {"nx": nx, "ny": ny, "nz": nz, "n_types": nt, "header2": h2.strip(),
                     "bead_total_from_counts": int(counts.sum()) if counts is not None else None,
                     "counts_integral": counts is not None,
                     "mean_phi": phi.mean(axis=0).round(6).tolist(), "mean_omega": omega.mean(axis=0).round(6).tolist(),
                     "first_line": [float(v) for v in np.concatenate([phi[0], omega[0]])]}
    with open(os.path.join(HERE, "density_invariants.json"), "w") as f:
        json.dump(inv, f, indent=1, sort_keys=True)
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    if len(sys.argv) > 1:
        main(sys.argv[1])
    else:
        sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
        from oracle.oracle import reference_dir
        ref = reference_dir()
        if ref is None:
            sys.exit("reference checkout not found (set REF)")
        main(ref)
