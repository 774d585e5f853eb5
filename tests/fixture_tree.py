"""Writes a project tree in the reference's layout (data/structures/*.cssr,
data/forcefields/*.def, data/masses.def, data/uc_replications/*.uc,
data/grids/, output_files/, simulation.input) for a synthetic framework, so
the drop-in tools (ours and the reference's) can run on it."""
import os

import numpy as np

import emptyroom_b200 as er

TYPE_LABELS = ["Zn", "O", "C", "H", "N", "Cu", "Al", "Si"]


def write_tree(root, fw, name="SYNFW", ff_name="SYNFF", resolution=0.8, insertions_per_a3=200,
               fmt="txt", temperature=298.0, rc=None):
    """fw: emptyroom_b200.synth.SynthFramework. Returns (framework name, adsorbate)."""
    for d in ["data/structures", "data/forcefields", "data/uc_replications", "data/grids",
              "output_files"]:
        os.makedirs(os.path.join(root, d), exist_ok=True)
    n_types = len(fw.type_eps)
    labels = TYPE_LABELS[:n_types]
    a, b, c = fw.abc
    al, be, ga = fw.angles
    with open(os.path.join(root, "data", "structures", name + ".cssr"), "w") as fh:
        fh.write(f"\t\t\t\t{a:.6f}  {b:.6f}  {c:.6f}\n")
        fh.write(f"\t\t{al:.6f}  {be:.6f}  {ga:.6f}  SPGR =  1 P 1\t\t OPT = 1\n")
        fh.write(f"{fw.n_atoms}  0\n0 {name}\t: {name}\n")
        for i, (xyz, ty) in enumerate(zip(fw.frac, fw.types)):
            fh.write(f" {i + 1} {labels[ty]} {xyz[0]:.17g} {xyz[1]:.17g} {xyz[2]:.17g}"
                     "  0  0  0  0  0  0  0  0  0.000000\n")
    probe = fw.probe
    from emptyroom_b200.synth import PROBES
    with open(os.path.join(root, "data", "forcefields", ff_name + ".def"), "w") as fh:
        fh.write("[Atom] [epsilon (K)] [sigma (A)]\n")
        for lab, e, s in zip(labels, fw.type_eps, fw.type_sig):
            fh.write(f"{lab} {e:.17g} {s:.17g}\n")
        for p, (e, s) in PROBES.items():
            fh.write(f"{p} {e} {s}\n")
    masses = {"Zn": 65.38, "O": 15.999, "C": 12.011, "H": 1.008, "N": 14.007, "Cu": 63.546,
              "Al": 26.982, "Si": 28.085, "CH4": 16.04, "Xe": 131.293, "Kr": 83.798}
    with open(os.path.join(root, "data", "masses.def"), "w") as fh:
        fh.write("[atom] [mass]\n")
        for k, v in masses.items():
            fh.write(f"{k} {v}\n")
    rcut = fw.rc if rc is None else rc
    t, _, _ = er.cell_matrices(a, b, c, al, be, ga)
    rep = er.replication_factors(t, rcut)
    with open(os.path.join(root, "data", "uc_replications", name + "_once.uc"), "w") as fh:
        fh.write(f"{rep[0]} {rep[1]} {rep[2]}\n")
    with open(os.path.join(root, "simulation.input"), "w") as fh:
        fh.write(f"Forcefield {ff_name} # store as .def\n\n")
        fh.write(f"GridResolution {resolution} A\nCutoffRadius {rcut} A\n")
        fh.write(f"GridOutputFormat {fmt}\nFeynmanHibbs 0\nTemperature {temperature} K\n")
        fh.write(f"NumberOfInsertionsPerA3 {insertions_per_a3}\nverbosemode 0\n")
    return name, probe


def particles_from_tree(root, name, ff_name, adsorbate):
    from emptyroom_b200 import files
    s = files.Structure(root, name)
    f = files.Forcefield(root, ff_name)
    eg, sg = f.find(adsorbate)
    return s, files.mix_particles(s, f, eg, sg), files.read_uc(root, name, "once")


def read_out(path):
    """.out lines without the date and timing lines."""
    skip = ("date:", "    Time to write grid", "    Simulation time")
    return [ln for ln in open(path).read().splitlines() if not ln.startswith(skip)]


def grid_file_values(path):
    from emptyroom_b200 import files
    return files.read_grid_txt(path)


def as_float_grid(values):
    return np.asarray(values, dtype=np.float64)
