"""Generate the golden fixtures under tests/golden from the reference's own data.

Run once where a checkout of the reference exists, giving its path; the GPU
box and the test suite only read the committed ``.npz`` outputs.

    python tests/golden/make_golden.py /path/to/attract-jax

Sources (all from sjdv1982/attract-jax):
* energy-init/make-energy-init.out + energy-init/score.out: 296 single-pair
  distances and the ATTRACT energies for type 15-15 (energy-init/energy-init.py).
* attract-original/attract.par: the type 15-15 parameters (rbc, abc, ipon).
* mono-leu/mono-leuc-pdb.npy: 1275 beads, all ATTRACT type 15 (receptor = ligand).
* mono-leu/minim-sorted.dat: Euler poses (receptor line, ligand line) and the
  ATTRACT scores computed from them: minim-sorted.score (all pairs,
  --rcut 9999999) and minim-sorted-nbgrid.score (neighbour grid only, plateau
  5 A: energies and gradients), mono-leu/dock.sh:13-30.
* mono-leu/minim-sorted.npy: the reference scripts' 4x4 poses; the first ten
  give the JAX outputs test-nb-energrad.out (no plateau shift) and
  test-nb-energrad-plateau.out (test5 plateau semantics): energies,
  -dE/dt and -dE/dmat[:3,:3].
"""
from __future__ import annotations

import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
N_POSES = 64


def parse_dat(fn):
    poses, cur = [], None
    for line in open(fn):
        if line.startswith("#"):
            if re.match(r"#\d+$", line.strip()):
                cur = []
                poses.append(cur)
            continue
        if cur is not None and line.strip():
            cur.append([float(x) for x in line.split()])
    return poses


def parse_score(fn):
    E, G = [], []
    for line in open(fn):
        if line.startswith(" Energy:"):
            E.append(float(line.split()[1]))
        elif line.startswith(" Gradients:"):
            G.append([float(x) for x in line.split()[1:]])
    return np.array(E), np.array(G)


def parse_out(fn):
    """Energies / translational / torque blocks printed by the JAX scripts."""
    text = open(fn).read()
    num = r"[-+]?\d+\.?\d*(?:[eE][-+]?\d+)?"

    def block(title, nxt):
        s = text.index(title) + len(title)
        e = text.index(nxt, s) if nxt else len(text)
        return np.array([float(x) for x in re.findall(num, text[s:e])])

    E = block("Energies:", "Gradients (translational):")
    T = block("Gradients (translational):", "Gradients (torque):").reshape(-1, 3)
    tail = text[text.index("Gradients (torque):"):]
    stop = tail.find("Run argsort")
    R = np.array([float(x) for x in re.findall(num, tail[len("Gradients (torque):"):stop if stop > 0 else None])])
    return E, T, R.reshape(-1, 3, 3)


def main(ref):
    out = {}
    # energy-init single pair known answers
    dis = np.array([float(x) for x in open(os.path.join(ref, "energy-init/make-energy-init.out"))])
    ene = np.array([float(x.split()[1]) for x in open(os.path.join(ref, "energy-init/score.out"))])
    assert len(dis) == len(ene)
    out["pair_dist"] = dis
    out["pair_energy_attract"] = ene
    lines = open(os.path.join(ref, "attract-original/attract.par")).read().splitlines()
    ntypes = int(lines[0].split()[1])
    vals = np.array(" ".join(lines[1:]).split(), dtype=np.float64)[: 3 * ntypes * ntypes].reshape(3, ntypes, ntypes)
    out["par15"] = np.array([vals[0, 14, 14], vals[1, 14, 14], vals[2, 14, 14]])  # rbc, abc, ipon
    # mono-leu
    lig = np.load(os.path.join(ref, "mono-leu/mono-leuc-pdb.npy"))
    out["beads"] = np.stack([lig["x"], lig["y"], lig["z"]], 1).astype(np.float64)
    out["bead_type"] = lig["occupancy"].astype(np.int32)
    dat = parse_dat(os.path.join(ref, "mono-leu/minim-sorted.dat"))
    rec_pose = np.array([d[0] for d in dat[:N_POSES]])
    lig_pose = np.array([d[1] for d in dat[:N_POSES]])
    out["dat_receptor_pose"] = rec_pose
    out["dat_ligand_pose"] = lig_pose
    out["score_allpairs"] = np.loadtxt(os.path.join(ref, "mono-leu/minim-sorted.score"))[:N_POSES]
    e, g = parse_score(os.path.join(ref, "mono-leu/minim-sorted-nbgrid.score"))
    out["score_nbgrid_energy"] = e[:N_POSES]
    out["score_nbgrid_grad"] = g[:N_POSES]
    out["mat10"] = np.load(os.path.join(ref, "mono-leu/minim-sorted.npy"))[:10]
    for name, key in (("test-nb-energrad.out", "jax_nb"), ("test-nb-energrad-plateau.out", "jax_nbplat")):
        E, T, R = parse_out(os.path.join(ref, name))
        out[key + "_energy"] = E
        out[key + "_negdt"] = T
        out[key + "_negdM"] = R
    np.savez_compressed(os.path.join(HERE, "attract_ref_golden.npz"), **out)
    print("wrote", os.path.join(HERE, "attract_ref_golden.npz"), {k: v.shape for k, v in out.items()})


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit(f"usage: python {sys.argv[0]} <path of the attract-jax checkout>")
    main(sys.argv[1])
