"""Shared pytest setup: the ``gpu`` marker, import paths and golden fixtures."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN = os.path.join(ROOT, "tests", "golden", "attract_ref_golden.npz")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built extension")


@pytest.fixture(scope="session")
def golden():
    return dict(np.load(GOLDEN))


def mono_leu_setup(g, plateau=5.0, spacing=1.5, shift_plateau=True):
    """Receptor = ligand = the mono-leu beads (ATTRACT type 15), an nbgrid that
    covers every bead within the plateau of the receptor, complete lists."""
    import attract_oracle as O

    rbc, abc, ipon = g["par15"]
    rc = np.array([[abc * rbc ** 8]])
    ac = np.array([[abc * rbc ** 6]])
    iv = np.array([[ipon]])
    pair = O.pair_table(rc, ac, iv, plateau, shift_plateau=shift_plateau)
    rec = g["beads"]
    pad = plateau + 2 * spacing
    origin = rec.min(0) - pad
    dim = np.ceil((rec.max(0) + pad - origin) / spacing).astype(int) + 2
    geom = dict(origin=origin, spacing=spacing, dim=dim, dim2=dim // 2 + 1, extension=0,
                plateau=plateau)
    hdr, lst = O.build_nbgrid(rec, geom, plateau + spacing * np.sqrt(3) / 2 + 1e-3)
    G = dict(geom=geom, nb_hdr=hdr, nb_list=lst, rec=rec, rtype=np.zeros(len(rec), np.int64), pair=pair)
    return G


def dat_poses(g):
    """Ligand poses of minim-sorted.dat relative to the (translated) receptor."""
    rp, lp = g["dat_receptor_pose"], g["dat_ligand_pose"]
    assert np.all(rp[:, :3] == 0)
    pose = lp.copy()
    pose[:, 3:] -= rp[:, 3:]
    return pose
