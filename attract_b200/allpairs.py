"""Explicit all-pairs rescoring (no grids): the reference's test-energy.py:46-58,
ATTRACT ``--score`` with an optional ``--rcut``.

Every ligand bead interacts with every receptor bead through the plain ATTRACT
pair potential of the force field (no plateau shift); ``rcut`` drops pairs at
or beyond that distance.  Poses are ``[B, 6]`` Euler + translation or
``[B, 4, 4]`` row-vector matrices; the optional gradient is dE/d(Euler, t) or
dE/dmat accordingly.
"""
from __future__ import annotations

import numpy as np
import torch

from . import _lib
from .engine import _stream, _used_on
from .forcefield import ForceField
from .grid import _dev, pack_receptor


class AllPairs:
    """A receptor and one ligand resident on the device for repeated rescoring."""

    def __init__(self, rec_xyz, rec_type, lig_xyz, lig_type, ff: ForceField, device=None):
        self.device = _dev(device)
        rec_type = np.asarray(rec_type, np.int64).reshape(-1)
        lig_type = np.asarray(lig_type, np.int64).reshape(-1)
        if len(rec_type) and (rec_type.min() < 0 or rec_type.max() >= ff.n_rtypes):
            raise ValueError("receptor type outside the force field")
        if len(lig_type) == 0 or lig_type.min() < 0 or lig_type.max() >= ff.n_ltypes:
            raise ValueError("ligand type outside the force field (or no ligand beads)")
        self.n_rec = len(rec_type)
        # receptor beads grouped by type: the kernel reloads a pair-table row
        # only when the receptor type changes (the sum does not depend on the order)
        order = np.argsort(rec_type, kind="stable")
        self.rec = pack_receptor(np.asarray(rec_xyz, np.float64).reshape(-1, 3)[order], rec_type[order], self.device)
        self.lig = pack_receptor(lig_xyz, lig_type, self.device)
        self.n_lig = len(lig_type)
        self.ff = ff
        self.pair = torch.from_numpy(ff.pair_table(1.0, shift_plateau=False)).to(self.device)

    def energy(self, poses: torch.Tensor, rcut: float | None = None, grad: bool = False, stream=None):
        """``(E [B], gradient or None)`` for ``poses`` on the device."""
        mat = poses.dim() == 3 or (poses.dim() == 2 and poses.shape[1] == 16)
        p2 = poses.reshape(len(poses), 16 if mat else 6)
        if p2.device != self.device or p2.dtype != torch.float32 or not p2.is_contiguous():
            raise ValueError("poses must be a contiguous float32 tensor on the receptor's device")
        B = len(p2)
        E = torch.empty(B, dtype=torch.float32, device=self.device)
        G = torch.empty((B, 16 if mat else 6), dtype=torch.float32, device=self.device) if grad else None
        rc = _lib.load().att_allpairs_energy(_lib.ptr(self.rec) if self.n_rec else None, self.n_rec,
                                             _lib.ptr(self.lig), self.n_lig, _lib.ptr(p2), B, 1 if mat else 0,
                                             _lib.ptr(self.pair), self.ff.n_rtypes, self.ff.n_ltypes,
                                             float(rcut or 0.0), _lib.ptr(E), _lib.ptr(G), _stream(stream))
        _lib.check(rc, "att_allpairs_energy")
        _used_on(stream, p2, E, G)
        if G is not None and mat:
            G = G.view(B, 4, 4)
        return E, G


def allpairs_energy(rec_xyz, rec_type, lig_xyz, lig_type, poses, ff: ForceField, rcut=None, grad=False,
                    device=None):
    """One-shot all-pairs energies (and gradients) of ``poses`` (NumPy or torch)."""
    ap = AllPairs(rec_xyz, rec_type, lig_xyz, lig_type, ff, device)
    P = torch.as_tensor(np.asarray(poses, np.float32) if not isinstance(poses, torch.Tensor) else poses,
                        dtype=torch.float32).to(ap.device).contiguous()
    return ap.energy(P, rcut, grad)
