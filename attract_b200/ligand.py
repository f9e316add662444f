"""Ligands (rigid bead sets) resident on the device.

Each bead is one float4 ``x, y, z, type word`` with ``type word = gtype |
ltype << 16`` (int32 bits): ``gtype`` is the bead's potential-grid slot (the
reference's ``lig_atomtype_pos``, test5.py:144-146) and ``ltype`` its ligand
type in the pair table (``lig_atomtypes``, test5.py:104).  A conformer
ensemble (test5.py:58-87) is a set of ligands with equal bead counts.
"""
from __future__ import annotations

import numpy as np
import torch

from . import _lib
from .grid import _dev


class LigandSet:
    def __init__(self, ligands, device=None):
        """``ligands``: list of ``(xyz [N,3], gtype [N], ltype [N])`` (ltype may be None = gtype)."""
        if len(ligands) == 0:
            raise ValueError("no ligands")
        self.device = _dev(device)
        rows, offs, self.sizes = [], [0], []
        self.host = []
        for xyz, gt, lt in ligands:
            xyz = np.asarray(xyz, np.float64).reshape(-1, 3)
            gt = np.asarray(gt, np.int64).reshape(-1)
            lt = gt if lt is None else np.asarray(lt, np.int64).reshape(-1)
            if not (len(xyz) == len(gt) == len(lt)):
                raise ValueError("ligand coordinates and types differ in length")
            if len(xyz) == 0:
                raise ValueError("empty ligand")
            if gt.min() < 0 or gt.max() > 0xFFFF or lt.min() < 0 or lt.max() > 0x7FFF:
                raise ValueError("ligand types out of range")
            a = np.zeros((len(xyz), 4), np.float32)
            a[:, :3] = xyz
            a[:, 3] = (gt | (lt << 16)).astype(np.int32).view(np.float32)
            rows.append(a)
            offs.append(offs[-1] + len(xyz))
            self.sizes.append(len(xyz))
            self.host.append((xyz, gt, lt))
        self.beads = torch.from_numpy(np.concatenate(rows)).to(self.device)
        self.offset = torch.tensor(offs, dtype=torch.int32, device=self.device)
        self.max_gtype = max(int(h[1].max()) for h in self.host)
        self.max_ltype = max(int(h[2].max()) for h in self.host)
        self._att = None

    def __len__(self):
        return len(self.sizes)

    def att(self) -> _lib.AttLigands:
        if self._att is None:
            a = _lib.AttLigands()
            a.beads = _lib.ptr(self.beads)
            a.offset = _lib.ptr(self.offset)
            a.n_lig = len(self.sizes)
            a.max_beads = max(self.sizes)
            a.n_beads = int(sum(self.sizes))
            self._att = a
        return self._att
