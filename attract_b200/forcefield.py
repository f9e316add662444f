"""ATTRACT force-field tables (test5.py:122-146; attract-original/convert-attract-par.py).

A force field is the receptor-major triple ``rc, ac, ivor [n_rtypes, n_ltypes]``
of the reference's ``ff`` namedtuple, plus an optional per-pair energy cap.
The kernels read a per-grid pair table ``[n_ltypes][n_rtypes][8]`` =
``rc, ac, emin, rmin2, ivor, eplat, gplat, rcap2`` where emin/rmin2 follow
test5.py:132-133 and eplat/gplat are the plateau energy and d/d(d^2) of the
pair potential at the grid's plateau distance (test5.py:208-211).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np


def _nonbon(dsq, rc, ac, emin, rmin2, ivor, rcap2):
    d = np.maximum(dsq, rcap2)
    rr2 = 1.0 / d
    vlj = (rc * rr2 - ac) * rr2 ** 3
    return np.where(d < rmin2, vlj + (ivor - 1.0) * emin, ivor * vlj)


def _dnonbon(dsq, rc, ac, emin, rmin2, ivor, rcap2):
    d = np.maximum(dsq, rcap2)
    rr2 = 1.0 / d
    dv = rr2 ** 4 * (3.0 * ac - 4.0 * rc * rr2)
    g = np.where(d < rmin2, dv, ivor * dv)
    return np.where(dsq < rcap2, 0.0, g)


@dataclass
class ForceField:
    rc: np.ndarray      # [n_rtypes, n_ltypes]
    ac: np.ndarray
    ivor: np.ndarray
    rcap2: np.ndarray | None = None

    def __post_init__(self):
        self.rc = np.asarray(self.rc, np.float64)
        self.ac = np.asarray(self.ac, np.float64)
        self.ivor = np.asarray(self.ivor, np.float64)
        if self.rc.ndim != 2 or self.rc.shape != self.ac.shape or self.rc.shape != self.ivor.shape:
            raise ValueError("rc, ac, ivor must share one [n_rtypes, n_ltypes] shape")
        if np.any(self.rc <= 0) or np.any(self.ac <= 0):
            raise ValueError("rc and ac must be positive")
        if not np.all(np.isin(self.ivor, (-1.0, 1.0))):
            raise ValueError("ivor must be +1 or -1 (convert-attract-par.py:14)")
        if self.rcap2 is None:
            self.rcap2 = np.zeros_like(self.rc)
        self.rcap2 = np.broadcast_to(np.asarray(self.rcap2, np.float64), self.rc.shape).copy()

    @property
    def n_rtypes(self) -> int:
        return self.rc.shape[0]

    @property
    def n_ltypes(self) -> int:
        return self.rc.shape[1]

    def pair_table(self, plateau: float, shift_plateau: bool = True) -> np.ndarray:
        """float32 ``[n_ltypes, n_rtypes, 8]`` for a grid with this plateau distance.

        ``shift_plateau=False`` zeroes eplat/gplat: the pair term is then the plain
        nonbon of test-nb-energrad.py:143-146 (a neighbour grid without potentials).
        """
        rc, ac, iv, cap = self.rc, self.ac, self.ivor, self.rcap2
        emin = -27.0 * ac ** 4 / (256.0 * rc ** 3)
        rmin2 = 4.0 * rc / (3.0 * ac)
        p2 = float(plateau) ** 2
        if shift_plateau:
            ep = _nonbon(p2, rc, ac, emin, rmin2, iv, cap)
            gp = _dnonbon(p2, rc, ac, emin, rmin2, iv, cap)
        else:
            ep = np.zeros_like(rc)
            gp = np.zeros_like(rc)
        t = np.stack([rc, ac, emin, rmin2, iv, ep, gp, cap], -1)
        return np.ascontiguousarray(np.transpose(t, (1, 0, 2))).astype(np.float32)

    @classmethod
    def from_attract_par(cls, text: str, rec_types=None, lig_types=None) -> "ForceField":
        """Parse ``attract.par`` (potshape 8) and slice to the ATTRACT type numbers
        present, 1-based as in test5.py:128-130.  Without a selection all types
        are kept (index = ATTRACT type - 1)."""
        lines = text.splitlines()
        head = lines[0].split() if lines else []
        if len(head) < 2:
            raise ValueError("attract.par: the first line must hold potshape and the number of types")
        potshape, ntypes = int(head[0]), int(head[1])
        if potshape != 8:
            raise ValueError(f"potshape {potshape} not supported (coarse-grained ATTRACT uses 8)")
        if ntypes < 1:
            raise ValueError(f"attract.par: {ntypes} types")
        vals = np.array(" ".join(lines[1:]).split(), dtype=np.float64)
        if len(vals) < 3 * ntypes * ntypes:
            raise ValueError(f"attract.par: {len(vals)} values, {3 * ntypes * ntypes} expected for {ntypes} types")
        par = vals[: 3 * ntypes * ntypes].reshape(3, ntypes, ntypes)
        rbc, abc, ipon = par
        rc = abc * rbc ** 8
        ac = abc * rbc ** 6
        sel_r = np.arange(ntypes) if rec_types is None else np.asarray(rec_types) - 1
        sel_l = np.arange(ntypes) if lig_types is None else np.asarray(lig_types) - 1
        for name, sel in (("receptor", sel_r), ("ligand", sel_l)):
            if sel.size and (sel.min() < 0 or sel.max() >= ntypes):
                raise ValueError(f"attract.par: {name} types outside 1..{ntypes}")
        return cls(rc[np.ix_(sel_r, sel_l)], ac[np.ix_(sel_r, sel_l)], ipon[np.ix_(sel_r, sel_l)])

    @classmethod
    def from_eps_sigma(cls, eps, sigma, cap_sigma_frac: float | None = 0.6) -> "ForceField":
        """E = eps*((sigma/r)^8 - (sigma/r)^6): rc = eps*sigma^8, ac = eps*sigma^6,
        ivor = 1; optional energy cap below cap_sigma_frac*sigma."""
        eps = np.asarray(eps, np.float64)
        sigma = np.asarray(sigma, np.float64)
        cap = None if cap_sigma_frac is None else (cap_sigma_frac * sigma) ** 2
        return cls(eps * sigma ** 8, eps * sigma ** 6, np.ones_like(eps), cap)

    @classmethod
    def synthetic(cls, n_types: int = 32, seed: int = 0, cap_sigma_frac: float | None = 0.6) -> "ForceField":
        """Random symmetric per-type-pair parameters: sigma U(3,5) A, eps U(0.1,2) kcal/mol."""
        rng = np.random.default_rng(seed)
        s = rng.uniform(3.0, 5.0, (n_types, n_types))
        e = rng.uniform(0.1, 2.0, (n_types, n_types))
        s = np.triu(s) + np.triu(s, 1).T
        e = np.triu(e) + np.triu(e, 1).T
        return cls.from_eps_sigma(e, s, cap_sigma_frac)
