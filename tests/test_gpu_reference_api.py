"""The reference's call surface (attract_b200.reference_api: main, vgrad_main,
minimise_schema) against the oracle's restatement of test5.py, with the
receptor grid passed the reference's way: ATTRACT .grid bytes read by
read_grid(data, read_gradients=True).

Parity of the scorer is reported as in test_gpu_parity.py: the fraction of
poses within the north-star tolerance (energies 1e-5 relative or 1e-4
kcal/mol, gradients 1e-4 relative), every other pose within the counted
float32 bound of gpu_cases.float32_bounds (the force field is uncapped, as
the reference's is, so clashes reach large energies).  dE/dq sums the 9
entries of dE/dR times entries of 2|q| <= 2: its bound is 6 times the Euler
rotation bound."""
import numpy as np
import pytest
import torch

import attract_oracle as O
from gpu_cases import float32_bounds, north_star_report, oracle_scales, small_case

pytestmark = pytest.mark.gpu


def _setup(seed=60, n_poses=64):
    from scipy.spatial.transform import Rotation

    from attract_b200 import load_library
    from attract_b200.gridfile import read_grid, write_grid
    from attract_b200.reference_api import make_ff

    load_library()
    c = small_case(seed=seed, n_poses=n_poses, cap=False)  # the reference's force field has no cap
    G, g = c["G"], c["G"]["geom"]
    alphabet = np.zeros(99, bool)
    alphabet[[2, 7, 11, 20][: c["n_types"]]] = True
    data = write_grid(gridspacing=g["spacing"], gridextension=g["extension"], plateaudis=g["plateau"],
                      neighbourdis=g["plateau"] + 1.0, alphabet=alphabet, origin=g["origin"], dim=g["dim"],
                      dim2=g["dim2"], natoms=len(G["rec"]), inner_potential_grid=G["inner"],
                      outer_potential_grid=G["outer"], nb_hdr=G["nb_hdr"], nb_list=G["nb_list"])
    grid = read_grid(data, read_gradients=True)
    rng = np.random.default_rng(seed + 1)
    lig2 = c["lig"] + rng.normal(scale=0.3, size=c["lig"].shape).astype(np.float32)
    confs = np.stack([c["lig"], lig2])
    conformers = rng.integers(0, 2, n_poses)
    q = Rotation.from_matrix(O.pose_to_mat(c["poses"])[:, :3, :3]).as_quat()
    t = c["poses"][:, 3:6].copy()
    args = dict(coor_rec=G["rec"].astype(np.float32), rec_atomtypes=G["rtype"], coor_lig=confs.astype(np.float32),
                lig_atomtypes=c["lt"], conformers=conformers, lig_atomtype_pos=c["gt"],
                ff=make_ff(c["rc"], c["ac"], c["ivor"]), grid=grid)
    es = np.zeros(n_poses)
    gs = np.zeros(n_poses)
    for k in (0, 1):
        e, s = oracle_scales(dict(c, lig=confs[k]), c["poses"], position_term=True)
        es = np.where(conformers == k, e, es)
        gs = np.where(conformers == k, s, gs)
    es = es + 0.1 * (t * t).sum(1)
    return c, q, t, confs, conformers, args, es, gs


@pytest.fixture(scope="module")
def setup():
    return _setup()


def _bounds(c, confs, conformers, t, gravity):
    """float32 bounds per pose (its conformer), plus the gravity term's rounding."""
    n = len(conformers)
    bE, bR, bT = np.zeros(n), np.zeros(n), np.zeros(n)
    for k in range(len(confs)):
        sel = conformers == k
        b = float32_bounds(c["poses"], confs[k].astype(np.float64), c["gt"], c["lt"], c["G"], "reference")
        bE[sel], bR[sel], bT[sel] = b[0][sel], b[1][sel], b[2][sel]
    t2 = (t * t).sum(1)
    return bE + 8 * 2.0 ** -24 * gravity * t2, 6 * bR, bT + 16 * 2.0 ** -24 * gravity * np.sqrt(t2)


def test_vgrad_main_matches_oracle(setup):
    from attract_b200.reference_api import vgrad_main

    c, q, t, confs, conformers, args, es, gs = setup
    (tot, E), (gq, gt) = vgrad_main(q, t, **args, gravity=True)
    E, gq, gt = E.cpu().numpy(), gq.cpu().numpy(), gt.cpu().numpy()
    Eo, gqo, gto = O.energrad_quat(q, t, confs, conformers, c["gt"], c["lt"], c["G"], gravity=0.1)
    bE, bR, bT = _bounds(c, confs, conformers, t, 0.1)
    north_star_report("vgrad_main (quaternions, conformers, gravity)", E, np.concatenate([gq, gt], 1), Eo,
                      np.concatenate([gqo, gto], 1), (bE, bR, bT))
    assert abs(float(tot) - Eo.sum()) <= max(1e-5 * abs(Eo.sum()), bE.sum())


def test_main_matrices_and_no_gravity(setup):
    from scipy.spatial.transform import Rotation

    from attract_b200.reference_api import main

    c, q, t, confs, conformers, args, es, gs = setup
    R = Rotation.from_quat(q).as_matrix()
    tot, E = main(R, t, **args, gravity=False)
    Eo, _, _ = O.energrad_quat(q, t, confs, conformers, c["gt"], c["lt"], c["G"], gravity=0.0)
    north_star_report("main (rotation matrices, no gravity)", E.cpu().numpy(), None, Eo, None,
                      _bounds(c, confs, conformers, t, 0.0))


def test_single_conformer_and_errors(setup):
    from attract_b200.reference_api import main, vgrad_main

    c, q, t, confs, conformers, args, es, gs = setup
    one = dict(args, coor_lig=confs[0], conformers=None)
    _, E = main(q, t, **one, gravity=True)
    zero = np.zeros(len(q), int)
    Eo, _, _ = O.energrad_quat(q, t, confs[:1], zero, c["gt"], c["lt"], c["G"], gravity=0.1)
    north_star_report("main (one conformer)", E.cpu().numpy(), None, Eo, None, _bounds(c, confs[:1], zero, t, 0.1))
    with pytest.raises(AssertionError):
        main(q, t[:-1], **args, gravity=True)  # test5.py:412
    with pytest.raises(AssertionError):
        main(q, t, **dict(args, conformers=np.full(len(q), 2)), gravity=True)
    with pytest.raises(AssertionError):
        vgrad_main(np.zeros((len(q), 3, 3)), t, **args, gravity=True)


def test_schema_minimisation_reproduces_the_oracle_ranking():
    """A shortened SCHEMA (two stages, gravity then none) on poses without
    deep clashes: the float32 CUDA path follows the float64 oracle's
    trajectories, so final energies and their ranking agree."""
    from scipy.stats import spearmanr

    from attract_b200.reference_api import minimise_schema

    c, q, t, confs, conformers, args, es, gs = _setup(seed=61, n_poses=96)
    Eo0, _, _ = O.energrad_quat(q, t, confs, conformers, c["gt"], c["lt"], c["G"])
    keep = Eo0 < 1e3  # start outside deep clashes, where the uncapped 8-6 term is steep
    q, t, conformers = q[keep], t[keep], conformers[keep]
    args = dict(args, conformers=conformers)
    schema = ((4, 0.5, True), (6, 0.05, False))
    qg, tg, Eg = minimise_schema(q, t, **args, schema=schema)
    qo, to, Eo = O.minimise_schema(q, t, confs, conformers, c["gt"], c["lt"], c["G"], schema)
    Eg = Eg.cpu().numpy()
    assert np.all(np.isfinite(Eg))
    rho = spearmanr(Eg, Eo)[0]
    assert rho > 0.98, rho
    close = np.abs(Eg - Eo) <= 1e-3 * np.abs(Eo) + 1e-2
    assert close.mean() >= 0.9, close.mean()


def test_fused_schema_kernel_matches_the_per_epoch_path():
    """att_minimise_schema (the whole protocol in one launch) against the
    per-epoch path (one energy/gradient launch per epoch, adabelief in torch
    ops): the same float32 arithmetic in a different order, so the
    trajectories agree closely; every stage boundary (fresh optimiser state,
    gravity switched off) is crossed."""
    from attract_b200.reference_api import minimise_schema

    c, q, t, confs, conformers, args, es, gs = _setup(seed=62, n_poses=64)
    Eo0, _, _ = O.energrad_quat(q, t, confs, conformers, c["gt"], c["lt"], c["G"])
    keep = Eo0 < 1e3
    q, t = q[keep], t[keep]
    args = dict(args, conformers=conformers[keep])
    schema = ((3, 0.5, True), (0, 1.0, True), (4, 0.1, False), (3, 0.02, False))
    qf, tf, Ef = minimise_schema(q, t, **args, schema=schema, fused=True)
    qh, th, Eh = minimise_schema(q, t, **args, schema=schema, fused=False)
    qf, tf, Ef = qf.cpu().numpy(), tf.cpu().numpy(), Ef.cpu().numpy()
    qh, th, Eh = qh.cpu().numpy(), th.cpu().numpy(), Eh.cpu().numpy()
    assert np.allclose(np.linalg.norm(qf, axis=1), 1.0, atol=1e-5)
    same = (np.abs(tf - th).max(1) < 1e-3) & (np.minimum(np.abs(qf - qh), np.abs(qf + qh)).max(1) < 1e-3)
    assert same.mean() >= 0.9, same.mean()
    assert np.all(np.abs(Ef - Eh)[same] <= 1e-3 * np.abs(Eh[same]) + 1e-2)
