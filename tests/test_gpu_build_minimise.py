"""GPU builders (K3/K4/K5), the fused minimiser and batching against the oracle."""
import numpy as np
import pytest
import torch

import attract_oracle as O
from gpu_cases import small_case, to_device_grid

pytestmark = pytest.mark.gpu


def _A():
    import attract_b200 as A

    A.load_library()
    return A


def _small_receptor(seed=0, n=40, n_types=4):
    A = _A()
    rng = np.random.default_rng(seed)
    ff = A.ForceField.synthetic(n_types, seed)
    geom = A.GridGeom((-8.0, -7.5, -7.0), 1.0, (17, 16, 15), (12, 12, 11), 4, 3.0, n_types)
    xyz = rng.uniform(-5, 5, (n, 3)).astype(np.float32).astype(np.float64)
    t = rng.integers(0, n_types, n)
    return A, ff, geom, xyz, t


def test_potential_grid_builder_vs_oracle():
    A, ff, geom, xyz, t = _small_receptor()
    g = A.Grid.build(xyz, t, ff, geom, cutoff=6.0, keep_dense=True)
    inner, outer, _, _ = g.dense_host()
    pair = O.pair_table(ff.rc, ff.ac, ff.ivor, geom.plateau, True, ff.rcap2)
    gd = geom.as_dict()
    ref_in = O.build_potential_grid(xyz, t, pair, gd, geom.n_types, 6.0, outer=False)
    ref_out = O.build_potential_grid(xyz, t, pair, gd, geom.n_types, 6.0, outer=True)
    for got, ref in ((inner, ref_in), (outer, ref_out)):
        scale = np.abs(ref).max(axis=(1, 2, 3), keepdims=True)
        # grid points exactly at the cutoff radius are the only float32/float64 disagreements
        bad = np.abs(got - ref) > 1e-6 * scale + 1e-6
        assert bad.mean() < 1e-4, bad.mean()


def _device_lists(g):
    """The grid's neighbour lists as the kernels read them (receptor beads
    named by device position) and the device-order float32 receptor."""
    hdr = g.nb_hdr.cpu().numpy().view(np.uint32)
    lst = g.nb_list.cpu().numpy().view(np.uint16)
    rec = g.rec.cpu().numpy()[: g.n_rec, :3]
    return hdr, lst, rec


def _f32_lists(g, rec32, radius):
    c = g.nb_geom.to_c()
    return O.build_nbgrid_f32(rec32, np.array(c.origin[:], np.float32), c.spacing, c.dim[:], np.float32(radius))


def test_nbgrid_builder_vs_oracle():
    """Neighbour lists are index work: the GPU builder's lists equal, bit for
    bit, the oracle's float32 restatement of the same membership test; and
    that restatement differs from the float64 lists only for pairs within
    float32 rounding of the radius."""
    A, ff, geom, xyz, t = _small_receptor(seed=1)
    radius = 3.0 + np.sqrt(3) / 2 + 0.01
    g = A.Grid.build(xyz, t, ff, geom, list_radius=radius, potentials=False, nb_refine=1)
    hdr, lst, rec32 = _device_lists(g)
    ref_hdr, ref_lst = _f32_lists(g, rec32, radius)
    assert np.array_equal(hdr, ref_hdr)
    assert np.array_equal(lst[: len(ref_lst)], ref_lst)
    # the float32 test against the exact one (caller order, float64)
    _, _, h64, l64 = g.dense_host()
    ref_hdr64, ref_lst64 = O.build_nbgrid(xyz, geom.as_dict(), radius)
    if not (np.array_equal(h64, ref_hdr64) and np.array_equal(l64[: len(ref_lst64)], ref_lst64)):
        pts = O.grid_points(geom.as_dict()).reshape(-1, 3)
        d = np.linalg.norm(pts[:, None, :] - xyz[None], axis=2)
        got = np.zeros_like(d, dtype=bool)
        for v in range(len(h64)):
            s0, n = h64[v]
            got[v, l64[s0:s0 + n]] = True
        mismatch = got != (d <= radius)
        assert np.all(np.abs(d[mismatch] - radius) < 1e-4)


@pytest.mark.parametrize("refine", [2, 4])
def test_refined_list_grid_finds_the_same_pairs(refine):
    """Lists on the inner grid refined 2x / 4x per axis (radius plateau + the
    refined half-diagonal): the refined builder matches the oracle's lists on
    the refined points, holds fewer entries per lookup, and the energies and
    gradients equal those of the unrefined lists and the oracle's."""
    A, ff, geom, xyz, t = _small_receptor(seed=2)
    g1 = A.Grid.build(xyz, t, ff, geom, cutoff=6.0, nb_refine=1, keep_dense=True)
    gr = A.Grid.build(xyz, t, ff, geom, cutoff=6.0, nb_refine=refine)
    fine = geom.refined(refine)
    radius = geom.plateau + fine.spacing * np.sqrt(3) / 2 + 1e-3
    dh, dl, rec32 = _device_lists(gr)
    ref_dh, ref_dl = _f32_lists(gr, rec32, radius)
    assert np.array_equal(dh, ref_dh) and np.array_equal(dl[: len(ref_dl)], ref_dl)  # bit-exact
    _, _, hdr, lst = gr.dense_host()
    ref_hdr, ref_lst = O.build_nbgrid(xyz, fine.as_dict(), radius)
    assert hdr.shape == ref_hdr.shape
    pts = O.grid_points(fine.as_dict()).reshape(-1, 3)
    for v in np.flatnonzero(hdr[:, 1] != ref_hdr[:, 1]):  # float64 vs float32: only rounding at the radius
        d = np.linalg.norm(pts[v] - xyz, axis=1)
        got = set(lst[hdr[v, 0]:hdr[v, 0] + hdr[v, 1]].tolist())
        want = set(np.flatnonzero(d <= radius).tolist())
        assert all(abs(d[j] - radius) < 1e-4 for j in got ^ want)
    rng = np.random.default_rng(5)
    lig = rng.normal(size=(12, 3)) * 1.6
    lt = rng.integers(0, geom.n_types, 12)
    poses = np.concatenate([rng.uniform(-np.pi, np.pi, (96, 3)), rng.uniform(-4, 4, (96, 3))], 1)
    P = torch.tensor(poses, dtype=torch.float32, device="cuda")
    out = []
    for g in (g1, gr):
        wl = A.Workload([g], A.LigandSet([(lig, lt, lt)]), [A.Segment(0, 0, 96)], lanes_per_pose=32)
        E, Gd, _ = A.energrad(wl, P)
        _, _, _, st = A.minimise(wl, P, 1, stats=True)
        out.append((E.cpu().numpy(), Gd.cpu().numpy(), st.cpu().numpy()))
    (E1, G1, s1), (Er, Gr, sr) = out
    scale = np.abs(E1) + 1.0
    assert np.all(np.abs(Er - E1) <= 2e-5 * scale)
    assert np.all(np.abs(Gr - G1) <= 2e-4 * (np.abs(G1) + 1.0))
    assert sr[2] < s1[2]  # fewer list entries visited
    inner, outer, h1, l1 = g1.dense_host()
    Go = dict(geom=dict(geom.as_dict(), nb_refine=refine), inner=inner.astype(np.float64),
              outer=outer.astype(np.float64), nb_hdr=hdr, nb_list=lst, rec=xyz, rtype=t,
              pair=O.pair_table(ff.rc, ff.ac, ff.ivor, geom.plateau, True, ff.rcap2))
    Eo, _ = O.energrad(poses.astype(np.float32).astype(np.float64), np.asarray(lig, np.float32).astype(np.float64),
                       lt, lt, Go)
    assert np.all(np.abs(Er - Eo) <= 2e-5 * (np.abs(Eo) + 1.0))


def test_repack_bricks_exact():
    A = _A()
    c = small_case(seed=11, n_poses=4)
    grid = to_device_grid(c)
    ref = O.repack_bricks(c["G"]["inner"].astype(np.float32), c["G"]["outer"].astype(np.float32))
    got = grid.bricks.cpu().numpy()
    assert got.shape == ref.shape
    assert np.array_equal(got, ref)


def _minimise_case(seed=12, n_poses=64, lanes=8):
    A = _A()
    c = small_case(seed=seed, n_poses=n_poses)
    grid = to_device_grid(c)
    ligs = A.LigandSet([(c["lig"], c["gt"], c["lt"])])
    wl = A.Workload([grid], ligs, [A.Segment(0, 0, n_poses)], lanes_per_pose=lanes)
    return A, c, wl


def test_minimise_one_step_matches_oracle():
    A, c, wl = _minimise_case()
    P = torch.tensor(c["poses"], dtype=torch.float32, device="cuda")
    out, E, S, _ = A.minimise(wl, P, 1)
    xo, Eo, fo = O.minimise(c["poses"], c["lig"], c["gt"], c["lt"], c["G"], 1)
    d = np.abs(out.cpu().numpy() - xo)
    # one ADAM step moves each DOF by ~lr*sign(g): a sign decided by float32
    # noise (|g| tiny) may flip; everything else agrees to float32 precision
    assert np.mean(d < 1e-4) > 0.97, np.mean(d < 1e-4)


def test_minimise_many_steps_ranking():
    A, c, wl = _minimise_case(seed=13, n_poses=128)
    P = torch.tensor(c["poses"], dtype=torch.float32, device="cuda")
    out, E, S, _ = A.minimise(wl, P, 40)
    xo, Eo, fo = O.minimise(c["poses"], c["lig"], c["gt"], c["lt"], c["G"], 40)
    E = E.cpu().numpy()
    assert np.all(np.isfinite(E))
    from scipy.stats import spearmanr

    assert spearmanr(E, Eo).correlation > 0.98
    close = np.abs(E - Eo) <= 1e-3 * np.maximum(np.abs(Eo), 1.0)
    assert close.mean() > 0.8, close.mean()
    # the energy reported is the energy of the pose returned
    Ef, _, _ = A.energrad(wl, out.contiguous())
    assert np.allclose(Ef.cpu().numpy(), E, rtol=1e-6, atol=1e-5)


def test_minimise_lanes_identical():
    res = []
    for lanes in (8, 16, 32):
        A, c, wl = _minimise_case(seed=14, n_poses=50, lanes=lanes)
        P = torch.tensor(c["poses"], dtype=torch.float32, device="cuda")
        out, E, _, _ = A.minimise(wl, P, 10)
        res.append((out.cpu().numpy(), E.cpu().numpy()))
    for o, e in res[1:]:
        assert np.allclose(o, res[0][0], rtol=1e-5, atol=1e-5)
        assert np.allclose(e, res[0][1], rtol=1e-4, atol=1e-4)


def test_minimise_resume_with_adam_state_is_exact():
    A, c, wl = _minimise_case(seed=15, n_poses=40)
    P = torch.tensor(c["poses"], dtype=torch.float32, device="cuda")
    full, Ef, _, _ = A.minimise(wl, P, 10)
    st = torch.zeros((40, 12), dtype=torch.float32, device="cuda")
    half, _, _, _ = A.minimise(wl, P, 5, adam_state=st)
    rest, Er, _, _ = A.minimise(wl, half.clone(), 5, A.AdamOptions(step0=5), adam_state=st)
    assert torch.equal(full, rest)
    assert torch.equal(Ef, Er)


def test_batched_uneven_equals_alone():
    """Many ligands of uneven sizes in one launch give bit-identical results to
    each ligand minimised alone."""
    A = _A()
    base = small_case(seed=16, n_poses=8)
    grid = to_device_grid(base)
    rng = np.random.default_rng(3)
    ligs, segs, poses = [], [], []
    for i, n in enumerate((3, 9, 17, 30)):
        lig = rng.normal(size=(n, 3)) * 1.5
        lig -= lig.mean(0)
        ligs.append((lig, rng.integers(0, 4, n), rng.integers(0, 4, n)))
        k = 5 + 7 * i
        segs.append(A.Segment(0, i, k))
        poses.append(small_case(seed=20 + i, n_poses=k)["poses"])
    L = A.LigandSet(ligs)
    wl = A.Workload([grid], L, segs)
    P = torch.tensor(np.concatenate(poses), dtype=torch.float32, device="cuda")
    out, E, _, _ = A.minimise(wl, P, 12)
    out, E = out.cpu().numpy(), E.cpu().numpy().copy()
    off = 0
    for i, s in enumerate(segs):
        wl1 = A.Workload([grid], A.LigandSet([ligs[i]]), [A.Segment(0, 0, s.n_poses)])
        o1, E1, _, _ = A.minimise(wl1, P[off:off + s.n_poses].contiguous(), 12)
        assert np.array_equal(o1.cpu().numpy(), out[off:off + s.n_poses])
        assert np.array_equal(E1.cpu().numpy(), E[off:off + s.n_poses])
        off += s.n_poses


def test_graph_capture_replay_matches_direct():
    A, c, wl = _minimise_case(seed=17, n_poses=64)
    plan = A.MinimisePlan(wl, 8)
    plan.pose_in.copy_(torch.tensor(c["poses"], dtype=torch.float32))
    out1, E1, _, _ = plan.run()
    o1, e1 = out1.clone(), E1.clone()
    plan.capture()
    for _ in range(2):
        out2, E2, _ = plan.replay()
    torch.cuda.synchronize()
    assert torch.equal(o1, out2) and torch.equal(e1, E2)


def test_side_stream_launches_equal_current_stream():
    """energrad / minimise / backward on a caller-given stream (a torch Stream
    or a raw handle) equal the current-stream results; the temporaries they
    allocate are recorded on that stream, so repeated launches whose buffers
    are dropped right away stay correct."""
    A, c, wl = _minimise_case(seed=18, n_poses=48)
    P = torch.tensor(c["poses"], dtype=torch.float32, device="cuda")
    E0, G0, _ = A.energrad(wl, P)
    o0, m0, _, _ = A.minimise(wl, P, 6)
    b0 = A.energrad_backward(wl, P, torch.ones(48, device="cuda"))
    side = torch.cuda.Stream()
    side.wait_stream(torch.cuda.current_stream())
    for s in (side, side.cuda_stream):
        for _ in range(3):  # every buffer of the earlier iterations is already released
            E1, G1, _ = A.energrad(wl, P, stream=s)
            o1, m1, _, _ = A.minimise(wl, P, 6, stream=s)
            b1 = A.energrad_backward(wl, P, torch.ones(48, device="cuda"), stream=s)
        side.synchronize()
        assert torch.equal(E0, E1) and torch.equal(G0, G1)
        assert torch.equal(o0, o1) and torch.equal(m0, m1) and torch.equal(b0, b1)


def test_minimise_stats_counts():
    A, c, wl = _minimise_case(seed=18, n_poses=32)
    P = torch.tensor(c["poses"], dtype=torch.float32, device="cuda")
    _, _, _, st = A.minimise(wl, P, 3, stats=True)
    st = st.cpu().numpy()
    n_lig = len(c["lig"])
    assert 0 < st[0] <= 4 * 32 * n_lig
    assert 0 < st[1] <= 4 * 32 * n_lig
    assert st[2] >= 0
    # copies only when a slot's brick / record changed: at least one per pose
    # and bead with data, at most one per evaluation
    assert 0 < st[3] <= st[0] and 0 < st[4] <= st[1]


def test_large_ligands_and_chunking():
    """Ligands up to 8 beads per lane (256 at 32 lanes per pose) and larger
    ones, evaluated in chunks, match the oracle; teams of one warp with
    different chunk counts (conformers of mixed size are not allowed, so mixed
    segments) also do."""
    A = _A()
    c = small_case(seed=19, n_poses=16)
    grid = to_device_grid(c)
    rng = np.random.default_rng(5)
    for n, lanes in ((200, 32), (64, 8), (33, 16), (65, 8), (300, 32), (150, 16)):
        lig = (rng.normal(size=(n, 3)) * 2.0).astype(np.float32).astype(np.float64)
        gt = rng.integers(0, 4, n)
        wl = A.Workload([grid], A.LigandSet([(lig, gt, gt)]), [A.Segment(0, 0, 16)], lanes_per_pose=lanes)
        P = torch.tensor(c["poses"], dtype=torch.float32, device="cuda")
        E, G, _ = A.energrad(wl, P)
        Eo, Go = O.energrad(c["poses"], lig, gt, gt, c["G"])
        assert np.allclose(E.cpu().numpy(), Eo, rtol=2e-5, atol=2e-3), (n, lanes)
    # one warp, teams with 1 and 3 chunks (8 lanes x 8 beads = 64 per chunk)
    ligs = [((rng.normal(size=(n, 3)) * 2.0).astype(np.float32).astype(np.float64), rng.integers(0, 4, n))
            for n in (20, 150)]
    wl = A.Workload([grid], A.LigandSet([(x, t, t) for x, t in ligs]), [A.Segment(0, 0, 3), A.Segment(0, 1, 5)],
                    lanes_per_pose=8)
    P = torch.tensor(c["poses"][:8], dtype=torch.float32, device="cuda")
    E, _, _ = A.minimise(wl, P, 2)[1], None, None
    for seg, (x, t), sl in ((0, ligs[0], slice(0, 3)), (1, ligs[1], slice(3, 8))):
        w1 = A.Workload([grid], A.LigandSet([(x, t, t)]), [A.Segment(0, 0, sl.stop - sl.start)], lanes_per_pose=8)
        E1 = A.minimise(w1, P[sl].contiguous(), 2)[1]
        assert torch.equal(E1, E[sl])


def test_zz_kernel_error_word_is_clear():
    """No kernel above set the device error word."""
    from attract_b200 import _lib

    torch.cuda.synchronize()
    assert _lib.kernel_status(clear=True) == 0


def test_record_size_does_not_change_results():
    """Neighbour records of 32 B (13 entries inline, the rest read from the CSR
    tail) and of 128 B (everything inline here) hold the same lists in the
    same order: identical results, bit for bit."""
    A = _A()
    c = small_case(seed=96, n_poses=48)
    res = []
    for rb in (32, 128):
        grid = to_device_grid(c)
        grid._pack_records(rec_bytes=rb)
        grid._att = None
        if rb == 32:
            assert int((grid.nb_hdr[:, 1] > 13).sum()) > 0
        wl = A.Workload([grid], A.LigandSet([(c["lig"], c["gt"], c["lt"])]), [A.Segment(0, 0, 48)],
                        lanes_per_pose=32)
        P = torch.tensor(c["poses"], dtype=torch.float32, device="cuda")
        out, E, _, _ = A.minimise(wl, P, 6)
        res.append((out.cpu().numpy(), E.cpu().numpy()))
    assert np.array_equal(res[0][0], res[1][0]) and np.array_equal(res[0][1], res[1][1])
