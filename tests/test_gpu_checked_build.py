"""The bounds-checked build (-DATT_BOUNDS_CHECK; compute-sanitizer is not
available here): every grid, list and receptor index of the scoring kernels
is checked before its access.  On cases that reach every index path -- inner
and outer grids, neighbour lists that overflow their 32-byte records into the
CSR tail, dense lists that fill the pair buffers many times over, two
receptors and ligands of 5 to 60 beads in one launch, a chunked large ligand, the adjoint's grid scatter, the 4x4 and quaternion modes -- no
check fails, and the results equal the regular build's."""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)

SCRIPT = r'''
import json, sys
import numpy as np, torch
sys.path.insert(0, {root!r}); sys.path.insert(0, {tests!r}); sys.path.insert(0, {oracle!r})
import attract_b200 as A
from attract_b200 import _lib
from gpu_cases import small_case, to_device_grid
A.load_library()
c = small_case(seed=95, n_poses=64)
grid = to_device_grid(c)
grid._pack_records(rec_bytes=32)  # 13 inline entries: longer lists continue in the CSR tail
grid._att = None
rng = np.random.default_rng(4)
big = rng.normal(size=(70, 3)) * 2.5
ligs = A.LigandSet([(c["lig"], c["gt"], c["lt"]), (big, rng.integers(0, 4, 70), rng.integers(0, 4, 70))])
wl = A.Workload([grid], ligs, [A.Segment(0, 0, 64), A.Segment(0, 1, 16)], lanes_per_pose=8)
P = torch.tensor(np.concatenate([c["poses"], c["poses"][:16]]), dtype=torch.float32, device="cuda")
E, G, S = A.energrad(wl, P)
out, Em, Sm, st = A.minimise(wl, P, 5, stats=True)
di = torch.zeros((*grid.inner.shape[:4], 4), device="cuda"); do = torch.zeros((*grid.outer.shape[:4], 4), device="cuda")
dP = A.energrad_backward(wl, P, torch.ones(80, device="cuda"), A.EvalOptions(grad_mode="analytic"),
                         dgrid_inner=di, dgrid_outer=do)
mats = torch.tensor(__import__("attract_oracle").pose_to_mat(c["poses"]).reshape(64, 16), dtype=torch.float32,
                    device="cuda")
wl1 = A.Workload([grid], A.LigandSet([(c["lig"], c["gt"], c["lt"])]), [A.Segment(0, 0, 64)], lanes_per_pose=32)
Ex, Gx, _ = A.energrad(wl1, mats)
qt = torch.zeros((64, 8), device="cuda"); qt[:, 3] = 1.0; qt[:, 4:7] = P[:64, 3:6]
oq, Eq, _ = A.minimise_schema(wl1, qt, ((3, 0.1, True), (2, 0.05, False)))
# dense lists (~100 entries, mostly in the CSR tail): every team's pair buffer
# fills many times over, at 2 and 8 beads per lane
cd = small_case(seed=31, n_rec=400, n_lig_beads=60, n_poses=16)
gd = to_device_grid(cd)
Ed = []
for lanes in (32, 8):
    wd = A.Workload([gd], A.LigandSet([(cd["lig"], cd["gt"], cd["lt"])]), [A.Segment(0, 0, 16)], lanes_per_pose=lanes)
    Pd = torch.tensor(cd["poses"], dtype=torch.float32, device="cuda")
    Ed += A.energrad(wd, Pd)[0].cpu().tolist() + A.minimise(wd, Pd, 3)[1].cpu().tolist()
# two receptors in one launch (segments on either grid) and ligands of 5 to 60 beads,
# as the serving rounds launch them
c2 = small_case(seed=96, n_rec=120, n_poses=16)
g2 = to_device_grid(c2)
rngm = np.random.default_rng(8)
mix = [(rngm.normal(size=(n, 3)) * 2.0, rngm.integers(0, 4, n)) for n in (5, 17, 33, 60)]
Emix = []
for lanes in (8, 32):
    wm = A.Workload([grid, g2], A.LigandSet([(x, t, t) for x, t in mix]),
                    [A.Segment(i % 2, i, 16) for i in range(len(mix))], lanes_per_pose=lanes)
    Pm = torch.tensor(np.concatenate([c["poses"][:16]] * len(mix)), dtype=torch.float32, device="cuda")
    Emix += A.energrad(wm, Pm)[0].cpu().tolist() + A.minimise(wm, Pm, 3)[1].cpu().tolist()
torch.cuda.synchronize()
import ctypes as C
info = (C.c_ulonglong * 3)()
_lib.check(_lib.load().att_kernel_debug_info(info, 1, torch.cuda.current_stream().cuda_stream), "debug")
res = dict(word=_lib.kernel_status(clear=True), debug=[int(v) for v in info], n_overflow=int((grid.nb_hdr[:, 1] > 13).sum()),
           entries=int(st[2]), E=E.cpu().tolist(), G=G.cpu().reshape(-1).tolist(), Em=Em.cpu().tolist(),
           dP=dP.cpu().reshape(-1).tolist(), di=float(di.abs().sum()), do=float(do.abs().sum()),
           Ex=Ex.cpu().tolist(), Eq=Eq.cpu().tolist(), Ed=Ed, Emix=Emix)
print("RESULT " + json.dumps(res))
'''


def _run(lib):
    env = dict(os.environ)
    if lib:
        env["ATTRACT_B200_LIB"] = lib
    code = SCRIPT.format(root=ROOT, tests=HERE, oracle=os.path.join(ROOT, "oracle"))
    p = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stderr[-3000:]
    line = [x for x in p.stdout.splitlines() if x.startswith("RESULT ")][-1]
    return json.loads(line[7:])


def test_bounds_checked_build_finds_no_bad_index_and_matches():
    from attract_b200 import build as B

    checked = B.build(checked=True)  # prebuilt by the package build; rebuilt here only if stale
    got = _run(checked)
    ref = _run(None)
    assert got["word"] == 0 and got["debug"] == [0, 0, 0], (got["word"], got["debug"])
    assert got["n_overflow"] > 0  # the overflow path was exercised
    for k in ("E", "G", "Em", "dP", "Ex", "Eq", "Ed", "Emix"):
        a, b = np.asarray(got[k]), np.asarray(ref[k])
        assert np.allclose(a, b, rtol=1e-5, atol=1e-4), k
    assert np.isclose(got["di"], ref["di"], rtol=1e-5) and np.isclose(got["do"], ref["do"], rtol=1e-5)
