"""Golden vectors for the ATTRACT .grid reader (tests/test_gridfile.py).

Writes a small synthetic grid with attract_b200.gridfile.write_grid (3 potential
types at ATTRACT alphabet positions 1, 5 and 31, inner 6x5x7, outer 5x4x6 with
absent points, ragged neighbour lists, one point with the -32768 count
sentinel), reads it back with the reference's own reader (read_grid2.read_grid,
imported from the reference checkout, which needs only NumPy), checks that the
reference reads back what was written, and stores the bytes and the reference
reader's arrays in attract_grid_golden.npz.

    python tests/golden/make_grid_golden.py /path/to/attract-jax
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from attract_b200.gridfile import write_grid  # noqa: E402


def make():
    rng = np.random.default_rng(7)
    alphabet = np.zeros(99, bool)
    alphabet[[0, 4, 30]] = True
    T, dim, dim2 = 3, (6, 5, 7), (5, 4, 6)
    V = int(np.prod(dim))
    inner = rng.normal(size=(T, *dim, 4)).astype(np.float32)
    outer = rng.normal(size=(T, *dim2, 4)).astype(np.float32)
    outer[:, 1:3, 1:3, 1:4] = 0.0  # points covered by the inner grid: stored as absent
    cnt = rng.integers(0, 7, V)
    cnt[rng.choice(V, 20, replace=False)] = 0
    start = np.cumsum(cnt) - cnt
    lst = rng.integers(0, 400, int(cnt.sum())).astype(np.uint16)
    nr = cnt.astype(np.int64).copy()
    nr[np.flatnonzero(cnt == 0)[0]] = -32768
    rec_type = rng.integers(1, 32, 400)
    data = write_grid(gridspacing=0.9, gridextension=4, plateaudis=5.0, neighbourdis=7.5, alphabet=alphabet,
                      origin=(-3.5, 2.25, 10.0), dim=dim, dim2=dim2, natoms=400, inner_potential_grid=inner,
                      outer_potential_grid=outer, nb_hdr=np.stack([start, cnt], 1), nb_list=lst,
                      nr_neighbours=nr, rec_type=rec_type, pivot=(1.0, 2.0, 3.0))
    return data, inner, outer, cnt, start, lst, nr


def main(ref_root):
    sys.path.insert(0, ref_root)
    from read_grid2 import read_grid as ref_read_grid

    data, inner, outer, cnt, start, lst, nr = make()
    g = ref_read_grid(data, read_gradients=True)
    e = ref_read_grid(data, read_gradients=False)
    assert np.array_equal(g.inner_potential_grid, inner)
    assert np.array_equal(g.outer_potential_grid, outer)
    assert np.array_equal(e.inner_potential_grid, inner[..., 0])
    assert np.array_equal(g.nr_neighbours.reshape(-1), nr)
    out = dict(
        grid_bytes=np.frombuffer(data, np.uint8),
        fields=np.array(g._fields),
        gridspacing=g.gridspacing, gridextension=g.gridextension, plateaudis=g.plateaudis,
        neighbourdis=g.neighbourdis, alphabet=g.alphabet, origin=g.origin, dim=g.dim, dim2=g.dim2,
        natoms=g.natoms, inner_potential_grid=g.inner_potential_grid, outer_potential_grid=g.outer_potential_grid,
        nr_neighbours=g.nr_neighbours, max_nr_neighbours=g.max_nr_neighbours, neighbour_grid=g.neighbour_grid,
        inner_energies=e.inner_potential_grid, outer_energies=e.outer_potential_grid)
    path = os.path.join(HERE, "attract_grid_golden.npz")
    np.savez_compressed(path, **out)
    print(path, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit(f"usage: python {sys.argv[0]} <path of the attract-jax checkout>")
    main(sys.argv[1])
