"""ATTRACT .grid reader/writer against the reference reader's golden output
(tests/golden/make_grid_golden.py ran read_grid2.read_grid on the bytes)."""
import os
import struct

import numpy as np
import pytest

from attract_b200 import gridfile as gf

GOLD = os.path.join(os.path.dirname(__file__), "golden", "attract_grid_golden.npz")


@pytest.fixture(scope="module")
def gold():
    return dict(np.load(GOLD))


def test_read_grid_matches_reference_reader(gold):
    data = gold["grid_bytes"].tobytes()
    g = gf.read_grid(data, read_gradients=True)
    assert list(g._fields) == list(gold["fields"])
    for f in ("alphabet", "origin", "dim", "dim2", "inner_potential_grid", "outer_potential_grid",
              "nr_neighbours", "neighbour_grid"):
        a, b = getattr(g, f), gold[f]
        assert a.shape == b.shape and a.dtype == b.dtype, f
        assert np.array_equal(a, b), f
    for f in ("gridspacing", "gridextension", "plateaudis", "neighbourdis", "natoms", "max_nr_neighbours"):
        assert getattr(g, f) == gold[f][()], f
    assert g.neighbour_grid_ravel is None
    e = gf.read_grid(data, read_gradients=False)
    assert np.array_equal(e.inner_potential_grid, gold["inner_energies"])
    assert np.array_equal(e.outer_potential_grid, gold["outer_energies"])


def test_csr_form_matches_padded_grid(gold):
    data = gold["grid_bytes"].tobytes()
    d, hdr, lst = gf.read_grid_csr(data)
    ng = gold["neighbour_grid"].reshape(len(hdr), -1)
    for v in range(len(hdr)):
        s, c = hdr[v]
        assert np.array_equal(lst[s:s + c], ng[v, :c])
        assert np.all(ng[v, c:] == 65535)
    assert np.array_equal(d["inner_potential_grid"], gold["inner_potential_grid"])


def test_write_of_read_reproduces_the_bytes(gold):
    """read -> write gives the same file except for the per-entry atom-type
    byte of the neighbour records, which the reader drops."""
    data = gold["grid_bytes"].tobytes()
    g = gf.read_grid(data, read_gradients=True)
    _, hdr, lst = gf.read_grid_csr(data)
    again = gf.write_grid(gridspacing=g.gridspacing, gridextension=g.gridextension, plateaudis=g.plateaudis,
                          neighbourdis=g.neighbourdis, alphabet=g.alphabet, origin=g.origin, dim=g.dim,
                          dim2=g.dim2, natoms=g.natoms, inner_potential_grid=g.inner_potential_grid,
                          outer_potential_grid=g.outer_potential_grid, nb_hdr=hdr, nb_list=lst,
                          nr_neighbours=g.nr_neighbours, pivot=(1.0, 2.0, 3.0))
    a = np.frombuffer(data, np.uint8)
    b = np.frombuffer(again, np.uint8)
    assert len(a) == len(b)
    diff = np.flatnonzero(a != b)
    n_eg = struct.unpack_from("=i", data, gf._HEAD.size)[0]
    nb0 = gf._HEAD.size + 8 + 16 * n_eg + 8  # first neighbour record
    assert np.all((diff - nb0) % 8 == 0)  # only the type bytes of neighbour records differ


def test_unsupported_grids_are_rejected(gold):
    data = gold["grid_bytes"].tobytes()
    with pytest.raises(gf.GridFileError, match="torque"):
        gf.read_grid(bytes([1]) + data[1:])
    with pytest.raises(gf.GridFileError, match="32-bit"):
        gf.read_grid(data[:1] + struct.pack("=h", 32) + data[3:])
    with pytest.raises(gf.GridFileError):
        gf.read_grid(data[: len(data) // 2])
    with pytest.raises(gf.GridFileError):
        gf.read_grid(data[:100])


def test_grid_without_potentials_has_no_potential_fields():
    hdr = np.zeros((27, 2), np.int64)
    hdr[5] = (0, 2)
    data = gf.write_grid(gridspacing=1.0, gridextension=2, plateaudis=5.0, neighbourdis=6.0,
                         alphabet=np.zeros(99, bool), origin=(0, 0, 0), dim=(3, 3, 3), dim2=(2, 2, 2), natoms=3,
                         nb_hdr=hdr, nb_list=np.array([2, 0], np.uint16))
    g = gf.read_grid(data)
    assert "inner_potential_grid" not in g._fields and "outer_potential_grid" not in g._fields
    assert g.neighbour_grid.shape == (3, 3, 3, 2)
    assert list(g.neighbour_grid.reshape(27, 2)[5]) == [2, 0]


from hypothesis import given, settings, HealthCheck
from hypothesis import strategies as st


@settings(max_examples=300, deadline=None, suppress_health_check=[HealthCheck.function_scoped_fixture])
@given(flips=st.lists(st.tuples(st.floats(0.0, 1.0, exclude_max=True), st.integers(0, 255)), max_size=6),
       cut=st.one_of(st.none(), st.floats(0.0, 1.0)), head=st.booleans())
def test_corrupted_grid_files_fail_cleanly(gold, flips, cut, head):
    """Random byte changes (biased to the header, where the counts and
    dimensions live) and truncations of a valid file: the reader returns a
    grid or raises GridFileError, never another exception."""
    data = bytearray(gold["grid_bytes"].tobytes())
    span = 400 if head else len(data)
    for where, byte in flips:
        data[int(where * span)] = byte
    if cut is not None:
        data = data[:int(cut * len(data))]
    for csr in (False, True):
        try:
            if csr:
                gf.read_grid_csr(bytes(data))
            else:
                gf.read_grid(bytes(data), read_gradients=True)
        except gf.GridFileError:
            pass


def test_negative_dimensions_are_rejected(gold):
    """Dimensions whose signs cancel in the size check are still rejected."""
    data = bytearray(gold["grid_bytes"].tobytes())
    h = list(gf._HEAD.unpack_from(data, 0))
    h[108], h[109] = -h[108], -h[109]   # dim x, y negated: same product
    data[:gf._HEAD.size] = gf._HEAD.pack(*h)
    with pytest.raises(gf.GridFileError, match="dimensions"):
        gf.read_grid(bytes(data), read_gradients=True)
