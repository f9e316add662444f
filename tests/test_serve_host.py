"""Host logic of the serving loop, on CPU: the pose-pool allocator under
random allocation / release sequences, and the launch-shape policy."""
import pytest
from hypothesis import given, settings
from hypothesis import strategies as st

from attract_b200.serve import PosePool, launch_shape, lanes_by_size


def _check_invariants(pool, live):
    free = pool.free
    # free ranges sorted, disjoint, not adjacent (merged), inside the pool
    for (a, la), (b, lb) in zip(free, free[1:]):
        assert a + la < b
    assert all(ln > 0 and 0 <= a and a + ln <= pool.capacity for a, ln in free)
    # live allocations disjoint from each other and from free space
    spans = sorted(list(live.items()) + free)
    for (a, la), (b, lb) in zip(spans, spans[1:]):
        assert a + la <= b
    assert pool.used == sum(live.values())


@settings(max_examples=200, deadline=None)
@given(cap=st.integers(1, 500), ops=st.lists(st.tuples(st.booleans(), st.integers(1, 120)), max_size=60))
def test_pose_pool_random_alloc_release(cap, ops):
    pool = PosePool(cap)
    live = {}
    for do_alloc, n in ops:
        if do_alloc or not live:
            s = pool.alloc(n)
            if s < 0:
                # first fit failed: no free range of n poses
                assert all(ln < n for _, ln in pool.free)
            else:
                live[s] = n
        else:
            s = sorted(live)[n % len(live)]
            pool.release(s, live.pop(s))
        _check_invariants(pool, live)
    for s in list(live):
        pool.release(s, live.pop(s))
    assert pool.free == [(0, cap)] and pool.used == 0


def test_pose_pool_rejects_double_and_foreign_release():
    pool = PosePool(100)
    a = pool.alloc(30)
    b = pool.alloc(30)
    pool.release(a, 30)
    with pytest.raises(ValueError):
        pool.release(a, 30)          # released twice
    with pytest.raises(ValueError):
        pool.release(a + 10, 30)     # overlaps the free range [0, 30)
    with pytest.raises(ValueError):
        pool.release(90, 20)         # beyond the pool
    pool.release(b, 30)
    assert pool.free == [(0, 100)]


@pytest.mark.parametrize("n", range(1, 130))
def test_launch_shape_covers_the_ligand(n):
    lanes = lanes_by_size(n)
    s, k = launch_shape(n, lanes)
    assert s == lanes and k in (1, 2, 4)
    # every bead has a slot, or the ligand runs in chunks of 4 beads per lane
    assert s * k >= n or k == 4
    # the smallest power-of-two beads per lane that holds the ligand
    assert k == 1 or s * (k // 2) < n
