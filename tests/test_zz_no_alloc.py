"""The allocation-free Morton sort (jt_morton_sort_static) against the
existing entry point that produces the same arrays (jt_debug_tree), over two
calls in a row with different inputs and sizes: the static scratch array
keeps the first call's contents, and the second call must not depend on them.
Bit-exact: sorted 30-bit codes and permutation.

The file name sorts last so that it also runs after every other test in the
same process; it passes alone in a fresh process too.
"""
import numpy as np
import pytest

import janus_treepm as J

pytestmark = pytest.mark.gpu


def _positions(seed, n, L, collide=False):
    rng = np.random.default_rng(seed)
    if collide:
        # many equal Morton codes: points on a coarse lattice of 8^3 cells
        cells = rng.integers(0, 8, (n, 3))
        return ((cells + 0.5) * (L / 8) - L / 2).astype(np.float32)
    return rng.uniform(-L / 2, L / 2, (n, 3)).astype(np.float32)


def _reference(pos, L):
    s = J.Solver(J.Config(box_L=L, pm_grid=32))
    s.set_state(pos, None, None, None)
    t = s.debug_tree(0)
    s.close()
    return t["morton"], t["perm"]


def _static(pos, L):
    import torch
    n = len(pos)
    d = torch.from_numpy(pos).cuda()
    mo = torch.full((n,), -1, dtype=torch.int32, device="cuda")
    pe = torch.full((n,), -1, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    J.morton_sort_static(d.data_ptr(), n, L, mo.data_ptr(), pe.data_ptr(), None)
    return mo.cpu().numpy().view(np.uint32), pe.cpu().numpy()


def test_static_sort_matches_debug_tree_two_calls_in_a_row():
    cases = [(21, 200_000, 64.0, False), (22, 3_001, 250.0, True)]
    for seed, n, L, collide in cases:
        pos = _positions(seed, n, L, collide)
        ref_m, ref_p = _reference(pos, L)
        got_m, got_p = _static(pos, L)
        assert np.array_equal(got_m, ref_m), (seed, n)
        assert np.array_equal(got_p, ref_p), (seed, n)


def test_static_sort_ties_follow_row_order():
    # rows in a shuffled order with many equal codes: the permutation must be
    # the stable order of the codes (ties by row), computed by the oracle
    import oracle as O
    L = 80.0
    pos = _positions(24, 50_000, L, collide=True)
    pos = pos[np.random.default_rng(5).permutation(len(pos))]
    codes = O.morton30(pos, np.float32(L / 2)).astype(np.uint32)
    order = np.argsort(codes, kind="stable")
    got_m, got_p = _static(pos, L)
    assert np.array_equal(got_m, codes[order])
    assert np.array_equal(got_p, order.astype(np.int32))


def test_static_sort_limits():
    L = J.library()
    assert L.jt_morton_sort_static(None, 10, 64.0, None, None, None) == J.JT_EINVAL
    # more than the static array holds: rejected on the host before any
    # device work (the pointers are never dereferenced on this path)
    fake = 256
    assert L.jt_morton_sort_static(fake, J.JT_STATIC_SORT_MAX + 1, 64.0, fake, fake, None) == J.JT_EINVAL
    pos = _positions(23, J.JT_STATIC_SORT_MAX, 100.0)
    ref_m, ref_p = _reference(pos, 100.0)
    got_m, got_p = _static(pos, 100.0)
    assert np.array_equal(got_m, ref_m) and np.array_equal(got_p, ref_p)
