"""CPU tests of Lexi-order renumbering: the oracle's restatement against the
reference library's own orderit (src/sptensor/orderit.c, compiled from its
sources) on tensors whose indices all have distinct row sets, where the
ordering is unique; the reference defect that keeps its other driver,
ptiIndexRenumber, from being a parity target; and the host-side shuffles."""
import ctypes as C

import numpy as np
import pytest

from hiparti_b200 import COOTensor, ffi, lib


def random_tensor(dims, nnz, seed):
    rng = np.random.default_rng(seed)
    lin = rng.choice(int(np.prod(dims)), nnz, replace=False)
    return [i.astype(np.uint32) for i in np.unravel_index(lin, dims)], rng.random(nnz).astype(np.float32)


def tie_free(dims, inds):
    """No two indices of any mode have the same set of other-mode tuples."""
    N = len(dims)
    for m in range(N):
        others = [k for k in range(N) if k != m]
        sets = {}
        for z in range(inds[0].size):
            sets.setdefault(int(inds[m][z]), set()).add(tuple(int(inds[k][z]) for k in others))
        v = [frozenset(x) for x in sets.values()]
        if len(set(v)) != len(v):
            return False
    return True


CASES = [((6, 5, 5), 40, 1), ((10, 8, 8), 150, 2), ((20, 25, 30), 3000, 3), ((8, 9, 10, 11), 2500, 2)]


@pytest.mark.parametrize("dims,nnz,its", CASES)
@pytest.mark.parametrize("seed", [0, 1])
def test_oracle_matches_reference_orderit(ref, dims, nnz, its, seed):
    from oracle.oracle import lexi_order
    inds, vals = random_tensor(dims, nnz, seed)
    assert tie_free(dims, inds)
    want = ref.orderit(dims, inds, vals, its)
    got = lexi_order(dims, inds, its)
    for a, b in zip(got, want):
        np.testing.assert_array_equal(a, b)


def test_reference_renumber_sort_is_not_a_sort(ref):
    """ptiSparseTensorSortIndexExceptSingleMode (used by the reference's
    ptiIndexRenumber) leaves the nonzeros unsorted, so that driver's output
    depends on the nonzero order; orderit's does not."""
    dims = (20, 25, 30)
    inds, vals = random_tensor(dims, 3000, 0)
    t, keep = ref._coo(dims, inds, vals)
    mode_order = (C.c_uint32 * 2)(1, 2)
    ref.L.ptiSparseTensorSortIndexExceptSingleMode(C.byref(t), C.c_int(1), mode_order, C.c_int(1))
    from oracle.oracle import _np_from
    key = _np_from(t.inds[1].data, 3000, np.uint32).astype(np.int64) * 100 + \
        _np_from(t.inds[2].data, 3000, np.uint32)
    assert (np.diff(key) < 0).any()
    perm = np.random.default_rng(1).permutation(3000)
    shuffled = [i[perm].copy() for i in inds]
    a, b = ref.orderit(dims, inds, vals, 1), ref.orderit(dims, shuffled, vals, 1)
    assert all(np.array_equal(x, y) for x, y in zip(a, b))


def test_shuffle_and_inverse_shuffle(lib):
    dims = (7, 5, 6)
    inds, vals = random_tensor(dims, 60, 3)
    t = COOTensor(dims, inds, vals)
    rng = np.random.default_rng(4)
    maps = [rng.permutation(d).astype(np.uint32) for d in dims]
    s = t.shuffled(maps)
    for m in range(3):
        np.testing.assert_array_equal(s.inds[m], maps[m][inds[m]])
    # a factor computed in the new numbering, brought back to the old one
    L = lib
    mat = ffi.new("ptiMatrix *")
    assert L.ptiNewMatrix(mat, 7, 3) == 0
    a = np.frombuffer(ffi.buffer(mat.values, 4 * 7 * mat.stride), np.float32).reshape(7, mat.stride)
    a[:, :3] = np.arange(21, dtype=np.float32).reshape(7, 3)
    before = a[:, :3].copy()
    mp = np.ascontiguousarray(maps[0])
    L.ptiMatrixInverseShuffleIndices(mat, ffi.cast("ptiIndex *", mp.ctypes.data))
    a = np.frombuffer(ffi.buffer(mat.values, 4 * 7 * mat.stride), np.float32).reshape(7, mat.stride)
    np.testing.assert_array_equal(a[:, :3], before[maps[0]])
    L.ptiFreeMatrix(mat)


# ---------------------------------------------------------------------------
# BFS-like renumbering (renumber == 2, src/sptensor/renumber.c:534-839)
# ---------------------------------------------------------------------------
def _bfs_cases():
    from conftest import load_golden
    g = load_golden("bfs_like.npz")
    for c in range(int(g["ncases"])):
        dims = [int(x) for x in g[f"c{c}_dims"]]
        yield (dims, [g[f"c{c}_ind{m}"] for m in range(len(dims))], g[f"c{c}_vals"],
               [g[f"c{c}_map{m}"] for m in range(len(dims))])


def test_bfs_oracle_matches_golden_reference_vectors():
    """The restatement against maps the reference's own ptiBFSLike produced
    (compiled with the 0xFF-filling allocator, tests/golden/make_bfs_golden.py)."""
    from oracle.oracle import bfs_like
    n = 0
    for dims, inds, vals, want in _bfs_cases():
        got = bfs_like(dims, inds)
        for a, b in zip(got, want):
            np.testing.assert_array_equal(a, b)
        n += 1
    assert n >= 5


@pytest.mark.parametrize("seed", [7, 8])
def test_bfs_oracle_matches_reference_library(ref, seed):
    from oracle.oracle import Ref, bfs_like
    if not Ref.bfs_available():
        pytest.skip("BFS-like oracle build of the reference not present")
    dims = (70, 40, 30) if seed == 7 else (25, 20, 15, 10)
    inds, vals = random_tensor(dims, 1500, seed)
    want = ref.bfs_like(list(dims), inds, vals)
    for a, b in zip(bfs_like(list(dims), inds), want):
        np.testing.assert_array_equal(a, b)


def test_reference_bfs_like_is_not_reproducible(ref):
    """The reference's ptiBFSLike as built plainly reads visit marks it never
    set (renumber.c:768): repeated calls on one tensor in one process give
    different numberings, which is why parity is pinned on the 0xFF build."""
    dims = (200, 150, 100)
    inds, vals = random_tensor(dims, 3000, 2)
    outs = []
    for rep in range(4):
        t, keep = ref._coo(dims, inds, vals)
        maps = [np.zeros(d, np.uint32) for d in dims]
        arr = (C.c_void_p * 3)(*[m.ctypes.data for m in maps])
        ref.L.ptiIndexRenumber(C.byref(t), arr, C.c_int(2), C.c_uint32(1), C.c_uint8(7), C.c_int(1), C.c_int(1))
        outs.append(maps)
        _ = [np.full(1000 + 37 * rep, rep, np.int32) for _ in range(5)]  # heap traffic between calls
    same = [all(np.array_equal(a, b) for a, b in zip(outs[0], o)) for o in outs[1:]]
    assert not all(same)


def test_lexi_impl_num_2_is_orderit(ref):
    """impl_num 2 compares block indices before indices, which orders the
    coordinates exactly as comparing the indices does, and sorts with a correct
    quicksort: the reference's own results equal orderit's."""
    for dims, nnz, seed, its in [((30, 20, 10), 300, 1, 1), ((200, 150, 100), 3000, 2, 2),
                                 ((40, 30, 20, 10), 2000, 4, 2)]:
        inds, vals = random_tensor(dims, nnz, seed)
        a = ref.renumber(list(dims), inds, vals, its, impl_num=2)
        b = ref.orderit(list(dims), inds, vals, its)
        assert all(np.array_equal(x, y) for x, y in zip(a, b))
