"""uph_search_neighbors_noalloc: the neighbour search for callers that cannot
allocate GPU memory (a host application's own memory pool, a real-time loop,
a plugin host that forbids cudaMalloc).  Its scratch is a fixed __device__
array inside the library, so the test hands it only caller-owned device
buffers and checks its pairs against uph_search_neighbors on two calls in a
row -- the second call must not see leftovers of the first.

Named to be collected last, so a run that stops at the first failure has
already run every other test."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _positions(seed, n):
    rng = np.random.default_rng(seed)
    return rng.uniform(0.0, 2.0, size=(n, 2))


@pytest.mark.parametrize("sizes", [(5000, 3500), (20000, 12000)])
def test_noalloc_search_matches_allocating_search_twice(sizes):
    torch = pytest.importorskip("torch")
    from uph_b200 import _lib
    from uph_b200.sim import search_neighbors

    n, nf = sizes
    dist = 0.03 ** 2
    pb = n - 1
    lib = _lib.lib()
    lo = (C.c_double * 2)(-0.1, -0.1)
    hi = (C.c_double * 2)(2.1, 2.1)
    stream = torch.cuda.current_stream().cuda_stream
    # second call: different positions and a different fluid count
    for call, (seed, nfl) in enumerate([(11, nf), (12, nf // 2)]):
        pos = _positions(seed + n, n)
        pos[7] = pos[8]  # coincident points are never partners
        want_i, want_j, want_r2 = search_neighbors(pos, nfl, pb, dist, number_of_neighbors=0)
        cap = want_i.size + 16
        d_pos = torch.from_numpy(pos).cuda()
        d_i = torch.full((cap,), -1, dtype=torch.int32, device="cuda")
        d_j = torch.full((cap,), -1, dtype=torch.int32, device="cuda")
        d_r2 = torch.zeros(cap, dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        niac = C.c_int64(-1)
        st = lib.uph_search_neighbors_noalloc(C.c_void_p(d_pos.data_ptr()), nfl, n, pb, dist, C.byref(lo),
                                              C.byref(hi), cap, C.c_void_p(d_i.data_ptr()),
                                              C.c_void_p(d_j.data_ptr()), C.c_void_p(d_r2.data_ptr()),
                                              C.byref(niac), C.c_void_p(stream))
        assert st == 0, lib.uph_last_error()
        k = niac.value
        assert k == want_i.size, f"call {call}: {k} pairs, {want_i.size} expected"
        # integer and distance outputs of a search are exact
        assert np.array_equal(d_i[:k].cpu().numpy(), want_i), f"call {call}: i_pair"
        assert np.array_equal(d_j[:k].cpu().numpy(), want_j), f"call {call}: j_pair"
        assert np.array_equal(d_r2[:k].cpu().numpy(), want_r2), f"call {call}: rij2"


def test_noalloc_search_rejects_sizes_beyond_its_limit():
    torch = pytest.importorskip("torch")
    from uph_b200 import _lib

    lib = _lib.lib()
    n = (1 << 18) + 1
    d_pos = torch.zeros((n, 2), dtype=torch.float64, device="cuda")
    lo = (C.c_double * 2)(-1.0, -1.0)
    hi = (C.c_double * 2)(1.0, 1.0)
    niac = C.c_int64(0)
    st = lib.uph_search_neighbors_noalloc(C.c_void_p(d_pos.data_ptr()), 10, n, n - 1, 0.01, C.byref(lo),
                                          C.byref(hi), 0, None, None, None, C.byref(niac), None)
    assert st == 1  # UPH_BAD_ARG
    assert b"exceed the limit" in lib.uph_last_error()
    # too many cells for the fixed scratch
    hi2 = (C.c_double * 2)(100.0, 100.0)
    st = lib.uph_search_neighbors_noalloc(C.c_void_p(d_pos.data_ptr()), 10, 1000, 999, 1e-4, C.byref(lo),
                                          C.byref(hi2), 0, None, None, None, C.byref(niac), None)
    assert st == 1
    assert b"cells" in lib.uph_last_error()


def test_noalloc_search_reports_an_overcrowded_cell():
    """5000 points in one search cell (more than the 4096 ids a cell may hold):
    a neighbour overflow, with no pair walk, and the next call works again."""
    torch = pytest.importorskip("torch")
    from uph_b200 import _lib

    lib = _lib.lib()
    pos = np.random.default_rng(5).uniform(0.0, 0.01, (5000, 2))
    d_pos = torch.from_numpy(pos).cuda()
    lo = (C.c_double * 2)(-0.1, -0.1)
    hi = (C.c_double * 2)(0.2, 0.2)
    niac = C.c_int64(-1)
    st = lib.uph_search_neighbors_noalloc(C.c_void_p(d_pos.data_ptr()), 5000, 5000, 4999, 1.0, C.byref(lo),
                                          C.byref(hi), 0, None, None, None, C.byref(niac), None)
    assert st == 3, lib.uph_last_error()  # UPH_NEIGHBOR_OVERFLOW
    assert niac.value == 0
    # a sane call right after it
    pos2 = np.random.default_rng(6).uniform(0.0, 0.2, (500, 2))
    d_pos2 = torch.from_numpy(pos2).cuda()
    cap = 100000
    d_i = torch.zeros(cap, dtype=torch.int32, device="cuda")
    d_j = torch.zeros(cap, dtype=torch.int32, device="cuda")
    d_r2 = torch.zeros(cap, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    st = lib.uph_search_neighbors_noalloc(C.c_void_p(d_pos2.data_ptr()), 500, 500, 499, 0.02 ** 2, C.byref(lo),
                                          C.byref(hi), cap, C.c_void_p(d_i.data_ptr()), C.c_void_p(d_j.data_ptr()),
                                          C.c_void_p(d_r2.data_ptr()), C.byref(niac), None)
    assert st == 0, lib.uph_last_error()
    assert 0 < niac.value < cap


def test_noalloc_search_dense_queries_and_short_capacity():
    """A dense cluster: every query has about a thousand partners, so each
    query's pairs come from the merge of nine long cell lists.  The pairs
    equal the allocating search's; with a capacity below the total the call
    reports the full 64-bit count, writes exactly the first `cap` pairs and
    returns UPH_NEIGHBOR_OVERFLOW."""
    torch = pytest.importorskip("torch")
    from uph_b200 import _lib
    from uph_b200.sim import search_neighbors

    lib = _lib.lib()
    n = 3000
    pos = np.random.default_rng(21).uniform(0.0, 0.06, (n, 2))
    dist = 0.03 ** 2
    want_i, want_j, want_r2 = search_neighbors(pos, n, n - 1, dist, number_of_neighbors=0)
    assert want_i.size > 500 * n
    lo = (C.c_double * 2)(-0.01, -0.01)
    hi = (C.c_double * 2)(0.07, 0.07)
    d_pos = torch.from_numpy(pos).cuda()
    for cap in (want_i.size, want_i.size // 3):
        d_i = torch.full((cap,), -1, dtype=torch.int32, device="cuda")
        d_j = torch.full((cap,), -1, dtype=torch.int32, device="cuda")
        d_r2 = torch.zeros(cap, dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        niac = C.c_int64(-1)
        st = lib.uph_search_neighbors_noalloc(C.c_void_p(d_pos.data_ptr()), n, n, n - 1, dist, C.byref(lo),
                                              C.byref(hi), cap, C.c_void_p(d_i.data_ptr()),
                                              C.c_void_p(d_j.data_ptr()), C.c_void_p(d_r2.data_ptr()),
                                              C.byref(niac), None)
        assert niac.value == want_i.size
        assert st == (0 if cap == want_i.size else 3), lib.uph_last_error()
        assert np.array_equal(d_i.cpu().numpy(), want_i[:cap])
        assert np.array_equal(d_j.cpu().numpy(), want_j[:cap])
        assert np.array_equal(d_r2.cpu().numpy(), want_r2[:cap])
