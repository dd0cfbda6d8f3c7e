"""Scan / compaction / tile-list primitives (PrefixSum, StreamCompact, IncrementalTileList)
through the C ABI, against the oracle restatements and the reference's own checks
(test_PrefixSum.py:35, test_StreamCompact.py:40-41, test_IncrementalTileList.py:38-40)."""
import numpy as np
import pytest

from IncrementalTileList import IncrementalTileList, Logical, Operator, PrefixSum, StreamCompact

pytestmark = pytest.mark.gpu


def _dev(a, torch):
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.int32)).cuda()


@pytest.mark.parametrize("n", [0, 1, 2, 511, 512, 513, 4095, 4096, 4097, 65536, 1 << 20, 3000017])
def test_prefix_sum(cuda, oracle, n):
    torch = cuda
    rng = np.random.default_rng(n)
    h = rng.integers(0, 20, n).astype(np.int32)
    ps = PrefixSum(max(n, 1))
    d = ps.factory(max(n, 1))
    d[:n] = _dev(h, torch)
    tot = torch.zeros(1, dtype=torch.int32, device="cuda")
    ps.scan(d, tot, n)
    ref, ref_tot = oracle.exclusive_scan(h)
    assert int(tot.item()) == h.sum() == ref_tot            # test_PrefixSum.py:35
    assert np.array_equal(d[:n].cpu().numpy(), ref)          # element-wise (stronger)


def test_prefix_sum_negative_values(cuda, oracle):
    torch = cuda
    h = np.random.default_rng(3).integers(-1000, 1000, 100000).astype(np.int32)
    d = _dev(h, torch)
    tot = torch.zeros(1, dtype=torch.int32, device="cuda")
    PrefixSum(h.size).scan(d, tot, h.size)
    ref, ref_tot = oracle.exclusive_scan(h)
    assert np.array_equal(d.cpu().numpy(), ref) and int(tot.item()) == ref_tot


@pytest.mark.parametrize("n", [0, 1, 4096, 4097, 65536, 1000003])
def test_stream_compact(cuda, oracle, n):
    torch = cuda
    flags = np.random.default_rng(n + 1).integers(0, 2, n).astype(np.int32)
    sc = StreamCompact(max(n, 1))
    dF = sc.flagFactory(max(n, 1)); dF[:n] = _dev(flags, torch)
    dL = sc.listFactory(max(n, 1))
    dN = torch.zeros(1, dtype=torch.int32, device="cuda")
    sc.compact(dF, dL, dN, n)
    m = int(dN.item())
    ref, ref_n = oracle.compact(flags)
    assert m == ref_n
    assert np.array_equal(np.where(flags == 1)[0], dL[:m].cpu().numpy())  # test_StreamCompact.py:40


def test_stream_compact_capacity_error(cuda):
    sc = StreamCompact(100)
    with pytest.raises(ValueError):
        sc.flagFactory(101)
    with pytest.raises(ValueError):
        sc.listFactory(101)


def test_tile_list_reference_check(cuda):
    """test_IncrementalTileList.py:18-40: 4096^2 image, 16^2 tiles, stamps in [0,20),
    build(GTE, 10) == row-major ids of np.where(tiles >= 10)."""
    torch = cuda
    tl = IncrementalTileList((4096, 4096), (16, 16))
    dim = tl.dim
    h = np.random.default_rng(0).integers(0, 20, (dim[1], dim[0])).astype(np.int32)
    tl.d_tiles.copy_(_dev(h, torch))
    tl.build(Operator.GTE, 10)
    ys, xs = np.where(h >= 10)
    ref = ys * dim[0] + xs
    assert tl.length == ref.size
    assert np.array_equal(ref, tl.d_list[:tl.length].cpu().numpy())


@pytest.mark.parametrize("op", [Operator.EQUAL, Operator.GT, Operator.LT, Operator.GTE, Operator.LTE])
def test_tile_list_operators(cuda, oracle, op):
    torch = cuda
    tl = IncrementalTileList((2048, 1024), (32, 32))
    h = np.random.default_rng(op).integers(-3, 4, (tl.dim[1], tl.dim[0])).astype(np.int32)
    tl.d_tiles.copy_(_dev(h, torch))
    tl.build(op, 1)
    ref, n = oracle.compact(oracle.flag(h.reshape(-1), op, 1))
    assert tl.length == n and np.array_equal(tl.d_list[:n].cpu().numpy(), ref)


def test_tile_list_incorporate_and_logical(cuda, oracle):
    torch = cuda
    tl = IncrementalTileList((1024, 1024), (32, 32))
    rng = np.random.default_rng(7)
    a = rng.integers(-2, 6, (tl.dim[1], tl.dim[0])).astype(np.int32)
    b = rng.integers(0, 30, (tl.dim[1], tl.dim[0])).astype(np.int32)
    tl.d_tiles.copy_(_dev(a, torch))
    d2 = _dev(b, torch)
    it = tl.increment()
    tl.incorporate(d2, Operator.LTE, 0, Operator.GTE, 12, Logical.AND)
    ref = oracle.increment_logical(a.reshape(-1), b.reshape(-1), Operator.LTE, Operator.GTE,
                                   0, 12, Logical.AND, it)
    assert np.array_equal(tl.d_tiles.cpu().numpy().reshape(-1), ref)
    tl.buildLogical(d2, Operator.EQUAL, it, Operator.LT, 20, Logical.OR)
    refl, n = oracle.compact(oracle.flag_logical(ref, b.reshape(-1), Operator.EQUAL, Operator.LT,
                                                 it, 20, Logical.OR))
    assert tl.length == n and np.array_equal(tl.d_list[:n].cpu().numpy(), refl)
    tl.reset()
    assert (tl.d_tiles.cpu().numpy() == -1).all() and tl.iteration == 0


def test_repeated_calls_reuse_lookback_state(cuda, oracle):
    """Many back-to-back launches: the look-back tags must not leak between launches."""
    torch = cuda
    rng = np.random.default_rng(11)
    sc = StreamCompact(200000)
    dL = sc.listFactory()
    dN = torch.zeros(1, dtype=torch.int32, device="cuda")
    for k in range(50):
        n = int(rng.integers(1, 200000))
        f = (rng.random(n) < rng.random()).astype(np.int32)
        dF = _dev(f, torch)
        sc.compact(dF, dL, dN, n)
        m = int(dN.item())
        assert m == int(f.sum())
        assert np.array_equal(np.flatnonzero(f), dL[:m].cpu().numpy())


@pytest.mark.parametrize("global_dim,tiles_dim", [((4096, 4096), (16, 16)), ((800, 608), (32, 32)),
                                                  ((100, 37), (16, 16)), ((1, 1), (16, 16))])
def test_tile_list_execute_view(cuda, oracle, global_dim, tiles_dim):
    """IncrementalTileList.execute (IncrementalTileList.pyx:191-208): the display layer of the
    tiles stamped with the current iteration equals the oracle's, bit for bit."""
    torch = cuda
    tl = IncrementalTileList(global_dim, tiles_dim)
    dim = tl.dim
    h = np.random.default_rng(3).integers(0, 4, (dim[1], dim[0])).astype(np.int32)
    if h.size:
        tl.d_tiles.copy_(_dev(h, torch))
    for it in (tl.iteration, 2):
        tl.iteration = it
        got = tl.execute().cpu().numpy().view(np.uint32)
        want = oracle.tiles_view(h, tiles_dim[0], tiles_dim[1], it, *global_dim)
        assert np.array_equal(got, want)
    out = torch.zeros((global_dim[1], global_dim[0]), dtype=torch.int32, device="cuda")
    assert tl.execute(out=out) is out


def test_lookback_wait_runs_out_and_reports(cuda):
    """A bounded look-back wait made to run out on purpose (a predecessor that never
    publishes, a short poll limit) records error 1; the state reports it once, is clear
    afterwards and still compacts correctly."""
    import _gcut
    torch = cuda
    st = _gcut.ScanState(0, 1 << 16)
    assert st.selftest(spins=2000) == 1
    assert st.error() == 0
    flags = (np.random.default_rng(5).random(50000) < 0.4).astype(np.int32)
    dF = _dev(flags, torch)
    dL = torch.zeros(50000, dtype=torch.int32, device="cuda")
    dN = torch.zeros(1, dtype=torch.int32, device="cuda")
    _gcut.check(_gcut.lib().gc_compact(st.handle, _gcut.ptr(dF), _gcut.ptr(dL), _gcut.ptr(dN),
                                       flags.size, _gcut.stream_handle()))
    m = int(dN.item())
    assert m == int(flags.sum()) and np.array_equal(np.flatnonzero(flags), dL[:m].cpu().numpy())
    assert st.error() == 0
    st.close()


def test_lookback_error_surfaces_at_next_call(cuda):
    """An error left on a state by an earlier launch makes the next call on it return
    GC_ERR_INTERNAL (after which the state is clear again)."""
    import _gcut
    torch = cuda
    st = _gcut.ScanState(0, 1 << 16)
    L = _gcut.lib()
    s = _gcut.stream_handle()
    # the wait runs out and its error word is left on the state, unread
    assert L.gc_scan_state_selftest(st.handle, 1000, None, s) == 0
    torch.cuda.synchronize()
    flags = np.ones(10000, np.int32)
    dF = _dev(flags, torch)
    dL = torch.zeros(10000, dtype=torch.int32, device="cuda")
    dN = torch.zeros(1, dtype=torch.int32, device="cuda")
    assert L.gc_compact(st.handle, _gcut.ptr(dF), _gcut.ptr(dL), _gcut.ptr(dN), 10000, s) == \
        _gcut.GC_ERR_INTERNAL
    assert b"look-back" in L.gc_last_error()
    # reported once: the same call now runs and is right
    assert L.gc_compact(st.handle, _gcut.ptr(dF), _gcut.ptr(dL), _gcut.ptr(dN), 10000, s) == 0
    torch.cuda.synchronize()
    assert int(dN.item()) == 10000
    assert np.array_equal(dL.cpu().numpy(), np.arange(10000))
    assert st.error() == 0
    st.close()


def test_objects_on_different_streams_do_not_interfere(cuda):
    """Two StreamCompact objects compacting at the same time on two streams (each with its
    own look-back state) both return np.flatnonzero of their flags, many times over."""
    torch = cuda
    rng = np.random.default_rng(17)
    n = 1_500_000
    objs = [StreamCompact(n), StreamCompact(n)]
    streams = [torch.cuda.Stream(), torch.cuda.Stream()]
    flags = [(rng.random(n) < p).astype(np.int32) for p in (0.2, 0.6)]
    dF = [_dev(f, torch) for f in flags]
    dL = [o.listFactory() for o in objs]
    dN = [torch.zeros(1, dtype=torch.int32, device="cuda") for _ in objs]
    torch.cuda.synchronize()
    for _ in range(20):
        for k in range(2):
            with torch.cuda.stream(streams[k]):
                objs[k].compact(dF[k], dL[k], dN[k], n, stream=streams[k])
    torch.cuda.synchronize()
    for k in range(2):
        m = int(dN[k].item())
        assert m == int(flags[k].sum())
        assert np.array_equal(np.flatnonzero(flags[k]), dL[k][:m].cpu().numpy())
        assert objs[k].state.error() == 0
