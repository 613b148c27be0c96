"""The serving loop on the GPU: results equal the single-grid evaluation,
each request's result is the same alone and in a mix of concurrent requests,
LRU eviction under the byte cap, submissions from several host threads."""
import threading

import numpy as np
import pytest

import adaptive_sparse_grid_bench_b200 as sg
from adaptive_sparse_grid_bench_b200 import _lib, inputs

pytestmark = pytest.mark.gpu

# the last two have >= 4096 subspaces: the server splits their sums into
# parts (3 and 8) evaluated by separate CTAs and added in part order
SHAPES = [(4, 8, _lib.SG_FN_PROD4, ()), (10, 5, _lib.SG_FN_GAUSS, ()), (2, 9, _lib.SG_FN_BUMP, (0.3, 50.0)),
          (7, 6, _lib.SG_FN_GAUSS, ()), (12, 4, _lib.SG_FN_PROD4, ()), (10, 7, _lib.SG_FN_GAUSS, ()),
          (8, 9, _lib.SG_FN_BUMP, (0.3, 50.0))]
SPLIT_SUBSPACES = 4096
# split sums are added in another order than the single-grid kernel's:
# same tolerance as the parity tests against the FP64 oracle
RTOL_NORM, ATOL = 1e-5, 2e-7


def assert_same_or_close(got, want, split):
    if not split:
        assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
        return
    scale = max(float(np.max(np.abs(want))), 1e-30)
    err = np.abs(got.astype(np.float64) - want.astype(np.float64))
    assert np.all(err <= RTOL_NORM * scale + ATOL), f"max err {err.max():.3e}"


def _server(cap=8 << 30, zero_copy=0):
    srv = sg.Server(cap, max_batch_points=1 << 18)
    srv.set_option(_lib.SG_SRV_OPT_ZERO_COPY, zero_copy)
    ids = [srv.add_grid(d, n, fn, p) for d, n, fn, p in SHAPES]
    return srv, ids


@pytest.mark.parametrize("zero_copy", [0, 1])
def test_server_results_equal_single_grid(cuda, zero_copy):
    srv, ids = _server(zero_copy=zero_copy)
    rng_seed = 40
    tickets = []
    for q in range(40):
        g = q % len(ids)
        m = [1, 17, 512, 513, 3000, 65536][q % 6]
        X = inputs.uniform_points(rng_seed + q, m, SHAPES[g][0])
        tickets.append((g, X, srv.submit(ids[g], X)))
    for g, X, t in tickets:
        out, lat = srv.wait(t)
        want = srv.evaluate_now(ids[g], X)
        assert lat >= 0
        d, n = SHAPES[g][:2]
        assert_same_or_close(out, want, d >= 4 and sg.Grid(d, n).num_subspaces >= SPLIT_SUBSPACES)
    st = srv.stats()
    assert st["requests"] == 40 and st["failed"] == 0 and st["batches"] >= 1
    srv.close()


@pytest.mark.parametrize("zero_copy", [0, 1])
@pytest.mark.parametrize("mine_g", [1, 5, 6])
def test_same_result_alone_and_in_mix(cuda, mine_g, zero_copy):
    # bit for bit, split grids (5, 6) included: a grid's parts are fixed at
    # admission, whatever else is in the batch; the same with the batches
    # reading and writing pinned host memory in place
    srv, ids = _server(zero_copy=zero_copy)
    X = inputs.uniform_points(7, 20000, SHAPES[mine_g][0])
    X[:3] = [[0.0] * X.shape[1], [1.0] * X.shape[1], [np.nan] * X.shape[1]]  # edges and NaN
    alone, _ = srv.wait(srv.submit(ids[mine_g], X))
    mix = []
    for q in range(64):
        g = q % len(ids)
        mix.append(srv.submit(ids[g], inputs.uniform_points(100 + q, 1 + 997 * q % 40000, SHAPES[g][0])))
        if q == 31:
            mine = srv.submit(ids[mine_g], X)
    for t in mix:
        srv.wait(t)
    in_mix, _ = srv.wait(mine)
    assert np.array_equal(alone.view(np.uint32), in_mix.view(np.uint32))
    assert alone[1] == 0.0 and np.isnan(alone[2])
    assert srv.stats()["batches"] >= 2
    srv.close()


def test_split_sums_match_oracle(cuda):
    # the split evaluation against the FP64 oracle directly
    from oracle.oracle import Oracle
    srv, ids = _server()
    for g in (5, 6):
        d, n = SHAPES[g][:2]
        grid = sg.Grid(d, n)
        grid.sample_function(SHAPES[g][2], SHAPES[g][3])
        vals = grid.get_values()
        o = Oracle(d, n)
        s64 = o.hierarchize_f64(vals.astype(np.float64))
        X = inputs.uniform_points(900 + g, 700, d)
        out, _ = srv.wait(srv.submit(ids[g], X))
        ref = o.evaluate_f64(s64, X)
        scale = max(float(np.max(np.abs(ref))), 1e-30)
        assert np.max(np.abs(out - ref)) <= RTOL_NORM * scale + ATOL
    srv.close()


def test_lru_eviction_under_cap(cuda):
    probe = sg.Grid(6, 10)
    probe.sample_function(_lib.SG_FN_GAUSS)
    probe.hierarchize()
    one = probe.device_bytes()  # about 8 MB
    srv = sg.Server(int(2.5 * one), max_batch_points=1 << 16)
    a = srv.add_grid(6, 10, _lib.SG_FN_GAUSS)
    b = srv.add_grid(6, 10, _lib.SG_FN_PROD4)
    X = inputs.uniform_points(1, 100, 6)
    srv.wait(srv.submit(a, X))  # a is now the most recently used
    c = srv.add_grid(6, 10, _lib.SG_FN_GAUSS)  # evicts b (least recently used)
    st = srv.stats()
    assert st["evictions"] == 1 and st["resident_grids"] == 2
    srv.wait(srv.submit(a, X))
    srv.wait(srv.submit(c, X))
    with pytest.raises(sg.SgError):
        srv.submit(b, X)
    with pytest.raises(sg.SgError) as e:
        srv.add_grid(10, 10, _lib.SG_FN_GAUSS)  # larger than the whole cap
    assert e.value.code == _lib.SG_ERR_NOMEM
    srv.close()


def test_submissions_from_several_threads(cuda):
    srv, ids = _server()
    errors = []

    def client(k):
        try:
            for q in range(25):
                g = (k + q) % len(ids)
                X = inputs.uniform_points(1000 * k + q, 1 + (q * 131) % 5000, SHAPES[g][0])
                out, _ = srv.wait(srv.submit(ids[g], X))
                want = srv.evaluate_now(ids[g], X)
                scale = max(float(np.max(np.abs(want))), 1e-30)
                if not np.all(np.abs(out - want) <= RTOL_NORM * scale + ATOL):
                    errors.append((k, q))
        except Exception as exc:  # pragma: no cover - reported below
            errors.append(repr(exc))

    th = [threading.Thread(target=client, args=(k,)) for k in range(4)]
    for t in th:
        t.start()
    for t in th:
        t.join(timeout=120)
    assert not errors
    srv.close()


def test_request_larger_than_batch_is_rejected(cuda):
    srv = sg.Server(1 << 30, max_batch_points=1024)
    g = srv.add_grid(3, 4, _lib.SG_FN_PROD4)
    with pytest.raises(sg.SgError) as e:
        srv.submit(g, np.zeros((1025, 3), np.float32))
    assert e.value.code == _lib.SG_ERR_RANGE
    srv.close()


def test_reserved_range_reused_across_evictions(cuda):
    # a tight cap and grids of mixed size: ranges freed by evictions are
    # merged and handed to later grids; every admitted grid still evaluates
    # exactly like a standalone grid of the same shape and function
    shapes = [(6, 9, _lib.SG_FN_GAUSS, ()), (3, 7, _lib.SG_FN_PROD4, ()), (8, 7, _lib.SG_FN_BUMP, (0.3, 50.0)),
              (2, 12, _lib.SG_FN_GAUSS, ()), (5, 8, _lib.SG_FN_PROD4, ())]
    probe = sg.Grid(6, 9)
    probe.sample_function(_lib.SG_FN_GAUSS)
    probe.hierarchize()
    cap = 3 * probe.device_bytes()
    srv = sg.Server(cap, max_batch_points=1 << 16)
    want = {}
    for i, (d, n, fn, p) in enumerate(shapes):
        g = sg.Grid(d, n)
        g.sample_function(fn, p)
        g.hierarchize()
        X = inputs.uniform_points(300 + i, 4000, d)
        want[i] = (X, g.evaluate(X))
    for q in range(30):
        i = (q * 7) % len(shapes)
        d, n, fn, p = shapes[i]
        gid = srv.add_grid(d, n, fn, p)
        X, ref = want[i]
        out, _ = srv.wait(srv.submit(gid, X))
        assert np.array_equal(out.view(np.uint32), ref.view(np.uint32)), (q, shapes[i])
        st = srv.stats()
        assert st["bytes_in_use"] <= cap
    assert srv.stats()["evictions"] > 0 and srv.stats()["failed"] == 0
    srv.close()


def test_zero_copy_ring_wraps_and_matches(cuda):
    """Many zero-copy requests in flight: the staging ring wraps around and
    frees out of order; every result equals the copying path's."""
    srv, ids = _server(zero_copy=1)
    ref, _ = _server(zero_copy=0)
    window = []

    def check_oldest():
        g, X, t = window.pop(0)
        out, _ = srv.wait(t)
        want, _ = ref.wait(ref.submit(ids[g], X))
        assert np.array_equal(out.view(np.uint32), want.view(np.uint32))

    for q in range(300):  # about 450 MB of coordinates through an 84 MB ring
        g = q % len(ids)
        m = 1 + (7919 * q) % 60000
        X = inputs.uniform_points(500 + q, m, SHAPES[g][0])
        window.append((g, X, srv.submit(ids[g], X)))
        if len(window) > 24:
            check_oldest()
    while window:
        check_oldest()
    with pytest.raises(sg.SgError):
        srv.set_option(_lib.SG_SRV_OPT_ZERO_COPY, 2)
    srv.close()
    ref.close()


@pytest.mark.parametrize("heavy_pairs,light_slots,sort,zero_copy",
                         [(1, 3, 1, 1), (1, 3, 0, 1), (1, 2, 1, 0), (1 << 22, 3, 1, 1), (1 << 22, 1, 1, 1),
                          (1 << 62, 2, 1, 1)])
def test_lanes_keep_results(cuda, heavy_pairs, light_slots, sort, zero_copy):
    """Requests split between the light and heavy lanes by their work give
    the same results as the plain call, whichever lane they take (all heavy,
    mixed, all light), however many light batches run at once, with the
    heavy requests' points spatially ordered or not, zero-copy or copied."""
    srv, ids = _server(zero_copy=zero_copy)
    srv.set_option(_lib.SG_SRV_OPT_HEAVY_PAIRS, heavy_pairs)
    srv.set_option(_lib.SG_SRV_OPT_LIGHT_SLOTS, light_slots)
    srv.set_option(_lib.SG_SRV_OPT_SORT_HEAVY, sort)
    tickets = []
    for q in range(48):
        g = (5 * q) % len(ids)
        m = [3, 700, 5000, 40000][q % 4]
        X = inputs.uniform_points(900 + q, m, SHAPES[g][0])
        tickets.append((g, X, srv.submit(ids[g], X)))
    for g, X, t in tickets:
        out, _ = srv.wait(t)
        d, n = SHAPES[g][:2]
        assert_same_or_close(out, srv.evaluate_now(ids[g], X),
                             d >= 4 and sg.Grid(d, n).num_subspaces >= SPLIT_SUBSPACES)
    with pytest.raises(sg.SgError):
        srv.set_option(_lib.SG_SRV_OPT_HEAVY_PAIRS, 0)
    with pytest.raises(sg.SgError):
        srv.set_option(_lib.SG_SRV_OPT_LIGHT_SLOTS, 4)
    with pytest.raises(sg.SgError):
        srv.set_option(_lib.SG_SRV_OPT_SORT_HEAVY, 2)
    srv.close()
