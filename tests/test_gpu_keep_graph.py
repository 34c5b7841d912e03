"""Device copies kept between calls (ag_pr_opts.keep_graph, AG_KEEP_GRAPH,
ag_graph_forget).

A kept upload is shown to be reused by changing the host graph in place: the
next kept call still answers for the graph as it was uploaded, and after
ag_graph_forget the call answers for the changed graph.  Every answer is
checked bit for bit against the oracle (EXACT order) on the arrays the
device copy was made from.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _pull(ag, g, keep, iterations=50, epsilon=1e-7):
    args = ag.default_arguments(iterations, epsilon)
    opts = ag.make_opts(order=ag.AG_ORDER_EXACT, quiet=True)
    opts.keep_graph = int(keep)
    out = C.POINTER(ag.PageRankStats)()
    ag.check(ag.lib.ag_pagerank_pull_ex(C.byref(args), g.ptr, C.byref(opts), C.byref(out)), "ag_pagerank_pull_ex")
    ranks = ag.stats_ranks(out)
    its = out.contents.iterations
    ag.lib.freePageRankStats(out)
    return ranks, its


def _oracle(oracle, g, iterations=50, epsilon=1e-7):
    return oracle.pagerank_pull(g.in_edges_idx(), g.in_degree(), g.in_neighbours().copy(), g.out_degree(),
                                iterations, epsilon)


def test_kept_upload_is_reused_until_forgotten(gpu, oracle):
    ag = gpu
    g = ag.Graph.rmat(13, 16, seed=5)
    try:
        want = _oracle(oracle, g)
        r0, it0 = _pull(ag, g, keep=True)
        assert np.array_equal(r0, want["ranks"]) and it0 == want["iterations"]
        r1, it1 = _pull(ag, g, keep=True)
        assert np.array_equal(r1, r0) and it1 == it0

        # change the host graph in place: the kept copy does not see it
        nb = g.in_neighbours()
        j = int(np.argmax(g.in_degree()))
        row = int(g.in_edges_idx()[j])
        old = int(nb[row])
        nb[row] = (old + 1) % g.num_vertices
        changed = _oracle(oracle, g)
        assert not np.array_equal(changed["ranks"], want["ranks"])
        r2, _ = _pull(ag, g, keep=True)
        assert np.array_equal(r2, r0)
        # a call without keep uploads afresh
        r3, it3 = _pull(ag, g, keep=False)
        assert np.array_equal(r3, changed["ranks"]) and it3 == changed["iterations"]

        # forgotten: the next kept call uploads the changed graph
        ag.check(ag.lib.ag_graph_forget(g.ptr), "ag_graph_forget")
        r4, it4 = _pull(ag, g, keep=True)
        assert np.array_equal(r4, changed["ranks"]) and it4 == changed["iterations"]
        nb[row] = old
    finally:
        ag.lib.ag_graph_forget(None)


def test_keep_table_evicts_least_recently_used(gpu, oracle):
    """Nine graphs through an eight-entry table: every answer stays the
    oracle's, whichever entries were evicted."""
    ag = gpu
    gs = [ag.Graph.rmat(9, 8, seed=100 + i) for i in range(9)]
    try:
        for rnd in range(2):
            for g in gs:
                want = _oracle(oracle, g, 30, 1e-6)
                r, it = _pull(ag, g, keep=True, iterations=30, epsilon=1e-6)
                assert np.array_equal(r, want["ranks"]) and it == want["iterations"]
    finally:
        ag.check(ag.lib.ag_graph_forget(None), "ag_graph_forget")


def test_spmv_keeps_its_upload_under_the_environment_switch(gpu, oracle, monkeypatch):
    ag = gpu
    monkeypatch.setenv("AG_KEEP_GRAPH", "1")
    rng = np.random.default_rng(9)
    n = 3000
    g = ag.Graph.from_edges(n, rng.integers(0, n, 40000), rng.integers(0, n, 40000),
                            rng.random(40000).astype(np.float32), flags=ag.AG_BUILD_DEDUPE)
    args = ag.default_arguments(2)
    try:
        ys = []
        for _ in range(2):
            sp = C.POINTER(ag.SPMVStats)()
            ag.check(ag.lib.ag_spmv_pull_ex(C.byref(args), g.ptr, 1, C.byref(sp)), "ag_spmv_pull_ex")
            ys.append(np.ctypeslib.as_array(sp.contents.vector_output, shape=(n,)).copy())
            ag.lib.freeSPMVStats(sp)
        x = oracle.spmv_input(g.out_degree())
        yo = oracle.spmv_pull(g.in_edges_idx(), g.in_degree(), g.in_neighbours(), g.in_weights(), x)
        assert np.array_equal(ys[0], ys[1])
        assert np.abs(ys[0].astype(np.float64) - yo).sum() <= 1e-5 * np.abs(yo.astype(np.float64)).sum()
    finally:
        ag.check(ag.lib.ag_graph_forget(None), "ag_graph_forget")


def test_csr_entry_points_serialise_concurrent_callers(gpu, oracle):
    """Four host threads call ag_pagerank_pull_ex (the entry under
    pageRankPullGraphCSR) at once; ctypes releases the GIL, so the library's
    lock is what keeps them apart.  Each gets the oracle's ranks bit for
    bit."""
    import threading

    ag = gpu
    gs = [ag.Graph.rmat(12, 16, seed=40 + i) for i in range(4)]
    want = [_oracle(oracle, g, 40, 1e-7) for g in gs]
    got = [None] * 4

    def run(i):
        args = ag.default_arguments(40, 1e-7)
        opts = ag.make_opts(order=ag.AG_ORDER_EXACT, quiet=True)
        out = C.POINTER(ag.PageRankStats)()
        st = ag.lib.ag_pagerank_pull_ex(C.byref(args), gs[i].ptr, C.byref(opts), C.byref(out))
        if st == 0:
            got[i] = (ag.stats_ranks(out), out.contents.iterations)
            ag.lib.freePageRankStats(out)

    ts = [threading.Thread(target=run, args=(i,)) for i in range(4)]
    for t in ts:
        t.start()
    for t in ts:
        t.join(timeout=300)
    for i in range(4):
        assert got[i] is not None
        assert np.array_equal(got[i][0], want[i]["ranks"]) and got[i][1] == want[i]["iterations"]
