"""Work lists planned on the device: equal, item for item, to a Python
statement of the planning rules, for both orders, several tile shapes and a
block-diagonal union of graphs.

Rules (the pull kernel's contract): rows above `cap` in-edges are long items;
in FAST order rows above `whub` are split into whub-edge hub chunks numbered
by a running slot; every other row joins an item of at most 32 consecutive
rows and `cap` in-edges that never crosses a 512-row planning segment or the
first row of a graph.  FAST lists hub chunks, then long rows, then row items;
EXACT lists long rows (split ones included), then row items."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SEG = 512


def plan(off, cap, whub, exact, gstart=None):
    n = len(off) - 1
    hubs, longs, rows = [], [], []
    pbase = 0
    r = 0
    while r < n:
        d = int(off[r + 1] - off[r])
        if d > cap:
            if d > whub:
                nch = (d + whub - 1) // whub
                for c in range(nch):
                    cb = int(off[r]) + c * whub
                    hubs.append(((2 << 30) | r, pbase | (c << 20), cb, min(int(off[r + 1]), cb + whub)))
                pbase += nch
            else:
                longs.append(((1 << 30) | r, r + 1, int(off[r]), int(off[r + 1])))
            r += 1
            continue
        rb, eb = r, int(off[r])
        limit = min(n, (rb // SEG + 1) * SEG)
        if gstart is not None:
            above = [s for s in gstart if s > rb]
            if above:
                limit = min(limit, above[0])
        r += 1
        while r < limit and r - rb < 32 and off[r + 1] - off[r] <= cap and off[r + 1] - eb <= cap:
            r += 1
        rows.append((rb, r, eb, int(off[r])))
    return np.array(hubs + longs + rows, dtype=np.uint32).reshape(-1, 4)


def device_offsets(g):
    """Row starts after the upload's relabelling (stable, descending out-degree)."""
    perm = np.argsort(-g.out_degree().astype(np.int64), kind="stable")
    deg = g.in_degree().astype(np.int64)[perm]
    return np.concatenate([[0], np.cumsum(deg)]).astype(np.int64)


@pytest.mark.parametrize("scale,ef", [(12, 16), (13, 8)])
def test_device_plan_matches_rules(gpu, scale, ef):
    ag = gpu
    g = ag.Graph.rmat(scale, ef, seed=scale)
    dg = ag.DeviceGraph(g)
    off = device_offsets(g)
    for cap, whub in ((256, 2048), (64, 256), (128, 1024), (32, 32)):
        dg.set_tiles(cap, whub, 0, 0)
        for exact in (False, True):
            got = dg.tasks(exact)
            want = plan(off, cap, whub, exact)
            assert got.shape == want.shape, (cap, whub, exact)
            assert np.array_equal(got, want), (cap, whub, exact)
    dg.release()


def test_device_plan_covers_every_row_once(gpu):
    ag = gpu
    g = ag.Graph.rmat(14, 16, seed=5)
    dg = ag.DeviceGraph(g)
    n = g.num_vertices
    off = device_offsets(g)
    for exact in (False, True):
        t = dg.tasks(exact)
        kind = t[:, 0] >> 30
        first = t[:, 0] & 0x3FFFFFFF
        seen = np.zeros(n, np.int64)
        for k, r0, y, eb, ee in zip(kind, first, t[:, 1], t[:, 2], t[:, 3]):
            if k == 0:
                seen[r0:y] += 1
                assert eb == off[r0] and ee == off[y] and ee - eb <= 256 and y - r0 <= 32
            elif k == 1:
                seen[r0] += 1
                assert eb == off[r0] and ee == off[r0 + 1]
            else:
                if eb == off[r0]:
                    seen[r0] += 1
                assert off[r0] <= eb < ee <= off[r0 + 1]
        assert (seen == 1).all()
    # one list serves both orders: the kernel's order decides how items sum
    assert np.array_equal(dg.tasks(False), dg.tasks(True))
    dg.release()


def test_multigraph_plan_respects_graph_starts(gpu):
    ag = gpu
    gs = [ag.Graph.rmat(s, 8, seed=s) for s in (6, 9, 7, 10, 5)]
    mg = ag.MultiGraph(gs)
    sizes = [g.num_vertices for g in gs]
    gstart = np.concatenate([[0], np.cumsum(sizes)])
    off = np.concatenate([[0], np.cumsum(np.concatenate([g.in_degree() for g in gs]).astype(np.int64))])
    t = mg.tasks(False)
    want = plan(off, 256, 2048, False, list(gstart))
    assert np.array_equal(t, want)
