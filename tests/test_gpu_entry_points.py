"""Every CSR entry point of the reference's pageRank.h:69-86 is exported and
runs its form on the GPU, compared with the reference's own function of the
same name (pageRank.c compiled with stand-in OpenGraph and libcxl headers and
an emulated accelerator gather, oracle/_ref) on the same graph and arguments.

The pull forms are deterministic in the reference: iterations and ranks must be
equal bit for bit (the entry points sum in the reference's stream order by
default).  The reference's push forms add with unsynchronised OpenMP threads;
its code runs on one thread here, which fixes the order: the 64-bit
fixed-point push is exact, the binary32 and quantised pushes agree within
1e-5 relative L1, the residual forms within 1e-4."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

# symbol, pushpull code the dispatcher maps to it, kind of comparison
FORMS = [
    ("pageRankPullGraphCSR", 0, "exact"),
    ("pageRankPushGraphCSR", 1, "rel1e-5"),
    ("pageRankPullFixedPoint64BitGraphCSR", 2, "exact"),
    ("pageRankPushFixedPointGraphCSR", 3, "exact"),
    ("pageRankPullQuant32BitGraphCSR", 4, "exact"),
    ("pageRankPushQuantGraphCSR", 5, "rel1e-5"),
    ("pageRankDataDrivenPullGraphCSR", 6, "exact"),
    ("pageRankDataDrivenPushGraphCSR", 7, "rel1e-4"),
    ("pageRankDataDrivenPullPushGraphCSR", 8, "rel1e-4"),
    ("pageRankPullFixedPoint32BitGraphCSR", 9, "exact"),
    ("pageRankPullFixedPoint16BitGraphCSR", 10, "exact"),
    ("pageRankPullFixedPoint8BitGraphCSR", 11, "exact"),
    ("pageRankPullQuant16BitGraphCSR", 12, "exact"),
    ("pageRankPullQuant8BitGraphCSR", 13, "exact"),
]


def _reference(refcode, name, args, g):
    n = g.num_vertices
    if name == "pageRankPullGraphCSR":
        return refcode.pagerank_pull(C.byref(args), g.ptr, n)
    if name == "pageRankDataDrivenPullGraphCSR":
        return refcode.pagerank_dd(C.byref(args), g.ptr, n)
    if name == "pageRankPullFixedPoint64BitGraphCSR":
        return refcode.pagerank_fixed64(C.byref(args), g.ptr, n)
    for (quant, width), sym in refcode._NARROW.items():
        if sym == name:
            return refcode.pagerank_narrow(quant, width, C.byref(args), g.ptr, n)
    for kind, sym in refcode._PUSH.items():
        if sym == name:
            return refcode.pagerank_push(kind, C.byref(args), g.ptr, n)
    for pull_push, sym in refcode._RESIDUAL.items():
        if sym == name:
            return refcode.pagerank_residual(pull_push, C.byref(args), g.ptr, n)
    raise KeyError(name)


@pytest.mark.parametrize("name,pushpull,kind", FORMS)
def test_entry_point_matches_reference_function(gpu, name, pushpull, kind, capfd):
    ag = gpu
    from oracle import refcode
    if not refcode.available():
        pytest.skip("the reference's own code is not built (oracle/_ref)")
    g = ag.Graph.rmat(12, 8, seed=78)
    args = ag.default_arguments(300, 1e-6)
    args.pushpull = pushpull
    args.ker_numThreads = 1
    st = getattr(ag.lib, name)(C.byref(args), g.ptr)
    ranks = ag.stats_ranks(st)
    iters = int(st.contents.iterations)
    ag.lib.freePageRankStats(st)
    capfd.readouterr()
    tol = 1e-5 if kind == "rel1e-5" else 1e-4

    def rel(a, b):
        return np.abs(a.astype(np.float64) - b).sum() / np.abs(b.astype(np.float64)).sum()

    # the dispatcher runs the same form for the symbol's pushpull code (the
    # residual forms add with atomics, so their bits vary from run to run)
    st = ag.lib.pageRankGraphCSR(C.byref(args), g.ptr)
    again = ag.stats_ranks(st)
    ag.lib.freePageRankStats(st)
    capfd.readouterr()
    if kind == "exact":
        assert np.array_equal(again.view(np.uint32), ranks.view(np.uint32))
    else:
        assert rel(again, ranks) <= tol
    ref = _reference(refcode, name, args, g)
    if kind == "exact":
        assert iters == ref["iterations"]
        assert np.array_equal(ranks.view(np.uint32), ref["ranks"].view(np.uint32))
    else:
        assert rel(ranks, ref["ranks"]) <= tol
