"""Failure detection without a GPU fault (the reference's watchdog tests,
03_capi_integration/accelerator_verification/host/test_accelerator_verification.c:19-158,
check that a stuck accelerator is reported, not waited on forever).

- Host side: every wait on the library stream polls against a deadline
  (AG_WAIT_TIMEOUT_S) and returns AG_ERR_TIMEOUT when it passes with work still
  queued; the work itself is not disturbed, and a later wait collects it.
- Device side: the pull kernel's wait for its hot-table copy is bounded
  (AG_MBAR_SPINS polls).  When it runs out the kernel flags ctl->fault, then
  waits again (bounded, long) for the copies before it reads the table, so the
  pass completes; the fetch reports AG_ERR_DEVICE_WAIT.  With 0 polls the first
  wait runs out at once: nothing hangs and nothing faults.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _oracle(oracle, g, it, eps):
    return oracle.pagerank_pull(g.in_edges_idx(), g.in_degree(), g.in_neighbours(), g.out_degree(), it, eps)


def test_host_deadline_returns_timeout_then_work_completes(gpu, oracle, monkeypatch):
    ag = gpu
    g = ag.Graph.rmat(20, 16, seed=5)
    ref = _oracle(oracle, g, 300, 1e-6)
    dg = ag.DeviceGraph(g)
    dg.pagerank(300, 1e-6, order=ag.AG_ORDER_EXACT)  # builds the launch graph
    monkeypatch.setenv("AG_WAIT_TIMEOUT_S", "1e-7")
    dg.launch(300, 1e-6, order=ag.AG_ORDER_EXACT)
    with pytest.raises(ag.AGError) as err:
        dg.fetch()
    assert err.value.status == ag.AG_ERR_TIMEOUT
    assert ag.lib.ag_synchronize(C.c_double(120.0)) == ag.AG_OK
    monkeypatch.delenv("AG_WAIT_TIMEOUT_S")
    r, res, _ = dg.fetch()
    assert res.iterations == ref["iterations"] and np.array_equal(r.view(np.uint32), ref["ranks"].view(np.uint32))
    dg.release()


def test_device_wait_limit_reports_fault_and_context_stays_usable(gpu, oracle, monkeypatch):
    ag = gpu
    g = ag.Graph.rmat(14, 16, seed=3)
    ref = _oracle(oracle, g, 100, 1e-6)
    monkeypatch.setenv("AG_MBAR_SPINS", "0")
    dg = ag.DeviceGraph(g)
    assert dg.tiles().hot_entries > 0
    dg.launch(100, 1e-6, order=ag.AG_ORDER_EXACT)
    with pytest.raises(ag.AGError) as err:
        dg.fetch()
    assert err.value.status == ag.AG_ERR_DEVICE_WAIT
    dg.release()
    monkeypatch.delenv("AG_MBAR_SPINS")
    dg = ag.DeviceGraph(g)
    r, res, _ = dg.pagerank(100, 1e-6, order=ag.AG_ORDER_EXACT)
    assert res.iterations == ref["iterations"] and np.array_equal(r.view(np.uint32), ref["ranks"].view(np.uint32))
    dg.release()
