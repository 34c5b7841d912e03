"""Learned warm start for the pull PageRank, driven through the C ABI.

The network, its features and its training and inference kernels are the
library's own CUDA code (accelgraph_b200/csrc/ag_mlp.cu); this module only
assembles training sets from this GPU's PageRank results, runs training, and
compares warm-started solves against uniform starting ranks.  Device buffers
are held as torch tensors (plumbing only); every call into the library is
bracketed by stream synchronisation so that torch's stream and the library's
stream never race.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import (AG_ORDER_FAST, AG_PREC_FP32, DeviceGraph, Graph, check, f32p, lib)

NUM_FEATURES = 8


def _torch():
    import torch
    return torch


def _sync():
    _torch().cuda.synchronize()
    check(lib.ag_synchronize(0.0), "ag_synchronize")


class MLP:
    """8 -> 64 -> 64 -> 1 MLP with bfloat16 weights (ag_mlp_t)."""

    def __init__(self, seed: int = 1):
        h = C.c_void_p()
        check(lib.ag_mlp_create(seed, C.byref(h)), "ag_mlp_create")
        self.h = h
        self.num_params = lib.ag_mlp_num_params()

    def release(self) -> None:
        if self.h:
            lib.ag_mlp_release(self.h)
            self.h = None

    def __del__(self):
        try:
            self.release()
        except Exception:
            pass

    @property
    def params(self) -> np.ndarray:
        p = np.empty(self.num_params, np.float32)
        check(lib.ag_mlp_get_params(self.h, p.ctypes.data_as(f32p)), "ag_mlp_get_params")
        return p

    @params.setter
    def params(self, p) -> None:
        p = np.ascontiguousarray(p, np.float32)
        assert p.size == self.num_params
        check(lib.ag_mlp_set_params(self.h, p.ctypes.data_as(f32p)), "ag_mlp_set_params")

    def save(self, path) -> None:
        np.save(path, self.params)

    @classmethod
    def load(cls, path) -> "MLP":
        m = cls()
        m.params = np.load(path)
        return m

    def forward(self, X):
        """X: device tensor (n x 8) -> device tensor (n)."""
        torch = _torch()
        n = X.shape[0]
        Y = torch.empty(n, dtype=torch.float32, device=X.device)
        _sync()
        check(lib.ag_mlp_forward(self.h, X.data_ptr(), n, Y.data_ptr()), "ag_mlp_forward")
        _sync()
        return Y

    def predict(self, X):
        """The warm start's prediction on the tensor cores (ag_mlp_predict):
        bfloat16 head and tail of every feature and activation, binary32
        accumulation."""
        torch = _torch()
        n = X.shape[0]
        Y = torch.empty(n, dtype=torch.float32, device=X.device)
        _sync()
        check(lib.ag_mlp_predict(self.h, X.data_ptr(), n, Y.data_ptr()), "ag_mlp_predict")
        _sync()
        return Y

    def gradients(self, X, T):
        g = np.empty(self.num_params, np.float32)
        loss = C.c_float()
        _sync()
        check(lib.ag_mlp_gradients(self.h, X.data_ptr(), T.data_ptr(), X.shape[0], g.ctypes.data_as(f32p),
                                   C.byref(loss)), "ag_mlp_gradients")
        return g, loss.value

    def train(self, X, T, epochs=20, batch=4096, lr=2e-3) -> float:
        loss = C.c_float()
        _sync()
        check(lib.ag_mlp_train(self.h, X.data_ptr(), T.data_ptr(), X.shape[0], epochs, batch, lr, C.byref(loss)),
              "ag_mlp_train")
        return loss.value

    def warm_start(self, dg: DeviceGraph) -> np.ndarray:
        init = np.empty(dg.num_vertices, np.float32)
        check(lib.ag_mlp_warm_start(dg.h, self.h, init.ctypes.data_as(f32p)), "ag_mlp_warm_start")
        return init


def features(dg: DeviceGraph):
    torch = _torch()
    X = torch.empty((dg.num_vertices, NUM_FEATURES), dtype=torch.float32, device="cuda")
    _sync()
    check(lib.ag_features(dg.h, X.data_ptr()), "ag_features")
    _sync()
    return X


def training_graph_specs(count=200, scales=(14, 18), seed=27491095):
    """Seeded R-MAT / power-law graphs: scale uniform in [14, 18], edge
    factor in [8, 24], quadrant skew a in [0.45, 0.65] (b = c = (1-a)/3 +-)."""
    rng = np.random.default_rng(seed)
    specs = []
    for i in range(count):
        s = int(rng.integers(scales[0], scales[1] + 1))
        ef = int(rng.integers(8, 25))
        a = float(rng.uniform(0.45, 0.65))
        b = c = (1.0 - a) / 3.0
        specs.append((s, ef, a, b, c, 1 + i))
    return specs


def build_training_set(specs, per_graph=4096, epsilon=1e-6, iterations=300, seed=0):
    """Features and targets log(un-normalised rank) from this GPU's FP32
    PageRank on every graph of `specs`; `per_graph` vertices sampled per graph.
    Returns device tensors (X n x 8, T n), shuffled."""
    torch = _torch()
    rng = np.random.default_rng(seed)
    xs, ts = [], []
    for (s, ef, a, b, c, gseed) in specs:
        g = Graph.rmat(s, ef, a, b, c, seed=gseed)
        dg = DeviceGraph(g)
        ranks, res, _ = dg.pagerank(iterations, epsilon, precision=AG_PREC_FP32, order=AG_ORDER_FAST)
        n = g.num_vertices
        X = features(dg)
        t = np.log(ranks.astype(np.float64) * n).astype(np.float32)
        idx = np.sort(rng.choice(n, size=min(per_graph, n), replace=False))
        ti = torch.from_numpy(idx).to(X.device)
        xs.append(X[ti])
        ts.append(torch.from_numpy(t[idx]).to(X.device))
        dg.release()
        g.free()
    X = torch.cat(xs)
    T = torch.cat(ts)
    perm = torch.from_numpy(rng.permutation(X.shape[0])).to(X.device)
    return X[perm].contiguous(), T[perm].contiguous()


def compare(dg: DeviceGraph, model: MLP, iterations=300, epsilon=1e-6):
    """Uniform start vs learned warm start on one graph: passes, device
    milliseconds (warm: features + MLP on the device, then the solve), ranks
    of both."""
    torch = _torch()
    r_u, res_u, _ = dg.pagerank(iterations, epsilon)
    init = torch.empty(dg.num_vertices, dtype=torch.float32, device="cuda")
    _sync()
    stream = torch.cuda.ExternalStream(lib.ag_stream(), device=init.device)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    check(lib.ag_mlp_warm_start_device(dg.h, model.h, init.data_ptr()), "ag_mlp_warm_start_device")
    e1.record(stream)
    e1.synchronize()
    t_pred = e0.elapsed_time(e1)
    r_w, res_w, _ = dg.pagerank(iterations, epsilon, init_ranks=init)
    return {
        "uniform": {"passes": res_u.passes, "iterations": res_u.iterations, "device_ms": res_u.device_ms},
        "warm": {"passes": res_w.passes, "iterations": res_w.iterations, "device_ms": res_w.device_ms,
                 "predict_ms": t_pred},
        "ranks_uniform": r_u, "ranks_warm": r_w, "init": init.cpu().numpy(),
    }
