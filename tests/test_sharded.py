"""CP-ALS sharded by mode-0 slabs (tenrso_b200.sharded), dense and sparse, the
slab-sharded loss/gradient and the batched instance partition, against the
single-process oracle: gloo ranks as CPU processes with the oracle as each
rank's compute (the partition, the all-reduces and the final all-gather are
the real ones), and on a GPU the library's kernels as each rank's compute
(two gloo processes sharing the one GPU: no kernel of one waits on the
other; the exchanges go through host memory).

Parity: with the FP64 oracle as compute the sharded history equals cp_als's
(core.rs:59-182) up to the summation order of the all-reduce (1e-10); with
the fp32 GPU kernels within 1e-4 (cp_als's fit bar), the same iteration
count and stop reason."""
import json
import os
import socket
import subprocess
import sys

import numpy as np
import pytest

from tenrso_b200.sharded import slab_rows

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

WORKER = r"""
import datetime, json, os, sys
import numpy as np
sys.path.insert(0, os.environ["SHARD_ROOT"])
import torch.distributed as dist
from tenrso_b200 import synth
from tenrso_b200.sharded import cp_als_sharded, slab_rows

cfg = json.loads(os.environ["SHARD_CFG"])
dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=120))
me, world = dist.get_rank(), dist.get_world_size()
shape, R = tuple(cfg["shape"]), cfg["rank"]
kind = cfg.get("kind", "cp_als")
if kind == "sparse_cp_als":
    sys.path.insert(0, os.path.join(os.environ["SHARD_ROOT"], "tests"))
    from test_sharded import merged_zipf_coo
    X = merged_zipf_coo(shape, cfg["nnz"], cfg["seed"])
elif kind != "batched":  # the batched instances are drawn below
    X, _ = synth.dense_lowrank(shape, R, seed=cfg["seed"], dist="normal", noise=0.01)
init = synth.init_factors(shape, R, cfg["seed"]) if kind != "batched" else None
r0, r1 = slab_rows(shape[0], world, me)

if kind == "loss_grad":
    from tenrso_b200.sharded import loss_grad_sharded, DeviceBackend
    if cfg["backend"] == "oracle":
        from oracle import oracle as orc

        class OracleBackend:
            put = staticmethod(lambda a: np.asarray(a, dtype=np.float64))
            to_host = staticmethod(lambda a: a)
            norm_sq = staticmethod(lambda X: float(np.sum(X * X)))

            @staticmethod
            def mttkrp(X, factors, mode):
                if X.shape[0] == 0:
                    return np.zeros((X.shape[mode], factors[0].shape[1]))
                return orc.mttkrp(X, factors, mode)

        be = OracleBackend()
        slab = X.astype(np.float64)[r0:r1]
    else:
        be = DeviceBackend()
        slab = X[r0:r1]
    rng = np.random.default_rng(cfg["seed"])
    fs = [rng.standard_normal((n, R)).astype(np.float32) for n in shape]
    loss, grads = loss_grad_sharded(slab, shape[0], fs, cfg["reg"], backend=be)
    dist.barrier()
    dist.destroy_process_group()
    print(json.dumps({"rank": me, "loss": loss, "grads": [g.tolist() for g in grads]}))
    sys.exit(0)

if kind == "batched":
    from tenrso_b200.sharded import batched_cp_als_sharded
    inst = synth.batched_instances(cfg["n_inst"], cfg["seed"])
    ids, res = batched_cp_als_sharded([t for t, _, _ in inst], [r for _, r, _ in inst],
                                      cfg["iters"], 0.0, [i for _, _, i in inst])
    dist.barrier()
    dist.destroy_process_group()
    print(json.dumps({"rank": me, "ids": ids, "fits": [c.fit for c in res],
                      "iters": [c.iters for c in res]}))
    sys.exit(0)

if kind == "sparse_cp_als":
    from tenrso_b200.sharded import cp_als_sparse_sharded, SparseDeviceBackend
    idx, vals = X
    if cfg["backend"] == "oracle":
        from oracle import oracle as orc

        class Slab:
            def __init__(self, idx, vals, shape, r0, r1):
                keep = (idx[:, 0] >= r0) & (idx[:, 0] < r1)
                self.idx = idx[keep].copy()
                self.idx[:, 0] -= r0
                self.vals = vals[keep].astype(np.float64)
                self.shape = [r1 - r0] + list(shape[1:])
                self.ndim = len(shape)

        class OracleSparseBackend:
            put = staticmethod(lambda a: np.asarray(a, dtype=np.float64))
            to_host = staticmethod(lambda a: a)
            norm_sq = staticmethod(lambda X: float(np.sum(X.vals ** 2)))
            slab = staticmethod(Slab)

            @staticmethod
            def mttkrp(X, factors, mode):
                # FP64 COO MTTKRP: M[i_mode] += v * prod_{m != mode} U_m[i_m]
                out = np.zeros((X.shape[mode], factors[0].shape[1]))
                w = X.vals[:, None] * np.ones((1, factors[0].shape[1]))
                for m in range(X.ndim):
                    if m != mode:
                        w = w * factors[m][X.idx[:, m]]
                np.add.at(out, X.idx[:, mode], w)
                return out

            @staticmethod
            def solve(M, H):
                U = orc.solve(M, H) if M.shape[0] else np.zeros_like(M)
                return U, U.T @ U, float(np.sum(M * U))

        be = OracleSparseBackend()
    else:
        be = SparseDeviceBackend()
    res = cp_als_sparse_sharded(idx, vals, shape, R, cfg["iters"], cfg["tol"], init, backend=be)
    dist.barrier()
    dist.destroy_process_group()
    print(json.dumps({"rank": me, "fit": res.fit, "iters": res.iters,
                      "hist": [float(v) for v in res.convergence.fit_history],
                      "reason": res.convergence.reason}))
    sys.exit(0)

if cfg["backend"] == "oracle":
    from oracle import oracle as orc

    class OracleBackend:
        put = staticmethod(lambda a: np.asarray(a, dtype=np.float64))
        to_host = staticmethod(lambda a: a)
        norm_sq = staticmethod(lambda X: float(np.sum(X * X)))

        @staticmethod
        def mttkrp(X, factors, mode):
            if X.shape[0] == 0:
                return np.zeros((X.shape[mode], factors[0].shape[1]))
            return orc.mttkrp(X, factors, mode)

        @staticmethod
        def solve(M, H):
            U = orc.solve(M, H) if M.shape[0] else np.zeros_like(M)
            return U, U.T @ U, float(np.sum(M * U))

    be = OracleBackend()
    slab = X.astype(np.float64)[r0:r1]
else:
    from tenrso_b200.sharded import DeviceBackend
    be = DeviceBackend(precision="fp32")
    slab = X[r0:r1]
res = cp_als_sharded(slab, shape[0], R, cfg["iters"], cfg["tol"], init, backend=be)
dist.barrier()
dist.destroy_process_group()
print(json.dumps({"rank": me, "fit": res.fit, "iters": res.iters,
                  "hist": [float(v) for v in res.convergence.fit_history],
                  "reason": res.convergence.reason,
                  "factors": [np.asarray(f, dtype=np.float64).tolist() for f in res.factors]}))
"""


def merged_zipf_coo(shape, nnz, seed):
    """The seeded Zipf COO (synth.zipf_coo) with its duplicates summed in fp32
    in draw order: (indices with distinct coordinates, values)."""
    from tenrso_b200 import synth
    idx, vals, _ = synth.zipf_coo(shape, nnz, seed)
    keys = np.ravel_multi_index(tuple(idx.T), shape)
    order = np.argsort(keys, kind="stable")
    _, starts = np.unique(keys[order], return_index=True)
    return (np.ascontiguousarray(idx[order][starts]),
            np.add.reduceat(vals[order], starts).astype(np.float32))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def run_ranks(world, cfg):
    port = _free_port()
    procs = []
    for r in range(world):
        env = dict(os.environ, MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(r),
                   WORLD_SIZE=str(world), LOCAL_RANK="0", SHARD_ROOT=ROOT,
                   SHARD_CFG=json.dumps(cfg))
        procs.append(subprocess.Popen([sys.executable, "-c", WORKER], env=env,
                                      stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True))
    results = []
    for p in procs:
        out, err = p.communicate(timeout=600)
        assert p.returncode == 0, err[-3000:]
        results.append(json.loads(out.strip().splitlines()[-1]))
    return sorted(results, key=lambda d: d["rank"])


def oracle_reference(orc, cfg):
    from tenrso_b200 import synth
    shape, R = tuple(cfg["shape"]), cfg["rank"]
    X, _ = synth.dense_lowrank(shape, R, seed=cfg["seed"], dist="normal", noise=0.01)
    init = synth.init_factors(shape, R, cfg["seed"])
    return orc.cp_als(X.astype(np.float64), R, cfg["iters"], cfg["tol"],
                      [f.astype(np.float64) for f in init])


def test_slab_rows_partition():
    for n, w in ((10, 3), (2, 3), (256, 8), (7, 1)):
        parts = [slab_rows(n, w, p) for p in range(w)]
        assert parts[0][0] == 0 and parts[-1][1] == n
        assert all(a[1] == b[0] for a, b in zip(parts, parts[1:]))
        sizes = [b - a for a, b in parts]
        assert max(sizes) - min(sizes) <= 1


@pytest.mark.parametrize("world,shape,rank", [(2, (12, 9, 8), 3), (3, (10, 7, 6, 5), 2),
                                              (3, (2, 6, 5), 2)])
def test_gloo_ranks_equal_single_process_oracle(orc, world, shape, rank):
    """CPU ranks (oracle compute): uneven slabs, a 4-way tensor, and a rank
    that holds no rows at all."""
    cfg = dict(shape=list(shape), rank=rank, seed=0xE5, iters=8, tol=0.0, backend="oracle")
    res = run_ranks(world, cfg)
    factors, info = oracle_reference(orc, cfg)
    for r in res:
        assert r["iters"] == info["iters"] and r["reason"] == info["reason"]
        assert np.allclose(r["hist"], info["fit_history"], rtol=0, atol=1e-10)
        for f, g in zip(r["factors"], factors):
            assert np.allclose(np.asarray(f), g, rtol=1e-7, atol=1e-9)


def test_gloo_ranks_stop_rule(orc):
    """A tolerance stop reached on every rank at the oracle's iteration."""
    cfg = dict(shape=[14, 9, 8], rank=3, seed=0xE6, iters=40, tol=1e-4, backend="oracle")
    res = run_ranks(2, cfg)
    _, info = oracle_reference(orc, cfg)
    for r in res:
        assert r["iters"] == info["iters"] and r["reason"] == info["reason"]


@pytest.mark.gpu
def test_device_ranks_vs_oracle(orc):
    """Two processes on the one GPU, the library's fp32 kernels as compute."""
    cfg = dict(shape=[64, 48, 40], rank=8, seed=0xE7, iters=10, tol=0.0, backend="device")
    res = run_ranks(2, cfg)
    factors, info = oracle_reference(orc, cfg)
    for r in res:
        assert r["iters"] == info["iters"] == 10
        assert np.abs(np.asarray(r["hist"]) - info["fit_history"]).max() <= 1e-4
    assert res[0]["hist"] == res[1]["hist"]


@pytest.mark.gpu
def test_device_single_process_matches_cp_als():
    import tenrso_b200 as tb
    from tenrso_b200 import synth
    from tenrso_b200.sharded import cp_als_sharded
    shape, R = (40, 32, 24), 6
    X, _ = synth.dense_lowrank(shape, R, seed=3, dist="normal", noise=0.01)
    init = synth.init_factors(shape, R, 3)
    sh = cp_als_sharded(X, shape[0], R, 8, 0.0, init)
    ref = tb.cp_als(X, R, 8, 0.0, init=init)
    assert np.abs(sh.convergence.fit_history - ref.convergence.fit_history).max() <= 1e-5


def dense_of(shape, idx, vals):
    X = np.zeros(shape, np.float64)
    X[tuple(idx.T)] = vals.astype(np.float64)
    return X


@pytest.mark.parametrize("world", [2, 3])
def test_gloo_sparse_ranks_equal_dense_oracle(orc, world):
    """CPU ranks holding the nonzeros of their mode-0 slabs (FP64 COO MTTKRP as
    compute) take cp_als's steps on the tensor with its zeros."""
    shape, R = (30, 20, 16), 4
    cfg = dict(kind="sparse_cp_als", shape=list(shape), rank=R, seed=0xE8, nnz=1500, iters=8,
               tol=0.0, backend="oracle")
    res = run_ranks(world, cfg)
    from tenrso_b200 import synth
    idx, vals = merged_zipf_coo(shape, 1500, 0xE8)
    init = [f.astype(np.float64) for f in synth.init_factors(shape, R, 0xE8)]
    _, info = orc.cp_als(dense_of(shape, idx, vals), R, 8, 0.0, init)
    for r in res:
        assert r["iters"] == info["iters"] and r["reason"] == info["reason"]
        assert np.allclose(r["hist"], info["fit_history"], rtol=0, atol=1e-10)


@pytest.mark.parametrize("world,shape", [(2, (12, 9, 8, 5)), (3, (2, 6, 5, 4))])
def test_gloo_loss_grad_equals_vjp(orc, world, shape):
    """Slab-sharded loss and gradients (FP64 oracle compute) against the
    oracle's VJP on the whole tensor; the second case has a rank without rows."""
    R, reg = 3, 1e-3
    cfg = dict(kind="loss_grad", shape=list(shape), rank=R, seed=0xE9, reg=reg,
               backend="oracle")
    res = run_ranks(world, cfg)
    from tenrso_b200 import synth
    X, _ = synth.dense_lowrank(shape, R, seed=0xE9, dist="normal", noise=0.01)
    rng = np.random.default_rng(0xE9)
    fs = [rng.standard_normal((n, R)).astype(np.float32) for n in shape]
    loss_ref, grads_ref = orc.cp_loss_grad_vjp(X, fs, reg)
    for r in res:
        assert abs(r["loss"] - loss_ref) <= 1e-10 * abs(loss_ref)
        for g, gr in zip(r["grads"], grads_ref):
            g = np.asarray(g)
            assert np.linalg.norm(g - gr) <= 1e-10 * np.linalg.norm(gr)


def test_partition_instances():
    from tenrso_b200.sharded import partition_instances
    work = [5.0, 1.0, 9.0, 3.0, 3.0, 7.0, 2.0]
    for world in (1, 2, 3, 8):
        parts = partition_instances(work, world)
        assert sorted(i for p in parts for i in p) == list(range(len(work)))
        assert all(p == sorted(p) for p in parts)
        assert partition_instances(work, world) == parts
    loads = [sum(work[i] for i in p) for p in partition_instances(work, 2)]
    assert max(loads) - min(loads) <= max(work)


@pytest.mark.gpu
def test_device_sparse_ranks_vs_oracle(orc):
    """Two processes on the one GPU, the CSF MTTKRP and FP64 solve as compute."""
    shape, R = (48, 40, 32), 6
    cfg = dict(kind="sparse_cp_als", shape=list(shape), rank=R, seed=0xEA, nnz=20000, iters=8,
               tol=0.0, backend="device")
    res = run_ranks(2, cfg)
    idx, vals = merged_zipf_coo(shape, 20000, 0xEA)
    from tenrso_b200 import synth
    init = [f.astype(np.float64) for f in synth.init_factors(shape, R, 0xEA)]
    _, info = orc.cp_als(dense_of(shape, idx, vals), R, 8, 0.0, init)
    for r in res:
        assert r["iters"] == info["iters"] == 8
        assert np.abs(np.asarray(r["hist"]) - info["fit_history"]).max() <= 1e-4
    assert res[0]["hist"] == res[1]["hist"]


@pytest.mark.gpu
def test_device_loss_grad_ranks(orc):
    """Two processes on the one GPU, the dense MTTKRP as compute (fp32 path):
    within 1e-5 of the oracle's VJP."""
    shape, R, reg = (40, 24, 16, 8), 8, 1e-3
    cfg = dict(kind="loss_grad", shape=list(shape), rank=R, seed=0xEB, reg=reg, backend="device")
    res = run_ranks(2, cfg)
    from tenrso_b200 import synth
    X, _ = synth.dense_lowrank(shape, R, seed=0xEB, dist="normal", noise=0.01)
    rng = np.random.default_rng(0xEB)
    fs = [rng.standard_normal((n, R)).astype(np.float32) for n in shape]
    loss_ref, grads_ref = orc.cp_loss_grad_vjp(X, fs, reg)
    for r in res:
        assert abs(r["loss"] - loss_ref) <= 1e-6 * abs(loss_ref)
        for g, gr in zip(r["grads"], grads_ref):
            g = np.asarray(g)
            assert np.linalg.norm(g - gr) <= 1e-5 * np.linalg.norm(gr)


@pytest.mark.gpu
def test_device_batched_ranks_partition():
    """Two processes on the one GPU split 24 instances by work; each instance's
    result matches the single-process batched run's within the 1e-4 fit bar
    (the autotuned launch configuration depends on the batch's composition,
    and with it the fp32 summation order)."""
    import tenrso_b200 as tb
    from tenrso_b200 import synth
    cfg = dict(kind="batched", shape=[1], rank=1, seed=0xEC, n_inst=24, iters=10)
    res = run_ranks(2, cfg)
    inst = synth.batched_instances(24, 0xEC)
    b = tb.BatchedCpAls([t for t, _, _ in inst], [r for _, r, _ in inst])
    ref = b.cp_als(10, 0.0, init=[i for _, _, i in inst])
    b.close()
    seen = sorted(i for r in res for i in r["ids"])
    assert seen == list(range(24))
    for r in res:
        for i, fit, it in zip(r["ids"], r["fits"], r["iters"]):
            assert it == ref[i].iters and abs(fit - ref[i].fit) <= 1e-4
