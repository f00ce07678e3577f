"""CP-ALS sharded by mode-0 slabs (tenrso_b200.sharded) against the
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
X, _ = synth.dense_lowrank(shape, R, seed=cfg["seed"], dist="normal", noise=0.01)
init = synth.init_factors(shape, R, cfg["seed"])
r0, r1 = slab_rows(shape[0], world, me)

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
