"""The multi-GPU partition on CPU: two gloo ranks split a solve's tiles.

Each rank takes its share from the host planner (pd_plan_tiles), evaluates the
pairs of its tiles in FP64 numpy exactly as the kernels partition them (i in
the 128-atom block, j in the tile's range, j > i), adds the i = j terms only
on rank 0, and the ranks all-reduce the six-term partials over gloo. The sum
must equal the oracle, and the shares must cover every pair exactly once.
"""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from conftest import ROOT


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _request(solvent):
    from pripps_b200.debye import DebyeRequest
    rng = np.random.default_rng(5)
    n, nq = 413, 29
    xyz = rng.uniform(-9, 9, (n, 3))
    sp = rng.integers(0, 3, n)
    ffA = rng.uniform(1, 8, (3, nq))
    if not solvent:
        return DebyeRequest(xyz, sp, ffA, None, None, None, 0.0, 0.6, nq, None, "fp32")
    ffC = rng.uniform(0.2, 3, (3, nq))
    w = np.where(rng.random(n) < 0.4, 1.3, 0.0)
    fw = rng.uniform(5, 10, nq)
    return DebyeRequest(xyz, sp, ffA, ffC, w, fw, 0.0, 0.6, nq, None, "fp32")


def _partial_terms(req, tiles, perm, K, rank):
    """FP64 six-term partial sums over the pairs of the given tiles."""
    nq = req.nq
    q = np.array([req.qmin + (req.qmax - req.qmin) * k / max(nq - 1, 1) for k in range(nq)])
    A = req.ff_atoms[req.species]                        # [N, nq]
    Cx = req.ff_excluded[req.species] if req.ff_excluded is not None else np.zeros_like(A)
    B = (req.hyd_weights[:, None] * req.ff_water[None, :]) if req.hyd_weights is not None \
        else np.zeros_like(A)
    out = np.zeros((6, nq))
    for i0, j0, j1, qb, _frame in tiles:
        ks = np.arange(qb * K, min((qb + 1) * K, nq))
        if len(ks) == 0:
            continue
        ii = np.arange(i0, i0 + 128)
        jj = np.arange(j0, j1)
        I, J = np.meshgrid(ii, jj, indexing="ij")
        m = (J > I) & (perm[I] >= 0) & (perm[J] >= 0)
        a, b = perm[I[m]], perm[J[m]]
        r = np.linalg.norm(req.xyz[a] - req.xyz[b], axis=1)
        x = q[None, ks] * r[:, None]
        with np.errstate(invalid="ignore", divide="ignore"):
            d = np.where(np.abs(x) < 1e-8, 1.0, np.sin(x) / x)
        Aa, Ab = A[a][:, ks], A[b][:, ks]
        Ca, Cb = Cx[a][:, ks], Cx[b][:, ks]
        Ba, Bb = B[a][:, ks], B[b][:, ks]
        out[0, ks] += (2 * Aa * Ab * d).sum(0)
        out[1, ks] += (2 * Ca * Cb * d).sum(0)
        out[2, ks] += (2 * Ba * Bb * d).sum(0)
        out[3, ks] += ((Aa * Cb + Ca * Ab) * d).sum(0)
        out[4, ks] += ((Aa * Bb + Ba * Ab) * d).sum(0)
        out[5, ks] += ((Ca * Bb + Ba * Cb) * d).sum(0)
    if rank == 0:
        out[0] += (A * A).sum(0)
        out[1] += (Cx * Cx).sum(0)
        out[2] += (B * B).sum(0)
        out[3] += (A * Cx).sum(0)
        out[4] += (A * B).sum(0)
        out[5] += (Cx * B).sum(0)
    return out


def _worker(rank, world, port, solvent, result_path):
    import sys
    import ctypes as C
    import torch
    sys.path.insert(0, str(ROOT))
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    from pripps_b200 import _lib, shard
    req = _request(solvent)
    tiles, perm = shard.tiles(req, rank, world)
    k = C.c_uint32()
    _lib.lib().pd_get_tuning(None, req.n_atoms, req.nq, 0, C.byref(k), None, None)
    part = torch.from_numpy(_partial_terms(req, tiles, perm, k.value, rank))
    # pair coverage of this share (q-block 0 tiles)
    cover = 0
    for i0, j0, j1, qb, _ in tiles:
        if qb != 0:
            continue
        ii = np.arange(i0, i0 + 128)[:, None]
        jj = np.arange(j0, j1)[None, :]
        cover += int(((jj > ii) & (perm[ii] >= 0) & (perm[jj] >= 0)).sum())
    cnt = torch.tensor([cover, len(tiles)], dtype=torch.int64)
    dist.all_reduce(part, op=dist.ReduceOp.SUM)
    dist.all_reduce(cnt, op=dist.ReduceOp.SUM)
    if rank == 0:
        np.savez(result_path, terms=part.numpy(), cover=cnt.numpy())
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("solvent", [False, True])
def test_two_rank_partition_sums_to_oracle(tmp_path, solvent):
    from oracle import oracle as O
    from pripps_b200 import shard
    from conftest import term_errors
    world = 2
    path = str(tmp_path / "res.npz")
    mp.start_processes(_worker, args=(world, _free_port(), solvent, path), nprocs=world,
                       join=True, start_method="spawn")
    res = np.load(path)
    req = _request(solvent)
    n = req.n_atoms
    assert res["cover"][0] == n * (n - 1) // 2
    all_tiles, _ = shard.tiles(req, 0, 1)
    assert res["cover"][1] == len(all_tiles)
    ref = O.terms_for_request(req, precise=True)
    err = term_errors(res["terms"], ref)
    assert np.all(err < 1e-12), err


def test_shares_are_disjoint_and_balanced():
    from pripps_b200 import shard
    req = _request(True)
    full, _ = shard.tiles(req, 0, 1)
    parts = [shard.tiles(req, r, 3)[0] for r in range(3)]
    key = lambda t: tuple(t)
    union = sorted(map(key, np.concatenate(parts)))
    assert union == sorted(map(key, full))
    cost = [int(((p[:, 2] - p[:, 1]).astype(np.int64)).sum()) for p in parts]
    assert max(cost) - min(cost) <= max(full[:, 2] - full[:, 1])
