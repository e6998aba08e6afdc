"""Monte Carlo group split and the rank-ordered group reduction (CPU, gloo).

The product's reduction (tensum_b200.mc.reduce_groups) runs here over two gloo
ranks, each holding one group's raw moments computed by the oracle on its
shard of the reference MC fixture's samples; the merge arithmetic injected
into it is the oracle's restatement of reduce_moments.  Rank 0's reduced,
finalised moments must equal a single-process merge of the same groups bit for
bit, and the reference driver's single-group result to rounding.
"""
import json
import os
import socket

import numpy as np
import pytest

from tests.golden.cases_spec import MC_CASE, MC_EXTRAS, build_mc_case
from tests.helpers import GOLDEN
from tensum_b200 import abi, mc, preproc

import oracle as O  # noqa: E402


def test_group_range_matches_reference_split():
    # src/parameter.cc:831-842 for 10 samples over 3 groups: 4, 3, 3
    assert [mc.group_range(10, 3, g) for g in range(3)] == [(0, 3), (4, 6), (7, 9)]
    assert [mc.group_range(4, 4, g) for g in range(4)] == [(0, 0), (1, 1), (2, 2), (3, 3)]
    assert [mc.group_range(7, 2, g) for g in range(2)] == [(0, 3), (4, 6)]
    with pytest.raises(ValueError):
        mc.group_range(2, 3, 0)
    covered = []
    for g in range(5):
        s, e = mc.group_range(23, 5, g)
        covered += list(range(s, e + 1))
    assert covered == list(range(23))


def _problem():
    mesh, cfg, rows = build_mc_case()
    core = {k: v for k, v in cfg.items() if k not in ("samples", "rnd_per_sample", "ic", "variables")}
    return abi.Problem(preproc.preprocess(mesh), core)


def _to_block(fm, sm, m2):
    """(n_vertex, nvar) arrays -> one [3][nvar][n_vertex] block."""
    return np.stack([fm.T, sm.T, m2.T])


def _worker(rank, world, port, out_dir):
    import datetime
    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        d = dict(np.load(f"{GOLDEN}/mc_kh.npz"))
        n_inst = len(d["time_instance"])
        ics = list(d["ics"])
        mine = [ics[i] for i in range(*[a + b for a, b in zip(mc.group_range(len(ics), world, rank), (0, 1))])]
        fm, sm, m2 = O.run_mc(_problem(), mine, n_inst, MC_EXTRAS)

        def local_block(t):
            return torch.from_numpy(_to_block(fm[t], sm[t], m2[t]))

        def merge(t, n_self, n_other, blk):
            b = blk.numpy()
            O.moments_merge(n_self, fm[t], sm[t], m2[t], n_other, b[0].T.copy(), b[1].T.copy(), b[2].T.copy())

        n = mc.reduce_groups(local_block, len(mine), merge, dist=dist, n_instances=n_inst)
        if rank == 0:
            for t in range(n_inst):
                O.moments_finalize(n, sm[t], m2[t])
            np.savez(os.path.join(out_dir, "reduced.npz"), fm=fm, sm=sm, m2=m2, n=n)
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_rank_reduction_matches_serial_merge_and_reference(tmp_path):
    import torch.multiprocessing as tmp
    tmp.start_processes(_worker, args=(2, _free_port(), str(tmp_path)), nprocs=2, join=True, start_method="spawn")
    r = dict(np.load(tmp_path / "reduced.npz"))
    assert int(r["n"]) == len(MC_CASE["samples"])

    d = dict(np.load(f"{GOLDEN}/mc_kh.npz"))
    n_inst = len(d["time_instance"])
    ics = list(d["ics"])
    P = _problem()
    s0, e0 = mc.group_range(len(ics), 2, 0)
    a = O.run_mc(P, ics[s0:e0 + 1], n_inst, MC_EXTRAS)
    b = O.run_mc(P, ics[e0 + 1:], n_inst, MC_EXTRAS)
    for t in range(n_inst):
        fm, sm, m2 = a[0][t].copy(), a[1][t].copy(), a[2][t].copy()
        n = O.moments_merge(e0 + 1, fm, sm, m2, len(ics) - e0 - 1, b[0][t], b[1][t], b[2][t])
        O.moments_finalize(n, sm, m2)
        assert np.array_equal(r["fm"][t], fm) and np.array_equal(r["sm"][t], sm) and np.array_equal(r["m2"][t], m2)
        for got, key, tol in ((fm, "fm", 1e-14), (sm, "sm", 1e-14), (m2, "var", 1e-11)):
            ref = d[f"m{t}_{key}"].reshape(got.shape)
            assert np.all(np.abs(got - ref) <= tol * np.abs(ref).max(axis=0)), (key, t)
