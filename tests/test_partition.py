"""Domain decomposition on the host: partition plans and the exchange over gloo.

The plan (tg_part_plan, no device) must cover every vertex exactly once, pair
each sender's entries with the receiver's entry for entry, and give every
partition the ghosts its owned vertices reach.  The exchange itself
(tensum_b200.partition.DistTransport, the code path the NCCL ranks run) moves
halo records and the step scalars between gloo ranks here; the device kernels
that pack and unpack them are covered by the GPU tests.
"""
import os
import socket

import numpy as np
import pytest

from tensum_b200 import abi, cases, gpu, partition, preproc

pytestmark = pytest.mark.skipif(gpu.load() is None, reason="library not loadable")


def _kh(n=17):
    g = preproc.preprocess(cases.kh_mesh(n, 0))
    return abi.Problem(g, dict(flux="kepes_tecno_rusanov", reconstruct="minmod",
                               boundary={t: ("periodic", {}) for t in (1, 2, 3, 4)}))


def _cyl():
    m = cases.cylinder_mesh(8, 16, 0)
    T, u, v, p = cases.cylinder_freestream(0.3, 1.0)
    far = {"temperature": T, "xvelocity": u, "yvelocity": v, "zvelocity": 0.0, "pressure": p}
    return abi.Problem(preproc.preprocess(m), dict(flux="kepes_tecno_roe", reconstruct="minmod", model="euler",
                                                   boundary={1: ("slip", {}), 2: ("farfield", far)}))


def _cyl_ns():
    m = cases.cylinder_mesh(8, 16, 0)
    return abi.Problem(preproc.preprocess(m), cases.cylinder_config(0.2, 100.0, 0.0, 1.0, 1))


@pytest.mark.parametrize("make", [_kh, _cyl, _cyl_ns])
@pytest.mark.parametrize("n_parts", [1, 2, 3, 5])
def test_plans_cover_and_pair(make, n_parts):
    P = make()
    nv = P.geom.n_vertex
    plans = [partition.plan(P, n_parts, q) for q in range(n_parts)]
    owned = np.concatenate([p["local"][:p["n_owned"]] for p in plans])
    assert np.array_equal(np.sort(owned), np.arange(nv))          # every vertex owned exactly once
    owner = np.empty(nv, int)
    for q, p in enumerate(plans):
        owner[p["local"][:p["n_owned"]]] = q
        ghosts = p["local"][p["n_owned"]:]
        assert np.all(owner[ghosts] != q) if len(ghosts) else True
        assert len(np.unique(p["local"])) == len(p["local"])
        assert p["recv_counts"][q] == 0 and p["send_counts"][q] == 0
        assert p["recv_counts"].sum() == p["n_ghost"]
    for q, p in enumerate(plans):
        # ghosts arrive grouped by owner, ascending
        r_off = np.concatenate([[0], np.cumsum(p["recv_counts"])])
        for s in range(n_parts):
            ids = p["local"][p["recv_idx"][r_off[s]:r_off[s + 1]]]
            assert np.all(owner[ids] == s)
            # the sender's list names the same vertices in the same order
            ps = plans[s]
            s_off = np.concatenate([[0], np.cumsum(ps["send_counts"])])
            sent = ps["local"][ps["send_idx"][s_off[q]:s_off[q + 1]]]
            assert np.array_equal(sent, ids)
            assert np.all(ps["send_idx"][s_off[q]:s_off[q + 1]] < ps["n_owned"])


def test_ghosts_are_the_owned_vertices_neighbours():
    """Every edge neighbour of an owned vertex is local, periodic partners' included."""
    P = _kh(17)
    g = P.geom
    fv = np.asarray(g.face_vertex).reshape(-1, 2)
    part_of = {}
    plans = [partition.plan(P, 3, q) for q in range(3)]
    sets = []
    for q, p in enumerate(plans):
        sets.append(set(p["local"].tolist()))
        for v in p["local"][:p["n_owned"]]:
            part_of[int(v)] = q
    groups = {}
    for s in g.periodic_sets:
        for v in s:
            groups[int(v)] = [int(x) for x in s]
    for a, b in fv:
        for x, y in ((a, b), (b, a)):
            for member in groups.get(int(x), [int(x)]):
                assert int(y) in sets[part_of[member]]


def test_plan_refuses_bad_indices():
    P = _cyl()
    assert partition.plan(P, 2, 1)["n_owned"] > 0
    for n_parts, part in ((2, 2), (2, -1), (0, 0), (P.geom.n_vertex + 1, 0)):
        with pytest.raises(gpu.TensumError) as e:
            partition.plan(P, n_parts, part)
        assert abi.STATUS[e.value.status] == "TG_INVALID_ARG"


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _value(ids, c):
    return ids.astype(np.float64) * 10.0 + c


def _worker(rank, world, port, out_dir):
    import datetime
    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        P = {2: _kh(17), 3: _cyl(), 4: _cyl_ns()}[world]
        p = partition.plan(P, world, rank)
        n_own, local = p["n_owned"], p["local"]
        rec = np.full((len(local), partition.WIDTH), np.nan)
        for c in range(partition.WIDTH):
            rec[:n_own, c] = _value(local[:n_own], c)
        send = torch.from_numpy(rec[p["send_idx"]].reshape(-1).copy() if len(p["send_idx"]) else np.zeros(1))
        recv = torch.zeros(max(1, p["n_ghost"] * partition.WIDTH), dtype=torch.float64)
        t = partition.DistTransport()
        t.alltoall(send, recv, p["send_counts"], p["recv_counts"])
        if p["n_ghost"]:
            rec[p["recv_idx"]] = recv.numpy()[:p["n_ghost"] * partition.WIDTH].reshape(-1, partition.WIDTH)
        ok = all(np.array_equal(rec[:, c], _value(local, c)) for c in range(partition.WIDTH))
        # step scalars: dt minimum (bits) and norm sums, gathered in rank order
        mine = np.array([3.0 + rank, rank + 0.5, 1.0, 2.0, 4.0 * rank]).view(np.int64).copy()
        mine[0] = np.array([0.25 / (rank + 1)]).view(np.int64)[0]
        everyone = torch.zeros(world * partition.REC, dtype=torch.int64)
        t.allgather(torch.from_numpy(mine), everyone)
        np.save(os.path.join(out_dir, f"r{rank}.npy"), np.concatenate([[float(ok)], everyone.numpy().view(np.float64)]))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3, 4])
def test_exchange_over_gloo_fills_every_ghost(tmp_path, world):
    import torch.multiprocessing as tmp
    tmp.start_processes(_worker, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True,
                        start_method="spawn")
    rows = [np.load(tmp_path / f"r{r}.npy") for r in range(world)]
    for r in rows:
        assert r[0] == 1.0
        assert np.array_equal(r[1:], rows[0][1:])       # every rank holds the same gathered records
    rec = rows[0][1:].reshape(world, partition.REC)
    # the fixed-order reduction k_part_import applies: minimum dt, summed norms
    assert rec[:, 0].min() == 0.25 / world
    assert rec[:, 4].sum() == sum(4.0 * r for r in range(world))


class _Part:
    """Records the phases run_step issues (stands in for a partition handle)."""

    def __init__(self, log, grads, n_rks=3):
        self.log, self.grads, self.n_rks = log, grads, n_rks

    def begin(self):
        self.log.append("begin")

    def gradients(self, r, tiles=partition.TILES_ALL):
        self.log.append(f"grad{r}:{tiles}")

    def flux(self, r, tiles=partition.TILES_ALL):
        self.log.append(f"flux{r}:{tiles}")


class _Exchange:
    def __init__(self, log):
        self.log = log

    def start(self, field):
        self.log.append(f"start:{field}")

    def finish(self, field):
        self.log.append(f"finish:{field}")

    def halo(self, field):
        self.log.append(f"halo:{field}")

    def scalars(self):
        self.log.append("scalars")


@pytest.mark.parametrize("grads", [True, False])
def test_overlap_schedule_keeps_every_dependency(grads):
    """Interior tiles run while an exchange is in flight; frontier tiles and the next
    exchange of a field only after the previous one finished; the last state
    exchange completes before the step's scalar exchange."""
    log = []
    partition.run_step([_Part(log, grads)], _Exchange(log), overlap=True)
    I, F = partition.TILES_INTERIOR, partition.TILES_FRONTIER
    S, G = partition.HALO_STATE, partition.HALO_GRAD
    want = ["begin"]
    for r in range(3):
        if grads:
            want += [f"grad{r}:{I}"] + ([f"finish:{S}"] if r else []) + [f"grad{r}:{F}", f"start:{G}",
                                                                           f"flux{r}:{I}", f"finish:{G}"]
        else:
            want += [f"flux{r}:{I}"] + ([f"finish:{S}"] if r else [])
        want += [f"flux{r}:{F}", f"start:{S}"]
    want += [f"finish:{S}", "scalars"]
    assert log == want
    log.clear()
    partition.run_step([_Part(log, grads)], _Exchange(log), overlap=False)
    A = partition.TILES_ALL
    want = ["begin"]
    for r in range(3):
        want += ([f"grad{r}:{A}", f"halo:{G}"] if grads else []) + [f"flux{r}:{A}", f"halo:{S}"]
    assert log == want + ["scalars"]
