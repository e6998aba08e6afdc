"""Domain decomposition on the device: a mesh cut into partitions steps to the
same bits as the one-partition solve.

Each partition handle owns a range of the Hilbert-ordered vertices, computes
them with the unchanged gather lists and exchanges ghost states and gradients
after every phase (all partitions on one GPU here, exchanged by device copies;
across GPUs the same calls run with NCCL).  The reference instead sums the
partial residuals and gradients of shared vertices across MPI ranks
(src/reduce_residual.cc:14-104, src/fv.cc:827-1030), which reorders sums with
the partition count; owner-computes does not, so the comparison is bitwise.
"""
import numpy as np
import pytest

from tensum_b200 import abi, cases, gpu, partition, preproc

pytestmark = pytest.mark.gpu


def _kh_problem(n, flux, recon, **extra):
    g = preproc.preprocess(cases.kh_mesh(n, 0))
    cfg = dict(flux=flux, reconstruct=recon, boundary={t: ("periodic", {}) for t in (1, 2, 3, 4)},
               final_time=1e9, time_stamps=1, cfl=0.8, **extra)
    a, phi = cases.kh_coefficients(3)
    return abi.Problem(g, cfg), cases.kh_ic(g.coords, a, phi)


def _cyl_problem(flux="kepes_tecno_roe", recon="minmod"):
    m = cases.cylinder_mesh(12, 24, 0)
    g = preproc.preprocess(m)
    T, u, v, p = cases.cylinder_freestream(0.3, 1.0)
    far = {"temperature": T, "xvelocity": u, "yvelocity": v, "zvelocity": 0.0, "pressure": p}
    cfg = dict(flux=flux, reconstruct=recon, model="euler", boundary={1: ("slip", {}), 2: ("farfield", far)},
               final_time=1e9, time_stamps=1, cfl=0.8)
    return abi.Problem(g, cfg), cases.cylinder_ic(g.coords, 0.3, 1.0)


def _one_partition(P, ic, steps):
    s = gpu.Solver(P)
    s.set_state(ic)
    info = s.step(steps)
    out = s.get_state()
    s.close()
    return out, info


@pytest.mark.parametrize("graph,overlap", [(True, True), (False, True), (True, False), (False, False)])
@pytest.mark.parametrize("flux,recon,n_parts", [("kepes_tecno_rusanov", "minmod", 2),
                                                ("kepes_tecno_rusanov", "minmod", 3),
                                                ("kep", "first", 4),
                                                ("roe_ec", "first", 2)])
def test_periodic_partitions_match_one_partition(flux, recon, n_parts, graph, overlap):
    P, ic = _kh_problem(33, flux, recon)
    want, winfo = _one_partition(P, ic, 6)
    ps = partition.PartitionedSolver(P, n_parts, graph=graph, overlap=overlap)
    ps.set_state(ic)
    info = ps.step(6)
    got = ps.get_state()
    assert np.array_equal(got, want)
    assert info[0] == winfo[0] and info[1] == winfo[1] and info[3] == winfo[3]   # elapsed, dt, iterations
    assert abs(info[2] - winfo[2]) <= 1e-12 * abs(winfo[2])                      # norms: sums regrouped
    for p in ps.parts:                                                             # every partition agrees
        assert np.array_equal(p.scalars()[:2], info[:2])
    ps.close()


@pytest.mark.parametrize("n_parts", [1, 2, 5])
def test_boundary_partitions_match_one_partition(n_parts):
    P, ic = _cyl_problem()
    want, winfo = _one_partition(P, ic, 5)
    ps = partition.PartitionedSolver(P, n_parts)
    ps.set_state(ic)
    info = ps.step(5)
    assert np.array_equal(ps.get_state(), want)
    assert info[1] == winfo[1]
    ps.close()


def test_rk4_and_fixed_time_step():
    for extra in (dict(time_scheme="rk4"), dict(time_step=2e-4)):
        P, ic = _kh_problem(17, "kepes_tecno_roe", "minmod", **extra)
        want, winfo = _one_partition(P, ic, 4)
        ps = partition.PartitionedSolver(P, 3)
        ps.set_state(ic, 0.0)
        info = ps.step(4)
        assert np.array_equal(ps.get_state(), want), extra
        assert info[0] == winfo[0]
        ps.close()


def test_restart_from_a_new_state():
    """A new state mid-run takes the partitions back through prime and the dt exchange."""
    P, ic = _kh_problem(17, "kepes_tecno_rusanov", "minmod")
    ps = partition.PartitionedSolver(P, 2)
    ps.set_state(ic)
    ps.step(3)                  # captures the step graph; the restart replays it
    mid = ps.get_state()
    ps.set_state(mid, 0.5)
    ps.step(2)
    got = ps.get_state()
    s = gpu.Solver(P)
    s.set_state(mid, 0.5)
    s.step(2)
    assert np.array_equal(got, s.get_state())


def test_partition_handles_refuse_whole_mesh_calls():
    P, ic = _kh_problem(17, "kep", "first")
    p = partition.Partition(P, 2, 0)
    p.set_state(ic)
    for call in (lambda: p._call("tg_step", 1, None), lambda: p._call("tg_advance", 1, 1, None)):
        with pytest.raises(gpu.TensumError) as e:
            call()
        assert abi.STATUS[e.value.status] == "TG_NOT_SUPPORTED"
    with pytest.raises(gpu.TensumError) as e:
        p.begin()                                   # prime and the dt exchange come first
    assert abi.STATUS[e.value.status] == "TG_INVALID_ARG"
    p.close()
    m = cases.cylinder_mesh(8, 16, 0)
    strong = abi.Problem(preproc.preprocess(m), dict(cases.cylinder_config(0.2, 100.0, 0.0, 1.0, 1), bc_scheme="strong"))
    with pytest.raises(gpu.TensumError) as e:
        partition.Partition(strong, 2, 0)
    assert abi.STATUS[e.value.status] == "TG_NOT_SUPPORTED"


@pytest.mark.parametrize("graph,overlap", [(False, False), (False, True), (True, False), (True, True)])
def test_torch_distributed_path_on_one_rank(graph, overlap):
    """DistPartitionedSolver over a one-rank NCCL group: the collectives run on the
    partition's stream (eagerly, or captured with the phases as one CUDA graph) and
    the result is the one-partition solve."""
    import datetime
    import socket

    import torch.distributed as dist
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1,
                            timeout=datetime.timedelta(seconds=60))
    try:
        P, ic = _kh_problem(17, "kepes_tecno_rusanov", "minmod")
        want, winfo = _one_partition(P, ic, 3)
        d = partition.DistPartitionedSolver(P, device=0, graph=graph, overlap=overlap)
        d.set_state(ic)
        info = d.step(3)
        assert np.array_equal(d.get_state(), want)
        assert info[1] == winfo[1]
        d.close()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("name", ["sq_roe_minmod_voronoi", "sq_kepec_axi_long", "cyl_slip_axi_voronoi"])
def test_voronoi_and_axisymmetric_partitions(name):
    """Voronoi duals (gradient-only edges) and axisymmetric radii go with the
    partition's edges and vertices: partitions repeat the one-partition solve,
    which the fixture pins to the reference."""
    from tests.golden.cases_spec import CASES, build_case
    from tests.helpers import geometry
    mesh, cfg, prim0 = build_case(CASES[name])
    P = abi.Problem(geometry(mesh, cfg), dict(cfg, final_time=1e9, time_stamps=1))
    want, winfo = _one_partition(P, prim0, 4)
    ps = partition.PartitionedSolver(P, 3)
    ps.set_state(prim0)
    info = ps.step(4)
    assert np.array_equal(ps.get_state(), want)
    assert info[1] == winfo[1]
    ps.close()


def test_frontier_tiles_are_the_ones_reading_ghosts():
    """The tile order puts the tiles with a ghost among their vertices first; a single
    partition has none, a mesh cut in two keeps interior tiles."""
    P, ic = _kh_problem(65, "kep", "first")
    for n in (1, 2, 4):
        parts = [partition.Partition(P, n, q) for q in range(n)]
        for p in parts:
            assert 0 <= p.n_frontier <= p.n_tiles
            assert (p.n_frontier == 0) == (n == 1)
            if n == 2:
                assert p.n_frontier < p.n_tiles
            p.close()


@pytest.mark.parametrize("name,n_parts", [("cyl_ns", 2), ("cyl_ns", 3), ("cyl_ns", 4), ("cyl_ns_isothermal", 3),
                                          ("cyl_ns_rusanov_va", 2), ("cyl_ns_axi", 3), ("cyl_ns_voronoi", 2),
                                          ("cyl_ns_rk4", 3)])
def test_navier_stokes_partitions_match_one_partition_and_oracle(name, n_parts):
    """Navier-Stokes meshes with walls and far field: each partition computes the
    viscous units its owned vertices gather (interior cells) and the boundary units
    of its boundary faces from its owned and ghost states (src/fv.cc:1197-1461 splits
    them over MPI partitions and sums shared vertices, src/reduce_residual.cc:14-104).
    The partitioned solve repeats the one-partition solve bit for bit, and both
    follow the oracle."""
    from tests.golden.cases_spec import CASES, build_case
    from tests.helpers import geometry, rel_l2
    import oracle as O
    mesh, cfg, prim0 = build_case(CASES[name])
    P = abi.Problem(geometry(mesh, cfg), dict(cfg, final_time=1e9, time_stamps=1))
    want, winfo = _one_partition(P, prim0, 6)
    ps = partition.PartitionedSolver(P, n_parts)
    ps.set_state(prim0)
    info = ps.step(6)
    got = ps.get_state()
    assert np.array_equal(got, want)
    assert info[1] == winfo[1]
    ps.close()
    o = O.Oracle(P)
    o.set_prim(prim0)
    o.step(6)
    assert rel_l2(got, o.get_prim()) <= 1e-10


@pytest.mark.parametrize("graph,overlap", [(True, True), (False, False)])
def test_navier_stokes_cylinder_partitions_over_many_steps(graph, overlap):
    """The 16 x 32 Navier-Stokes cylinder (adiabatic wall, far field) in 3 partitions
    over 25 steps: bit-identical to one partition and within 1e-10 of the oracle."""
    from tests.helpers import rel_l2
    import oracle as O
    from tensum_b200 import mesh as M
    m = M.annulus(16, 32, 0.5, 20.0, 0.05, seed=2)
    prim0 = cases.cylinder_ic(m.coords)
    prim0[:, 3] += 0.02 * np.cos(m.coords[:, 0])
    cfg = dict(flux="kepes_tecno_roe", reconstruct="minmod", model="ns", mu_ref=0.002,
               boundary={1: ("noslip", {"xvelocity": 0.0, "yvelocity": 0.0, "zvelocity": 0.0}),
                         2: ("farfield", {"temperature": 1 / 1.4, "xvelocity": 0.2, "yvelocity": 0.0,
                                          "zvelocity": 0.0, "pressure": 1 / 1.4})},
               final_time=1e9, time_stamps=1, cfl=0.8)
    P = abi.Problem(preproc.preprocess(m), cfg)
    want, _ = _one_partition(P, prim0, 25)
    ps = partition.PartitionedSolver(P, 3, graph=graph, overlap=overlap)
    ps.set_state(prim0)
    ps.step(25)
    got = ps.get_state()
    ps.close()
    assert np.array_equal(got, want)
    o = O.Oracle(P)
    o.set_prim(prim0)
    o.step(25)
    assert rel_l2(got, o.get_prim()) <= 1e-10
