"""Synthetic meshes: sizes of the benchmark configurations, periodic sets, part-file round trip."""
import os

import numpy as np
import pytest

from tensum_b200 import cases, mesh as M, preproc


def n_edges(m):
    e = np.concatenate([m.cells[:, [0, 1]], m.cells[:, [1, 2]], m.cells[:, [2, 0]]])
    e.sort(axis=1)
    return np.unique(e, axis=0).shape[0]


def test_cfg0_sizes():
    m = cases.vortex_mesh(65, 0)
    assert (m.n_vertex, m.n_cell, n_edges(m)) == (4225, 8192, 12416)
    assert len(m.periodic_sets) == 2 * 63 + 1


def test_cfg2_sizes():
    m = cases.cylinder_mesh(256, 512, 0)
    assert (m.n_vertex, m.n_cell, n_edges(m)) == (131072, 261120, 392192)
    r = np.hypot(m.coords[:, 0], m.coords[:, 1])
    assert r.min() == pytest.approx(0.5) and r.max() == pytest.approx(20.0)


def test_cells_are_counter_clockwise_and_jitter_bounded():
    m = M.periodic_square(33, 0.0, 1.0, 0.0, 1.0, seed=1)
    g = preproc.preprocess(m)
    assert np.all(g.cell_area > 0)
    h = 1.0 / 32
    ij = np.stack(np.meshgrid(np.arange(33), np.arange(33), indexing="xy"), -1).reshape(-1, 2) * h
    assert np.abs(m.coords - ij).max() <= 0.15 * h + 1e-15


def test_periodic_copies_share_coordinates_modulo_period():
    m = M.periodic_square(17, 0.0, 1.0, 0.0, 1.0, seed=2)
    for s in m.periodic_sets:
        xy = m.coords[s]
        d = np.abs(xy - xy[0]) % 1.0
        assert np.all(np.minimum(d, 1.0 - d) < 1e-14)


def test_dual_areas_tile_the_domain():
    m = M.periodic_square(17, 0.0, 1.0, 0.0, 1.0, seed=2)
    g = preproc.preprocess(m)
    w = np.ones(m.n_vertex)
    for s in m.periodic_sets:
        w[s] = 1.0 / len(s)
    assert (g.dcarea * w).sum() == pytest.approx(1.0, rel=1e-13)


def test_part_file_round_trip(tmp_path):
    m = M.annulus(5, 10, 0.5, 3.0, 0.2, seed=3)
    p = M.write_part_file(m, str(tmp_path))
    r = M.read_part_file(p)
    assert np.array_equal(r.coords, m.coords)
    assert np.array_equal(r.cells, m.cells)
    assert np.array_equal(r.bfaces, m.bfaces)
