"""The rounded-box loudspeaker enclosure generator (mesh.rounded_box_enclosure):
the mesh behind the batched-sweep and adjoint-gradient workloads (a rounded
box 0.2 x 0.3 x 0.25 m with a 0.05 m piston on the front face, seeded jitter).
CPU only."""
import math

import numpy as np
import pytest

from beat_engine_b200 import mesh as M

SIZE = np.array([0.2, 0.3, 0.25])
FILLET = 0.02


def rounded_box_distance(p):
    """Signed distance to the rounded box (0 on its surface)."""
    q = np.abs(p) - (SIZE / 2 - FILLET)
    return np.linalg.norm(np.maximum(q, 0.0), axis=1) + np.minimum(q.max(axis=1), 0.0) - FILLET


@pytest.mark.parametrize("target", [2000, 6000, 12000])
def test_closed_outward_and_on_the_surface(target):
    m = M.rounded_box_enclosure(target, seed=3)
    F, V = m.num_faces, m.num_vertices
    assert abs(F - target) <= 0.1 * target
    assert V == F // 2 + 2  # closed surface of genus 0
    # every edge shared by exactly two faces, once in each direction
    edges = {}
    for a, b, c in np.asarray(m.faces):
        for e in ((a, b), (b, c), (c, a)):
            edges[e] = edges.get(e, 0) + 1
    assert all(n == 1 for n in edges.values())
    assert all((b, a) in edges for a, b in edges)
    v = np.asarray(m.vertices)
    f = np.asarray(m.faces)
    vol = np.einsum("ij,ij->i", v[f[:, 0]], np.cross(v[f[:, 1]], v[f[:, 2]])).sum() / 6.0
    box = np.prod(SIZE)
    assert 0.95 * box < vol < box  # the fillets and the inscribed facets take a little
    assert np.abs(rounded_box_distance(v)).max() <= 1e-12
    piston = m.areas[m.physical_tags == 2].sum()
    assert abs(piston - math.pi * 0.05 ** 2) <= 0.06 * math.pi * 0.05 ** 2
    assert np.all(m.centroids[m.physical_tags == 2][:, 2] > SIZE[2] / 2 - 1e-9)


def test_seeded_jitter():
    a = M.rounded_box_enclosure(2000, seed=5)
    b = M.rounded_box_enclosure(2000, seed=5)
    c = M.rounded_box_enclosure(2000, seed=6)
    plain = M.rounded_box_enclosure(2000, jitter=0.0)
    assert np.array_equal(a.vertices, b.vertices) and not np.array_equal(a.vertices, c.vertices)
    h = math.sqrt(2 * 2 * (0.2 * 0.3 + 0.3 * 0.25 + 0.2 * 0.25) / 2000)
    shift = np.linalg.norm(a.vertices - plain.vertices, axis=1)
    assert 0 < shift.max() <= 0.05 * h * math.sqrt(2) * 1.5
