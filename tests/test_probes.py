"""Probe sampling for the field-evaluation workload: the exact point-to-panel
distance against brute force over every panel, and the rejection radius."""
import numpy as np


def test_panel_distance_matches_brute_force(fp):
    m = fp.meshes.swept_wing("0012", 10, 6)
    rng = np.random.default_rng(0)
    P = rng.uniform([-0.5, -3, -0.3], [3.5, 3, 0.3], size=(200, 3))
    # brute force: every panel, triangles densely sampled as a check of the closed form
    d_all = np.stack([fp.meshes.panel_distance(m, P, np.full(len(P), j)) for j in range(m.npanels)], axis=1)
    d_min = d_all.min(axis=1)
    for j in range(0, m.npanels, 7):
        idx = m.panel_nodes[m.panel_offsets[j]:m.panel_offsets[j + 1]]
        X = m.nodes[idx]
        s = np.linspace(0, 1, 41)
        pts = []
        for a in s:
            for b in s:
                if a + b <= 1:
                    pts.append(X[0] + a * (X[1] - X[0]) + b * (X[2] - X[0]))
                    if len(idx) == 4:
                        pts.append(X[0] + a * (X[2] - X[0]) + b * (X[3] - X[0]))
        pts = np.array(pts)
        dense = np.linalg.norm(P[:, None, :] - pts[None], axis=2).min(axis=1)
        # the sampled surface can only be farther than the exact distance
        assert np.all(d_all[:, j] <= dense + 1e-12)
        assert np.all(dense - d_all[:, j] <= 0.05 * 0.025 * np.linalg.norm(X[1] - X[0]) + 0.02)
    assert np.all(d_min >= 0)


def test_probe_box_rejects_points_near_the_surface(fp):
    m = fp.meshes.swept_wing("0012", 10, 6)
    P = fp.meshes.probe_box(m, 3000, lo=(-0.5, -3, -0.3), hi=(3.5, 3, 0.3), min_dist=0.05, seed=5)
    assert P.shape == (3000, 3)
    d = np.stack([fp.meshes.panel_distance(m, P, np.full(len(P), j)) for j in range(m.npanels)], axis=1).min(axis=1)
    assert d.min() >= 0.05
    Q = fp.meshes.probe_box(m, 3000, lo=(-0.5, -3, -0.3), hi=(3.5, 3, 0.3), min_dist=0.05, seed=5)
    np.testing.assert_array_equal(P, Q)   # seeded
