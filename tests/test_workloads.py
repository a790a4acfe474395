"""Synthetic workload generators (CPU only): the shapes, ranges and seeding that stand in
for the benchmark configurations, at small scales."""
import numpy as np

from rtnn_b200 import workloads as wl


def test_seeded_and_deterministic():
    for f in (lambda s: wl.uniform_cube(500, seed=s), lambda s: wl.gmm(scale=0.001, seed=s)[0],
              lambda s: wl.multicloud(n_clouds=6, lo=64, hi=512, seed=s)[0],
              lambda s: wl.surfaces(scale=0.0005, seed=s)):
        a, b, c = f(1), f(1), f(2)
        assert a.dtype == np.float32 and a.shape[1] == 3
        assert np.array_equal(a, b) and not np.array_equal(a, c)


def test_uniform_cube_range():
    p = wl.uniform_cube(2000, 100.0, seed=0)
    assert p.shape == (2000, 3) and p.min() >= 0.0 and p.max() <= 100.0


def test_multicloud_sizes_and_unit_cube():
    p, off = wl.multicloud(n_clouds=64, seed=3)
    sizes = np.diff(off.astype(np.int64))
    assert len(off) == 65 and off[0] == 0 and int(off[-1]) == len(p)
    assert sizes.min() >= 512 and sizes.max() <= 65536
    for c in range(64):
        q = p[int(off[c]):int(off[c + 1])]
        # each cloud normalised to the unit cube: it touches 0 and 1 on every axis
        assert np.allclose(q.min(0), 0.0, atol=1e-6) and np.allclose(q.max(0), 1.0, atol=1e-6)
    # scale shrinks the cloud count, not the cloud sizes
    _, off2 = wl.multicloud(scale=0.01, seed=3)
    assert len(off2) - 1 == 40


def test_gmm_queries_cover_the_mixture_box():
    p, q = wl.gmm(scale=0.002, seed=1)
    assert len(p) == 2000 and len(q) == 2000
    lo, hi = p.min(0), p.max(0)
    assert (q.min(0) >= lo - 1e-3).all() and (q.max(0) <= hi + 1e-3).all()


def test_sph_lattice_and_step():
    p = wl.sph_lattice(scale=0.001, seed=4)
    n_lat = int(round(len(p) / 1.05))
    # the lattice block holds spacing-1 points with jitter of at most 0.1
    frac = np.abs(p[:n_lat] - np.round(p[:n_lat]))
    assert frac.max() <= 0.1 + 1e-4
    s = wl.sph_step(p, seed=1)
    d = s - p
    assert s.shape == p.shape and 0.03 < d.std() < 0.07   # N(0, 0.05 h) per axis


def test_configs_name_the_benchmark_parameters():
    assert wl.CONFIGS["knn_multicloud_4096"] == dict(mode="knn", radius=0.2, k=32)
    assert wl.CONFIGS["sph_lattice_5e7"]["k"] == 64
    assert set(wl.CONFIGS) == {"radius_uniform_1e5", "knn_gmm_1e6", "knn_surface_1e7",
                               "knn_multicloud_4096", "sph_lattice_5e7"}
