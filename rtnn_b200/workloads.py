"""Seeded synthetic point clouds for the benchmark configurations (numpy PCG64).

The reference ships no datasets beyond an 8-point sample (src/samplepc.txt); its
comments name clouds that are not in the project (util.cpp:587, 653). These generators
stand in for them with the shapes, sizes and value distributions of the five
configurations the engine is measured on. Every generator takes a `scale` in (0, 1] that
shrinks the point counts (not the geometry's extent) for parity tests.
"""
import numpy as np

CONFIGS = {
    "radius_uniform_1e5": dict(mode="radius", radius=4.0, k=50),
    "knn_gmm_1e6": dict(mode="knn", radius=10.0, k=5),
    "knn_surface_1e7": dict(mode="knn", radius=2.0, k=16),
    "knn_multicloud_4096": dict(mode="knn", radius=0.2, k=32),
    "sph_lattice_5e7": dict(mode="radius", radius=2.0, k=64),
}


def _rng(seed):
    return np.random.Generator(np.random.PCG64(seed))


def uniform_cube(n=100_000, side=100.0, seed=0, scale=1.0):
    """N points i.i.d. uniform in [0, side]^3 (queries = points)."""
    n = max(1, int(n * scale))
    return _rng(seed).uniform(0.0, side, size=(n, 3)).astype(np.float32)


def gmm(n=1_000_000, n_comp=64, box=1000.0, sigma=(5.0, 40.0), seed=1, scale=1.0,
        n_queries=None):
    """Isotropic Gaussian mixture (centers U[0, box]^3, sigma U[sigma], equal weights)
    plus separate queries uniform over the mixture's bounding box."""
    rng = _rng(seed)
    n = max(1, int(n * scale))
    nq = n if n_queries is None else max(1, int(n_queries * scale))
    centers = rng.uniform(0.0, box, size=(n_comp, 3))
    sig = rng.uniform(sigma[0], sigma[1], size=n_comp)
    comp = rng.integers(0, n_comp, size=n)
    pts = centers[comp] + rng.standard_normal((n, 3)) * sig[comp, None]
    pts = pts.astype(np.float32)
    lo, hi = pts.min(axis=0), pts.max(axis=0)
    qs = rng.uniform(lo, hi, size=(nq, 3)).astype(np.float32)
    return pts, qs


def surfaces(n=10_000_000, n_spheres=200, n_quads=200, box=1000.0, seed=2, scale=1.0,
             noise=0.05):
    """Surface-like cloud: points on random spheres (radius U[5, 50]) and planar quads
    (side U[20, 200], random orientation) in [0, box]^3, sampled in proportion to area,
    with Gaussian noise of `noise` along each surface normal."""
    rng = _rng(seed)
    n = max(1, int(n * scale))
    sc = rng.uniform(0.0, box, size=(n_spheres, 3))
    sr = rng.uniform(5.0, 50.0, size=n_spheres)
    qc = rng.uniform(0.0, box, size=(n_quads, 3))
    qside = rng.uniform(20.0, 200.0, size=n_quads)
    # random orthonormal frames for quads
    a = rng.standard_normal((n_quads, 3))
    a /= np.linalg.norm(a, axis=1, keepdims=True)
    b = rng.standard_normal((n_quads, 3))
    b -= (b * a).sum(axis=1, keepdims=True) * a
    b /= np.linalg.norm(b, axis=1, keepdims=True)
    nrm = np.cross(a, b)
    areas = np.concatenate([4.0 * np.pi * sr ** 2, qside ** 2])
    prob = areas / areas.sum()
    which = rng.choice(n_spheres + n_quads, size=n, p=prob)
    out = np.empty((n, 3), dtype=np.float64)
    isph = which < n_spheres
    ns = int(isph.sum())
    if ns:
        s = which[isph]
        d = rng.standard_normal((ns, 3))
        d /= np.linalg.norm(d, axis=1, keepdims=True)
        rad = sr[s] + rng.standard_normal(ns) * noise
        out[isph] = sc[s] + d * rad[:, None]
    iq = ~isph
    nqd = n - ns
    if nqd:
        q = which[iq] - n_spheres
        u = rng.uniform(-0.5, 0.5, size=(nqd, 2)) * qside[q, None]
        out[iq] = (qc[q] + u[:, :1] * a[q] + u[:, 1:] * b[q] +
                   (rng.standard_normal(nqd) * noise)[:, None] * nrm[q])
    return out.astype(np.float32)


def multicloud(n_clouds=4096, lo=512, hi=65536, seed=3, scale=1.0):
    """Independent clouds, sizes log-uniform in [lo, hi], each a 1-8 component isotropic
    Gaussian mixture normalised to the unit cube. Returns (points, offsets[n_clouds+1])."""
    rng = _rng(seed)
    n_clouds = max(1, int(n_clouds * scale))
    sizes = np.exp(rng.uniform(np.log(lo), np.log(hi), size=n_clouds)).astype(np.int64)
    sizes = np.maximum(sizes, 1)
    offsets = np.zeros(n_clouds + 1, dtype=np.uint64)
    offsets[1:] = np.cumsum(sizes)
    pts = np.empty((int(offsets[-1]), 3), dtype=np.float32)
    for c in range(n_clouds):
        m = int(sizes[c])
        nc = int(rng.integers(1, 9))
        centers = rng.uniform(0.0, 1.0, size=(nc, 3))
        sig = rng.uniform(0.02, 0.2, size=nc)
        comp = rng.integers(0, nc, size=m)
        p = centers[comp] + rng.standard_normal((m, 3)) * sig[comp, None]
        pmin, pmax = p.min(axis=0), p.max(axis=0)
        p = (p - pmin) / np.maximum(pmax - pmin, 1e-12)
        pts[int(offsets[c]):int(offsets[c + 1])] = p.astype(np.float32)
    return pts, offsets


def sph_lattice(nx=500, ny=200, nz=500, h=1.0, jitter=0.1, splash=0.05,
                domain=(2000.0, 1000.0, 2000.0), seed=4, scale=1.0):
    """Jittered cubic lattice (spacing h, jitter U[-jitter, jitter]*h) filling an
    nx*ny*nz block at the bottom centre of the domain, plus `splash` * lattice-size
    particles uniform in the whole domain. `scale` shrinks the block edge-wise."""
    rng = _rng(seed)
    f = scale ** (1.0 / 3.0)
    nx, ny, nz = max(1, int(nx * f)), max(1, int(ny * f)), max(1, int(nz * f))
    dom = np.array(domain, dtype=np.float64) * f
    x0 = np.array([(dom[0] - nx * h) / 2.0, 0.0, (dom[2] - nz * h) / 2.0])
    n_lat = nx * ny * nz
    out = np.empty((n_lat + int(splash * n_lat), 3), dtype=np.float32)
    # build the lattice slab by slab to bound memory
    yy, xx = np.meshgrid(np.arange(ny), np.arange(nx), indexing="ij")
    base = np.stack([xx.ravel(), yy.ravel()], axis=1).astype(np.float64)
    per = nx * ny
    for z in range(nz):
        s = slice(z * per, (z + 1) * per)
        blk = np.empty((per, 3))
        blk[:, 0] = base[:, 0]
        blk[:, 1] = base[:, 1]
        blk[:, 2] = z
        blk = x0 + (blk + rng.uniform(-jitter, jitter, size=(per, 3))) * h
        out[s] = blk.astype(np.float32)
    ns = out.shape[0] - n_lat
    out[n_lat:] = rng.uniform(0.0, 1.0, size=(ns, 3)) * dom
    return out


def sph_step(points, h=1.0, sigma=0.05, seed=0):
    """One time step of the SPH configuration: positions perturbed by N(0, sigma*h)."""
    rng = _rng(seed)
    return (points + rng.standard_normal(points.shape) * (sigma * h)).astype(np.float32)


def training_clouds(name, scale=1.0, rank=0, count=None):
    """Clouds of other seeds (never a measured one) whose exact K-th neighbor distances
    train the width model of workload `name`: [(points, queries or None)], at most
    `count` of them when given."""
    s = 1000 * rank + 100
    out = []
    if name == "knn_multicloud_4096":
        p, off = multicloud(n_clouds=96 if count is None else count, seed=s + 7)
        for c in range(len(off) - 1):
            out.append((p[int(off[c]):int(off[c + 1])], None))
    elif name == "knn_surface_1e7":
        for i in range(20 if count is None else count):
            out.append((surfaces(seed=s + i, scale=0.05 * max(scale, 0.02)), None))
    elif name == "knn_gmm_1e6":
        for i in range(4 if count is None else count):
            out.append(gmm(seed=s + i, scale=0.25 * scale))
    elif name == "radius_uniform_1e5":
        for i in range(4 if count is None else count):
            out.append((uniform_cube(seed=s + i, scale=scale), None))
    elif name == "sph_lattice_5e7":
        for i in range(2 if count is None else count):
            out.append((sph_lattice(seed=s + i, scale=0.02 * scale), None))
    else:
        raise ValueError(f"unknown workload {name}")
    return out


def train_width_model(ctx, name, scale=1.0, rank=0, epochs=32, count=None):
    """Trains the context's width model for workload `name` on the GPU: exact K-th
    distances from the plain search over training_clouds(), then the library's own
    forward/backward/Adam kernels. Returns sample count and first/last epoch loss."""
    import torch
    cfg = CONFIGS[name]
    feats, tgts = [], []
    for p, q in training_clouds(name, scale, rank, count):
        tp = torch.from_numpy(np.ascontiguousarray(p)).cuda()
        tq = None if q is None else torch.from_numpy(np.ascontiguousarray(q)).cuda()
        f, t = ctx.collect_training(tp, tq, cfg["mode"], cfg["radius"], cfg["k"])
        feats.append(f)
        tgts.append(t)
    f = torch.cat(feats)
    t = torch.cat(tgts)
    gen = torch.Generator(device=f.device).manual_seed(0)
    perm = torch.randperm(f.shape[0], device=f.device, generator=gen)
    f = f[perm].contiguous()
    t = t[perm].contiguous()
    losses = ctx.train_model(f, t, epochs=epochs, batch=16384, lr=3e-3, seed=rank)
    return {"samples": int(f.shape[0]), "loss_first": float(losses[0]),
            "loss_last": float(losses[-1])}
