"""Seeded synthetic workloads with the shapes of the benchmark configurations.

Each generator returns closed polylines as (loop_offsets, xyz) float64 arrays
(xyz rounded through float32, as a BCC file stores it) or, for the spline
case, control points. ``write_bcc`` stores any of them as a BCC file.

  ring_chain   64 rings of radius 1 centred at (1.6 i, 0, 0), planes
               alternating xy / xz, each the composite of 8 cubic Bezier arcs
               (control points jittered +-0.02) sampled at 4 points per arc.
  chain_mail   100 x 100 rings of radius 1 on a square grid of spacing 1.3;
               the ring planes of successive x-rows are tilted +-25 degrees
               about x, which links each ring to its x-row neighbours;
               48-gons, vertices jittered +-0.01.
  polymer      closed Gaussian random walks (sigma = 1 per axis, mean step
               subtracted so the walk closes), centres uniform in a cube.
  mixed_batch  torus knots (p, q coprime in [2, 9]) and closed random walks,
               50/50, segment counts log-uniform in [16, 2^18].
"""
from __future__ import annotations

import math
import struct

import numpy as np


def _f32(x):
    return np.asarray(x, dtype=np.float32).astype(np.float64)


def _pack(loops):
    off = np.zeros(len(loops) + 1, dtype=np.int64)
    off[1:] = np.cumsum([len(l) for l in loops])
    xyz = np.concatenate(loops, axis=0) if loops else np.zeros((0, 3))
    return off, _f32(xyz)


def bezier_ring_controls(rng, jitter=0.02, arcs=8):
    """Control points (3 per arc, closed) of a unit circle made of `arcs`
    cubic Bezier arcs, each control point jittered uniformly."""
    k = 4.0 / 3.0 * math.tan(math.pi / (2 * arcs))
    pts = []
    for a in range(arcs):
        t0 = 2 * math.pi * a / arcs
        t1 = 2 * math.pi * (a + 1) / arcs
        p0 = np.array([math.cos(t0), math.sin(t0)])
        p3 = np.array([math.cos(t1), math.sin(t1)])
        d0 = np.array([-math.sin(t0), math.cos(t0)])
        d3 = np.array([-math.sin(t1), math.cos(t1)])
        pts += [p0, p0 + k * d0, p3 - k * d3]
    c = np.array(pts)
    c = np.concatenate([c, np.zeros((len(c), 1))], axis=1)
    return c + rng.uniform(-jitter, jitter, size=c.shape)


def sample_composite_bezier(ctrl, per_arc=4):
    """Samples the closed composite Bezier (arcs share endpoints) at per_arc
    points per arc (t = 0, 1/per_arc, ...)."""
    n = len(ctrl) // 3
    out = []
    for a in range(n):
        p0, p1, p2 = ctrl[3 * a], ctrl[3 * a + 1], ctrl[3 * a + 2]
        p3 = ctrl[(3 * a + 3) % len(ctrl)]
        for s in range(per_arc):
            t = s / per_arc
            u = 1 - t
            out.append(u ** 3 * p0 + 3 * u * u * t * p1 + 3 * u * t * t * p2 + t ** 3 * p3)
    return np.array(out)


def ring_chain(seed=1, n_rings=64, spacing=1.6, per_arc=4, as_bezier=False):
    """Ring chain: linked neighbours, expected certificate (i, i+1) = +-1."""
    rng = np.random.default_rng(seed)
    loops = []
    for i in range(n_rings):
        c = bezier_ring_controls(rng)
        pts = c if as_bezier else sample_composite_bezier(c, per_arc)
        if i % 2 == 1:  # xz plane
            pts = np.stack([pts[:, 0], pts[:, 2], pts[:, 1]], axis=1)
        pts = pts + np.array([spacing * i, 0.0, 0.0])
        loops.append(pts)
    return _pack(loops)


def chain_mail(seed=2, rows=100, cols=100, spacing=1.3, tilt_deg=25.0, ngon=48, jitter=0.01):
    rng = np.random.default_rng(seed)
    th = 2 * np.pi * np.arange(ngon) / ngon
    base = np.stack([np.cos(th), np.sin(th), np.zeros(ngon)], axis=1)
    loops = []
    for a in range(rows):
        phi = math.radians(tilt_deg if a % 2 == 0 else -tilt_deg)
        R = np.array([[1, 0, 0], [0, math.cos(phi), -math.sin(phi)], [0, math.sin(phi), math.cos(phi)]])
        ring = base @ R.T
        for b in range(cols):
            pts = ring + np.array([spacing * a, spacing * b, 0.0])
            loops.append(pts + rng.uniform(-jitter, jitter, size=pts.shape))
    return _pack(loops)


def random_walk_loop(rng, n, sigma=1.0):
    steps = rng.normal(0.0, sigma, size=(n, 3))
    steps -= steps.mean(axis=0)
    pts = np.cumsum(steps, axis=0)
    return pts - pts.mean(axis=0)


def polymer(seed=3, n_loops=200, n_steps=50_000, cube=400.0):
    rng = np.random.default_rng(seed)
    loops = []
    for _ in range(n_loops):
        centre = rng.uniform(0.0, cube, size=3)
        loops.append(random_walk_loop(rng, n_steps) + centre)
    return _pack(loops)


def torus_knot(p, q, n, R=1.0, r=0.4, scale=1.0):
    t = 2 * np.pi * np.arange(n) / n
    x = (R + r * np.cos(q * t)) * np.cos(p * t)
    y = (R + r * np.cos(q * t)) * np.sin(p * t)
    z = r * np.sin(q * t)
    return scale * np.stack([x, y, z], axis=1)


def mixed_batch(seed=5, n_loops=5000, lo=16, hi=2 ** 18, cube=None):
    """Torus knots and closed random walks, sizes log-uniform in [lo, hi].

    The default cube side (35.1 x n_loops^(1/3), 600 for 5,000 loops) gives
    35,717 potentially linked pairs for seed 5 (1.37e8 segments after
    Discretize)."""
    rng = np.random.default_rng(seed)
    sizes = np.exp(rng.uniform(math.log(lo), math.log(hi), size=n_loops)).astype(np.int64)
    if cube is None:
        cube = 600.0 * (n_loops / 5000.0) ** (1 / 3)
    loops = []
    pq = [(p, q) for p in range(2, 10) for q in range(2, 10) if math.gcd(p, q) == 1 and p != q]
    for k in range(n_loops):
        n = int(sizes[k])
        centre = rng.uniform(0.0, cube, size=3)
        if rng.random() < 0.5:
            p, q = pq[rng.integers(len(pq))]
            scale = 0.5 * math.sqrt(n) ** 0.5 + 1.0
            pts = torus_knot(p, q, max(n, 8), scale=scale)
        else:
            pts = random_walk_loop(rng, max(n, 8), sigma=0.3)
        loops.append(pts + centre)
    return _pack(loops)


def walk_pairs(seed=11, n_pairs=20, n_steps=100_000, offset=20.0):
    """Training set of the learned criterion: n_pairs pairs of closed random
    walks whose centres lie `offset` apart (so their trees interleave).
    Returns (offsets, xyz, pairs)."""
    rng = np.random.default_rng(seed)
    loops, pairs = [], []
    for k in range(n_pairs):
        centre = rng.uniform(0.0, 1000.0, size=3)
        d = rng.normal(size=3)
        d *= offset / np.linalg.norm(d)
        loops.append(random_walk_loop(rng, n_steps) + centre)
        loops.append(random_walk_loop(rng, n_steps) + centre + d)
        pairs.append((2 * k, 2 * k + 1))
    off, xyz = _pack(loops)
    return off, xyz, np.array(pairs, dtype=np.int32)


def write_bcc(path, loops_or_packed, seg_type="PL"):
    """BCC writer: closed curves (negative counts), float32 xyz."""
    if isinstance(loops_or_packed, tuple):
        off, xyz = loops_or_packed
        loops = [xyz[off[i]:off[i + 1]] for i in range(len(off) - 1)]
    else:
        loops = loops_or_packed
    total = sum(len(l) for l in loops)
    hdr = b"BCC" + bytes([0x44]) + seg_type.encode() + bytes([3, 1])
    hdr += struct.pack("<QQ", len(loops), total) + b"\0" * 40
    with open(path, "wb") as f:
        f.write(hdr)
        for l in loops:
            f.write(struct.pack("<i", -len(l)))
            f.write(np.asarray(l, dtype=np.float32).tobytes())


def named(name: str, seed: int = 3):
    """The benchmark workloads by name: (loop_offsets, xyz, description).

      ring_chain    64 rings x 32 segments
      chain_mail    100 x 100 rings, 48-gons (480k segments)
      polymer       200 x 50,000-step closed walks (10M segments), cube 400
      held_out_20M  1,000 x 20,000-step closed walks (20M segments), cube 504:
                    the polymer density, the learned criterion's held-out set
      mixed_batch   5,000 torus knots and walks, 16 to 2^18 segments (134M
                    segments), cube 600
    """
    if name == "polymer":
        off, xyz = polymer(seed=seed, n_loops=200, n_steps=50_000, cube=400.0)
        d = "polymer loops: 200 x 50000-step closed Gaussian walks (10M segments), cube 400"
    elif name == "held_out_20M":
        off, xyz = polymer(seed=seed, n_loops=1000, n_steps=20_000, cube=504.0)
        d = "held-out polymer: 1000 x 20000-step closed Gaussian walks (20M segments), cube 504"
    elif name == "mixed_batch":
        off, xyz = mixed_batch(seed=seed)
        d = ("mixed batch: 5000 loops, half (p,q) torus knots, half closed walks, sizes log-uniform in "
             "[16, 2^18] (134M segments), cube 600")
    elif name == "chain_mail":
        off, xyz = chain_mail(seed=seed)
        d = "chain-mail sheet: 100 x 100 rings, 48-gons (480k segments)"
    elif name == "ring_chain":
        off, xyz = ring_chain(seed=seed)
        d = "ring chain: 64 rings x 32 segments"
    else:
        raise ValueError(f"unknown workload {name}")
    return off, xyz, d


def digest(*arrays) -> str:
    """SHA-256 (hex, first 32 digits) of the arrays' bytes: pins a prepared
    workload (polylines and pairs) between machines."""
    import hashlib
    h = hashlib.sha256()
    for a in arrays:
        a = np.ascontiguousarray(a)
        h.update(str(a.dtype).encode() + str(a.shape).encode())
        mv = memoryview(a).cast("B")
        for k in range(0, len(mv), 1 << 28):
            h.update(mv[k:k + (1 << 28)])
    return h.hexdigest()[:32]


def certificate_text(ncurves: int, pairs, lk) -> str:
    """Certificate text from per-pair real sums, as ExportToFile writes it
    (linking_number_certificate.cpp:185-213, :441-454): the curve count, then
    `i,j,lk` for every pair whose std::round (half away from zero) is
    nonzero, with i < j, sorted by (i, j)."""
    pairs = np.asarray(pairs).reshape(-1, 2)
    lk = np.asarray(lk, dtype=np.float64)
    r = np.sign(lk) * np.floor(np.abs(lk) + 0.5)
    if not np.all(np.isfinite(r)):
        raise ValueError("non-finite linking number")
    keep = np.abs(r) >= 0.25
    i = np.minimum(pairs[keep, 0], pairs[keep, 1])
    j = np.maximum(pairs[keep, 0], pairs[keep, 1])
    v = r[keep].astype(np.int64)
    o = np.lexsort((j, i))
    lines = [str(int(ncurves))] + [f"{a},{b},{c}" for a, b, c in zip(i[o], j[o], v[o])]
    return "\n".join(lines) + "\n"


def pair_work(off, pairs):
    """Sum over pairs of n_i * n_j (direct-sum-equivalent segment pairs)."""
    n = np.diff(off).astype(np.float64)
    pairs = np.asarray(pairs).reshape(-1, 2)
    return float(np.sum(n[pairs[:, 0]] * n[pairs[:, 1]]))
