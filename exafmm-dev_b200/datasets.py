"""Seeded synthetic body distributions for the benchmark workloads.

The reference generates bodies with drand48 in ``Dataset`` (include/dataset.h:51-164):
cube [-pi, pi]^3, sphere surface of radius pi, Plummer scaled by 3 pi / 16 and clipped at
r < 100, charges U[-.5, .5] minus their mean or 1/N under MASS.  The workloads here use the
same constructions at the sizes and scales the solver is benchmarked on, drawn from numpy's
counter-based Philox generator in FP64 and rounded to the working precision:

* ``cube``:    x ~ U[-1, 1]^3, q ~ U[-1, 1] minus its mean
* ``plummer``: a = 1, r = a / sqrt(u^(-2/3) - 1) rejected when r > 10 a, isotropic
               direction (dataset.h:117-131), recentred on the centre of mass, q = 1/N
* ``sphere``:  x = g / |g|, g ~ N(0, I3) (uniform on the unit sphere), q ~ U[0, 1]

Positions are returned as float64 arrays holding values exactly representable in the
requested working precision, so every consumer (solver, oracle, reference) sees the same
bodies.
"""
import numpy as np


def _rng(seed):
    return np.random.Generator(np.random.Philox(seed))


def cube(n, seed=42):
    g = _rng(seed)
    x = g.uniform(-1.0, 1.0, (n, 3))
    q = g.uniform(-1.0, 1.0, n)
    q -= q.mean()
    return x, q


def plummer(n, seed=43, clip=10.0):
    g = _rng(seed)
    out = np.empty((0, 3))
    while len(out) < n:
        m = int((n - len(out)) * 1.1) + 16
        u = g.random((m, 3))
        with np.errstate(divide="ignore", invalid="ignore"):
            r = 1.0 / np.sqrt(u[:, 0] ** (-2.0 / 3.0) - 1.0)
        ok = np.isfinite(r) & (r < clip)
        r, u2, u3 = r[ok], u[ok, 1], u[ok, 2]
        z = (1.0 - 2.0 * u2) * r
        s = np.sqrt(np.maximum(r * r - z * z, 0.0))
        p = np.stack([s * np.cos(2 * np.pi * u3), s * np.sin(2 * np.pi * u3), z], axis=1)
        out = np.concatenate([out, p])[:n]
    out -= out.mean(axis=0)
    q = np.full(n, 1.0 / n)
    return out, q


def sphere(n, seed=44):
    g = _rng(seed)
    v = g.standard_normal((n, 3))
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    q = g.uniform(0.0, 1.0, n)
    return v, q


DISTRIBUTIONS = {"cube": cube, "plummer": plummer, "sphere": sphere}


def make(dist, n, seed=None, precision="f32"):
    """Bodies (x: (n, 3) float64, q: (n,) float64) rounded to the working precision."""
    f = DISTRIBUTIONS[dist]
    x, q = f(n) if seed is None else f(n, seed)
    if precision == "f32":
        x = x.astype(np.float32).astype(np.float64)
        q = q.astype(np.float32).astype(np.float64)
    return np.ascontiguousarray(x), np.ascontiguousarray(q)


def sample_targets(n, count):
    """Stride sampling of targets (Dataset::sampleBodies, include/dataset.h:268-276)."""
    if count >= n:
        return np.arange(n)
    stride = n // count
    return np.arange(count) * stride
