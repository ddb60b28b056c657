"""Seeded synthetic point sets for the benchmark configurations.

No public dataset is involved: every workload is generated from a counter-based
splitmix64 stream (53-bit uniform doubles), so the CPU oracle and the GPU see
identical bits.

  c1  1,000 points i.i.d. uniform in [0,1]^2, seed 1, texture 512
  c2  4,194,304 points i.i.d. uniform in [0,1]^2, texture 8192
  c3  16,777,216 points: 50% from 64 Gaussian blobs (sigma 0.01, centres
      uniform, Box-Muller), 30% uniform, 20% snapped to the 1024 x 1024
      lattice floor(1024 u) / 1024; texture 8192
  c4  4,096 sets, sizes floor(exp(U[ln 64, ln 65536])), each a unit square,
      unit disk (r = sqrt(u)) or annulus r in [0.8, 1] (r = sqrt(0.64 + 0.36 u))
"""
import numpy as np

_GAMMA = np.uint64(0x9E3779B97F4A7C15)
_M1 = np.uint64(0xBF58476D1CE4E5B9)
_M2 = np.uint64(0x94D049BB133111EB)


def splitmix64(seed, n, offset=0):
    """n outputs of splitmix64 for state seed, counter positions offset..offset+n-1."""
    with np.errstate(over="ignore"):
        x = np.uint64(seed) + _GAMMA * (np.arange(offset, offset + n, dtype=np.uint64) + np.uint64(1))
        z = x
        z = (z ^ (z >> np.uint64(30))) * _M1
        z = (z ^ (z >> np.uint64(27))) * _M2
        return z ^ (z >> np.uint64(31))


def uniform01(seed, n, offset=0):
    """n doubles in [0, 1) with 53 random bits each."""
    return (splitmix64(seed, n, offset) >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


def uniform_points(n, seed):
    u = uniform01(seed, 2 * n)
    return u.reshape(n, 2)


def gaussian_blobs(n, seed, nblobs=64, sigma=0.01):
    centres = uniform01(seed ^ 0xB10B, 2 * nblobs).reshape(nblobs, 2)
    pick = (splitmix64(seed ^ 0xC0DE, n) % np.uint64(nblobs)).astype(np.int64)
    u1 = uniform01(seed ^ 0x1111, n)
    u2 = uniform01(seed ^ 0x2222, n)
    r = np.sqrt(-2.0 * np.log(1.0 - u1))
    g = np.stack([r * np.cos(2 * np.pi * u2), r * np.sin(2 * np.pi * u2)], axis=1)
    return centres[pick] + sigma * g


def degenerate_mix(n, seed):
    """c3 recipe: 50% blobs, 30% uniform, 20% lattice-snapped (duplicates, cocircular quads)."""
    nb, nu = n // 2, (3 * n) // 10
    nl = n - nb - nu
    blobs = gaussian_blobs(nb, seed)
    unif = uniform_points(nu, seed ^ 0x3333)
    lat = np.floor(uniform_points(nl, seed ^ 0x4444) * 1024.0) / 1024.0
    return np.concatenate([blobs, unif, lat], axis=0)


def c4_sets(nsets=4096, seed=4, lo=64, hi=65536):
    sizes = np.floor(np.exp(np.log(lo) + (np.log(hi) - np.log(lo)) * uniform01(seed, nsets))).astype(np.int64)
    kinds = (splitmix64(seed ^ 0x5555, nsets) % np.uint64(3)).astype(np.int64)
    sets = []
    for k in range(nsets):
        n = int(sizes[k])
        s = seed * 1000003 + k
        if kinds[k] == 0:
            p = uniform_points(n, s)
        else:
            u = uniform01(s, n)
            th = 2 * np.pi * uniform01(s ^ 0x7777, n)
            r = np.sqrt(u) if kinds[k] == 1 else np.sqrt(0.64 + 0.36 * u)
            p = np.stack([r * np.cos(th), r * np.sin(th)], axis=1)
        sets.append(p)
    return sets


CONFIGS = {
    "c1": dict(n=1000, seed=1, fbo=512, kind="uniform"),
    "c2": dict(n=4194304, seed=2, fbo=8192, kind="uniform"),
    "c3": dict(n=16777216, seed=3, fbo=8192, kind="degenerate"),
}


def make(config, n=None):
    c = CONFIGS[config]
    n = c["n"] if n is None else n
    if c["kind"] == "uniform":
        return uniform_points(n, c["seed"]), c["fbo"]
    return degenerate_mix(n, c["seed"]), c["fbo"]
