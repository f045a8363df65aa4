"""Seeded synthetic point sets with the shapes of the F2M benchmark configs.

A counter-based splitmix64 stream gives the same points on every machine:
value(seed, stream, i) = splitmix64(seed * 2**32 + stream * 2**24 + i).

  config1: 1,000 points, integer coordinates uniform in [0, 10^4)^2
  config2: 100,000 points from 64 Gaussian clusters (centres uniform in
           [0, 10^6)^2, sigma = 0.5% of the box) plus 10% uniform background,
           rounded and clamped to integers
  config3: 4,096 instances, sizes log-uniform in [50, 5000], integer
           coordinates uniform in [0, 10^4)^2
  config4: 10,000 FP32 points uniform in [0, 1)^2 (smoothed bound)
  config5: 1,024 instances, sizes uniform in [200, 2000], FP32 points on a
           jittered unit square lattice (jitter uniform in +-0.3) (smoothed
           bound, batched)
"""
import numpy as np

_M64 = np.uint64(0xFFFFFFFFFFFFFFFF)


def splitmix64(x):
    x = np.asarray(x, dtype=np.uint64)
    with np.errstate(over="ignore"):
        z = x + np.uint64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        return z ^ (z >> np.uint64(31))


def uniform(seed, stream, n, start=0):
    """n doubles in [0,1) from stream `stream` of `seed`."""
    idx = np.arange(start, start + n, dtype=np.uint64)
    with np.errstate(over="ignore"):
        key = np.uint64(seed) * np.uint64(1 << 32) + np.uint64(stream) * np.uint64(1 << 24) + idx
    return (splitmix64(key) >> np.uint64(11)).astype(np.float64) * (1.0 / (1 << 53))


def normal(seed, stream, n):
    u1 = uniform(seed, stream, n)
    u2 = uniform(seed, stream + 1, n)
    return np.sqrt(-2.0 * np.log1p(-u1)) * np.cos(2.0 * np.pi * u2)


def uniform_int_points(n, seed, box=10_000, stream=0):
    x = np.floor(uniform(seed, stream, n) * box)
    y = np.floor(uniform(seed, stream + 1, n) * box)
    return x, y


def config1(seed=1):
    return uniform_int_points(1000, seed)


def config2(seed=2, n=100_000, clusters=64, box=1_000_000, background=0.10):
    sigma = 0.005 * box
    nb = int(round(background * n))
    nc = n - nb
    cx = uniform(seed, 0, clusters) * box
    cy = uniform(seed, 1, clusters) * box
    which = np.minimum((uniform(seed, 2, nc) * clusters).astype(np.int64), clusters - 1)
    x = cx[which] + sigma * normal(seed, 3, nc)
    y = cy[which] + sigma * normal(seed, 5, nc)
    bx = uniform(seed, 7, nb) * box
    by = uniform(seed, 8, nb) * box
    x = np.clip(np.rint(np.concatenate([x, bx])), 0, box - 1)
    y = np.clip(np.rint(np.concatenate([y, by])), 0, box - 1)
    return x, y


def batch_sizes(n_inst, seed, lo=50, hi=5000):
    u = uniform(seed, 100, n_inst)
    return np.floor(np.exp(np.log(lo) + u * (np.log(hi) - np.log(lo)))).astype(np.int64).clip(lo, hi)


def config3(seed=3, n_inst=4096, lo=50, hi=5000, box=10_000):
    """Returns (offs, x, y) for n_inst instances."""
    sizes = batch_sizes(n_inst, seed, lo, hi)
    offs = np.zeros(n_inst + 1, np.int64)
    offs[1:] = np.cumsum(sizes)
    n = int(offs[-1])
    x = np.floor(uniform(seed, 101, n) * box)
    y = np.floor(uniform(seed, 102, n) * box)
    return offs, x, y


def config4(seed=4, n=10_000):
    x = uniform(seed, 300, n).astype(np.float32)
    y = uniform(seed, 301, n).astype(np.float32)
    return x, y


def jittered_lattice(n, seed, stream=310, jitter=0.3):
    """n FP32 points: the first n sites of a square unit lattice (row-major,
    side ceil(sqrt n)), each moved by a uniform offset in +-jitter."""
    side = int(np.ceil(np.sqrt(n)))
    i = np.arange(n)
    x = (i % side) + (2 * uniform(seed, stream, n) - 1) * jitter
    y = (i // side) + (2 * uniform(seed, stream + 1, n) - 1) * jitter
    return x.astype(np.float32), y.astype(np.float32)


def config5(seed=5, n_inst=1024, lo=200, hi=2000):
    """(offs, x, y) of n_inst jittered-lattice instances."""
    sizes = lo + np.floor(uniform(seed, 320, n_inst) * (hi - lo + 1)).astype(np.int64)
    offs = np.zeros(n_inst + 1, np.int64)
    offs[1:] = np.cumsum(sizes)
    xs, ys = [], []
    for b in range(n_inst):
        x, y = jittered_lattice(int(sizes[b]), seed * 100_000 + b)
        xs.append(x)
        ys.append(y)
    return offs, np.concatenate(xs), np.concatenate(ys)


def lattice_points(n, seed, side=None, keep=0.7):
    """Integer points on a square lattice with a random subset kept: many
    equal distances, as in the VLSI instances (exercises ties and the
    comb repair path)."""
    if side is None:
        side = int(np.ceil(np.sqrt(n / keep)))
    u = uniform(seed, 200, side * side)
    idx = np.argsort(u)[:n]
    return (idx % side).astype(np.float64), (idx // side).astype(np.float64)


def write_tsplib(path, x, y, labels=None, name="synthetic"):
    n = len(x)
    if labels is None:
        labels = np.arange(1, n + 1)
    with open(path, "w") as f:
        f.write(f"NAME : {name}\nTYPE : TSP\nDIMENSION : {n}\nEDGE_WEIGHT_TYPE : EUC_2D\n")
        f.write("NODE_COORD_SECTION\n")
        for k, a, b in zip(labels, x, y):
            f.write(f"{int(k)} {a:.10g} {b:.10g}\n")
        f.write("EOF\n")
