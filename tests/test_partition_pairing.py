"""The pairing form of the reference's list partition (qpart_ptr_B,
graph_cuda_partition.hpp:3-25), which both solvers run on the device: on
finite values a pass of the Hoare loop swaps the t-th entry above the
threshold among the first Lc positions (ascending) with the t-th entry at or
below it among the rest (descending), Lc being the count at or below the
threshold, and returns Lc (a one-entry list is returned as it is).  This
test restates the Hoare loop and the pairing in Python and compares the
final order and count on seeded lists with many ties; the device forms are
compared with the serial loop on the device by `f2m_partition_selfcheck`."""
import random


def hoare(vals, avg):
    """qpart_ptr_B's loop: returns (count, order of original positions)."""
    v = list(vals)
    pl = list(range(len(v)))
    size = len(v)
    low, high, i, j = 0, size - 1, 0, size - 1
    passes = 0
    while i < j and passes <= size:
        while i <= high and v[i] <= avg:
            i += 1
        while j >= low and v[j] > avg:
            j -= 1
        if i < j:
            v[i], v[j] = v[j], v[i]
            pl[i], pl[j] = pl[j], pl[i]
        passes += 1
    return j + 1, pl


def pairing(vals, avg):
    size = len(vals)
    pl = list(range(size))
    if size <= 1:
        return size, pl
    lc = sum(1 for x in vals if x <= avg)
    above_low = [k for k in range(lc) if vals[k] > avg]             # ascending
    below_high = [k for k in range(size - 1, lc - 1, -1) if vals[k] <= avg]  # descending
    assert len(above_low) == len(below_high)
    for a, b in zip(above_low, below_high):
        pl[a], pl[b] = pl[b], pl[a]
    return lc, pl


def test_pairing_equals_the_hoare_loop():
    rng = random.Random(17)
    for it in range(20000):
        size = rng.choice([0, 1, 2, 3, 5, 31, 32, 33, 64, rng.randint(0, 128)])
        kind = it % 3
        if kind == 0:
            vals = [rng.random() for _ in range(size)]
        elif kind == 1:
            vals = [float(rng.randint(0, 4)) for _ in range(size)]  # ties
        else:
            vals = sorted(rng.random() for _ in range(size))
            if rng.random() < 0.5:
                vals.reverse()
        avg = rng.choice([0.5, 2.0, -1.0, 10.0, rng.random()])
        assert hoare(vals, avg) == pairing(vals, avg), (vals, avg)
