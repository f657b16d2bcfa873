"""The summation orders of the ring sums, restated in numpy on the CPU.

The reference sums a ring's 1024-cell block with a halving tree in shared
memory (output_lv1, device_func.cu:49-76): list[t] += list[t + half] for
half = 512, 256, ..., 1.  The library's warp form of the mass sums
(k_reduce_mass_w) gives lane L the cells L + 32 m, m = 0..31, adds
v[m] += v[m + h] for h = 16, 8, 4, 2, 1 inside the lane (the levels 512..32)
and then x += shuffle_down(x, d) for d = 16..1 across lanes (the levels
16..1).  Every addition there has the same two operands as in the tree, so
the two orders give the same bits; these tests check that argument on random
blocks, in IEEE double arithmetic as numpy does it (one rounding per add).
The kernels themselves are compared bit for bit on the GPU."""
import numpy as np


def tree1024(vals):
    lst = [np.float64(x) for x in vals]
    half = 512
    while half >= 1:
        for t in range(half):
            lst[t] = lst[t] + lst[t + half]
        half //= 2
    return lst[0]


def warp_tree1024(vals):
    # lane L holds list[L + 32 m]
    v = [[np.float64(vals[lane + 32 * m]) for m in range(32)] for lane in range(32)]
    h = 16
    while h >= 1:
        for lane in range(32):
            for m in range(h):
                v[lane][m] = v[lane][m] + v[lane][m + h]
        h //= 2
    x = [v[lane][0] for lane in range(32)]
    d = 16
    while d >= 1:
        y = [x[lane + d] if lane + d < 32 else x[lane] for lane in range(32)]   # shuffle down
        x = [x[lane] + y[lane] if lane < d else x[lane] for lane in range(32)]
        d //= 2
    return x[0]


def test_warp_order_equals_tree_order_bitwise():
    rng = np.random.default_rng(7)
    for trial in range(20):
        # cell masses of very different magnitudes make the order visible
        vals = rng.standard_normal(1024) * np.exp(rng.uniform(-30.0, 30.0, 1024))
        a, b = tree1024(vals), warp_tree1024(vals)
        assert a.tobytes() == b.tobytes(), (trial, a, b)


def test_other_orders_differ():
    """A different pairing (sequential sum) gives other bits on the same
    blocks, so the test above can tell orders apart."""
    rng = np.random.default_rng(8)
    differ = 0
    for _ in range(20):
        vals = rng.standard_normal(1024) * np.exp(rng.uniform(-30.0, 30.0, 1024))
        seq = np.float64(0.0)
        for x in vals:
            seq = seq + np.float64(x)
        differ += seq.tobytes() != tree1024(vals).tobytes()
    assert differ >= 15, differ


def test_padded_block():
    """A ring shorter than 1024 cells pads the block with zeros in both forms."""
    rng = np.random.default_rng(9)
    vals = np.zeros(1024)
    vals[:768] = rng.uniform(0.5, 2.0, 768) * 1e-3
    assert tree1024(vals).tobytes() == warp_tree1024(vals).tobytes()
