"""The CPU FP64 oracle of the learned proposal's training step, pinned by
central finite differences of its own loss (no GPU).  The GPU gradients are
then checked against this oracle in tests/test_gpu_learned.py."""
import numpy as np

from oracle import mlp_oracle as MO


def _setup(seed=0, n=6, hidden=8, C=5):
    rng = np.random.Generator(np.random.PCG64(seed))
    bits = rng.integers(0, 256, size=(n, 32), dtype=np.uint8)
    labels = rng.integers(0, C, size=n)
    w1 = rng.normal(size=(hidden, 256)) * 0.1
    b1 = rng.normal(size=hidden) * 0.1
    w2 = rng.normal(size=(C, hidden)) * 0.3
    b2 = rng.normal(size=C) * 0.1
    return bits, labels, {"w1": w1, "b1": b1, "w2": w2, "b2": b2}


def test_pm1_bit_order():
    bits = np.zeros((1, 32), dtype=np.uint8)
    bits[0, 0] = 0b00000101
    bits[0, 31] = 0b10000000
    x = MO.pm1(bits)[0]
    assert x[0] == 1 and x[1] == -1 and x[2] == 1 and x[255] == 1 and x[254] == -1


def test_gradients_match_finite_differences():
    bits, labels, w = _setup()
    _, g = MO.forward_backward(bits, labels, w["w1"], w["b1"], w["w2"], w["b2"])
    rng = np.random.Generator(np.random.PCG64(1))
    eps = 1e-6
    for name in ("w1", "b1", "w2", "b2"):
        for _ in range(12):
            idx = tuple(int(rng.integers(0, s)) for s in w[name].shape)
            wp = {k: v.copy() for k, v in w.items()}
            wm = {k: v.copy() for k, v in w.items()}
            wp[name][idx] += eps
            wm[name][idx] -= eps
            lp, _ = MO.forward_backward(bits, labels, wp["w1"], wp["b1"], wp["w2"], wp["b2"])
            lm, _ = MO.forward_backward(bits, labels, wm["w1"], wm["b1"], wm["w2"], wm["b2"])
            num = (lp - lm) / (2 * eps)
            assert abs(num - g[name][idx]) < 1e-6 + 1e-5 * abs(num), (name, idx, num, g[name][idx])


def test_bf16_round_ties_to_even():
    vals = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, 1.0 + 2 ** -9, -2.5], dtype=np.float32)
    r = MO.bf16_round(vals)
    assert r[0] == 1.0
    assert r[1] == 1.0                      # halfway, rounds to even mantissa
    assert r[2] == 1.0 + 2 ** -6            # halfway, rounds up to even
    assert r[3] == 1.0
    assert r[4] == -2.5


def test_knn1_bruteforce_ties_smallest_index():
    db = np.zeros((3, 32), dtype=np.uint8)
    db[1, 0] = 1
    q = np.zeros((1, 32), dtype=np.uint8)
    d, i = MO.knn1_bruteforce(q, np.vstack([db[1:2], db[0:1], db[0:1]]))
    assert d[0] == 0 and i[0] == 1


def test_label_set_gradients_match_finite_differences():
    """The listed-cluster target: loss -log(softmax mass on the set), sets of
    up to 3 distinct clusters with unused (-1) entries."""
    bits, labels, w = _setup()
    rng = np.random.Generator(np.random.PCG64(2))
    C = w["b2"].shape[0]
    sets = np.full((len(labels), 3), -1, dtype=np.int64)
    for r, l in enumerate(labels):
        k = int(rng.integers(1, 4))
        others = rng.permutation([c for c in range(C) if c != l])[: k - 1]
        sets[r, :k] = [l] + list(others)
    loss, g = MO.forward_backward(bits, sets, w["w1"], w["b1"], w["w2"], w["b2"])
    loss1, _ = MO.forward_backward(bits, labels, w["w1"], w["b1"], w["w2"], w["b2"])
    assert loss <= loss1 + 1e-12  # a superset of the label has at least its mass
    eps = 1e-6
    for name in ("w1", "b1", "w2", "b2"):
        for _ in range(8):
            idx = tuple(int(rng.integers(0, s)) for s in w[name].shape)
            wp = {k: v.copy() for k, v in w.items()}
            wm = {k: v.copy() for k, v in w.items()}
            wp[name][idx] += eps
            wm[name][idx] -= eps
            lp, _ = MO.forward_backward(bits, sets, wp["w1"], wp["b1"], wp["w2"], wp["b2"])
            lm, _ = MO.forward_backward(bits, sets, wm["w1"], wm["b1"], wm["w2"], wm["b2"])
            num = (lp - lm) / (2 * eps)
            assert abs(num - g[name][idx]) < 1e-6 + 1e-5 * abs(num), (name, idx, num, g[name][idx])
