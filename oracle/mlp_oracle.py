"""CPU FP64 restatement of one training step of the learned matching proposal.

TEST INFRASTRUCTURE ONLY: the checker for the library's MLP gradients
(orbx_learned_gradients) and GEMM.  Nothing in the product imports it.  The
learned proposal has no counterpart in the reference (CUDA-ORB only has exact
brute-force matching, orbd.cu:1471-1559), so there is nothing to pin against
there; this module states the mathematics directly:

    x_k     = +1 if bit (k % 8) of byte (k // 8) is set, else -1     (k < 256)
    H       = relu(X W1^T + b1)
    logits  = H W2^T + b2
    loss    = mean_r ( logsumexp(logits_r) - logits_r[label_r] )
    dL      = (softmax(logits) - onehot(label)) / n
    (label sets, labels of shape (n, S) with -1 unused, as ORBX_LABEL_LISTED:
     loss = mean_r -log P_r with P_r the softmax mass on the set, and
     dL   = (softmax - softmax * [c in set] / P_r) / n; S = 1 is the line above)
    dW2     = dL^T H,        db2 = sum_r dL
    dH      = (dL W2) * [H > 0]
    dW1     = dH^T X,        db1 = sum_r dH

With bf16=True the intermediates the GPU stores in bf16 (H, dL, dH) are
rounded to bf16 (round to nearest even) at the same points.
"""
import numpy as np


def pm1(bits):
    """(n, 32) uint8 -> (n, 256) float64 of +-1, bit order LSB first."""
    b = np.unpackbits(np.ascontiguousarray(bits, dtype=np.uint8), axis=1, bitorder="little")
    return b.astype(np.float64) * 2.0 - 1.0


def bf16_round(a):
    """Round to the nearest bf16 (ties to even), returned as float64."""
    f = np.ascontiguousarray(a, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    r = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def forward(bits, w1, b1, w2, b2, bf16=False):
    X = pm1(bits)
    H = np.maximum(X @ w1.astype(np.float64).T + b1, 0.0)
    if bf16:
        H = bf16_round(H)
    logits = H @ w2.astype(np.float64).T + b2
    return X, H, logits


def forward_backward(bits, labels, w1, b1, w2, b2, bf16=False):
    """Returns (mean loss, {"w1", "b1", "w2", "b2"} gradients) in float64."""
    n = bits.shape[0]
    X, H, logits = forward(bits, w1, b1, w2, b2, bf16)
    m = logits.max(axis=1, keepdims=True)
    e = np.exp(logits - m)
    s = e.sum(axis=1, keepdims=True)
    lab = np.asarray(labels, dtype=np.int64)
    if lab.ndim == 1:
        lab = lab[:, None]
    member = np.zeros_like(logits, dtype=bool)
    rows, cols = np.nonzero(lab >= 0)
    member[rows, lab[rows, cols]] = True
    p = e / s
    mass = (p * member).sum(axis=1)
    loss = float(np.mean(-np.log(mass)))
    dL = p - p * member / mass[:, None]
    dL /= n
    if bf16:
        dL = bf16_round(dL)
    dW2 = dL.T @ H
    db2 = dL.sum(axis=0)
    dH = (dL @ w2.astype(np.float64)) * (H > 0)
    if bf16:
        dH = bf16_round(dH)
    dW1 = dH.T @ X
    db1 = dH.sum(axis=0)
    return loss, {"w1": dW1, "b1": db1, "w2": dW2, "b2": db2}


def knn1_bruteforce(q, db):
    """Exact nearest (distance, smallest index among ties) per query, numpy popcount."""
    qb = np.unpackbits(q, axis=1).astype(np.int32)
    dbb = np.unpackbits(db, axis=1).astype(np.int32)
    # Hamming = popcount(q) + popcount(d) - 2 * (q . d)
    d = qb.sum(1)[:, None] + dbb.sum(1)[None, :] - 2 * (qb @ dbb.T)
    idx = d.argmin(axis=1)
    return d[np.arange(len(q)), idx], idx
