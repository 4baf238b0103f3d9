"""CPU restatement of the target-shard cut of ``pacman_b200_plan_shard``
(test infrastructure, the checker of the CUDA cut).

Per target: cost = 1 + sum over the patches holding it of max(1, (n^3 // m) >> 8)
(n sources, m targets of the patch, n capped at 2^21); Morton key of 21 bits
per axis over the source bounding box, (x - lo) * ((2^21 - 1) / (hi - lo))
truncated and clamped; stable sort by key; position i goes to rank
min(world - 1, P_{i-1} * world // total) with P the inclusive cost prefix."""
import numpy as np

BITS = 21


def morton_keys(tgt, lo, hi, dim):
    keys = np.zeros(tgt.shape[0], dtype=np.uint64)
    qmax = float((1 << BITS) - 1)
    for a in range(dim):
        e = hi[a] - lo[a]
        sc = qmax / e if e > 0.0 else 0.0
        q = (tgt[:, a] - lo[a]) * sc
        q = np.where(q > 0.0, q, 0.0)
        q = np.minimum(q, qmax)
        v = q.astype(np.uint64)
        for b in range(BITS):
            keys |= ((v >> np.uint64(b)) & np.uint64(1)) << np.uint64(b * dim + a)
    return keys


def target_costs(m, src_off, tgt_off, tgt_idx):
    cost = np.ones(m, dtype=np.uint64)
    n = np.minimum(np.diff(src_off), 1 << 21).astype(np.uint64)
    mm = np.diff(tgt_off).astype(np.uint64)
    for k in np.nonzero(mm)[0]:
        share = max(1, int((n[k] * n[k] * n[k]) // mm[k]) >> 8)
        cost[tgt_idx[tgt_off[k]:tgt_off[k + 1]]] += np.uint64(share)
    return cost


def shard_ranks(tgt, src, dim, src_off, tgt_off, tgt_idx, world):
    """Rank of every target."""
    lo, hi = src[:, :dim].min(axis=0), src[:, :dim].max(axis=0)
    keys = morton_keys(tgt, lo, hi, dim)
    cost = target_costs(tgt.shape[0], src_off, tgt_off, tgt_idx)
    order = np.argsort(keys, kind="stable")
    sc = cost[order]
    prefix = np.cumsum(sc, dtype=np.uint64)
    total = int(prefix[-1])
    before = (prefix - sc).astype(object)
    r = np.array([min(world - 1, int(b) * world // total) for b in before], dtype=np.int64)
    ranks = np.empty(tgt.shape[0], dtype=np.int64)
    ranks[order] = r
    return ranks
