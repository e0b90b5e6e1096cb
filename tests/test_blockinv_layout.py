"""The block-inverse sweep's arithmetic on the CPU (numpy), on a real
subdomain factor from the oracle: rows cut into blocks of at most 32 rows
whose left parts + N + pivots fit a staging capacity (the rule of
build_inv_blocks in csrc/fw_capi.cu), N = (I + L_bb)^-1 - I of each block's
own unit lower triangle built row by row as inv_relayout_kernel does, and
the forward/backward sweeps of subsolve_staged_kernel<T, true>: row passes
left of the block, y_b = v + N v, z = y / d, x_b = w + N^T w, then the
column updates left of the block.  The result equals the reference's
row-oriented substitution (advlas_skyline.c:134-167, restated by the
oracle's skyline_solve) to rounding."""
import numpy as np

from oracle import oracle
from adventure_fullwave_b200 import meshgen


def plain_solve(lo, pos, S, b):
    n = len(lo)
    v = b.copy()
    for i in range(1, n):
        v[i] -= sum(S[pos[i] + j] * v[j] for j in range(lo[i], i))
    for i in range(n):
        v[i] *= S[pos[i] + i]
    for i in range(n - 1, 0, -1):
        for j in range(lo[i], i):
            v[j] -= S[pos[i] + j] * v[i]
    return v


def cut_blocks(lo, cap):
    n, blocks, r = len(lo), [], 0
    while r < n:
        r0, lsum, rows = r, 0, 0
        while r < n and rows < 32:
            left = max(0, r0 - lo[r])
            if rows > 0 and lsum + left + (rows + 1) * rows // 2 + rows + 1 > cap - 2:
                break
            lsum += left
            r += 1
            rows += 1
        blocks.append((r0, r))
    return blocks


def block_inverse(lo, pos, S, r0, r1):
    nb = r1 - r0
    M = np.zeros((nb, nb), complex)
    for t in range(nb):
        for j in range(t):
            if r0 + j >= lo[r0 + t]:
                M[t, j] = S[pos[r0 + t] + r0 + j]
    N = np.zeros((nb, nb), complex)
    for i in range(1, nb):
        for j in range(i):
            acc = M[i, j]
            for k in range(j + 1, i):
                acc += M[i, k] * N[k, j]
            N[i, j] = -acc
    return N


def blockinv_solve(lo, pos, S, b, blocks):
    y = b.astype(complex).copy()
    Ns = [block_inverse(lo, pos, S, r0, r1) for r0, r1 in blocks]
    for (r0, r1), N in zip(blocks, Ns):
        v = np.array([y[t] - sum(S[pos[t] + c] * y[c] for c in range(lo[t], r0)) for t in range(r0, r1)])
        y[r0:r1] = v + N @ v
    y *= np.array([S[pos[i] + i] for i in range(len(lo))])
    for (r0, r1), N in reversed(list(zip(blocks, Ns))):
        w = y[r0:r1].copy()
        y[r0:r1] = w + N.T @ w
        for t in range(r1 - 1, r0 - 1, -1):
            for c in range(lo[t], r0):
                y[c] -= S[pos[t] + c] * y[t]
    return y


def test_block_inverse_sweep_equals_substitution():
    model = meshgen.make_model("x", n=6, size=1.0, npml=1, nleaves=2, seed=3)
    meshgen.round_trip_material(model)
    part = oracle.partition(model)
    sub = max(part.subs, key=lambda s: s.edge_gid.shape[0])
    lo, pos, _, S = oracle.factor_sub(model, sub)
    n = len(lo)
    assert n > 100 and max(i - lo[i] for i in range(n)) > 32  # rows reach past one block
    b = np.random.default_rng(0).standard_normal(n) + 1j * np.random.default_rng(1).standard_normal(n)
    want = plain_solve(lo, pos, S, b)
    for cap in (256, 1024):
        blocks = cut_blocks(lo, cap)
        assert blocks[0][0] == 0 and blocks[-1][1] == n and len(blocks) > 3
        assert all(r1 - r0 <= 32 for r0, r1 in blocks)
        got = blockinv_solve(lo, pos, S, b, blocks)
        assert np.linalg.norm(got - want) <= 1e-12 * np.linalg.norm(want)
