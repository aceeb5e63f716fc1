"""Seeded systems for the sparse-LU route's tests: upper block triangular
systems of sparse irreducible blocks (a cyclic chain plus random entries,
every magnitude in [0.5, 2] with random sign, so the diagonal preference of
the reference's pivot test holds for most block orderings), coupled above the
blocks and randomly permuted.  Canonical COO (rows sorted, no duplicates)."""
import numpy as np
import scipy.sparse as sp


def sparse_block(rng, m, extra):
    rows = list(range(m)) + list(range(m))
    cols = list(range(m)) + [(i + 1) % m for i in range(m)]
    k = int(extra * m)
    rows += list(rng.integers(0, m, k))
    cols += list(rng.integers(0, m, k))
    vals = rng.uniform(0.5, 2.0, len(rows)) * rng.choice([-1.0, 1.0], len(rows))
    A = sp.csr_matrix((vals, (rows, cols)), shape=(m, m))
    A.sum_duplicates()
    A.eliminate_zeros()
    return A


def sparse_block_system(seed, sizes, extra=0.5):
    """(n, rows, cols, vals) of the seeded system with diagonal blocks of
    the given sizes."""
    rng = np.random.default_rng(seed)
    n = int(sum(sizes))
    A = sp.block_diag([sparse_block(rng, m, extra) for m in sizes], format="lil")
    off = 0
    for m in sizes[:-1]:
        for i in range(off, off + m, 3):
            A[i, rng.integers(off + m, n)] = 0.1 * rng.standard_normal()
        off += m
    A = A.tocsr()
    p, q = rng.permutation(n), rng.permutation(n)
    A = A[p][:, q].tocoo()
    order = np.lexsort((A.col, A.row))
    return n, A.row[order].astype(np.int32), A.col[order].astype(np.int32), A.data[order].astype(np.float64)


def no_pivot_fill(block):
    """Entries of L + U of the elimination without pivoting of a dense block's
    pattern (boolean, row-major)."""
    f = np.asarray(block) != 0
    m = f.shape[0]
    for k in range(m):
        rows = np.nonzero(f[k + 1:, k])[0] + k + 1
        if rows.size:
            f[np.ix_(rows, np.arange(k + 1, m))] |= f[k, k + 1:]
    return int(f.sum())
