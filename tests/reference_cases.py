"""Matrix builders and tolerances of the reference's test program
(blockdaglu/apps/tests/main.cpp), restated for the Python tests."""
import numpy as np

# main.cpp:117 golden solution of small_matrix() for b = {1, 2, 3}.
GOLDEN_X = np.array([0.2222222222222222, 0.1111111111111111, 1.4444444444444444])


def small_matrix():
    """main.cpp:85-91."""
    return [(0, 0, 4.0), (0, 1, 1.0),
            (1, 0, 1.0), (1, 1, 3.0), (1, 2, 1.0),
            (2, 1, 1.0), (2, 2, 2.0)]


def cache_matrix(n, changed_column):
    """main.cpp:130-143: diagonal 4.0, one 0.25 per row, duplicate diagonal
    (4.0 + 0.5) in the last two rows."""
    out = []
    for row in range(n):
        out.append((row, row, 4.0))
        if row + 2 < n:
            col = changed_column if row == n // 2 else row + 1
            out.append((row, col, 0.25))
        else:
            out.append((row, row, 0.5))
    return out


def export_matrix():
    """main.cpp:175-181."""
    return [(0, 0, 100.0), (0, 1, 20.0), (0, 2, 7.0),
            (1, 0, 30.0), (1, 1, 80.0), (1, 3, 5.0),
            (2, 2, 0.25), (2, 3, 0.05),
            (3, 2, 0.10), (3, 3, 0.50)]


def multiply(coo, n, x):
    """main.cpp:36-43."""
    out = np.zeros(n)
    for r, c, v in coo:
        out[r] += v * x[c]
    return out


def dense(coo, n):
    """main.cpp:45-52."""
    a = np.zeros((n, n))
    for r, c, v in coo:
        a[r, c] += v
    return a


def close(a, b, tol=1e-9):
    """main.cpp:71-73."""
    return abs(a - b) <= tol * max(1.0, abs(a), abs(b))


def close_vec(actual, expected, tol=1e-9):
    actual = np.asarray(actual, dtype=np.float64).ravel()
    expected = np.asarray(expected, dtype=np.float64).ravel()
    if actual.shape != expected.shape:
        return False
    bound = tol * np.maximum(1.0, np.maximum(np.abs(actual), np.abs(expected)))
    return bool(np.all(np.abs(actual - expected) <= bound))
