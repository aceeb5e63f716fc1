/*
 * Block upper triangular form of a square sparse pattern, for the oracle and
 * the reference build under oracle/_ref (SuiteSparse's btf_order is absent
 * here).  Test infrastructure only.
 *
 * Contract (SuiteSparse BTF as the reference binds it,
 * blockdaglu/src/btf_dynamic.h:19-28, called at
 * blockdaglu/src/ubtf_block_solver.cpp:661-670, Q unflipped at :705-707):
 *   input  A in CSC (Ap[n+1], Ai[nnz]);
 *   output P[k] = row of A placed at position k, Q[k] = column of A placed at
 *          position k (BTF_FLIP(j) = -j-2 for a column that could not be
 *          matched to a row), R[0..nblocks] block boundaries, *nmatch = size of
 *          the maximum matching; returns nblocks.  A(P, Q) is block upper
 *          triangular and its diagonal blocks are the strongly connected
 *          components of the matched graph.
 *
 * Algorithm (own restatement of the published methods, not SuiteSparse's
 * code or traversal order):
 *   1. maximum transversal: a greedy pass (first free row of each column),
 *      then Hopcroft-Karp phases -- a breadth-first layering from all free
 *      columns, then vertex-disjoint augmenting paths by depth-first search
 *      along the layers with a per-column edge cursor kept for the whole
 *      phase (Hopcroft and Karp, SIAM J. Comput. 2(4), 1973);
 *   2. unmatched rows are paired with unmatched columns in increasing order
 *      (those columns are reported flipped);
 *   3. strongly connected components by Tarjan's algorithm (SIAM J. Comput.
 *      1(2), 1972), iterative, on the graph "column position k -> rows of
 *      that column": components come out in an order in which every entry
 *      A(P[i], Q[k]) has block(i) <= block(k).
 * Any maximum matching gives the same blocks (as sets of rows and columns);
 * the order of the blocks and of the rows inside a block may differ from
 * SuiteSparse's.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define OR_FLIP(j) (-(j)-2)

static int cmp_i32(const void* a, const void* b) {
  const int32_t x = *(const int32_t*)a, y = *(const int32_t*)b;
  return (x > y) - (x < y);
}

static int32_t* ialloc(int64_t count) { return (int32_t*)malloc(sizeof(int32_t) * (size_t)(count > 0 ? count : 1)); }

/* Maximum matching: col_match[j] = row or -1, row_match[i] = column or -1.
 * Returns the matching size, or -1 on allocation failure. */
static int32_t or_max_matching(int32_t n, const int32_t* Ap, const int32_t* Ai, int32_t* col_match,
                               int32_t* row_match) {
  int32_t i, j, size = 0;
  int32_t *dist = ialloc(n), *queue = ialloc(n), *cursor = ialloc(n), *stack = ialloc(n);
  if (!dist || !queue || !cursor || !stack) {
    free(dist);
    free(queue);
    free(cursor);
    free(stack);
    return -1;
  }
  for (i = 0; i < n; ++i) row_match[i] = -1;
  for (j = 0; j < n; ++j) {
    int32_t p;
    col_match[j] = -1;
    for (p = Ap[j]; p < Ap[j + 1]; ++p)
      if (row_match[Ai[p]] < 0) {
        row_match[Ai[p]] = j;
        col_match[j] = Ai[p];
        ++size;
        break;
      }
  }
  for (;;) {
    /* Layering: dist[j] for columns reachable from free columns by
     * alternating paths; `limit` is the layer at which a free row was met. */
    int32_t head = 0, tail = 0, limit = -1, augmented = 0;
    for (j = 0; j < n; ++j) {
      dist[j] = -1;
      if (col_match[j] < 0) {
        dist[j] = 0;
        queue[tail++] = j;
      }
    }
    while (head < tail) {
      const int32_t c = queue[head++];
      int32_t p;
      if (limit >= 0 && dist[c] >= limit) break;
      for (p = Ap[c]; p < Ap[c + 1]; ++p) {
        const int32_t r = Ai[p], c2 = row_match[r];
        if (c2 < 0) {
          if (limit < 0) limit = dist[c] + 1;
        } else if (dist[c2] < 0) {
          dist[c2] = dist[c] + 1;
          queue[tail++] = c2;
        }
      }
    }
    if (limit < 0) break;
    /* Disjoint shortest augmenting paths from each free column. */
    for (j = 0; j < n; ++j) cursor[j] = Ap[j];
    for (j = 0; j < n; ++j) {
      int32_t top = 0;
      if (col_match[j] >= 0 || dist[j] != 0) continue;
      stack[top++] = j;
      while (top > 0) {
        const int32_t c = stack[top - 1];
        int32_t found = -1;
        while (cursor[c] < Ap[c + 1]) {
          const int32_t r = Ai[cursor[c]++], c2 = row_match[r];
          if (c2 < 0) {
            if (dist[c] + 1 == limit) {
              found = r;
              break;
            }
          } else if (dist[c2] == dist[c] + 1 && dist[c2] < limit) {
            stack[top++] = c2;
            found = -2;
            break;
          }
        }
        if (found >= 0) {
          /* Flip the path: stack[0..top-1] are the columns; each column takes
           * the row the next column gives up, the last takes the free row. */
          int32_t r = found, k;
          for (k = top - 1; k >= 0; --k) {
            const int32_t c3 = stack[k], prev = col_match[c3];
            col_match[c3] = r;
            row_match[r] = c3;
            r = prev;
          }
          ++size;
          ++augmented;
          for (k = 0; k < top; ++k) dist[stack[k]] = -1; /* used in this phase */
          top = 0;
        } else if (found == -1) {
          dist[c] = -1; /* dead end for the rest of the phase */
          --top;
        }
      }
    }
    if (!augmented) break;
  }
  free(dist);
  free(queue);
  free(cursor);
  free(stack);
  return size;
}

int32_t or_btf_order(int32_t n, const int32_t* Ap, const int32_t* Ai, int32_t* P, int32_t* Q, int32_t* R,
                     int32_t* nmatch) {
  int32_t i, j, k, nblocks = 0, counter = 0, sp = 0, cp = 0, next_free_col = 0, matched;
  int32_t *col_match, *row_match, *qm, *index, *low, *stk, *cstack, *cursor;
  char *onstk, *flipped;
  if (n < 0) return -1;
  if (n == 0) {
    R[0] = 0;
    if (nmatch) *nmatch = 0;
    return 0;
  }
  col_match = ialloc(n);
  row_match = ialloc(n);
  qm = ialloc(n);
  index = ialloc(n);
  low = ialloc(n);
  stk = ialloc(n);
  cstack = ialloc(n);
  cursor = ialloc(n);
  onstk = (char*)calloc((size_t)n, 1);
  flipped = (char*)calloc((size_t)n, 1);
  if (!col_match || !row_match || !qm || !index || !low || !stk || !cstack || !cursor || !onstk || !flipped) {
    nblocks = -1;
    goto done;
  }
  matched = or_max_matching(n, Ap, Ai, col_match, row_match);
  if (matched < 0) {
    nblocks = -1;
    goto done;
  }
  if (nmatch) *nmatch = matched;
  /* qm[i] = column matched to row i; unmatched rows take the unmatched
   * columns in increasing order (flipped in Q). */
  for (i = 0; i < n; ++i) {
    if (row_match[i] >= 0) {
      qm[i] = row_match[i];
      continue;
    }
    while (col_match[next_free_col] >= 0) ++next_free_col;
    qm[i] = next_free_col;
    col_match[next_free_col] = i;
    flipped[i] = 1;
    ++next_free_col;
  }
  /* Tarjan on vertices = rows i (position of column qm[i]); out-edges of i:
   * the rows of column qm[i]. */
  for (i = 0; i < n; ++i) index[i] = -1;
  for (j = 0; j < n; ++j) {
    if (index[j] >= 0) continue;
    cstack[cp++] = j;
    index[j] = low[j] = counter++;
    stk[sp++] = j;
    onstk[j] = 1;
    cursor[j] = Ap[qm[j]];
    while (cp > 0) {
      const int32_t v = cstack[cp - 1];
      const int32_t c = qm[v];
      if (cursor[v] < Ap[c + 1]) {
        const int32_t w = Ai[cursor[v]++];
        if (index[w] < 0) {
          index[w] = low[w] = counter++;
          stk[sp++] = w;
          onstk[w] = 1;
          cursor[w] = Ap[qm[w]];
          cstack[cp++] = w;
        } else if (onstk[w] && index[w] < low[v]) {
          low[v] = index[w];
        }
        continue;
      }
      --cp;
      if (cp > 0 && low[v] < low[cstack[cp - 1]]) low[cstack[cp - 1]] = low[v];
      if (low[v] == index[v]) {
        /* Pop one component; its rows take the next positions. */
        const int32_t start = (nblocks == 0) ? 0 : R[nblocks];
        int32_t pos = start, w;
        if (nblocks == 0) R[0] = 0;
        do {
          w = stk[--sp];
          onstk[w] = 0;
          P[pos++] = w;
        } while (w != v);
        /* Rows of a component in increasing order. */
        qsort(P + start, (size_t)(pos - start), sizeof(int32_t), cmp_i32);
        R[++nblocks] = pos;
      }
    }
  }
  for (k = 0; k < n; ++k) Q[k] = flipped[P[k]] ? OR_FLIP(qm[P[k]]) : qm[P[k]];
done:
  free(col_match);
  free(row_match);
  free(qm);
  free(index);
  free(low);
  free(stk);
  free(cstack);
  free(cursor);
  free(onstk);
  free(flipped);
  return nblocks;
}
