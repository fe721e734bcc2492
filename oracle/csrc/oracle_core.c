/*
 * CPU oracle: C restatement of the reference algorithms the B200 backend
 * replaces.  TEST INFRASTRUCTURE ONLY -- used by tests/, the smoke check and
 * the CPU baseline of bench.py, never by the backend.
 *
 *  oracle_build_sparsity  follows build_sparsity_pattern_seq,
 *                         pyop2/sparsity_utils.cxx:5-51 (per-row ordered set
 *                         of columns; here: gather, sort, unique per row).
 *  oracle_plan_color      follows Plan._compute_coloring,
 *                         pyop2/plan.pyx:214-376 (greedy thread colouring in
 *                         element order per block, then greedy block
 *                         colouring in block order, 32-colour mask rounds).
 *  oracle_csr_addto_*     follow addto_scalar / addto_vector,
 *                         pyop2/mat_utils.cxx:4-28, with PETSc's
 *                         MatSetValuesLocal ADD/INSERT on a fixed CSR pattern.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

static int cmp_int(const void *a, const void *b) {
  int x = *(const int *)a, y = *(const int *)b;
  return (x > y) - (x < y);
}

/* rmaps[m] / cmaps[m]: [from_size[m]][rdims[m]] / [..][cdims[m]] int32.
 * Outputs are malloc'd; free with oracle_free. Returns 0 or -1 (bad index). */
int oracle_build_sparsity(int rmult, int cmult, int nrows, int nmaps, const int *const *rmaps,
                          const int *rdims, const int *const *cmaps, const int *cdims,
                          const int *from_size, int **nnz_out, int **rowptr_out,
                          int **colidx_out, int64_t *nz_out) {
  const int lsize = nrows * rmult;
  int64_t *cnt = (int64_t *)calloc((size_t)lsize + 1, sizeof(int64_t));
  for (int m = 0; m < nmaps; ++m)
    for (int e = 0; e < from_size[m]; ++e)
      for (int i = 0; i < rdims[m]; ++i)
        for (int r = 0; r < rmult; ++r) {
          int row = rmult * rmaps[m][i + e * rdims[m]] + r;
          if (row < 0 || row >= lsize) { free(cnt); return -1; }
          cnt[row + 1] += (int64_t)cdims[m] * cmult;
        }
  for (int r = 0; r < lsize; ++r) cnt[r + 1] += cnt[r];
  int *buf = (int *)malloc(sizeof(int) * (size_t)(cnt[lsize] > 0 ? cnt[lsize] : 1));
  int64_t *fill = (int64_t *)malloc(sizeof(int64_t) * ((size_t)lsize + 1));
  memcpy(fill, cnt, sizeof(int64_t) * ((size_t)lsize + 1));
  for (int m = 0; m < nmaps; ++m)
    for (int e = 0; e < from_size[m]; ++e)
      for (int i = 0; i < rdims[m]; ++i)
        for (int r = 0; r < rmult; ++r) {
          int row = rmult * rmaps[m][i + e * rdims[m]] + r;
          for (int d = 0; d < cdims[m]; ++d)
            for (int c = 0; c < cmult; ++c)
              buf[fill[row]++] = cmult * cmaps[m][d + e * cdims[m]] + c;
        }
  int *nnz = (int *)malloc(sizeof(int) * (size_t)(lsize > 0 ? lsize : 1));
  int *rowptr = (int *)malloc(sizeof(int) * ((size_t)lsize + 1));
  int64_t nz = 0;
  rowptr[0] = 0;
  for (int r = 0; r < lsize; ++r) {
    int *p = buf + cnt[r];
    int64_t k = cnt[r + 1] - cnt[r], u = 0;
    qsort(p, (size_t)k, sizeof(int), cmp_int);
    for (int64_t j = 0; j < k; ++j)
      if (j == 0 || p[j] != p[j - 1]) p[u++] = p[j];
    nnz[r] = (int)u;
    nz += u;
    rowptr[r + 1] = (int)nz;
  }
  int *colidx = (int *)malloc(sizeof(int) * (size_t)(nz > 0 ? nz : 1));
  for (int r = 0; r < lsize; ++r) memcpy(colidx + rowptr[r], buf + cnt[r], sizeof(int) * nnz[r]);
  free(buf);
  free(fill);
  free(cnt);
  *nnz_out = nnz;
  *rowptr_out = rowptr;
  *colidx_out = colidx;
  *nz_out = nz;
  return 0;
}

void oracle_free(void *p) { free(p); }

/* Race args: nrace targets (Dats / Mat row sets) of race_size[g] entries;
 * target g has race_count[g] (map, dim, idx) triples, flattened in maps/dims/
 * idxs.  thrcol[set_size] (filled -1 first), nthrcol[nblocks], pcolors[nblocks]. */
void oracle_plan_color(int nblocks, const int *nelems, int nrace, const int *race_size,
                       const int *race_count, const int *const *maps, const int *dims,
                       const int *idxs, int thread_coloring, int *thrcol, int *nthrcol,
                       int *pcolors) {
  unsigned **tmp = (unsigned **)malloc(sizeof(unsigned *) * (nrace > 0 ? nrace : 1));
  int *first = (int *)malloc(sizeof(int) * (nrace > 0 ? nrace : 1));
  int total = 0;
  for (int g = 0; g < nrace; ++g) {
    tmp[g] = (unsigned *)malloc(sizeof(unsigned) * (race_size[g] > 0 ? race_size[g] : 1));
    first[g] = total;
    total += race_count[g];
  }
  int set_size = 0;
  for (int p = 0; p < nblocks; ++p) set_size += nelems[p];
  for (int t = 0; t < set_size; ++t) thrcol[t] = -1;
#define MASK_OF(t, OPER)                                                  \
  for (int g = 0; g < nrace; ++g)                                         \
    for (int mi = 0; mi < race_count[g]; ++mi) {                          \
      int k = first[g] + mi;                                              \
      OPER(tmp[g][maps[k][(int64_t)(t) * dims[k] + idxs[k]]]);            \
    }
  if (thread_coloring) {
    int tid = 0;
    for (int p = 0; p < nblocks; ++p) {
      unsigned base = 0;
      int terminated = 0;
      while (!terminated) {
        terminated = 1;
        for (int g = 0; g < nrace; ++g) memset(tmp[g], 0, sizeof(unsigned) * race_size[g]);
        for (int t = tid; t < tid + nelems[p]; ++t) {
          if (thrcol[t] != -1) continue;
          unsigned mask = 0;
#define OR_INTO(x) mask |= (x)
          MASK_OF(t, OR_INTO)
          if (mask == 0xffffffffu) {
            terminated = 0;
          } else {
            unsigned c = 0;
            while (mask & 1u) { mask >>= 1; ++c; }
            thrcol[t] = (int)(base + c);
            unsigned bit = 1u << c;
#define SET_BIT(x) (x) |= bit
            MASK_OF(t, SET_BIT)
          }
        }
        base += 32;
      }
      int mx = -1;
      for (int t = tid; t < tid + nelems[p]; ++t) mx = thrcol[t] > mx ? thrcol[t] : mx;
      nthrcol[p] = mx + 1;
      tid += nelems[p];
    }
  } else {
    for (int p = 0; p < nblocks; ++p) nthrcol[p] = 0;
  }
  for (int p = 0; p < nblocks; ++p) pcolors[p] = -1;
  unsigned base = 0;
  int terminated = 0;
  while (!terminated) {
    terminated = 1;
    for (int g = 0; g < nrace; ++g) memset(tmp[g], 0, sizeof(unsigned) * race_size[g]);
    int tid = 0;
    for (int p = 0; p < nblocks; ++p) {
      if (pcolors[p] == -1) {
        unsigned mask = 0;
        for (int t = tid; t < tid + nelems[p]; ++t) { MASK_OF(t, OR_INTO) }
        if (mask == 0xffffffffu) {
          terminated = 0;
        } else {
          unsigned c = 0;
          while (mask & 1u) { mask >>= 1; ++c; }
          pcolors[p] = (int)(base + c);
          unsigned bit = 1u << c;
          for (int t = tid; t < tid + nelems[p]; ++t) { MASK_OF(t, SET_BIT) }
        }
      }
      tid += nelems[p];
    }
    base += 32;
  }
  for (int g = 0; g < nrace; ++g) free(tmp[g]);
  free(tmp);
  free(first);
}

/* PETSc ADD/INSERT on a CSR pattern.  Returns -1 if (row, col) is absent
 * (PETSc: NEW_NONZERO_ALLOCATION_ERR, pyop2/petsc_base.py:113-115). */
static int64_t csr_pos(const int *rowptr, const int *colidx, int row, int col) {
  int lo = rowptr[row], hi = rowptr[row + 1];
  while (lo < hi) {
    int mid = (lo + hi) / 2;
    if (colidx[mid] < col) lo = mid + 1; else hi = mid;
  }
  return (lo < rowptr[row + 1] && colidx[lo] == col) ? lo : -1;
}

int oracle_csr_addto_scalar(double *vals, const int *rowptr, const int *colidx, double v, int row,
                            int col, int insert) {
  if (v == 0.0 && !insert) return 0;   /* mat_utils.cxx:10 */
  int64_t k = csr_pos(rowptr, colidx, row, col);
  if (k < 0) return -1;
  if (insert) vals[k] = v; else vals[k] += v;
  return 0;
}

int oracle_csr_addto_block(double *vals, const int *rowptr, const int *colidx,
                           const double *values, int nrows, const int *rows, int ncols,
                           const int *cols, int insert) {
  for (int i = 0; i < nrows; ++i)
    for (int j = 0; j < ncols; ++j) {
      int64_t k = csr_pos(rowptr, colidx, rows[i], cols[j]);
      if (k < 0) return -1;
      if (insert) vals[k] = values[i * ncols + j]; else vals[k] += values[i * ncols + j];
    }
  return 0;
}
