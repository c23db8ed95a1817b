/*
 * ORACLE (test infrastructure only). CPU restatement of PyMatting's
 * thresholded incomplete Cholesky factorisation and its triangular solves,
 * used by tests/ and the CPU baseline of bench.py to check the CUDA path.
 * Nothing in the product links or calls this file.
 *
 * Follows pymatting/preconditioner/ichol.py:
 *   - _ichol :6-113: left-looking column factorisation with a dense work
 *     column, per-row linked lists of pending columns, candidate rows sorted
 *     before insertion, absolute and relative discard thresholds, optional
 *     diagonal compensation of discarded entries; returns nnz, -1 (matrix not
 *     positive definite for this shift) or -2 (more than max_nnz entries);
 *   - _backsub_L_csc_inplace :116-129 and _backsub_LT_csc_inplace :132-145.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

static int cmp_i64(const void *a, const void *b)
{
    int64_t x = *(const int64_t *)a, y = *(const int64_t *)b;
    return (x > y) - (x < y);
}

int64_t oracle_ichol(int64_t n, const double *Av, const int64_t *Ar,
                     const int64_t *Ap, double *Lv, int64_t *Lr, int64_t *Lp,
                     double discard_threshold, double shift, int64_t max_nnz,
                     double relative_discard_threshold, int diag_keep_discarded)
{
    int64_t nnz = 0, c_n = 0, result = 0;
    int64_t *s = (int64_t *)calloc((size_t)n + 1, sizeof(int64_t));
    int64_t *t = (int64_t *)calloc((size_t)n + 1, sizeof(int64_t));
    int64_t *l = (int64_t *)malloc(sizeof(int64_t) * ((size_t)n + 1));
    double *a = (double *)calloc((size_t)n + 1, sizeof(double));
    double *r = (double *)calloc((size_t)n + 1, sizeof(double));
    uint8_t *b = (uint8_t *)calloc((size_t)n + 1, 1);
    int64_t *c = (int64_t *)malloc(sizeof(int64_t) * ((size_t)n + 1));
    double *d = (double *)malloc(sizeof(double) * ((size_t)n + 1));
    if (!s || !t || !l || !a || !r || !b || !c || !d) {
        result = -3;
        goto done;
    }
    for (int64_t j = 0; j < n; ++j) {
        l[j] = -1;
        d[j] = shift;
    }
    for (int64_t j = 0; j < n; ++j) {
        for (int64_t idx = Ap[j]; idx < Ap[j + 1]; ++idx) {
            int64_t i = Ar[idx];
            if (i == j) {
                d[j] += Av[idx];
                t[j] = idx + 1;
            }
            if (i >= j)
                r[j] += fabs(Av[idx]);
        }
    }
    for (int64_t j = 0; j < n; ++j) {
        for (int64_t idx = t[j]; idx < Ap[j + 1]; ++idx) {
            int64_t i = Ar[idx];
            double L_ij = Av[idx];
            if (L_ij != 0.0 && i > j) {
                a[i] += L_ij;
                if (!b[i]) {
                    b[i] = 1;
                    c[c_n++] = i;
                }
            }
        }
        int64_t k = l[j];
        while (k != -1) {
            int64_t k0 = s[k];
            int64_t k1 = Lp[k + 1];
            int64_t k2 = l[k];
            double L_jk = Lv[k0];
            k0 += 1;
            if (k0 < k1) {
                s[k] = k0;
                int64_t i = Lr[k0];
                l[k] = l[i];
                l[i] = k;
                for (int64_t idx = k0; idx < k1; ++idx) {
                    int64_t ii = Lr[idx];
                    double L_ik = Lv[idx];
                    a[ii] -= L_ik * L_jk;
                    if (!b[ii]) {
                        b[ii] = 1;
                        c[c_n++] = ii;
                    }
                }
            }
            k = k2;
        }
        if (d[j] <= 0.0) {
            result = -1;
            goto done;
        }
        if (nnz + 1 + c_n > max_nnz) {
            result = -2;
            goto done;
        }
        d[j] = sqrt(d[j]);
        Lv[nnz] = d[j];
        Lr[nnz] = j;
        nnz += 1;
        s[j] = nnz;
        qsort(c, (size_t)c_n, sizeof(int64_t), cmp_i64);
        for (int64_t q = 0; q < c_n; ++q) {
            int64_t i = c[q];
            double L_ij = a[i] / d[j];
            if (diag_keep_discarded)
                d[i] -= L_ij * L_ij;
            double rel = relative_discard_threshold * r[j];
            if (fabs(L_ij) > discard_threshold && fabs(a[i]) > rel) {
                if (!diag_keep_discarded)
                    d[i] -= L_ij * L_ij;
                Lv[nnz] = L_ij;
                Lr[nnz] = i;
                nnz += 1;
            }
            a[i] = 0.0;
            b[i] = 0;
        }
        c_n = 0;
        Lp[j + 1] = nnz;
        if (Lp[j] + 1 < Lp[j + 1]) {
            int64_t i = Lr[Lp[j] + 1];
            l[j] = l[i];
            l[i] = j;
        }
    }
    result = nnz;
done:
    free(s); free(t); free(l); free(a); free(r); free(b); free(c); free(d);
    return result;
}

void oracle_backsub_L(const double *data, const int64_t *indices,
                      const int64_t *indptr, double *x, int64_t n)
{
    for (int64_t j = 0; j < n; ++j) {
        int64_t k = indptr[j];
        double L_jj = data[k];
        double temp = x[j] / L_jj;
        x[j] = temp;
        for (k = indptr[j] + 1; k < indptr[j + 1]; ++k)
            x[indices[k]] -= data[k] * temp;
    }
}

void oracle_backsub_LT(const double *data, const int64_t *indices,
                       const int64_t *indptr, double *x, int64_t n)
{
    for (int64_t i = n - 1; i >= 0; --i) {
        double s = x[i];
        for (int64_t k = indptr[i] + 1; k < indptr[i + 1]; ++k)
            s -= data[k] * x[indices[k]];
        x[i] = s / data[indptr[i]];
    }
}
