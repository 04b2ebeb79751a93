/*
 * CPU oracle: sparse kernels of the reference PDLP path, restated in C.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker's arithmetic: the
 * tests, the smoke check and the CPU-baseline leg of the benchmark load it;
 * the product never does.
 *
 * Every kernel accumulates in exactly the order the reference's Numba kernels
 * do (one row or column at a time, entries in storage order), and the build
 * forbids FMA contraction, so each result is bit-identical to the
 * reference's on the same inputs:
 *
 *   csr_spmv          src/sovopt/core/sparse.py:50-58   (_csr_spmv; also used for
 *                     A^T y through the CSC arrays, sparse.py:61-69 _csc_spmv_t)
 *   abs_max_by_slice  src/sovopt/core/sparse.py:102-112
 *   scale_csc         src/sovopt/core/sparse.py:128-135
 *   scale_csr         src/sovopt/core/sparse.py:138-145
 *   transpose         src/sovopt/core/sparse.py:148-172 (counting sort)
 *   residual_csr      src/sovopt/numerics/refine.py:49-87 (compensated b - A x)
 *   csr_spmm          src/sovopt/core/sparse.py:72-84
 *
 * Build: see oracle/Makefile (gcc -O2 -fopenmp -ffp-contract=off).
 */
#include <stdint.h>
#include <stdlib.h>
#include <math.h>

#ifdef _OPENMP
#include <omp.h>
#endif

int oracle_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

void oracle_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

/* out[i] = sum_p values[p] * x[indices[p]] over slice i, in storage order. */
void csr_spmv(int64_t m, const int64_t* indptr, const int32_t* indices,
              const double* values, const double* x, double* out) {
    #pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < m; ++i) {
        double acc = 0.0;
        for (int64_t p = indptr[i]; p < indptr[i + 1]; ++p)
            acc += values[p] * x[indices[p]];
        out[i] = acc;
    }
}

/* out[s] = max |values[p]| over slice s; 0.0 for an empty slice. */
void abs_max_by_slice(int64_t ns, const int64_t* indptr, const double* values,
                      double* out) {
    #pragma omp parallel for schedule(static)
    for (int64_t s = 0; s < ns; ++s) {
        double hi = 0.0;
        for (int64_t p = indptr[s]; p < indptr[s + 1]; ++p) {
            double v = fabs(values[p]);
            if (v > hi) hi = v;
        }
        out[s] = hi;
    }
}

/* CSC in place: values[p] *= rowscale[indices[p]] * colscale[j]. */
void scale_csc(int64_t n, const int64_t* indptr, const int32_t* indices,
               double* values, const double* rowscale, const double* colscale) {
    #pragma omp parallel for schedule(static)
    for (int64_t j = 0; j < n; ++j) {
        double cs = colscale[j];
        for (int64_t p = indptr[j]; p < indptr[j + 1]; ++p)
            values[p] *= rowscale[indices[p]] * cs;
    }
}

/* CSR in place: values[p] *= rowscale[i] * colscale[indices[p]]. */
void scale_csr(int64_t m, const int64_t* indptr, const int32_t* indices,
               double* values, const double* rowscale, const double* colscale) {
    #pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < m; ++i) {
        double rs = rowscale[i];
        for (int64_t p = indptr[i]; p < indptr[i + 1]; ++p)
            values[p] *= rs * colscale[indices[p]];
    }
}

/* Counting-sort transpose of compressed storage: the result lists, for every
 * target slice, its entries in increasing source-slice order. */
int transpose(int64_t n, const int64_t* indptr, const int32_t* indices,
              const double* values, int64_t n_other, int64_t* t_indptr,
              int32_t* t_indices, double* t_values) {
    int64_t nnz = indptr[n];
    for (int64_t i = 0; i <= n_other; ++i) t_indptr[i] = 0;
    for (int64_t p = 0; p < nnz; ++p) t_indptr[indices[p] + 1] += 1;
    for (int64_t i = 0; i < n_other; ++i) t_indptr[i + 1] += t_indptr[i];
    int64_t* cursor = (int64_t*)malloc(sizeof(int64_t) * (size_t)(n_other > 0 ? n_other : 1));
    if (!cursor) return -1;
    for (int64_t i = 0; i < n_other; ++i) cursor[i] = t_indptr[i];
    for (int64_t j = 0; j < n; ++j) {
        for (int64_t p = indptr[j]; p < indptr[j + 1]; ++p) {
            int32_t i = indices[p];
            int64_t q = cursor[i]++;
            t_indices[q] = (int32_t)j;
            t_values[q] = values[p];
        }
    }
    free(cursor);
    return 0;
}

/* out = b - A x with a compensated (Dekker two-product + two-sum) dot per row. */
void residual_csr(int64_t m, const int64_t* rp, const int32_t* ri,
                  const double* rx, const double* x, const double* b,
                  double* out) {
    const double split = 134217729.0; /* 2^27 + 1 */
    #pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < m; ++i) {
        double s = 0.0, comp = 0.0;
        for (int64_t p = rp[i]; p < rp[i + 1]; ++p) {
            double a = rx[p], xv = x[ri[p]];
            double prod = a * xv;
            double ca = split * a, ah = ca - (ca - a), al = a - ah;
            double cb = split * xv, bh = cb - (cb - xv), bl = xv - bh;
            double err = ((ah * bh - prod) + ah * bl + al * bh) + al * bl;
            double t = s + prod, bb = t - s;
            double e = (s - (t - bb)) + (prod - bb);
            s = t;
            comp += e + err;
        }
        double bi = b[i];
        double t = bi - s, bb = t - bi;
        double e = (bi - (t - bb)) + (-s - bb);
        out[i] = t + (e - comp);
    }
}

/* out[i, :] = sum_p values[p] * X[indices[p], :], X dense row-major (n, k). */
void csr_spmm(int64_t m, int64_t k, const int64_t* indptr, const int32_t* indices,
              const double* values, const double* X, double* out) {
    #pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < m; ++i) {
        double* o = out + i * k;
        for (int64_t t = 0; t < k; ++t) o[t] = 0.0;
        for (int64_t p = indptr[i]; p < indptr[i + 1]; ++p) {
            double a = values[p];
            const double* xr = X + (int64_t)indices[p] * k;
            for (int64_t t = 0; t < k; ++t) o[t] += a * xr[t];
        }
    }
}

/* Neumaier compensated sum of a[0..n): returns the sum in *s and the running
 * correction in *comp (src/sovopt/mip/safebound.py:161-171, _neumaier_sum). */
void neumaier_sum(int64_t n, const double* a, double* s_out, double* comp_out) {
    double s = 0.0, comp = 0.0;
    for (int64_t i = 0; i < n; ++i) {
        double v = a[i];
        double t = s + v;
        if (fabs(s) >= fabs(v)) comp += (s - t) + v;
        else comp += (v - t) + s;
        s = t;
    }
    *s_out = s;
    *comp_out = comp;
}
