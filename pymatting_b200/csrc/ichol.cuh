// Launch interface of the incomplete-Cholesky kernels (ichol.cu).
#pragma once

#include "pm_common.cuh"

namespace pmb {

void ichol_launch_init(int64_t n, const int64_t* Ap, const int64_t* Ar, const double* Av,
                       double shift, double* d, double* rsum, int* level, unsigned long long* band,
                       cudaStream_t s);
void ichol_launch_factor(int64_t n, int64_t W, const int64_t* Ap, const int64_t* Ar,
                         const double* Av, double* d, const double* rsum, int* level, double* F,
                         uint8_t* pat, int* cand, double* keptv, int64_t* kepti, int64_t* Lp,
                         int64_t* Lr, double* Lv, int64_t cap, double discard, int64_t max_nnz,
                         double rel, int diag_keep, int64_t* result, cudaStream_t s);
void ichol_launch_levels(int64_t n, const int* level, int64_t* cnt, int* maxlevel, cudaStream_t s);
void ichol_launch_level_scatter(int64_t n, const int* level, int64_t* fill, int* order,
                                const int64_t* lptr, int nlevels, cudaStream_t s);
void ichol_launch_rows(int64_t n, const int64_t* Lp, const int64_t* Lr, const double* Lv,
                       int64_t* rcnt, cudaStream_t s);
void ichol_launch_row_fill(int64_t n, const int64_t* Lp, const int64_t* Lr, const double* Lv,
                           int64_t* rfill, int64_t* Rc, double* Rv, const int64_t* Rp,
                           cudaStream_t s);
void ichol_prepare();
void ichol_launch_solve(int64_t n, int nlevels, const int64_t* lptr, const int* order,
                        const int64_t* Lp, const int64_t* Lr, const double* Lv, const int64_t* Rp,
                        const int64_t* Rc, const double* Rv, const double* b, double* x,
                        const InstState* st, cudaStream_t s);

}  // namespace pmb
