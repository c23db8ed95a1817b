// Launch interface of the general-CSR conjugate gradient kernels (csr.cu).
#pragma once

#include "pm_common.cuh"

namespace pmb {

enum : int { kCsrPrecNone = 0, kCsrPrecJacobi = 1, kCsrPrecOther = 2 };

struct CsrMat {
    const int64_t* indptr;
    const int64_t* indices;
    const double* data;
};

void csr_launch_init(int prec, const CsrMat& A, int64_t n, const double* b, const double* x0,
                     double* x, double* r, double* z, const double* invd, InstState* st,
                     double* part, double atol, double rtol, int maxiter, cudaStream_t s);
void csr_launch_iteration_head(const CsrMat& A, int64_t n, const double* z, double* p0,
                               double* p1, double* Ap, InstState* st, double* part,
                               cudaStream_t s);
void csr_launch_pupdate(int64_t n, const double* z, double* p0, double* p1, InstState* st,
                        cudaStream_t s);
void csr_launch_pap(int64_t n, const double* p0, const double* p1, const double* Ap, InstState* st,
                    double* part, cudaStream_t s);
void csr_launch_update(int prec, int64_t n, double* x, double* r, double* z, const double* p0,
                       const double* p1, const double* Ap, const double* invd, double* dr,
                       int reorth, InstState* st, double* part, cudaStream_t s);
void csr_launch_rz(int64_t n, const double* r, const double* z, const double* dr, int reorth,
                   InstState* st, double* part, cudaStream_t s);
void csr_launch_spmv(const CsrMat& A, int64_t n, const double* x, double* y, const InstState* st,
                     cudaStream_t s);
void csr_launch_inv_diag(const CsrMat& A, int64_t n, double* invd, cudaStream_t s);
void csr_launch_vec_mul(int64_t n, const double* a, const double* b, double* out, cudaStream_t s);
int csr_partials_count(int64_t n);
void csr_launch_dense_solve(const CsrMat& A, int64_t n, double* D, double* x, int* singular,
                            cudaStream_t s);
void csr_launch_add_diag_count(const CsrMat& A, int64_t n, const double* c, int64_t* counts,
                               int* overflow, cudaStream_t s);
void csr_launch_add_diag_fill(const CsrMat& A, int64_t n, const double* c, const int64_t* rowptr,
                              int64_t* cols, double* vals, cudaStream_t s);
// Half-stencil planes (pitched, 13 planes) of a grid matrix given as CSR,
// and the counts of entries outside the 5x5 pattern (bad[0]) and of
// forward/backward pairs that differ by more than rel_tol (bad[1]).
void csr_launch_to_planes(const CsrMat& A, int h, int w, int pitch, double* planes, double* back,
                          double rel_tol, unsigned long long* bad, cudaStream_t s);

}  // namespace pmb
