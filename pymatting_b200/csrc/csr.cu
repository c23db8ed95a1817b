// Conjugate gradient on a general CSR matrix (one system), for callers of
// cg() whose matrix is not a pixel-grid stencil: the compressed hard-
// constraint system L_U of estimate_alpha_cf, user matrices, dense arrays.
// Same step structure and device-side scalars as the stencil kernels
// (pymatting/solver/cg.py:64-117); vectors are contiguous of length n.
#include "pm_common.cuh"
#include "csr.cuh"

namespace pmb {

constexpr int kCsrBlock = 256;

__device__ __forceinline__ double row_dot(const CsrMat& A, int64_t i, const double* __restrict__ v) {
    double acc = 0.0;
    for (int64_t k = A.indptr[i]; k < A.indptr[i + 1]; ++k) acc += A.data[k] * v[A.indices[k]];
    return acc;
}

__device__ __forceinline__ void csr_finish_beta(InstState* st, double rz_new, double dz, int reorth) {
    if (st->flags & kFirst) {
        st->rz = rz_new;
        return;
    }
    if (reorth) {
        st->beta = dz / st->rz;
    } else {
        double beta = 1.0 / st->rz;
        beta *= rz_new;
        st->beta = beta;
    }
    st->rz = rz_new;
}

// Single-system tile reduction: tiles are blocks of kCsrBlock entries.
template <int NQ, typename Fin>
__device__ __forceinline__ void csr_reduce(double (&v)[NQ], double* partials, int ntiles,
                                           InstState* st, Fin fin) {
    __shared__ double s_red[NQ * 32];
    tile_reduce<NQ>(v, partials, ntiles, blockIdx.x, 0, ntiles, st, s_red, fin);
}

template <int PREC>
__global__ void __launch_bounds__(kCsrBlock)
k_csr_init(CsrMat A, int64_t n, const double* __restrict__ b, const double* __restrict__ x0,
           double* x, double* r, double* z, const double* __restrict__ invd, InstState* st,
           double* partials, double atol, double rtol, int maxiter) {
    const int64_t i = blockIdx.x * (int64_t)kCsrBlock + threadIdx.x;
    double v[3] = {0.0, 0.0, 0.0};
    if (i < n) {
        const double bi = b[i];
        double ri = bi;
        if (x0) {
            ri = bi - row_dot(A, i, x0);
            x[i] = x0[i];
        } else {
            x[i] = 0.0;
        }
        r[i] = ri;
        v[0] = bi * bi;
        v[1] = ri * ri;
        if (PREC == kCsrPrecJacobi) {
            const double zi = ri * invd[i];
            z[i] = zi;
            v[2] = ri * zi;
        } else if (PREC == kCsrPrecNone) {
            v[2] = v[1];
        }
    }
    csr_reduce<3>(v, partials, gridDim.x, st, [&](double* s) {
        st->norm_b = sqrt(s[0]);
        st->norm_r = sqrt(s[1]);
        st->tol = fmax(atol, rtol * st->norm_b);
        st->iters = 0;
        st->maxiter = maxiter;
        st->flags = kFirst;
        st->beta = 0.0;
        if (st->norm_r < atol || st->norm_r < rtol * st->norm_b) st->status = kConverged;
        else if (maxiter <= 0) st->status = kMaxIter;
        else st->status = kRunning;
        if (PREC == kCsrPrecJacobi || PREC == kCsrPrecNone) st->rz = s[2];
    });
}

// Build p_new = z + beta p_old into the other parity buffer (neighbours of
// the matrix read arbitrary entries, so the combination is a separate pass).
__global__ void __launch_bounds__(kCsrBlock)
k_csr_pupdate(int64_t n, const double* __restrict__ z, double* p0, double* p1, InstState* st) {
    if (st->status != kRunning) return;
    const int64_t i = blockIdx.x * (int64_t)kCsrBlock + threadIdx.x;
    if (i >= n) return;
    const int par = st->iters & 1;
    const double* pold = par ? p1 : p0;
    double* pnew = par ? p0 : p1;
    pnew[i] = (st->flags & kFirst) ? z[i] : z[i] + st->beta * pold[i];
}

__global__ void __launch_bounds__(kCsrBlock)
k_csr_apply(CsrMat A, int64_t n, const double* p0, const double* p1, double* Ap, InstState* st,
            double* partials) {
    if (st->status != kRunning) return;
    const int par = st->iters & 1;
    const double* p = par ? p0 : p1;
    const int64_t i = blockIdx.x * (int64_t)kCsrBlock + threadIdx.x;
    double v[1] = {0.0};
    if (i < n) {
        const double api = row_dot(A, i, p);
        Ap[i] = api;
        v[0] = p[i] * api;
    }
    csr_reduce<1>(v, partials, gridDim.x, st, [&](double* s) {
        st->pap = s[0];
        st->alpha = st->rz / s[0];
        st->flags &= ~kFirst;
    });
}

// p . Ap with Ap supplied by the caller (A given as a function).
__global__ void __launch_bounds__(kCsrBlock)
k_csr_pap(int64_t n, const double* p0, const double* p1, const double* __restrict__ Ap,
          InstState* st, double* partials) {
    if (st->status != kRunning) return;
    const double* p = (st->iters & 1) ? p0 : p1;
    const int64_t i = blockIdx.x * (int64_t)kCsrBlock + threadIdx.x;
    double v[1] = {0.0};
    if (i < n) v[0] = p[i] * Ap[i];
    csr_reduce<1>(v, partials, gridDim.x, st, [&](double* s) {
        st->pap = s[0];
        st->alpha = st->rz / s[0];
        st->flags &= ~kFirst;
    });
}

template <int PREC>
__global__ void __launch_bounds__(kCsrBlock)
k_csr_update(int64_t n, double* x, double* r, double* z, const double* p0, const double* p1,
             const double* __restrict__ Ap, const double* __restrict__ invd, double* dr,
             int reorth, InstState* st, double* partials) {
    if (st->status != kRunning) return;
    const double* p = (st->iters & 1) ? p0 : p1;
    const double alpha = st->alpha;
    const int64_t i = blockIdx.x * (int64_t)kCsrBlock + threadIdx.x;
    double v[3] = {0.0, 0.0, 0.0};
    if (i < n) {
        const double rold = r[i];
        x[i] += alpha * p[i];
        const double ri = rold - alpha * Ap[i];
        r[i] = ri;
        v[0] = ri * ri;
        if (PREC == kCsrPrecJacobi) {
            const double zi = ri * invd[i];
            z[i] = zi;
            v[1] = ri * zi;
            if (reorth) v[2] = (ri - rold) * zi;
        } else if (PREC == kCsrPrecNone) {
            v[1] = v[0];
            if (reorth) v[2] = (ri - rold) * ri;
        } else if (reorth) {
            dr[i] = ri - rold;
        }
    }
    csr_reduce<3>(v, partials, gridDim.x, st, [&](double* s) {
        const double nr = sqrt(s[0]);
        st->norm_r = nr;
        st->iters += 1;
        if (!isfinite(nr)) st->status = kNonFinite;
        else if (nr < st->tol) st->status = kConverged;
        else if (st->iters >= st->maxiter) st->status = kMaxIter;
        if (st->status == kRunning && (PREC == kCsrPrecJacobi || PREC == kCsrPrecNone))
            csr_finish_beta(st, s[1], s[2], reorth);
    });
}

__global__ void __launch_bounds__(kCsrBlock)
k_csr_rz(int64_t n, const double* __restrict__ r, const double* __restrict__ z,
         const double* __restrict__ dr, int reorth, InstState* st, double* partials) {
    if (st->status != kRunning) return;
    const int64_t i = blockIdx.x * (int64_t)kCsrBlock + threadIdx.x;
    double v[2] = {0.0, 0.0};
    if (i < n) {
        v[0] = r[i] * z[i];
        if (reorth) v[1] = dr[i] * z[i];
    }
    csr_reduce<2>(v, partials, gridDim.x, st, [&](double* s) {
        csr_finish_beta(st, s[0], s[1], reorth);
    });
}

// z = M r for a preconditioner given as a matrix (cg.py:58-62, M.dot).
__global__ void __launch_bounds__(kCsrBlock)
k_csr_spmv(CsrMat A, int64_t n, const double* __restrict__ x, double* y, const InstState* st) {
    if (st && st->status != kRunning) return;
    const int64_t i = blockIdx.x * (int64_t)kCsrBlock + threadIdx.x;
    if (i < n) y[i] = row_dot(A, i, x);
}

// 1 / diagonal, summing duplicate diagonal entries like scipy's diagonal()
// (jacobi.py:24-26).
__global__ void k_csr_inv_diag(CsrMat A, int64_t n, double* invd) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    double d = 0.0;
    for (int64_t k = A.indptr[i]; k < A.indptr[i + 1]; ++k)
        if (A.indices[k] == i) d += A.data[k];
    invd[i] = 1.0 / d;
}

__global__ void k_vec_mul(int64_t n, const double* __restrict__ a, const double* __restrict__ b,
                          double* out) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < n) out[i] = a[i] * b[i];
}

static inline int blocks_for(int64_t n) { return (int)((n + kCsrBlock - 1) / kCsrBlock); }

void csr_launch_init(int prec, const CsrMat& A, int64_t n, const double* b, const double* x0,
                     double* x, double* r, double* z, const double* invd, InstState* st,
                     double* part, double atol, double rtol, int maxiter, cudaStream_t s) {
    const int g = blocks_for(n);
    if (prec == kCsrPrecNone) k_csr_init<kCsrPrecNone><<<g, kCsrBlock, 0, s>>>(A, n, b, x0, x, r, z, invd, st, part, atol, rtol, maxiter);
    else if (prec == kCsrPrecJacobi) k_csr_init<kCsrPrecJacobi><<<g, kCsrBlock, 0, s>>>(A, n, b, x0, x, r, z, invd, st, part, atol, rtol, maxiter);
    else k_csr_init<kCsrPrecOther><<<g, kCsrBlock, 0, s>>>(A, n, b, x0, x, r, z, invd, st, part, atol, rtol, maxiter);
}

void csr_launch_iteration_head(const CsrMat& A, int64_t n, const double* z, double* p0,
                               double* p1, double* Ap, InstState* st, double* part,
                               cudaStream_t s) {
    const int g = blocks_for(n);
    k_csr_pupdate<<<g, kCsrBlock, 0, s>>>(n, z, p0, p1, st);
    k_csr_apply<<<g, kCsrBlock, 0, s>>>(A, n, p0, p1, Ap, st, part);
}

void csr_launch_pupdate(int64_t n, const double* z, double* p0, double* p1, InstState* st,
                        cudaStream_t s) {
    k_csr_pupdate<<<blocks_for(n), kCsrBlock, 0, s>>>(n, z, p0, p1, st);
}

void csr_launch_pap(int64_t n, const double* p0, const double* p1, const double* Ap, InstState* st,
                    double* part, cudaStream_t s) {
    k_csr_pap<<<blocks_for(n), kCsrBlock, 0, s>>>(n, p0, p1, Ap, st, part);
}

void csr_launch_update(int prec, int64_t n, double* x, double* r, double* z, const double* p0,
                       const double* p1, const double* Ap, const double* invd, double* dr,
                       int reorth, InstState* st, double* part, cudaStream_t s) {
    const int g = blocks_for(n);
    if (prec == kCsrPrecNone) k_csr_update<kCsrPrecNone><<<g, kCsrBlock, 0, s>>>(n, x, r, z, p0, p1, Ap, invd, dr, reorth, st, part);
    else if (prec == kCsrPrecJacobi) k_csr_update<kCsrPrecJacobi><<<g, kCsrBlock, 0, s>>>(n, x, r, z, p0, p1, Ap, invd, dr, reorth, st, part);
    else k_csr_update<kCsrPrecOther><<<g, kCsrBlock, 0, s>>>(n, x, r, z, p0, p1, Ap, invd, dr, reorth, st, part);
}

void csr_launch_rz(int64_t n, const double* r, const double* z, const double* dr, int reorth,
                   InstState* st, double* part, cudaStream_t s) {
    k_csr_rz<<<blocks_for(n), kCsrBlock, 0, s>>>(n, r, z, dr, reorth, st, part);
}

void csr_launch_spmv(const CsrMat& A, int64_t n, const double* x, double* y, const InstState* st,
                     cudaStream_t s) {
    if (n > 0) k_csr_spmv<<<blocks_for(n), kCsrBlock, 0, s>>>(A, n, x, y, st);
}

void csr_launch_inv_diag(const CsrMat& A, int64_t n, double* invd, cudaStream_t s) {
    if (n > 0) k_csr_inv_diag<<<blocks_for(n), kCsrBlock, 0, s>>>(A, n, invd);
}

void csr_launch_vec_mul(int64_t n, const double* a, const double* b, double* out, cudaStream_t s) {
    if (n > 0) k_vec_mul<<<blocks_for(n), kCsrBlock, 0, s>>>(n, a, b, out);
}

int csr_partials_count(int64_t n) { return blocks_for(n); }

}  // namespace pmb

namespace pmb {

constexpr int kRowMax = 64;

// One row of L + diag(c) in scipy's canonical form: entries sorted by
// column, duplicates summed in stored order, c_i added to the diagonal and
// explicit zeros dropped (what L + scipy.sparse.diags(c) followed by tocsr()
// and sum_duplicates() yields, pymatting/laplacian/laplacian.py:50-55).
// Rows of fewer than kRowMax stored entries only (longer rows take
// canonical_row_long); returns the number of entries.
__device__ int canonical_row(const CsrMat& A, int64_t i, const double* __restrict__ c,
                             int64_t* cols, double* vals) {
    int m = 0;
    for (int64_t k = A.indptr[i]; k < A.indptr[i + 1]; ++k) {
        if (m >= kRowMax) return -1;
        const int64_t col = A.indices[k];
        const double v = A.data[k];
        int q = m - 1;
        while (q >= 0 && cols[q] > col) {
            cols[q + 1] = cols[q];
            vals[q + 1] = vals[q];
            --q;
        }
        cols[q + 1] = col;
        vals[q + 1] = v;
        ++m;
    }
    // Merge duplicates (stable order keeps the stored summation order).
    int u = 0;
    for (int q = 0; q < m; ++q) {
        if (u > 0 && cols[u - 1] == cols[q]) vals[u - 1] += vals[q];
        else {
            cols[u] = cols[q];
            vals[u] = vals[q];
            ++u;
        }
    }
    // Diagonal term.
    bool found = false;
    for (int q = 0; q < u; ++q)
        if (cols[q] == i) {
            vals[q] = vals[q] + c[i];
            found = true;
        }
    if (!found && c[i] != 0.0) {
        if (u >= kRowMax) return -1;
        int q = u - 1;
        while (q >= 0 && cols[q] > i) {
            cols[q + 1] = cols[q];
            vals[q + 1] = vals[q];
            --q;
        }
        cols[q + 1] = i;
        vals[q + 1] = c[i];
        ++u;
    }
    int z = 0;
    for (int q = 0; q < u; ++q)
        if (vals[q] != 0.0) {
            cols[z] = cols[q];
            vals[z] = vals[q];
            ++z;
        }
    return z;
}

// The same canonical row for rows longer than kRowMax, without a row buffer:
// the distinct columns are visited in ascending order by repeated selection
// of the next larger column (O(m^2) per row), each column's stored entries
// are summed in stored order, then c_i is added on the diagonal and zeros
// are dropped — the arithmetic of canonical_row. Writes the entries to
// out_cols / out_vals when they are given; returns the entry count.
__device__ int64_t canonical_row_long(const CsrMat& A, int64_t i, const double* __restrict__ c,
                                      int64_t* out_cols, double* out_vals) {
    const int64_t k0 = A.indptr[i], k1 = A.indptr[i + 1];
    int64_t count = 0;
    int64_t last = INT64_MIN;
    bool diag_done = false;
    auto emit = [&](int64_t col, double v) {
        if (v == 0.0) return;
        if (out_cols) {
            out_cols[count] = col;
            out_vals[count] = v;
        }
        ++count;
    };
    for (;;) {
        int64_t col = INT64_MAX;
        for (int64_t k = k0; k < k1; ++k) {
            const int64_t q = A.indices[k];
            if (q > last && q < col) col = q;
        }
        // The diagonal comes in its place even if the row does not store it.
        if (!diag_done && i > last && i < col && c[i] != 0.0) {
            emit(i, c[i]);
            diag_done = true;
            last = i;
            continue;
        }
        if (col == INT64_MAX) break;
        double v = 0.0;
        bool first = true;
        for (int64_t k = k0; k < k1; ++k)
            if (A.indices[k] == col) {
                v = first ? A.data[k] : v + A.data[k];
                first = false;
            }
        if (col == i) {
            v = v + c[i];
            diag_done = true;
        }
        emit(col, v);
        last = col;
    }
    return count;
}

__global__ void k_add_diag_count(CsrMat A, int64_t n, const double* __restrict__ c, int64_t* counts,
                                 int* overflow) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    (void)overflow;
    if (A.indptr[i + 1] - A.indptr[i] >= kRowMax) {
        counts[i] = canonical_row_long(A, i, c, nullptr, nullptr);
        return;
    }
    int64_t cols[kRowMax];
    double vals[kRowMax];
    counts[i] = canonical_row(A, i, c, cols, vals);
}

__global__ void k_add_diag_fill(CsrMat A, int64_t n, const double* __restrict__ c,
                                const int64_t* __restrict__ rowptr, int64_t* out_cols,
                                double* out_vals) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int64_t at = rowptr[i];
    if (A.indptr[i + 1] - A.indptr[i] >= kRowMax) {
        canonical_row_long(A, i, c, out_cols + at, out_vals + at);
        return;
    }
    int64_t cols[kRowMax];
    double vals[kRowMax];
    const int m = canonical_row(A, i, c, cols, vals);
    for (int q = 0; q < m; ++q) {
        out_cols[at + q] = cols[q];
        out_vals[at + q] = vals[q];
    }
}

// Grid matrix -> half-stencil planes. Row i = (y, x) of an (h w) x (h w)
// matrix: an entry at column j = (yj, xj) with d = (yj - y, xj - x) inside
// the 5x5 block is a forward entry (stored in plane half_index(d) at pixel
// i) or a backward one (kept in `back` at pixel j for the symmetry check);
// duplicates are summed. Entries with |dy| > 2 or |dx| > 2 are counted in
// bad[0]. planes and back must be zero on entry.
__global__ void k_csr_to_planes(CsrMat A, int h, int w, int pitch, double* planes, double* back,
                                unsigned long long* bad) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int64_t n = (int64_t)h * w;
    if (i >= n) return;
    const int y = (int)(i / w), x = (int)(i % w);
    const int64_t ps = (int64_t)h * pitch;
    unsigned long long nbad = 0;
    for (int64_t k = A.indptr[i]; k < A.indptr[i + 1]; ++k) {
        const int64_t j = A.indices[k];
        const int yj = (int)(j / w), xj = (int)(j % w);
        const int dy = yj - y, dx = xj - x;
        if (j < 0 || j >= n || dy < -2 || dy > 2 || dx < -2 || dx > 2) {
            ++nbad;
            continue;
        }
        const int p = half_index(dy, dx);
        if (p >= 0) planes[p * ps + (int64_t)y * pitch + x] += A.data[k];
        else back[(half_index(-dy, -dx) - 1) * ps + (int64_t)yj * pitch + xj] += A.data[k];
    }
    if (nbad) atomicAdd(&bad[0], nbad);
}

// Symmetry: A[i, i + d] (plane p at pixel i) against A[i + d, i] (kept in
// back at pixel i), within rel_tol of |A_ii| + |A_jj| + both values (a
// Laplacian assembled window by window is symmetric up to rounding, and
// entries that are sums of cancelling terms keep rounding of the diagonal's
// size). Pairs whose partner pixel lies outside the grid must be zero.
__global__ void k_planes_symmetric(int h, int w, int pitch, const double* planes,
                                   const double* back, double rel_tol, unsigned long long* bad) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= (int64_t)h * w) return;
    const int y = (int)(i / w), x = (int)(i % w);
    const int64_t ps = (int64_t)h * pitch;
    unsigned long long nbad = 0;
    for (int p = 1; p < kNH; ++p) {
        const double f = planes[p * ps + (int64_t)y * pitch + x];
        const double b = back[(p - 1) * ps + (int64_t)y * pitch + x];
        const int yj = y + half_dy(p), xj = x + half_dx(p);
        const bool inside = yj >= 0 && yj < h && xj >= 0 && xj < w;
        if (!inside) {
            if (f != 0.0 || b != 0.0) ++nbad;
            continue;
        }
        const double di = planes[(int64_t)y * pitch + x];
        const double dj = planes[(int64_t)yj * pitch + xj];
        if (fabs(f - b) > rel_tol * (fabs(f) + fabs(b) + fabs(di) + fabs(dj))) ++nbad;
    }
    if (nbad) atomicAdd(&bad[1], nbad);
}

void csr_launch_to_planes(const CsrMat& A, int h, int w, int pitch, double* planes, double* back,
                          double rel_tol, unsigned long long* bad, cudaStream_t s) {
    const int64_t n = (int64_t)h * w;
    if (n <= 0) return;
    const unsigned g = (unsigned)((n + 255) / 256);
    k_csr_to_planes<<<g, 256, 0, s>>>(A, h, w, pitch, planes, back, bad);
    k_planes_symmetric<<<g, 256, 0, s>>>(h, w, pitch, planes, back, rel_tol, bad);
}

void csr_launch_add_diag_count(const CsrMat& A, int64_t n, const double* c, int64_t* counts,
                               int* overflow, cudaStream_t s) {
    if (n > 0) k_add_diag_count<<<(unsigned)((n + 127) / 128), 128, 0, s>>>(A, n, c, counts, overflow);
}

void csr_launch_add_diag_fill(const CsrMat& A, int64_t n, const double* c, const int64_t* rowptr,
                              int64_t* cols, double* vals, cudaStream_t s) {
    if (n > 0) k_add_diag_fill<<<(unsigned)((n + 127) / 128), 128, 0, s>>>(A, n, c, rowptr, cols, vals);
}

}  // namespace pmb

namespace pmb {

// Dense copy of a small CSR matrix (duplicates summed).
__global__ void k_csr_densify(CsrMat A, int64_t n, double* D) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    for (int64_t j = 0; j < n; ++j) D[i * n + j] = 0.0;
    for (int64_t k = A.indptr[i]; k < A.indptr[i + 1]; ++k) D[i * n + A.indices[k]] += A.data[k];
}

// x = A^-1 b by Gaussian elimination with partial pivoting (the exact
// small solve that replaces scipy.sparse.linalg.spsolve, vcycle.py:59-60).
// One CTA; D (n x n) and x (holding b on entry) are overwritten.
__global__ void k_dense_solve(int64_t n, double* D, double* x, int* singular) {
    for (int64_t k = 0; k < n; ++k) {
        if (threadIdx.x == 0) {
            int64_t best = k;
            double bv = fabs(D[k * n + k]);
            for (int64_t i = k + 1; i < n; ++i) {
                const double v = fabs(D[i * n + k]);
                if (v > bv) { bv = v; best = i; }
            }
            if (bv == 0.0) *singular = 1;
            if (best != k) {
                for (int64_t j = 0; j < n; ++j) {
                    const double t = D[k * n + j]; D[k * n + j] = D[best * n + j]; D[best * n + j] = t;
                }
                const double t = x[k]; x[k] = x[best]; x[best] = t;
            }
        }
        __syncthreads();
        const double piv = D[k * n + k];
        for (int64_t i = k + 1 + threadIdx.x; i < n; i += blockDim.x) {
            const double f = D[i * n + k] / piv;
            for (int64_t j = k; j < n; ++j) D[i * n + j] -= f * D[k * n + j];
            x[i] -= f * x[k];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        for (int64_t i = n - 1; i >= 0; --i) {
            double s = x[i];
            for (int64_t j = i + 1; j < n; ++j) s -= D[i * n + j] * x[j];
            x[i] = s / D[i * n + i];
        }
    }
}

void csr_launch_dense_solve(const CsrMat& A, int64_t n, double* D, double* x, int* singular,
                            cudaStream_t s) {
    k_csr_densify<<<(unsigned)((n + 127) / 128), 128, 0, s>>>(A, n, D);
    k_dense_solve<<<1, 256, 0, s>>>(n, D, x, singular);
}

}  // namespace pmb
