// k-nearest-neighbour matting Laplacian (knn_laplacian,
// pymatting/laplacian/knn_laplacian.py) on the device.
//
// Features per pixel: (r, g, b, dw x, dw y) in float32 with x, y the
// numpy.linspace(0, 1, .) grids, one pass per (k, dw). Neighbours come from
// an exact search with the reference k-d tree's distance
// (pymatting/util/kdtree.py:_find_knn: float32 squared differences summed in
// float64), keeping the k smallest by (distance, index). Candidate tiles of
// 256 pixels whose bounding box is farther than every query's k-th distance
// are skipped. The reference keeps the first found among equal distances in
// its tree order, so the two differ only where the k-th distance is tied.
//
// W = sum over passes of B + B^T (B_ij = 1, or 1 - |f_i - f_j|_1 / 5 for the
// soft kernel), assembled per row: the row's own neighbours, then the rows
// that list it. Each row is sorted by column, duplicates are summed in a
// fixed order, and the row is normalised: L = I - diag(1 / rowsum(W)) W.

#include <cuda_runtime.h>

#include "pm_common.cuh"
#include <stdint.h>

int pmb_scan_exclusive(int64_t* v, int64_t n, int64_t* chunk_scratch, int64_t* total,
                       cudaStream_t s);

namespace pmb {
namespace knn {

constexpr int kMaxK = 64;
constexpr int kDims = 5;

__global__ void k_features(const double* __restrict__ image, int h, int w, double dw,
                           float* __restrict__ f) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= (long long)h * w) return;
    const int y = (int)(i / w), x = (int)(i % w);
    // numpy.linspace(0, 1, num): j * (1 / (num - 1)), last element exactly 1
    const double sx = w > 1 ? 1.0 / (double)(w - 1) : 0.0;
    const double sy = h > 1 ? 1.0 / (double)(h - 1) : 0.0;
    const double xv = (w > 1 && x == w - 1) ? 1.0 : (double)x * sx;
    const double yv = (h > 1 && y == h - 1) ? 1.0 : (double)y * sy;
    float* o = f + i * kDims;
    o[0] = (float)image[i * 3 + 0];
    o[1] = (float)image[i * 3 + 1];
    o[2] = (float)image[i * 3 + 2];
    o[3] = (float)(dw * xv);
    o[4] = (float)(dw * yv);
}

constexpr int kTile = 256;

// Bounding box of every tile of kTile consecutive feature rows: lo[5], hi[5].
__global__ void k_tile_boxes(const float* __restrict__ f, long long n, float* __restrict__ box) {
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const long long ntiles = (n + kTile - 1) / kTile;
    if (t >= ntiles) return;
    float lo[kDims], hi[kDims];
    for (int d = 0; d < kDims; ++d) lo[d] = hi[d] = f[t * kTile * kDims + d];
    const long long end = min(n, (t + 1) * kTile);
    for (long long i = t * kTile + 1; i < end; ++i)
        for (int d = 0; d < kDims; ++d) {
            lo[d] = fminf(lo[d], f[i * kDims + d]);
            hi[d] = fmaxf(hi[d], f[i * kDims + d]);
        }
    for (int d = 0; d < kDims; ++d) {
        box[t * 2 * kDims + d] = lo[d];
        box[t * 2 * kDims + kDims + d] = hi[d];
    }
}

// One thread per query, one CTA per tile of queries. Candidate tiles are
// visited with the query tile first; a tile is skipped when, for every
// query of the CTA with a full list, the lower bound of the distance to the
// tile's box exceeds the k-th distance (with a 1e-5 relative margin over the
// float32 rounding of the computed distances). The k smallest by
// (distance, index) are kept, so the visiting order does not change them.
__global__ void __launch_bounds__(kTile) k_knn(const float* __restrict__ f,
                                               const float* __restrict__ box, long long n, int k,
                                               int64_t* __restrict__ nbr) {
    __shared__ float tile[kTile * kDims];
    const long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const long long ntiles = (n + kTile - 1) / kTile;
    float qf[kDims];
#pragma unroll
    for (int d = 0; d < kDims; ++d) qf[d] = q < n ? f[q * kDims + d] : 0.f;
    double D[kMaxK];
    int64_t I[kMaxK];
    int cnt = 0;
    for (long long vt = 0; vt < ntiles; ++vt) {
        // visiting order: own tile, then the others in index order
        const long long tt = vt == 0 ? blockIdx.x : (vt <= blockIdx.x ? vt - 1 : vt);
        bool need = q < n;
        if (need && cnt == k) {
            double lb = 0.0;
#pragma unroll
            for (int d = 0; d < kDims; ++d) {
                const double lo = box[tt * 2 * kDims + d], hi = box[tt * 2 * kDims + kDims + d];
                const double v = qf[d];
                const double e = v < lo ? lo - v : (v > hi ? v - hi : 0.0);
                lb += e * e;
            }
            need = !(lb > D[k - 1] * (1.0 + 1e-5));
        }
        if (!__syncthreads_or(need)) continue;
        const long long t0 = tt * kTile;
        const int m = (int)min((long long)kTile, n - t0);
        for (int e = threadIdx.x; e < m * kDims; e += blockDim.x) tile[e] = f[t0 * kDims + e];
        __syncthreads();
        if (need) {
            for (int c = 0; c < m; ++c) {
                double dist = 0.0;
#pragma unroll
                for (int d = 0; d < kDims; ++d) {
                    const float dd = __fsub_rn(qf[d], tile[c * kDims + d]);
                    dist = __dadd_rn(dist, (double)__fmul_rn(dd, dd));
                }
                const long long ci = t0 + c;
                if (cnt == k && !(dist < D[k - 1] || (dist == D[k - 1] && ci < I[k - 1])))
                    continue;
                int pos = cnt < k ? cnt : k - 1;
                while (pos > 0 && (D[pos - 1] > dist || (D[pos - 1] == dist && I[pos - 1] > ci))) {
                    if (pos < k) {
                        D[pos] = D[pos - 1];
                        I[pos] = I[pos - 1];
                    }
                    --pos;
                }
                D[pos] = dist;
                I[pos] = ci;
                if (cnt < k) ++cnt;
            }
        }
    }
    if (q < n)
        for (int j = 0; j < k; ++j) nbr[q * k + j] = j < cnt ? I[j] : q;
}

struct Pass {
    const int64_t* nbr;  // (n, k)
    const float* f;      // (n, 5)
    int k;
};
struct Passes {
    Pass p[4];
    int np;
    int soft;
};

__device__ __forceinline__ double edge_value(const Passes& P, int pi, long long i, long long j) {
    if (!P.soft) return 1.0;
    const float* a = P.p[pi].f + i * kDims;
    const float* b = P.p[pi].f + j * kDims;
    float s = 0.f;
    for (int d = 0; d < kDims; ++d) s = __fadd_rn(s, fabsf(__fsub_rn(a[d], b[d])));
    return __dsub_rn(1.0, (double)__fdiv_rn(s, (float)kDims));
}

// in-degree of every row (edges q -> j give row j an entry)
__global__ void k_indegree(Passes P, long long n, int64_t* cap) {
    const long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (q >= n) return;
    for (int pi = 0; pi < P.np; ++pi)
        for (int e = 0; e < P.p[pi].k; ++e)
            atomicAdd((unsigned long long*)(cap + P.p[pi].nbr[q * P.p[pi].k + e]), 1ull);
}

__global__ void k_add_outdegree(long long n, int kt, int64_t* cap) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i < n) cap[i] += kt;
}

// Scatter: own neighbours at the start of the row's slots, reverse edges
// after them (slot claimed with an atomic counter).
__global__ void k_scatter(Passes P, long long n, int kt, const int64_t* off, int64_t* fillc,
                          int64_t* cols, double* vals) {
    const long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (q >= n) return;
    long long o = off[q];
    for (int pi = 0; pi < P.np; ++pi)
        for (int e = 0; e < P.p[pi].k; ++e) {
            const long long j = P.p[pi].nbr[q * P.p[pi].k + e];
            const double v = edge_value(P, pi, q, j);
            cols[o] = j;
            vals[o] = v;
            ++o;
            const long long slot = off[j] + kt +
                                   (long long)atomicAdd((unsigned long long*)(fillc + j), 1ull);
            cols[slot] = q;
            vals[slot] = v;
        }
}

// Sort each row by (column, value), merge duplicates (sum in that order),
// count the unique columns.
__global__ void k_sort_merge(long long n, const int64_t* off, const int64_t* cap, int64_t* cols,
                             double* vals, int64_t* ucount) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const long long a = off[i], m = cap[i];
    for (long long s = 1; s < m; ++s) {
        const int64_t c = cols[a + s];
        const double v = vals[a + s];
        long long t = s - 1;
        while (t >= 0 && (cols[a + t] > c || (cols[a + t] == c && vals[a + t] > v))) {
            cols[a + t + 1] = cols[a + t];
            vals[a + t + 1] = vals[a + t];
            --t;
        }
        cols[a + t + 1] = c;
        vals[a + t + 1] = v;
    }
    long long u = 0;
    for (long long s = 0; s < m; ++s) {
        if (s > 0 && cols[a + s] == cols[a + u - 1]) {
            vals[a + u - 1] = __dadd_rn(vals[a + u - 1], vals[a + s]);
        } else {
            cols[a + u] = cols[a + s];
            vals[a + u] = vals[a + s];
            ++u;
        }
    }
    ucount[i] = u;
}

// L = I - diag(1 / rowsum(W)) W into the final CSR.
__global__ void k_normalize(long long n, const int64_t* off, const int64_t* rowptr,
                            const int64_t* wcols, const double* wvals, int64_t* cols,
                            double* vals) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const long long a = off[i], b = rowptr[i], u = rowptr[i + 1] - rowptr[i];
    double s = 0.0;
    for (long long t = 0; t < u; ++t) s = __dadd_rn(s, wvals[a + t]);
    const double fct = __ddiv_rn(1.0, s);
    for (long long t = 0; t < u; ++t) {
        const long long j = wcols[a + t];
        const double wp = __dmul_rn(fct, wvals[a + t]);
        cols[b + t] = j;
        vals[b + t] = (j == i) ? __dsub_rn(1.0, wp) : -wp;
    }
}

}  // namespace knn
}  // namespace pmb

using namespace pmb::knn;

// Scratch elements (int64) for pmb_launch_knn with n pixels, total
// neighbours per pixel kt and passes np: features, neighbour lists, row
// capacities / offsets / fill counters / unique counts, and the unmerged
// W (2 n kt columns + values).
int64_t pmb_launch_knn_scratch(long long n, int kt, int np) {
    if (n <= 0 || kt <= 0 || np <= 0 || np > 4) return -1;
    const long long feat = (n * kDims * np * 4 + 7) / 8;  // floats -> int64 slots
    const long long boxes = (((n + kTile - 1) / kTile) * 2 * kDims * 4 + 7) / 8;
    return feat + boxes + n * kt + 4 * (n + 1) + ((n + 1) + 1023) / 1024 + 2 + 2 * (2 * n * kt);
}

// Two calls on the same scratch and rowptr. First (cols / vals null): the
// neighbour search and the merged rows of W; writes rowptr and the number of
// stored entries of L to *nnz_out (synchronises the stream once). Second
// (cols / vals of *nnz_out entries): L from the state the first call left.
int pmb_launch_knn(const double* image, int h, int w, const int* ks, const double* dws, int np,
                   int soft, int64_t* scratch, int64_t* rowptr, int64_t* cols, double* vals,
                   int64_t* nnz_out, cudaStream_t st) {
    const long long n = (long long)h * w;
    if (!image || !ks || !dws || np <= 0 || np > 4 || !scratch || !rowptr || n <= 0) return -2;
    int kt = 0;
    for (int p = 0; p < np; ++p) {
        if (ks[p] <= 0 || ks[p] > kMaxK || ks[p] > n) return -2;
        kt += ks[p];
    }
    float* feat = (float*)scratch;
    int64_t* s = scratch + (n * kDims * np * 4 + 7) / 8;
    float* boxes = (float*)s;
    s += (((n + kTile - 1) / kTile) * 2 * kDims * 4 + 7) / 8;
    int64_t* nbr = s;
    s += n * kt;
    int64_t* cap = s;
    s += n + 1;
    int64_t* off = s;
    s += n + 1;
    int64_t* fillc = s;
    s += n + 1;
    int64_t* ucount = s;
    s += n + 1;
    int64_t* chunk = s;
    s += ((n + 1) + 1023) / 1024 + 2;
    int64_t* wcols = s;
    s += 2 * n * kt;
    double* wvals = (double*)s;
    const int blocks = (int)((n + 255) / 256);
    if (cols && vals) {
        k_normalize<<<blocks, 256, 0, st>>>(n, off, rowptr, wcols, wvals, cols, vals);
        return pmb::launch_status() ? 1 : 0;
    }
    Passes P{};
    P.np = np;
    P.soft = soft;
    int64_t* nb = nbr;
    for (int p = 0; p < np; ++p) {
        float* fp = feat + (long long)p * n * kDims;
        k_features<<<blocks, 256, 0, st>>>(image, h, w, dws[p], fp);
        const long long ntiles = (n + kTile - 1) / kTile;
        k_tile_boxes<<<(unsigned)((ntiles + 127) / 128), 128, 0, st>>>(fp, n, boxes);
        k_knn<<<(unsigned)ntiles, kTile, 0, st>>>(fp, boxes, n, ks[p], nb);
        P.p[p] = Pass{nb, fp, ks[p]};
        nb += n * ks[p];
    }
    if (cudaMemsetAsync(cap, 0, 3 * (n + 1) * sizeof(int64_t), st) != cudaSuccess) return 1;
    k_indegree<<<blocks, 256, 0, st>>>(P, n, cap);
    k_add_outdegree<<<blocks, 256, 0, st>>>(n, kt, cap);
    cudaMemcpyAsync(off, cap, n * sizeof(int64_t), cudaMemcpyDeviceToDevice, st);
    if (pmb_scan_exclusive(off, n, chunk, off + n, st)) return 1;
    cudaMemsetAsync(fillc, 0, (n + 1) * sizeof(int64_t), st);
    k_scatter<<<blocks, 256, 0, st>>>(P, n, kt, off, fillc, wcols, wvals);
    k_sort_merge<<<blocks, 256, 0, st>>>(n, off, cap, wcols, wvals, ucount);
    cudaMemcpyAsync(rowptr, ucount, n * sizeof(int64_t), cudaMemcpyDeviceToDevice, st);
    if (pmb_scan_exclusive(rowptr, n, chunk, rowptr + n, st)) return 1;
    int64_t nnz = 0;
    cudaMemcpyAsync(&nnz, rowptr + n, sizeof(int64_t), cudaMemcpyDeviceToHost, st);
    if (cudaStreamSynchronize(st) != cudaSuccess) return 1;
    if (nnz_out) *nnz_out = nnz;
    return pmb::launch_status() ? 1 : 0;
}
