// Closed-form matting Laplacian assembly on the device.
//
// Restates pymatting/laplacian/cf_laplacian.py:5-129 (_cf_laplacian) without
// its serial scatter: every thread owns one pixel i and gathers the entries
// of row i from the (2r+1)^2 windows that contain it. A CTA first computes
// the coefficients of every window touching its tile (colour mean and the
// inverse of the epsilon-regularised covariance, :38-92) into shared memory,
// then each thread walks its windows in raster order and adds
//     delta_ij - (1 + c_i' M c_j) / |w|                         (:95-129)
// to slot (j - i). Windows fully inside the known region are skipped (:34).
//
// This translation unit is compiled with -fmad=false and every expression
// keeps the reference's operation order, so each slot receives the same
// rounded terms in the same order as the reference loop: the values are
// bitwise identical to PyMatting's CSR data.
#include "pm_common.cuh"

namespace pmb {

enum { kModeEll = 0, kModeHalf = 1, kModeHard = 2 };

constexpr int kAT = 16;  // assembly tile (kAT x kAT pixels, one per thread)

struct AssembleArgs {
    const double* image;      // h*w*3, interleaved RGB
    const uint8_t* known;     // h*w (may be null: nothing known)
    int h, w;
    double epsilon;
    // kModeEll
    double* values;           // n * (4r+1)^2
    int64_t* indices;         // n * (4r+1)^2
    int64_t* indptr;          // n + 1
    // kModeHalf / kModeHard
    double* planes;           // kNH planes of h*pitch
    int pitch;
    const uint8_t* diag_mask; // kModeHalf: centre += diag_value where mask
    double diag_value;
    const uint8_t* fg;        // kModeHard: foreground mask (1 where trimap >= 0.9)
    double* rhs;              // kModeHard: pitched right-hand side -R m
};

template <int R, int MODE>
__global__ void __launch_bounds__(kAT * kAT)
cf_assemble_kernel(AssembleArgs a) {
    constexpr int SZ = 2 * R + 1;          // window side
    constexpr int WA = SZ * SZ;            // window area
    constexpr int S = 4 * R + 1;           // stencil side
    constexpr int NS = S * S;              // slots per row
    constexpr int IW = kAT + 4 * R;        // image tile side (halo 2R)
    constexpr int WW = kAT + 2 * R;        // window tile side (halo R)

    __shared__ double s_img[IW * IW * 3];
    __shared__ uint8_t s_known[IW * IW];
    __shared__ double s_mean[WW * WW * 3];
    __shared__ double s_m[WW * WW * 6];
    __shared__ uint8_t s_act[WW * WW];

    const int h = a.h, w = a.w;
    const int x0 = blockIdx.x * kAT, y0 = blockIdx.y * kAT;
    const int tid = threadIdx.x;

    for (int q = tid; q < IW * IW; q += blockDim.x) {
        int ly = q / IW, lx = q % IW;
        int y = y0 - 2 * R + ly, x = x0 - 2 * R + lx;
        bool in = (y >= 0 && y < h && x >= 0 && x < w);
        int64_t gi = (int64_t)y * w + x;
#pragma unroll
        for (int c = 0; c < 3; ++c) s_img[q * 3 + c] = in ? a.image[gi * 3 + c] : 0.0;
        s_known[q] = in ? (a.known ? a.known[gi] : 0) : 1;
    }
    __syncthreads();

    const double wa = (double)WA;
    for (int q = tid; q < WW * WW; q += blockDim.x) {
        int ly = q / WW, lx = q % WW;
        int ky = y0 - R + ly, kx = x0 - R + lx;
        bool act = (ky >= R && ky < h - R && kx >= R && kx < w - R);
        if (act) {
            bool all_known = true;
            for (int dy = 0; dy < SZ; ++dy)
                for (int dx = 0; dx < SZ; ++dx)
                    all_known = all_known && s_known[(ly + dy) * IW + (lx + dx)];
            act = !all_known;
        }
        s_act[q] = act;
        if (!act) continue;
        double mean[3];
        for (int c = 0; c < 3; ++c) {
            double s = 0.0;
            for (int dy = 0; dy < SZ; ++dy)
                for (int dx = 0; dx < SZ; ++dx)
                    s += s_img[((ly + dy) * IW + (lx + dx)) * 3 + c];
            mean[c] = s / wa;
            s_mean[q * 3 + c] = mean[c];
        }
        double a00 = a.epsilon, a01 = 0.0, a02 = 0.0;
        double a11 = a.epsilon, a12 = 0.0, a22 = a.epsilon;
        for (int dy = 0; dy < SZ; ++dy) {
            for (int dx = 0; dx < SZ; ++dx) {
                const double* p = s_img + ((ly + dy) * IW + (lx + dx)) * 3;
                double c0 = p[0] - mean[0], c1 = p[1] - mean[1], c2 = p[2] - mean[2];
                a00 += c0 * c0;
                a01 += c0 * c1;
                a02 += c0 * c2;
                a11 += c1 * c1;
                a12 += c1 * c2;
                a22 += c2 * c2;
            }
        }
        a00 /= wa; a01 /= wa; a02 /= wa;
        a11 /= wa; a12 /= wa; a22 /= wa;
        double det = a00 * a12 * a12 + a01 * a01 * a22 + a02 * a02 * a11
                     - a00 * a11 * a22 - 2 * a01 * a02 * a12;
        double inv_det = 1.0 / det;
        s_m[q * 6 + 0] = (a12 * a12 - a11 * a22) * inv_det;
        s_m[q * 6 + 1] = (a01 * a22 - a02 * a12) * inv_det;
        s_m[q * 6 + 2] = (a02 * a11 - a01 * a12) * inv_det;
        s_m[q * 6 + 3] = (a02 * a02 - a00 * a22) * inv_det;
        s_m[q * 6 + 4] = (a00 * a12 - a01 * a02) * inv_det;
        s_m[q * 6 + 5] = (a01 * a01 - a00 * a11) * inv_det;
    }
    __syncthreads();

    const int tx = tid % kAT, ty = tid / kAT;
    const int x = x0 + tx, y = y0 + ty;
    if (x >= w || y >= h) return;
    const int64_t i = (int64_t)y * w + x;

    // Row accumulators. In the half mode only forward slots are needed.
    double acc[NS];
#pragma unroll
    for (int q = 0; q < NS; ++q) acc[q] = 0.0;

    const double* Ii = s_img + ((ty + 2 * R) * IW + (tx + 2 * R)) * 3;
#pragma unroll
    for (int wy = 0; wy < SZ; ++wy) {          // window centre ky = y - R + wy
#pragma unroll
        for (int wx = 0; wx < SZ; ++wx) {      // window centre kx = x - R + wx
            const int q = (ty + wy) * WW + (tx + wx);
            if (!s_act[q]) continue;
            const double* mu = s_mean + q * 3;
            const double* m = s_m + q * 6;
            double s = Ii[0] - mu[0], t = Ii[1] - mu[1], u = Ii[2] - mu[2];
            double c0 = m[0] * s + m[1] * t + m[2] * u;
            double c1 = m[1] * s + m[3] * t + m[4] * u;
            double c2 = m[2] * s + m[4] * t + m[5] * u;
            // Window (wy, wx) covers rows y-2R+wy .. y+wy and columns
            // x-2R+wx .. x+wx; (jy, jx) walks them in raster order.
#pragma unroll
            for (int jy = 0; jy < SZ; ++jy) {
#pragma unroll
                for (int jx = 0; jx < SZ; ++jx) {
                    const int ddy = wy - 2 * R + jy;   // (yj - yi)
                    const int ddx = wx - 2 * R + jx;   // (xj - xi)
                    if (MODE == kModeHalf && half_index(ddy, ddx) < 0) continue;
                    const double* Ij = s_img + ((ty + 2 * R + ddy) * IW + (tx + 2 * R + ddx)) * 3;
                    double cj0 = Ij[0] - mu[0], cj1 = Ij[1] - mu[1], cj2 = Ij[2] - mu[2];
                    double temp = c0 * cj0 + c1 * cj1 + c2 * cj2;
                    double value = ((ddy == 0 && ddx == 0) ? 1.0 : 0.0) - (1 + temp) / wa;
                    acc[(ddy + 2 * R) * S + (ddx + 2 * R)] += value;
                }
            }
        }
    }

    if (MODE == kModeEll) {
        const int64_t base = i * NS;
#pragma unroll
        for (int dy = -2 * R; dy <= 2 * R; ++dy) {
#pragma unroll
            for (int dx = -2 * R; dx <= 2 * R; ++dx) {
                const int slot = (dy + 2 * R) * S + (dx + 2 * R);
                const int yj = y + dy, xj = x + dx;
                const bool in = (yj >= 0 && yj < h && xj >= 0 && xj < w);
                double v = acc[slot];
                if (dy == 0 && dx == 0 && a.diag_mask && a.diag_mask[i]) v = v + a.diag_value;
                a.values[base + slot] = v;
                a.indices[base + slot] = in ? ((int64_t)yj * w + xj) : 0;
            }
        }
        a.indptr[i + 1] = base + NS;
        if (i == 0) a.indptr[0] = 0;
    } else {
        const int64_t pstride = (int64_t)h * a.pitch;
        const int64_t pi = (int64_t)y * a.pitch + x;
        const bool ki = a.known ? a.known[i] != 0 : false;
#pragma unroll
        for (int p = 0; p < kNH; ++p) {
            const int dy = half_dy(p), dx = half_dx(p);
            const int slot = (dy + 2) * S + (dx + 2);
            const int yj = y + dy, xj = x + dx;
            const bool in = (yj >= 0 && yj < h && xj >= 0 && xj < w);
            double v = in ? acc[slot] : 0.0;
            if (MODE == kModeHalf) {
                if (p == 0 && a.diag_mask && a.diag_mask[i]) v = v + a.diag_value;
            } else {
                // Hard constraints: keep only unknown-unknown couplings; a
                // known pixel's row becomes the identity.
                if (p == 0) {
                    v = ki ? 1.0 : v;
                } else {
                    const bool kj = in ? a.known[(int64_t)yj * w + xj] != 0 : true;
                    v = (ki || kj) ? 0.0 : v;
                }
            }
            a.planes[p * pstride + pi] = v;
        }
        if (MODE == kModeHard) {
            // -R m with m = is_fg on the known columns, summed in column order
            // as scipy's CSR product does (estimate_alpha_cf.py:66-74).
            double sum = 0.0;
            if (!ki) {
#pragma unroll
                for (int dy = -2; dy <= 2; ++dy) {
#pragma unroll
                    for (int dx = -2; dx <= 2; ++dx) {
                        const int yj = y + dy, xj = x + dx;
                        if (yj < 0 || yj >= h || xj < 0 || xj >= w) continue;
                        const int64_t j = (int64_t)yj * w + xj;
                        if (!a.known[j]) continue;
                        const double m = a.fg[j] ? 1.0 : 0.0;
                        sum += acc[(dy + 2) * S + (dx + 2)] * m;
                    }
                }
            }
            a.rhs[pi] = ki ? 0.0 : -sum;
        }
    }
}

}  // namespace pmb

using namespace pmb;

// Launchers (called from the C-ABI layer in engine.cu).
int pmb_launch_cf_ell(const double* image, const uint8_t* known, int h, int w, int r,
                      double eps, const uint8_t* diag_mask, double diag_value, double* values,
                      int64_t* indices, int64_t* indptr, cudaStream_t s) {
    AssembleArgs a = {};
    a.image = image; a.known = known; a.h = h; a.w = w; a.epsilon = eps;
    a.values = values; a.indices = indices; a.indptr = indptr;
    a.diag_mask = diag_mask; a.diag_value = diag_value;
    dim3 grid((w + kAT - 1) / kAT, (h + kAT - 1) / kAT);
    if (r == 1) cf_assemble_kernel<1, kModeEll><<<grid, kAT * kAT, 0, s>>>(a);
    else if (r == 2) cf_assemble_kernel<2, kModeEll><<<grid, kAT * kAT, 0, s>>>(a);
    else return -1;
    return launch_status();
}

int pmb_launch_cf_half(const double* image, const uint8_t* known, int h, int w, double eps,
                       double* planes, int pitch, const uint8_t* diag_mask, double diag_value,
                       cudaStream_t s) {
    AssembleArgs a = {};
    a.image = image; a.known = known; a.h = h; a.w = w; a.epsilon = eps;
    a.planes = planes; a.pitch = pitch; a.diag_mask = diag_mask; a.diag_value = diag_value;
    dim3 grid((w + kAT - 1) / kAT, (h + kAT - 1) / kAT);
    cf_assemble_kernel<1, kModeHalf><<<grid, kAT * kAT, 0, s>>>(a);
    return launch_status();
}

int pmb_launch_cf_hard(const double* image, const uint8_t* known, const uint8_t* fg, int h,
                       int w, double eps, double* planes, int pitch, double* rhs,
                       cudaStream_t s) {
    AssembleArgs a = {};
    a.image = image; a.known = known; a.h = h; a.w = w; a.epsilon = eps;
    a.planes = planes; a.pitch = pitch; a.fg = fg; a.rhs = rhs;
    dim3 grid((w + kAT - 1) / kAT, (h + kAT - 1) / kAT);
    cf_assemble_kernel<1, kModeHard><<<grid, kAT * kAT, 0, s>>>(a);
    return launch_status();
}

// --------------------------------------------------------------------------
// Sparse-format conversions of the assembled rows
// --------------------------------------------------------------------------

namespace pmb {

// Exclusive scan of n int64 counts in place, one 1024-thread block per chunk
// of 1024 elements plus a sequential pass over the chunk totals.
__global__ void k_scan_chunks(int64_t* v, int64_t n, int64_t* chunk_sum) {
    __shared__ int64_t s[1024];
    const int64_t i = blockIdx.x * 1024ll + threadIdx.x;
    int64_t x = i < n ? v[i] : 0;
    s[threadIdx.x] = x;
    __syncthreads();
    for (int o = 1; o < 1024; o <<= 1) {
        int64_t t = threadIdx.x >= o ? s[threadIdx.x - o] : 0;
        __syncthreads();
        s[threadIdx.x] += t;
        __syncthreads();
    }
    if (i < n) v[i] = s[threadIdx.x] - x;
    if (threadIdx.x == 1023) chunk_sum[blockIdx.x] = s[1023];
}

__global__ void k_scan_totals(int64_t* chunk_sum, int64_t nchunks, int64_t* total) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    int64_t run = 0;
    for (int64_t c = 0; c < nchunks; ++c) {
        const int64_t t = chunk_sum[c];
        chunk_sum[c] = run;
        run += t;
    }
    *total = run;
}

__global__ void k_scan_add(int64_t* v, int64_t n, const int64_t* chunk_sum) {
    const int64_t i = blockIdx.x * 1024ll + threadIdx.x;
    if (i < n) v[i] += chunk_sum[blockIdx.x];
}

// Row counts for the canonical CSR of an assembled ELL: in-image slots with
// a non-zero value (scipy drops explicit zeros when forming L + C,
// pymatting/laplacian/laplacian.py:50-55).
__global__ void k_ell_count(const double* __restrict__ values, int h, int w, int r,
                            int64_t* counts) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= (int64_t)h * w) return;
    const int S = 4 * r + 1, y = (int)(i / w), x = (int)(i % w);
    int64_t c = 0;
    for (int dy = -2 * r; dy <= 2 * r; ++dy)
        for (int dx = -2 * r; dx <= 2 * r; ++dx) {
            const int yj = y + dy, xj = x + dx;
            if (yj < 0 || yj >= h || xj < 0 || xj >= w) continue;
            if (values[i * S * S + (dy + 2 * r) * S + (dx + 2 * r)] != 0.0) ++c;
        }
    counts[i] = c;
}

__global__ void k_ell_fill(const double* __restrict__ values, int h, int w, int r,
                           const int64_t* __restrict__ rowptr, int64_t* indices, double* data) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= (int64_t)h * w) return;
    const int S = 4 * r + 1, y = (int)(i / w), x = (int)(i % w);
    int64_t k = rowptr[i];
    for (int dy = -2 * r; dy <= 2 * r; ++dy)
        for (int dx = -2 * r; dx <= 2 * r; ++dx) {
            const int yj = y + dy, xj = x + dx;
            if (yj < 0 || yj >= h || xj < 0 || xj >= w) continue;
            const double v = values[i * S * S + (dy + 2 * r) * S + (dx + 2 * r)];
            if (v == 0.0) continue;
            indices[k] = (int64_t)yj * w + xj;
            data[k] = v;
            ++k;
        }
}

// Unknown-pixel compaction for the hard-constraint system.
__global__ void k_flag_unknown(const uint8_t* __restrict__ known, int64_t n, int64_t* flag) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < n) flag[i] = known[i] ? 0 : 1;
}

// Row counts of L_U = L[U, :][:, U] (estimate_alpha_cf.py:66): in-image
// slots whose column is unknown. cidx holds the compact index of every
// pixel (exclusive scan of the unknown flags).
__global__ void k_lu_count(const uint8_t* __restrict__ known, int h, int w, int r,
                           int64_t* counts_u, const int64_t* __restrict__ cidx) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= (int64_t)h * w || known[i]) return;
    const int y = (int)(i / w), x = (int)(i % w);
    int64_t c = 0;
    for (int dy = -2 * r; dy <= 2 * r; ++dy)
        for (int dx = -2 * r; dx <= 2 * r; ++dx) {
            const int yj = y + dy, xj = x + dx;
            if (yj < 0 || yj >= h || xj < 0 || xj >= w) continue;
            if (!known[(int64_t)yj * w + xj]) ++c;
        }
    counts_u[cidx[i]] = c;
}

// Fill L_U (CSR, compact indices) and b_U = -R m with m = is_fg on the known
// columns, summed in column order (estimate_alpha_cf.py:66-74).
__global__ void k_lu_fill(const double* __restrict__ values, const uint8_t* __restrict__ known,
                          const uint8_t* __restrict__ fg, int h, int w, int r,
                          const int64_t* __restrict__ cidx, const int64_t* __restrict__ rowptr,
                          int64_t* indices, double* data, double* rhs) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= (int64_t)h * w || known[i]) return;
    const int y = (int)(i / w), x = (int)(i % w);
    const int S = 4 * r + 1;   // ELL row: an S x S block of offsets
    const int64_t ci = cidx[i];
    int64_t k = rowptr[ci];
    double sum = 0.0;
    for (int dy = -2 * r; dy <= 2 * r; ++dy)
        for (int dx = -2 * r; dx <= 2 * r; ++dx) {
            const int yj = y + dy, xj = x + dx;
            if (yj < 0 || yj >= h || xj < 0 || xj >= w) continue;
            const int64_t j = (int64_t)yj * w + xj;
            const double v = values[i * S * S + (dy + 2 * r) * S + (dx + 2 * r)];
            if (known[j]) {
                sum += v * (fg[j] ? 1.0 : 0.0);
            } else {
                indices[k] = cidx[j];
                data[k] = v;
                ++k;
            }
        }
    rhs[ci] = -sum;
}

// alpha = clip(x, 0, 1) with x = trimap on known pixels and the solution
// on unknown ones (estimate_alpha_cf.py:72-76).
__global__ void k_alpha_compose(const double* __restrict__ trimap, const uint8_t* __restrict__ known,
                                const int64_t* __restrict__ cidx, const double* __restrict__ xu,
                                int64_t n, double* alpha) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    double v = known[i] ? trimap[i] : xu[cidx[i]];
    v = v < 0.0 ? 0.0 : (v > 1.0 ? 1.0 : v);
    alpha[i] = v;
}

// Trimap split (pymatting/util/util.py:510-525): fg = t >= fg_thr,
// bg = t <= bg_thr, known = fg | bg; counts[0] = #fg, counts[1] = #bg.
__global__ void k_trimap_masks(const double* __restrict__ trimap, int64_t n, double fg_thr,
                               double bg_thr, uint8_t* is_fg, uint8_t* is_known,
                               unsigned long long* counts) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    bool f = false, b = false;
    if (i < n) {
        const double t = trimap[i];
        f = t >= fg_thr;
        b = t <= bg_thr;
        is_fg[i] = f;
        is_known[i] = f || b;
    }
    const unsigned nf = __popc(__ballot_sync(0xffffffffu, f));
    const unsigned nb = __popc(__ballot_sync(0xffffffffu, b));
    if ((threadIdx.x & 31) == 0) {
        if (nf) atomicAdd(counts, (unsigned long long)nf);
        if (nb) atomicAdd(counts + 1, (unsigned long long)nb);
    }
}

}  // namespace pmb

int pmb_scan_exclusive(int64_t* v, int64_t n, int64_t* chunk_scratch, int64_t* total,
                       cudaStream_t s) {
    const int64_t nchunks = (n + 1023) / 1024;
    if (n <= 0) {
        return launch_status(cudaMemsetAsync(total, 0, sizeof(int64_t), s));
    }
    k_scan_chunks<<<(unsigned)nchunks, 1024, 0, s>>>(v, n, chunk_scratch);
    k_scan_totals<<<1, 32, 0, s>>>(chunk_scratch, nchunks, total);
    k_scan_add<<<(unsigned)nchunks, 1024, 0, s>>>(v, n, chunk_scratch);
    return launch_status();
}

int pmb_launch_ell_count(const double* values, int h, int w, int r, int64_t* counts, cudaStream_t s) {
    const int64_t n = (int64_t)h * w;
    k_ell_count<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(values, h, w, r, counts);
    return launch_status();
}

int pmb_launch_ell_fill(const double* values, int h, int w, int r, const int64_t* rowptr,
                        int64_t* indices, double* data, cudaStream_t s) {
    const int64_t n = (int64_t)h * w;
    k_ell_fill<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(values, h, w, r, rowptr, indices, data);
    return launch_status();
}

int pmb_launch_flag_unknown(const uint8_t* known, int64_t n, int64_t* flag, cudaStream_t s) {
    k_flag_unknown<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(known, n, flag);
    return launch_status();
}

int pmb_launch_lu_count(const uint8_t* known, int h, int w, int r, int64_t* counts_u,
                        const int64_t* cidx, cudaStream_t s) {
    const int64_t n = (int64_t)h * w;
    k_lu_count<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(known, h, w, r, counts_u, cidx);
    return launch_status();
}

int pmb_launch_lu_fill(const double* values, const uint8_t* known, const uint8_t* fg, int h, int w,
                       int r, const int64_t* cidx, const int64_t* rowptr, int64_t* indices,
                       double* data, double* rhs, cudaStream_t s) {
    const int64_t n = (int64_t)h * w;
    k_lu_fill<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(values, known, fg, h, w, r, cidx, rowptr,
                                                          indices, data, rhs);
    return launch_status();
}

int pmb_launch_alpha_compose(const double* trimap, const uint8_t* known, const int64_t* cidx,
                             const double* xu, int64_t n, double* alpha, cudaStream_t s) {
    k_alpha_compose<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(trimap, known, cidx, xu, n, alpha);
    return launch_status();
}

int pmb_launch_trimap_masks(const double* trimap, int64_t n, double fg_thr, double bg_thr,
                            uint8_t* is_fg, uint8_t* is_known, unsigned long long* counts,
                            cudaStream_t s) {
    if (launch_status(cudaMemsetAsync(counts, 0, 2 * sizeof(unsigned long long), s))) return -2;
    k_trimap_masks<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(trimap, n, fg_thr, bg_thr, is_fg,
                                                               is_known, counts);
    return launch_status();
}

// --------------------------------------------------------------------------
// Unknown-pixel index without caller scratch
// --------------------------------------------------------------------------
//
// For callers that must not allocate device memory, the chunk totals of the
// scan live in a fixed array of this file instead of a caller buffer. The
// array is 256 KB and exists on every device that loads the library, for the
// life of the process. The scan writes every element it reads within the same
// call (chunk sums, then the total), so nothing in it has to start at zero.
// All calls share the array: two calls whose work overlaps on the GPU (on
// different streams, or from different threads) race on it.

#include <mutex>

namespace pmb {

constexpr int64_t kStaticScanElems = 32768;
static __device__ __align__(256) int64_t g_static_scan[kStaticScanElems];

}  // namespace pmb

// Largest n: the scan of n + 1 entries needs one chunk sum per 1024 entries
// plus one slot for the total.
int64_t pmb_static_scan_max_n() { return (pmb::kStaticScanElems - 1) * 1024 - 1; }

// The driver's current context, as an opaque key (null if unavailable).
typedef int (*CtxGetCurrentFn)(void**);
static void* current_context() {
    static CtxGetCurrentFn fn = nullptr;
    static bool looked = false;
    if (!looked) {
        cudaDriverEntryPointQueryResult q;
        void* p = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) ==
                cudaSuccess && q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<CtxGetCurrentFn>(p);
        looked = true;
    }
    void* ctx = nullptr;
    if (fn && fn(&ctx) != 0) ctx = nullptr;
    return ctx;
}

// Device address of the array on the current device. Host code only knows a
// host-side stand-in for g_static_scan, so the address is looked up with
// cudaGetSymbolAddress, once per device and context: the first call on a
// device does it, and a call after the caller reset the device (a new
// primary context, where the module and its array are loaded again) looks
// it up anew.
static int static_scan_address(int64_t** out) {
    constexpr int kMaxDevices = 64;
    static std::mutex mu;
    static int64_t* addr[kMaxDevices] = {};
    static void* ctx_of[kMaxDevices] = {};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return -2;
    void* ctx = current_context();
    std::lock_guard<std::mutex> lock(mu);
    if (!addr[dev] || !ctx || ctx_of[dev] != ctx) {
        void* p = nullptr;
        if (cudaGetSymbolAddress(&p, pmb::g_static_scan) != cudaSuccess || !p) return -3;
        addr[dev] = static_cast<int64_t*>(p);
        // The lookup makes the runtime's context current if it was not yet.
        ctx_of[dev] = ctx ? ctx : current_context();
    }
    *out = addr[dev];
    return 0;
}

// cidx = exclusive scan of the unknown flags of is_known, cidx[n] = count,
// with the scan's scratch in g_static_scan. Returns 0, -1 (n too large),
// -2 (CUDA error) or -3 (the array's address could not be found).
int pmb_launch_unknown_index_static(const uint8_t* is_known, int64_t n, int64_t* cidx,
                                    cudaStream_t s) {
    if (n > pmb_static_scan_max_n()) return -1;
    int64_t* scratch = nullptr;
    if (int rc = static_scan_address(&scratch)) return rc;
    const int64_t nchunks = (n + 1 + 1023) / 1024;
    if (launch_status(cudaMemsetAsync(cidx + n, 0, sizeof(int64_t), s))) return -2;
    if (pmb_launch_flag_unknown(is_known, n, cidx, s)) return -2;
    return pmb_scan_exclusive(cidx, n + 1, scratch, scratch + nchunks, s);
}

// --------------------------------------------------------------------------
// Vector-Jacobian product of the Laplacian with respect to the image
// --------------------------------------------------------------------------
//
// grad[k] = d(mu' L(I) x) / d I_k for the radius-1 Laplacian of
// cf_laplacian.py (no counterpart in the reference, which has no gradients).
// Per active window w with centred colours c_i = I_i - mean_w,
// Delta_w = ((eps I + sum_i c_i c_i') / 9)^-1, u = sum_i mu_i c_i,
// v = sum_i x_i c_i, p = Delta u, q = Delta v, mu_bar / x_bar the window
// means of mu / x, the window's part of mu' L x is
//     sum_i mu_i x_i - 9 mu_bar x_bar - u' Delta v / 9,
// whose derivative with respect to I_k (the mean's contribution cancels
// because sum_i c_i = 0) is
//     -[(mu_k - mu_bar) q + (x_k - x_bar) p - (p (c_k . q) + q (c_k . p)) / 9] / 9.
// The window coefficients are recomputed from the image (same arithmetic as
// the assembly); each pixel gathers its windows in raster order, so the
// result is deterministic. One 16x16 tile of pixels per CTA.

namespace pmb {

__global__ void __launch_bounds__(kAT * kAT)
cf_vjp_kernel(const double* __restrict__ image, const uint8_t* __restrict__ known, int h, int w,
              double eps, const double* __restrict__ xs, const double* __restrict__ mus,
              double* __restrict__ grad) {
    constexpr int IW = kAT + 4;            // pixel tile with a 2-pixel halo
    constexpr int WW = kAT + 2;            // windows touching the tile
    __shared__ double s_img[IW * IW * 3];
    __shared__ double s_x[IW * IW];
    __shared__ double s_mu[IW * IW];
    __shared__ uint8_t s_known[IW * IW];
    __shared__ double s_mean[WW * WW * 3];
    __shared__ double s_p[WW * WW * 3];
    __shared__ double s_q[WW * WW * 3];
    __shared__ double s_bar[WW * WW * 2];
    __shared__ uint8_t s_act[WW * WW];
    const int x0 = blockIdx.x * kAT, y0 = blockIdx.y * kAT;
    const int tid = threadIdx.x;
    for (int q = tid; q < IW * IW; q += blockDim.x) {
        const int ly = q / IW, lx = q % IW;
        const int y = y0 - 2 + ly, x = x0 - 2 + lx;
        const bool in = (y >= 0 && y < h && x >= 0 && x < w);
        const int64_t gi = (int64_t)y * w + x;
#pragma unroll
        for (int c = 0; c < 3; ++c) s_img[q * 3 + c] = in ? image[gi * 3 + c] : 0.0;
        s_x[q] = in ? xs[gi] : 0.0;
        s_mu[q] = in ? mus[gi] : 0.0;
        s_known[q] = in ? (known ? known[gi] : 0) : 1;
    }
    __syncthreads();
    const double wa = 9.0;
    for (int q = tid; q < WW * WW; q += blockDim.x) {
        const int ly = q / WW, lx = q % WW;
        const int ky = y0 - 1 + ly, kx = x0 - 1 + lx;
        bool act = (ky >= 1 && ky < h - 1 && kx >= 1 && kx < w - 1);
        if (act) {
            bool all_known = true;
            for (int dy = 0; dy < 3; ++dy)
                for (int dx = 0; dx < 3; ++dx)
                    all_known = all_known && s_known[(ly + dy) * IW + (lx + dx)];
            act = !all_known;
        }
        s_act[q] = act;
        if (!act) continue;
        double mean[3];
        for (int c = 0; c < 3; ++c) {
            double s = 0.0;
            for (int dy = 0; dy < 3; ++dy)
                for (int dx = 0; dx < 3; ++dx) s += s_img[((ly + dy) * IW + (lx + dx)) * 3 + c];
            mean[c] = s / wa;
            s_mean[q * 3 + c] = mean[c];
        }
        double a00 = eps, a01 = 0.0, a02 = 0.0, a11 = eps, a12 = 0.0, a22 = eps;
        double u0 = 0.0, u1 = 0.0, u2 = 0.0, v0 = 0.0, v1 = 0.0, v2 = 0.0;
        double mb = 0.0, xb = 0.0;
        for (int dy = 0; dy < 3; ++dy) {
            for (int dx = 0; dx < 3; ++dx) {
                const int t = (ly + dy) * IW + (lx + dx);
                const double* p = s_img + t * 3;
                const double c0 = p[0] - mean[0], c1 = p[1] - mean[1], c2 = p[2] - mean[2];
                a00 += c0 * c0;
                a01 += c0 * c1;
                a02 += c0 * c2;
                a11 += c1 * c1;
                a12 += c1 * c2;
                a22 += c2 * c2;
                const double m = s_mu[t], xv = s_x[t];
                u0 += m * c0; u1 += m * c1; u2 += m * c2;
                v0 += xv * c0; v1 += xv * c1; v2 += xv * c2;
                mb += m;
                xb += xv;
            }
        }
        a00 /= wa; a01 /= wa; a02 /= wa;
        a11 /= wa; a12 /= wa; a22 /= wa;
        const double det = a00 * a12 * a12 + a01 * a01 * a22 + a02 * a02 * a11
                           - a00 * a11 * a22 - 2 * a01 * a02 * a12;
        const double inv_det = 1.0 / det;
        const double m00 = (a12 * a12 - a11 * a22) * inv_det;
        const double m01 = (a01 * a22 - a02 * a12) * inv_det;
        const double m02 = (a02 * a11 - a01 * a12) * inv_det;
        const double m11 = (a02 * a02 - a00 * a22) * inv_det;
        const double m12 = (a00 * a12 - a01 * a02) * inv_det;
        const double m22 = (a01 * a01 - a00 * a11) * inv_det;
        s_p[q * 3 + 0] = m00 * u0 + m01 * u1 + m02 * u2;
        s_p[q * 3 + 1] = m01 * u0 + m11 * u1 + m12 * u2;
        s_p[q * 3 + 2] = m02 * u0 + m12 * u1 + m22 * u2;
        s_q[q * 3 + 0] = m00 * v0 + m01 * v1 + m02 * v2;
        s_q[q * 3 + 1] = m01 * v0 + m11 * v1 + m12 * v2;
        s_q[q * 3 + 2] = m02 * v0 + m12 * v1 + m22 * v2;
        s_bar[q * 2 + 0] = mb / wa;
        s_bar[q * 2 + 1] = xb / wa;
    }
    __syncthreads();
    const int tx = tid % kAT, ty = tid / kAT;
    const int x = x0 + tx, y = y0 + ty;
    if (x >= w || y >= h) return;
    const int t = (ty + 2) * IW + (tx + 2);
    const double* Ik = s_img + t * 3;
    const double mk = s_mu[t], xk = s_x[t];
    double g0 = 0.0, g1 = 0.0, g2 = 0.0;
    for (int wy = 0; wy < 3; ++wy) {
        for (int wx = 0; wx < 3; ++wx) {
            const int q = (ty + wy) * WW + (tx + wx);
            if (!s_act[q]) continue;
            const double c0 = Ik[0] - s_mean[q * 3 + 0];
            const double c1 = Ik[1] - s_mean[q * 3 + 1];
            const double c2 = Ik[2] - s_mean[q * 3 + 2];
            const double p0 = s_p[q * 3 + 0], p1 = s_p[q * 3 + 1], p2 = s_p[q * 3 + 2];
            const double q0 = s_q[q * 3 + 0], q1 = s_q[q * 3 + 1], q2 = s_q[q * 3 + 2];
            const double dm = mk - s_bar[q * 2 + 0], dx = xk - s_bar[q * 2 + 1];
            const double cq = c0 * q0 + c1 * q1 + c2 * q2;
            const double cp = c0 * p0 + c1 * p1 + c2 * p2;
            g0 -= (dm * q0 + dx * p0 - (p0 * cq + q0 * cp) / wa) / wa;
            g1 -= (dm * q1 + dx * p1 - (p1 * cq + q1 * cp) / wa) / wa;
            g2 -= (dm * q2 + dx * p2 - (p2 * cq + q2 * cp) / wa) / wa;
        }
    }
    const int64_t gi = (int64_t)y * w + x;
    grad[gi * 3 + 0] = g0;
    grad[gi * 3 + 1] = g1;
    grad[gi * 3 + 2] = g2;
}

}  // namespace pmb

int pmb_launch_cf_vjp(const double* image, const uint8_t* known, int h, int w, double eps,
                      const double* x, const double* mu, double* grad, cudaStream_t s) {
    const dim3 grid((w + pmb::kAT - 1) / pmb::kAT, (h + pmb::kAT - 1) / pmb::kAT);
    pmb::cf_vjp_kernel<<<grid, pmb::kAT * pmb::kAT, 0, s>>>(image, known, h, w, eps, x, mu, grad);
    return launch_status();
}
