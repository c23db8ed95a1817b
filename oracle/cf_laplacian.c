/*
 * ORACLE (test infrastructure only). CPU restatement of PyMatting's
 * closed-form matting Laplacian assembly, used by tests/, the smoke check and
 * the CPU baseline of bench.py to check the CUDA path. Nothing in the product
 * links or calls this file.
 *
 * Follows pymatting/laplacian/cf_laplacian.py:5-129 (_cf_laplacian):
 *   - structure loop :12-25: slot k = i*(4r+1)^2 + (dy+2r)*(4r+1) + (dx+2r)
 *     holds column j = i + dy*w + dx when in bounds, else stays 0;
 *   - window loop :31-129: for every window centre not fully known, centred
 *     colours (:38-50), epsilon-regularised covariance / |w| (:53-74),
 *     adjugate inverse with the sign-flipped determinant (:76-92) and the
 *     pair scatter values[i, dy, dx] += delta_ij - (1 + c_i' M c_j) / |w|
 *     (:95-129).
 * Every floating-point operation is written in the same order as the
 * reference so that, compiled without FMA contraction, the values match it
 * bit for bit.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

int oracle_cf_laplacian(const double *image, int64_t h, int64_t w,
                        double epsilon, int64_t r, const uint8_t *is_known,
                        double *values, int64_t *indices, int64_t *indptr)
{
    const int64_t size = 2 * r + 1;
    const int64_t window_area = size * size;
    const int64_t S = 4 * r + 1;
    const int64_t slots = S * S;
    const int64_t n = h * w;

    memset(values, 0, sizeof(double) * (size_t)(n * slots));
    memset(indices, 0, sizeof(int64_t) * (size_t)(n * slots));
    indptr[0] = 0;
    for (int64_t yi = 0; yi < h; ++yi) {
        for (int64_t xi = 0; xi < w; ++xi) {
            int64_t i = xi + yi * w;
            int64_t k = i * slots;
            for (int64_t yj = yi - 2 * r; yj <= yi + 2 * r; ++yj) {
                for (int64_t xj = xi - 2 * r; xj <= xi + 2 * r; ++xj) {
                    if (xj >= 0 && xj < w && yj >= 0 && yj < h)
                        indices[k] = xj + yj * w;
                    ++k;
                }
            }
            indptr[i + 1] = k;
        }
    }

    double *c = (double *)malloc(sizeof(double) * (size_t)(window_area * 3));
    if (!c)
        return -1;
    const double wa = (double)window_area;

    for (int64_t y = r; y < h - r; ++y) {
        for (int64_t x = r; x < w - r; ++x) {
            int all_known = 1;
            for (int64_t dy = -r; dy <= r && all_known; ++dy)
                for (int64_t dx = -r; dx <= r; ++dx)
                    if (!is_known[(y + dy) * w + (x + dx)]) {
                        all_known = 0;
                        break;
                    }
            if (all_known)
                continue;

            for (int dc = 0; dc < 3; ++dc) {
                double s = 0.0;
                for (int64_t dy = 0; dy < size; ++dy)
                    for (int64_t dx = 0; dx < size; ++dx)
                        s += image[((y + dy - r) * w + (x + dx - r)) * 3 + dc];
                for (int64_t dy = 0; dy < size; ++dy)
                    for (int64_t dx = 0; dx < size; ++dx)
                        c[(dy * size + dx) * 3 + dc] =
                            image[((y + dy - r) * w + (x + dx - r)) * 3 + dc] - s / wa;
            }

            double a00 = epsilon, a01 = 0.0, a02 = 0.0;
            double a11 = epsilon, a12 = 0.0, a22 = epsilon;
            for (int64_t q = 0; q < window_area; ++q) {
                const double *cq = c + q * 3;
                a00 += cq[0] * cq[0];
                a01 += cq[0] * cq[1];
                a02 += cq[0] * cq[2];
                a11 += cq[1] * cq[1];
                a12 += cq[1] * cq[2];
                a22 += cq[2] * cq[2];
            }
            a00 /= wa; a01 /= wa; a02 /= wa;
            a11 /= wa; a12 /= wa; a22 /= wa;

            double det = a00 * a12 * a12 + a01 * a01 * a22 + a02 * a02 * a11
                         - a00 * a11 * a22 - 2 * a01 * a02 * a12;
            double inv_det = 1.0 / det;
            double m00 = (a12 * a12 - a11 * a22) * inv_det;
            double m01 = (a01 * a22 - a02 * a12) * inv_det;
            double m02 = (a02 * a11 - a01 * a12) * inv_det;
            double m11 = (a02 * a02 - a00 * a22) * inv_det;
            double m12 = (a00 * a12 - a01 * a02) * inv_det;
            double m22 = (a01 * a01 - a00 * a11) * inv_det;

            for (int64_t dyi = 0; dyi < size; ++dyi) {
                for (int64_t dxi = 0; dxi < size; ++dxi) {
                    const double *ci = c + (dyi * size + dxi) * 3;
                    double s = ci[0], t = ci[1], u = ci[2];
                    double c0 = m00 * s + m01 * t + m02 * u;
                    double c1 = m01 * s + m11 * t + m12 * u;
                    double c2 = m02 * s + m12 * t + m22 * u;
                    int64_t xi = x + dxi - r, yi = y + dyi - r;
                    int64_t i = xi + yi * w;
                    for (int64_t dyj = 0; dyj < size; ++dyj) {
                        for (int64_t dxj = 0; dxj < size; ++dxj) {
                            const double *cj = c + (dyj * size + dxj) * 3;
                            int64_t xj = x + dxj - r, yj = y + dyj - r;
                            int64_t j = xj + yj * w;
                            double temp = c0 * cj[0] + c1 * cj[1] + c2 * cj[2];
                            double value = (i == j ? 1.0 : 0.0) - (1 + temp) / wa;
                            int64_t ddx = xj - xi + 2 * r, ddy = yj - yi + 2 * r;
                            values[i * slots + ddy * S + ddx] += value;
                        }
                    }
                }
            }
        }
    }
    free(c);
    return 0;
}
