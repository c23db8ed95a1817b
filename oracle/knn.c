/* ORACLE — test infrastructure, not product code.
 *
 * Exact k-nearest-neighbour search with the distance of PyMatting's k-d
 * tree (pymatting/util/kdtree.py:_find_knn, :129-199): float32 squared
 * differences accumulated in float64 (numba types `distance = 0.0` as
 * float64). The k smallest by (distance, index) are kept, which is
 * independent of the visiting order. The reference keeps the first found
 * among equal (and float32-equal) distances in its tree order, so the two
 * differ only where the k-th distance is tied.
 */
#include <stdint.h>

void oracle_knn(const float* f, int64_t n, int dims, int k, int64_t* out) {
    double D[256];
    int64_t I[256];
    for (int64_t q = 0; q < n; ++q) {
        int cnt = 0;
        for (int64_t c = 0; c < n; ++c) {
            double dist = 0.0;
            for (int d = 0; d < dims; ++d) {
                float dd = f[q * dims + d] - f[c * dims + d];
                dist += (double)(dd * dd);
            }
            /* keep the k smallest by (distance, index) */
            if (cnt == k && !(dist < D[k - 1] || (dist == D[k - 1] && c < I[k - 1]))) continue;
            int pos = cnt < k ? cnt : k - 1;
            while (pos > 0 && (D[pos - 1] > dist || (D[pos - 1] == dist && I[pos - 1] > c))) {
                if (pos < k) {
                    D[pos] = D[pos - 1];
                    I[pos] = I[pos - 1];
                }
                --pos;
            }
            D[pos] = dist;
            I[pos] = c;
            if (cnt < k) ++cnt;
        }
        for (int j = 0; j < k; ++j) out[q * k + j] = I[j];
    }
}
