/* ORACLE — test infrastructure, not product code.
 *
 * Exact k-nearest-neighbour search with the insertion rule of PyMatting's
 * k-d tree (pymatting/util/kdtree.py:_find_knn, :129-199): the squared
 * distance accumulates float32 squared differences in float64 (numba types
 * `distance = 0.0` as float64), is stored as float32, and a candidate is
 * inserted before the first stored distance that is strictly larger.
 * Candidates are visited in index order here; the reference visits them in
 * its tree order, which only matters among points at equal distance.
 */
#include <stdint.h>

void oracle_knn(const float* f, int64_t n, int dims, int k, int64_t* out) {
    float D[256];
    int64_t I[256];
    for (int64_t q = 0; q < n; ++q) {
        int cnt = 0;
        for (int64_t c = 0; c < n; ++c) {
            double dist = 0.0;
            for (int d = 0; d < dims; ++d) {
                float dd = f[q * dims + d] - f[c * dims + d];
                dist += (double)(dd * dd);
            }
            int pos = cnt;
            for (int j = cnt - 1; j >= 0; --j)
                if ((double)D[j] > dist) pos = j;
            if (pos < k) {
                for (int j = (cnt < k - 1 ? cnt : k - 1); j > pos; --j) {
                    D[j] = D[j - 1];
                    I[j] = I[j - 1];
                }
                D[pos] = (float)dist;
                I[pos] = c;
                cnt = cnt + 1 < k ? cnt + 1 : k;
            }
        }
        for (int j = 0; j < k; ++j) out[q * k + j] = I[j];
    }
}
