// The Fisher classification shared by the CUDA-core (fisher.cu) and tensor-core
// (fisher_tc.cu) classified searches: the ORDERING / MAPPING tables, the reference's
// descending bubble sort, and the class / variance-class / isometry of a block from its
// exact quadrant sums (classify.rs:62-164, Mars 1 index_func.c).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace mars {
namespace {

// ORDERING (tables.rs:13-38): the 24 descending-order permutations of the quadrants, each
// with the isometry and class newclass assigns to it.  The table is data shared with the
// reference so that class numbers and bucket order agree.
__constant__ int8_t kOrdering[24][6] = {
    {3, 2, 1, 0, 3, 0}, {2, 3, 1, 0, 5, 1}, {2, 1, 3, 0, 5, 2}, {3, 1, 2, 0, 7, 0},
    {1, 3, 2, 0, 1, 1}, {1, 2, 3, 0, 1, 2}, {3, 2, 0, 1, 3, 1}, {2, 3, 0, 1, 5, 0},
    {2, 1, 0, 3, 2, 2}, {3, 1, 0, 2, 7, 1}, {1, 3, 0, 2, 1, 0}, {1, 2, 0, 3, 4, 2},
    {3, 0, 2, 1, 3, 2}, {2, 0, 3, 1, 2, 0}, {2, 0, 1, 3, 2, 1}, {3, 0, 1, 2, 7, 2},
    {1, 0, 2, 3, 4, 1}, {1, 0, 3, 2, 4, 0}, {0, 3, 2, 1, 6, 2}, {0, 2, 3, 1, 6, 1},
    {0, 2, 1, 3, 6, 0}, {0, 3, 1, 2, 0, 2}, {0, 1, 3, 2, 0, 1}, {0, 1, 2, 3, 0, 0},
};
// MAPPING (tables.rs:42-51): isometry composition, [range isometry][domain isometry].
__constant__ uint8_t kMapping[8][8] = {
    {0, 1, 2, 3, 4, 5, 6, 7}, {2, 0, 3, 1, 7, 6, 4, 5}, {1, 3, 0, 2, 6, 7, 5, 4},
    {3, 2, 1, 0, 5, 4, 7, 6}, {4, 7, 6, 5, 0, 3, 2, 1}, {5, 6, 7, 4, 3, 0, 1, 2},
    {6, 4, 5, 7, 1, 2, 0, 3}, {7, 5, 4, 6, 2, 1, 3, 0},
};

// flips(b, iso) reads out[i][j] = b[src(i, j)] (classify.rs:139-164); quadrant q of the
// flipped block (TL, TR, BL, BR) is quadrant kFlipQuad[iso][q] of the original.
__constant__ uint8_t kFlipQuad[8][4] = {
    {0, 1, 2, 3},  // identity
    {1, 3, 0, 2},  // src (j, s-1-i)
    {2, 0, 3, 1},  // src (s-1-j, i)
    {3, 2, 1, 0},  // src (s-1-i, s-1-j)
    {1, 0, 3, 2},  // src (i, s-1-j)
    {2, 3, 0, 1},  // src (s-1-i, j)
    {0, 2, 1, 3},  // src (j, i)
    {3, 1, 2, 0},  // src (s-1-j, s-1-i)
};

// The 3-pass descending bubble sort of index_func.c (classify.rs:62-73) and match().
template <class T>
__device__ __forceinline__ int sorted_row(T a0, T a1, T a2, T a3) {
    T a[4] = {a0, a1, a2, a3};
    int o[4] = {0, 1, 2, 3};
#pragma unroll
    for (int i = 2; i >= 0; --i)
#pragma unroll
        for (int j = 0; j <= i; ++j)
            if (a[j] < a[j + 1]) {
                const T t = a[j];
                a[j] = a[j + 1];
                a[j + 1] = t;
                const int u = o[j];
                o[j] = o[j + 1];
                o[j + 1] = u;
            }
    for (int r = 0; r < 24; ++r)
        if (kOrdering[r][0] == o[0] && kOrdering[r][1] == o[1] && kOrdering[r][2] == o[2] &&
            kOrdering[r][3] == o[3])
            return r;
    return 23;  // unreachable: o is a permutation of 0..3
}

// variance_2 (classify.rs:77-89) from exact quadrant sums: sum2/n - (sum/n)^2.
__device__ __forceinline__ double quad_variance(int64_t sum, int64_t sum2, double n) {
    const double m = __ddiv_rn((double)sum, n);
    return __dsub_rn(__ddiv_rn((double)sum2, n), __dmul_rn(m, m));
}

// (isometry, class * 24 + variance class) from the four quadrant sums and sums of squares.
__device__ __forceinline__ void fisher_classify(const int64_t q[4], const int64_t q2[4], int h,
                                         int* iso, int* bucket) {
    const int r = sorted_row<int64_t>(q[0], q[1], q[2], q[3]);
    const int is = kOrdering[r][4], clas = kOrdering[r][5];
    const double n = (double)(h * h);
    double v[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const int src = kFlipQuad[is][k];
        v[k] = quad_variance(q[src], q2[src], n);
    }
    const int var_class = sorted_row<double>(v[0], v[1], v[2], v[3]);
    *iso = is;
    *bucket = clas * 24 + var_class;
}

// MAPPING[range isometry][domain isometry]: the isometry of a classified candidate.
__device__ __forceinline__ int fisher_mapping(int range_iso, int domain_iso) {
    return kMapping[range_iso][domain_iso];
}

}  // namespace
}  // namespace mars
