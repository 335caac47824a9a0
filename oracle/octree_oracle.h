/* Test infrastructure: the CPU oracle (a plain-C restatement of the reference
 * algorithm for the point-cloud neighbour-search path).  Only tests/, the
 * golden-fixture script and bench.py's CPU-baseline leg load it; the product
 * never does.
 *
 * Conventions shared with the product's C ABI:
 *   encoder 1 = Morton 3D, 5 = Hilbert 3D (reference EncoderType values,
 *     inc/main_options.hpp:73-83)
 *   kernel  0 circle, 1 sphere, 2 square, 3 cube (reference Kernel_t,
 *     inc/main_options.hpp:97-103)
 *   algo    1 neighbors, 2 neighborsPrune, 3 neighborsStruct (SearchAlgo order,
 *     inc/main_options.hpp:29-34)
 *   box[12] = center xyz, radii xyz, min xyz, max xyz
 * Point arrays are AoS xyz doubles of the SFC-sorted cloud. */
#ifndef OCTREE_ORACLE_H
#define OCTREE_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_tree orc_tree;

void orc_bbox(const double* xyz, uint64_t n, double* box);
uint64_t orc_anchor(double p, double c, double r);
uint64_t orc_morton_encode(uint64_t x, uint64_t y, uint64_t z);
void orc_morton_decode(uint64_t key, uint64_t* x, uint64_t* y, uint64_t* z);
uint64_t orc_hilbert_encode(uint64_t x, uint64_t y, uint64_t z);
void orc_hilbert_decode(uint64_t key, uint64_t* x, uint64_t* y, uint64_t* z);
void orc_encode(int encoder, const double* xyz, uint64_t n, const double* box, uint64_t* keys);
void orc_sort(uint64_t* keys, uint64_t n, uint32_t* perm);

orc_tree* orc_build(int encoder, const uint64_t* keys, uint64_t n, uint64_t max_leaf, const double* box);
void orc_tree_info(const orc_tree* t, uint64_t* out);
void orc_tree_arrays(const orc_tree* t, uint32_t* offsets, uint64_t* ranges, double* centers, double* radii,
                     double* half);
void orc_tree_free(orc_tree* t);

void orc_radius_count(const orc_tree* t, const double* xyz, int kernel, int algo, const double* centers,
                      uint64_t nq, const double* radii, uint64_t* counts);
void orc_radius_fill(const orc_tree* t, const double* xyz, int kernel, int algo, const double* centers,
                     uint64_t nq, const double* radii, const uint64_t* offsets, uint64_t* idx);
void orc_struct_ranges_count(const orc_tree* t, const double* xyz, int kernel, const double* centers,
                             uint64_t nq, const double* radii, uint64_t* counts);
void orc_struct_ranges_fill(const orc_tree* t, const double* xyz, int kernel, const double* centers,
                            uint64_t nq, const double* radii, const uint64_t* offsets, uint64_t* pairs);
/* neighborsApprox (linear_octree.hpp:945-1035): neighborsStruct cut below depth `level`;
 * with `upper` the ranges of the cut octants are added */
void orc_approx_ranges_count(const orc_tree* t, const double* xyz, int kernel, const double* centers,
                             uint64_t nq, const double* radii, uint32_t level, int upper, uint64_t* counts);
void orc_approx_ranges_fill(const orc_tree* t, const double* xyz, int kernel, const double* centers,
                            uint64_t nq, const double* radii, uint32_t level, int upper, const uint64_t* offsets,
                            uint64_t* pairs);
void orc_knn(const orc_tree* t, const double* xyz, uint64_t n, const double* centers, uint64_t nq, uint64_t k,
             uint64_t* idx, double* d2, uint64_t* counts);

#ifdef __cplusplus
}
#endif
#endif
