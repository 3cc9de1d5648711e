/* Test infrastructure (oracle only) -- never linked into the product.
 *
 * A plain-C CPU restatement of the reference KIFMM pieces that parity is
 * checked against:
 *   - the kernel library and the FP64 direct sum
 *       Kernel3d::kernel   fmm3d/kernel3d.cpp:116-414
 *       Dense3d::eval      fmm3d/dense3d.cpp:38-57
 *   - the adaptive octree and its U/V/W/X interaction lists
 *       Let3d::srcdata     fmm3d/let3d.cpp:56-137
 *       Let3d::trgdata     fmm3d/let3d.cpp:140-211
 *       Let3d::calgnext    fmm3d/let3d.cpp:214-281
 *       findgnt/adjacent   fmm3d/let3d.cpp:325-352
 *   - the sampled relative error of FMM3d::check (fmm3d/fmm3d_check.cpp:61-71)
 *
 * Pinned against the reference itself (oracle/_ref/libkifmm_ref.so, built
 * from the reference's own sources) by tests/test_oracle.py and by the
 * committed fixtures in tests/golden/. */
#ifndef KIFMM_ORACLE_H
#define KIFMM_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* dof counts of a kernel id (fmm3d/kernel3d.cpp:24-86); returns 0 if known */
int ko_kernel_dofs(int kt, int* sdof, int* tdof);

/* Dense3d direct sum: trgval[t*tdof+i] = sum_s K(trg_t - src_s) den_s.
 * Positions/normals are 3 x n column-major (xyz interleaved), like the
 * reference's DblNumMat(3, n).  nthreads <= 0 picks the online CPU count. */
int ko_direct(int kt, int ncoef, const double* coefs, int ns, const double* srcpos,
              const double* srcnor, const double* srcden, int nt, const double* trgpos,
              double* trgval, int nthreads);

typedef struct ko_tree ko_tree;

/* Builds the tree and all lists.  *status = 0 on success, 3 if a point lies
 * outside the root box (the reference's iA at fmm3d/let3d.cpp:73,155). */
ko_tree* ko_tree_build(int ptsmax, int maxlevel, const double* ctr, int rootlvl, int ns,
                       const double* srcpos, int nt, const double* trgpos, int* status);
int ko_tree_nnodes(const ko_tree* t);
int ko_tree_nodes(const ko_tree* t, int* depth, int* path, int* par, int* chd, int* tag,
                  int* sbeg, int* snum, int* tbeg, int* tnum);
/* which: 0=U 1=V 2=W 3=X 4=source point ids per node 5=target point ids per node */
long ko_tree_list_total(const ko_tree* t, int which);
int ko_tree_lists(const ko_tree* t, int which, long* ptr, int* idx);
void ko_tree_free(ko_tree* t);

#ifdef __cplusplus
}
#endif
#endif
