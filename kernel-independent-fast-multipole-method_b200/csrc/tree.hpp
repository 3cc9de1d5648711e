// Adaptive octree and U/V/W/X interaction lists (host side of setup).
//
// Same tree and same lists as the reference's Let3d (fmm3d/let3d.cpp:56-281):
// nodes are numbered breadth first exactly like Let3d::ndevec, a node splits
// while it holds more than ptsmax source points and its depth is below
// maxlevel-1 (:86), a point goes to child octant (p >= centre) per axis with
// the centre computed by the same FP64 formula (:99, :309-318), and the lists
// follow Let3d::calgnext (:214-281).  The construction differs: points get a
// Morton key from those FP64 comparisons, are radix-sorted once, and every
// node's points are a contiguous range of the sorted order (the layout the
// device kernels read).  Lists are built in parallel over target nodes.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace kifmm {

enum : int { TAG_SRC = 1, TAG_TRG = 2 };  // LET_SRCNODE / LET_TRGNODE, fmm3d/let3d.hpp:27-30

struct Csr {
  std::vector<int64_t> ptr;  // nnodes + 1
  std::vector<int> idx;
};

struct Tree {
  double ctr[3] = {0, 0, 0};
  int rootlvl = 0;
  int ptsmax = 150;
  int maxlevel = 10;

  int nnodes = 0;
  int maxdepth = 0;
  std::vector<int> depth, par, chd, tag;
  std::vector<int> path;              // 3 per node
  std::vector<int> sbeg, scnt;        // source range in sorted order (every node)
  std::vector<int> tbeg, tcnt;        // target range in sorted order (every node)
  std::vector<double> center;         // 3 per node, Let3d::center formula
  std::vector<double> radius;         // Let3d::radius
  std::vector<int> level_beg;         // nodes of depth d: [level_beg[d], level_beg[d+1])
  std::vector<int> sperm, tperm;      // sorted position -> original point id
  Csr lists[4];                       // 0=U 1=V 2=W 3=X, per node (empty for non-target nodes)

  bool terminal(int g) const { return chd[g] == -1; }
  double rad() const;
};

// Returns 0, or 3 when a point lies outside the root box (the reference's
// iA at fmm3d/let3d.cpp:73,155), or 1 on bad parameters.
int build_tree(Tree& t, int ns, const double* srcpos, int nt, const double* trgpos, int nthreads,
               std::string* err);

// The same tree and lists built on the current GPU (tree_gpu.cu) and copied
// into t; returns as build_tree, or 4 on a CUDA error.
int build_tree_device(Tree& t, int ns, const double* srcpos, int nt, const double* trgpos, std::string* err);

}  // namespace kifmm
