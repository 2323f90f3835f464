// hr_engine.h — internal types shared by the host planner (C++) and the
// device kernels (CUDA). Not part of the public C ABI.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace hr {

// Evaluation kinds. Each one is a boundary sum of the reference:
enum Kind : int {
  K_SL_ON = 0,        // eval_Stokes_SL_onSurf(_tree)      2S/stokeslets.cpp:141-225, 2S/KITC.cpp:1389
  K_SL_OFF = 1,       // eval_Stokes_SL_offSurf(_tree)     2S/stokeslets.cpp:12-135, 2S/KITC.cpp:1496
  K_DL_ON = 2,        // eval_Stokes_DL_onSurf(_tree)      2S/stresslets.cpp:186-279, 2S/KITC.cpp:1606
  K_DL_OFF = 3,       // eval_Stokes_DL_offSurf(_tree)     2S/stresslets.cpp:13-179, 2S/KITC.cpp:1712
  K_E2G_SL_AWAY = 4,  // stokes_SL_away                    E2G/stokes.cpp:13-45
  K_E2G_P_AWAY = 5,   // stokes_pressure_away              E2G/stokes.cpp:102-126
  K_E2G_SL7 = 6,      // stokes_SL_7ord                    E2G/stokes.cpp:53-97
  K_E2G_P7 = 7,       // stokes_pressure_7ord              E2G/stokes.cpp:134-203
  K_E2G_UP_AWAY = 8,  // stokes_SL_away + stokes_pressure_away at the same targets, one pass
  K_E2G_UP7 = 9,      // stokes_SL_7ord + stokes_pressure_7ord at the same targets, one pass
};

constexpr int kTB = 128;  // targets per target block = threads per CTA

// One unit of a target block's work: a treecode node evaluated either through
// its proxy points (type 0, "far", Call_Treecode_*) or by a direct sum over its
// member sources (type 1, "near", Call_Ds_*). mask bit t of word w selects
// target 32*w + t of the block.
struct Entry {
  int node;
  int type;
  uint32_t mask[4];
};

// A treecode over one surface, built on the host with the reference's
// splitting rule (2S/KITC.cpp:30-348). Sources are stored in tree order;
// perm[p] is the reference index of the source at tree position p.
struct Tree {
  int P = 6, N0 = 1000;
  double theta = 0.6, sq_theta = 0.36;
  int n = 0;
  std::vector<int> perm;
  std::vector<int> m0, m1;        // member range per node, inclusive, tree order
  std::vector<double> xc, yc, zc, mac;
  std::vector<double> box;        // 6 per node: x0,x1,y0,y1,z0,z1
  std::vector<int> child_start, child_count, children;
  std::vector<double> tcheb;      // 3*(P+1) per node: Chebyshev points in x, y, z
  int nnodes() const { return (int)m0.size(); }
};

// Builds the tree of n points (interleaved xyz) with root box
// ctr + [-1-1e-8, 1+1e-8]^3. direct=true builds a single node spanning all points.
Tree build_tree(int n, const double* xyz, const double ctr[3], int P, int N0, double theta,
                bool direct);

// Interaction lists of one (tree, target set) pair in target-block form.
struct Lists {
  std::vector<int> tord;        // target order -> target index
  std::vector<int> blk_start;   // nblocks+1 offsets into entries
  std::vector<Entry> entries;
  std::vector<double> blk_cost; // estimated pair work per block
  long long near_pairs_reg = 0; // pairs evaluated with the regularized kernel (near targets)
  long long near_pairs_plain = 0;
  long long proxy_pairs = 0;
  int nblocks() const { return (int)blk_start.size() - 1; }
};

// Per-target traversal exactly as eval_{SL,DL}_Sum_cluster(_onSurf)
// (2S/KITC.cpp:1066-1386): far if node.MAC < |x - node centre|^2, else a
// direct sum if (m1 - m0) < N0, else recurse into the children in order.
// near[t] (may be null) marks targets that take the regularized branch.
// morton (optional): the targets' morton_order, when the caller has it already.
Lists build_lists(const Tree& T, int nt, const double* txyz, const uint8_t* near,
                  const std::vector<int>* morton = nullptr);

// Density-interpolation stencils (2S/main.cpp:682-1046): for every target with
// nrst != 0, the 6x6 source indices (reference order; unset slots read 0) and
// the offsets p, q of x0 in grid units.
struct Stencils {
  std::vector<int> tgt;     // targets that interpolate
  std::vector<int> idx;     // 36 per entry: idx[36*e + 6*ii + jj] = stencil slot (ii, jj)
  std::vector<double> pq;   // 2 per entry
};
Stencils build_stencils(double h, const double ctr[3], int nq, const double* xq, int nt,
                        const int* nrst, const double* x0, const int* i123);

// Morton order of points (stable), used to form spatially coherent target blocks.
std::vector<int> morton_order(int n, const double* xyz);

}  // namespace hr
