// hr_tree.cpp — host-side planning for the treecode and the density
// interpolation. Geometry-only work, done once per scene:
//
//  * build_tree: the KITC cluster tree (2S/KITC.cpp:30-348, 780-804): root box
//    centre + [-1-1e-8, 1+1e-8]^3, octant split at the box midpoint while a
//    node holds >= N0 points, children kept in octant order, MAC = (half
//    diagonal)^2 / theta^2, Chebyshev points cos(i pi / P) mapped to each box.
//    The reference reorders particles with a swap/address-table loop whose
//    effect is a stable partition by octant; the same order is produced here
//    so that leaf membership and order match.
//  * build_lists: the per-target traversal of eval_*_Sum_cluster
//    (2S/KITC.cpp:1066-1386), regrouped into blocks of 128 spatially sorted
//    targets with a bit mask per (block, node) telling which targets take that
//    node as far field or as a direct leaf. The decision per target is the
//    reference's, evaluated in the same floating-point expression.
//  * build_stencils: the 6x6 stencil search of sixPoint_stencil
//    (2S/main.cpp:682-748, 969-1016), done by hashing grid-line coordinates
//    instead of scanning all quadrature points per target; candidates are
//    verified with the reference's own tolerance test and the last matching
//    index wins, as in the reference's sequential scan.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <unordered_map>

#include "../csrc/hr_engine.h"

namespace hr {

namespace {

struct Build {
  Tree* T;
  std::vector<double> x, y, z;  // in current (tree) order
  std::vector<int> perm;
  std::vector<std::vector<int>> kids;
};

int push_node(Build& B, int m0, int m1, const double box[6], double xc, double yc, double zc,
              double mac) {
  Tree& T = *B.T;
  T.m0.push_back(m0);
  T.m1.push_back(m1);
  for (int k = 0; k < 6; k++) T.box.push_back(box[k]);
  T.xc.push_back(xc);
  T.yc.push_back(yc);
  T.zc.push_back(zc);
  T.mac.push_back(mac);
  B.kids.emplace_back();
  return (int)T.m0.size() - 1;
}

void split(Build& B, int pi) {
  Tree& T = *B.T;
  const double x0 = T.box[6 * pi], x1 = T.box[6 * pi + 1], y0 = T.box[6 * pi + 2],
               y1 = T.box[6 * pi + 3], z0 = T.box[6 * pi + 4], z1 = T.box[6 * pi + 5];
  const double mx = (x0 + x1) / 2.0, my = (y0 + y1) / 2.0, mz = (z0 + z1) / 2.0;
  const double xc0 = (x0 + mx) / 2.0, xc1 = (x1 + mx) / 2.0;
  const double yc0 = (y0 + my) / 2.0, yc1 = (y1 + my) / 2.0;
  const double zc0 = (z0 + mz) / 2.0, zc1 = (z1 + mz) / 2.0;
  const int a = T.m0[pi], b = T.m1[pi];
  const int n = b - a + 1;
  std::vector<int> oct(n);
  int cnt[8] = {0};
  for (int i = 0; i < n; i++) {
    int p = a + i;
    int o = (B.x[p] > mx) + 2 * (B.y[p] > my) + 4 * (B.z[p] > mz);
    oct[i] = o;
    cnt[o]++;
  }
  int start[8];
  int s = 0;
  for (int o = 0; o < 8; o++) {
    start[o] = s;
    s += cnt[o];
  }
  {
    std::vector<double> tx(n), ty(n), tz(n);
    std::vector<int> tp(n);
    int pos[8];
    memcpy(pos, start, sizeof(pos));
    for (int i = 0; i < n; i++) {
      int d = pos[oct[i]]++;
      tx[d] = B.x[a + i];
      ty[d] = B.y[a + i];
      tz[d] = B.z[a + i];
      tp[d] = B.perm[a + i];
    }
    std::copy(tx.begin(), tx.end(), B.x.begin() + a);
    std::copy(ty.begin(), ty.end(), B.y.begin() + a);
    std::copy(tz.begin(), tz.end(), B.z.begin() + a);
    std::copy(tp.begin(), tp.end(), B.perm.begin() + a);
  }
  for (int o = 0; o < 8; o++) {
    if (cnt[o] == 0) continue;
    int bx = o & 1, by = (o >> 1) & 1, bz = (o >> 2) & 1;
    double box[6] = {bx ? mx : x0, bx ? x1 : mx, by ? my : y0,
                     by ? y1 : my, bz ? mz : z0, bz ? z1 : mz};
    double ex = bx ? (x1 - xc1) : (mx - xc0);
    double ey = by ? (y1 - yc1) : (my - yc0);
    double ez = bz ? (z1 - zc1) : (mz - zc0);
    double mac = (ex * ex + ey * ey + ez * ez) / T.sq_theta;
    int ci = push_node(B, a + start[o], a + start[o] + cnt[o] - 1, box, bx ? xc1 : xc0,
                       by ? yc1 : yc0, bz ? zc1 : zc0, mac);
    B.kids[pi].push_back(ci);
  }
}

void build_rec(Build& B, int pi) {
  Tree& T = *B.T;
  int n = T.m1[pi] - T.m0[pi] + 1;
  if (n >= T.N0) {
    split(B, pi);
    std::vector<int> ch = B.kids[pi];
    for (int c : ch) build_rec(B, c);
  }
}

}  // namespace

Tree build_tree(int n, const double* xyz, const double ctr[3], int P, int N0, double theta,
                bool direct) {
  Tree T;
  T.P = P;
  T.N0 = N0;
  T.theta = theta;
  T.sq_theta = theta * theta;
  T.n = n;
  Build B;
  B.T = &T;
  B.x.resize(n);
  B.y.resize(n);
  B.z.resize(n);
  B.perm.resize(n);
  for (int i = 0; i < n; i++) {
    B.x[i] = xyz[3 * i];
    B.y[i] = xyz[3 * i + 1];
    B.z[i] = xyz[3 * i + 2];
    B.perm[i] = i;
  }
  const double eps = 1.e-8;
  double box[6] = {-1.0 - eps + ctr[0], 1.0 + eps + ctr[0], -1.0 - eps + ctr[1],
                   1.0 + eps + ctr[1], -1.0 - eps + ctr[2], 1.0 + eps + ctr[2]};
  double xc = 0.5 * (box[0] + box[1]), yc = 0.5 * (box[2] + box[3]), zc = 0.5 * (box[4] + box[5]);
  // Direct mode: one node holding every source that is never taken as far field.
  push_node(B, 0, n - 1, box, xc, yc, zc,
            direct ? INFINITY : (3 * 10 * 10 / 4) / T.sq_theta);
  if (!direct && n > 0) build_rec(B, 0);
  T.perm = B.perm;
  // flatten children
  int nn = T.nnodes();
  T.child_start.resize(nn);
  T.child_count.resize(nn);
  for (int i = 0; i < nn; i++) {
    T.child_start[i] = (int)T.children.size();
    T.child_count[i] = (int)B.kids[i].size();
    for (int c : B.kids[i]) T.children.push_back(c);
  }
  // Chebyshev points (Cluster_Chev_Points, 2S/KITC.cpp:780-804)
  int P1 = P + 1;
  std::vector<double> t(P1);
  double hh = 3.14159265358979323846 / P;
  for (int i = 0; i < P1; i++) t[i] = cos(i * hh);
  T.tcheb.resize((size_t)3 * P1 * nn);
  for (int c = 0; c < nn; c++) {
    const double* bx = &T.box[6 * c];
    double* tc = &T.tcheb[(size_t)3 * P1 * c];
    for (int i = 0; i < P1; i++) {
      tc[i] = bx[0] + (t[i] + 1) / 2 * (bx[1] - bx[0]);
      tc[P1 + i] = bx[2] + (t[i] + 1) / 2 * (bx[3] - bx[2]);
      tc[2 * P1 + i] = bx[4] + (t[i] + 1) / 2 * (bx[5] - bx[4]);
    }
  }
  return T;
}

std::vector<int> morton_order(int n, const double* xyz) {
  std::vector<int> ord(n);
  std::iota(ord.begin(), ord.end(), 0);
  if (n <= 1) return ord;
  double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
  for (int i = 0; i < n; i++)
    for (int k = 0; k < 3; k++) {
      lo[k] = std::min(lo[k], xyz[3 * i + k]);
      hi[k] = std::max(hi[k], xyz[3 * i + k]);
    }
  double ext = std::max(hi[0] - lo[0], std::max(hi[1] - lo[1], hi[2] - lo[2]));
  if (!(ext > 0)) ext = 1.0;
  auto spread = [](uint64_t v) {
    v &= 0x1fffff;
    v = (v | v << 32) & 0x1f00000000ffffULL;
    v = (v | v << 16) & 0x1f0000ff0000ffULL;
    v = (v | v << 8) & 0x100f00f00f00f00fULL;
    v = (v | v << 4) & 0x10c30c30c30c30c3ULL;
    v = (v | v << 2) & 0x1249249249249249ULL;
    return v;
  };
  std::vector<uint64_t> code(n), code2(n);
#pragma omp parallel for schedule(static)
  for (int i = 0; i < n; i++) {
    uint64_t q[3];
    for (int k = 0; k < 3; k++) {
      double u = (xyz[3 * i + k] - lo[k]) / ext;
      u = std::min(std::max(u, 0.0), 1.0);
      q[k] = (uint64_t)(u * 2097151.0);
    }
    code[i] = spread(q[0]) | (spread(q[1]) << 1) | (spread(q[2]) << 2);
  }
  // stable LSD radix sort of the 63-bit codes, 11 bits per pass
  std::vector<int> ord2(n);
  for (int shift = 0; shift < 63; shift += 11) {
    int cnt[2049] = {0};
    for (int i = 0; i < n; i++) cnt[((code[i] >> shift) & 2047) + 1]++;
    for (int d = 0; d < 2048; d++) cnt[d + 1] += cnt[d];
    for (int i = 0; i < n; i++) {
      const int d = (int)((code[i] >> shift) & 2047);
      const int p = cnt[d]++;
      code2[p] = code[i];
      ord2[p] = ord[i];
    }
    code.swap(code2);
    ord.swap(ord2);
  }
  return ord;
}

Lists build_lists(const Tree& T, int nt, const double* txyz, const uint8_t* near,
                  const std::vector<int>* morton) {
  Lists L;
  L.tord = morton ? *morton : morton_order(nt, txyz);
  const int nb = (nt + kTB - 1) / kTB;
  const int nn = T.nnodes();
  const int P1 = T.P + 1;
  const long long Pf = (long long)P1 * P1 * P1;
  std::vector<std::vector<Entry>> per(nb);
  std::vector<double> cost(nb, 0.0);
  std::vector<long long> reg(nb, 0), plain(nb, 0), prox(nb, 0);
#pragma omp parallel
  {
    std::vector<int> slot(2 * (size_t)nn, -1);
    std::vector<int> touched;
    std::vector<std::vector<int>> keys(kTB);  // each target's entries, in traversal order
    std::vector<int> order(kTB), tsave(kTB);
    std::vector<double> tx(kTB), ty(kTB), tz(kTB);
    std::vector<uint8_t> treg(kTB);
    std::vector<std::vector<int>> sub(2, std::vector<int>(kTB));  // targets reaching a node, per depth
#pragma omp for schedule(dynamic, 4)
    for (int b = 0; b < nb; b++) {
      std::vector<Entry>& E = per[b];
      touched.clear();
      const int cnt_t = std::min(kTB, nt - b * kTB);
      // One depth-first traversal per block carries the block's targets that
      // reach each node. A node whose centre is farther from the block's
      // bounding box than its MAC radius is far for all of them, and one that
      // holds the whole box within it is far for none: rounding is monotone, so
      // every target's R_sq lies between the box's rounded extremes (a 1e-13
      // margin on top). Only the other nodes test targets one by one, with the
      // per-target expression. A target's keys come out in the per-target
      // traversal's order (children in order), so the lists are unchanged.
      double bmin[3] = {0, 0, 0}, bmax[3] = {0, 0, 0};
      for (int tt = 0; tt < cnt_t; tt++) {
        keys[tt].clear();
        const int t = L.tord[b * kTB + tt];
        tx[tt] = txyz[3 * t];
        ty[tt] = txyz[3 * t + 1];
        tz[tt] = txyz[3 * t + 2];
        treg[tt] = near ? near[t] != 0 : true;
        const double v[3] = {tx[tt], ty[tt], tz[tt]};
        for (int d = 0; d < 3; d++) {
          bmin[d] = tt == 0 ? v[d] : std::min(bmin[d], v[d]);
          bmax[d] = tt == 0 ? v[d] : std::max(bmax[d], v[d]);
        }
      }
      for (int tt = 0; tt < cnt_t; tt++) sub[0][tt] = tt;
      auto visit = [&](auto&& self, int c, int depth, int ns) -> void {
        const int* S = sub[depth].data();
        const double ctr[3] = {T.xc[c], T.yc[c], T.zc[c]};
        double lo[3], hi[3];
        for (int d = 0; d < 3; d++) {
          lo[d] = ctr[d] < bmin[d] ? bmin[d] - ctr[d] : (ctr[d] > bmax[d] ? ctr[d] - bmax[d] : 0.0);
          hi[d] = std::max(std::fabs(bmin[d] - ctr[d]), std::fabs(bmax[d] - ctr[d]));
        }
        const double dmin2 = lo[0] * lo[0] + lo[1] * lo[1] + lo[2] * lo[2];
        const double dmax2 = hi[0] * hi[0] + hi[1] * hi[1] + hi[2] * hi[2];
        const bool leaf = (T.m1[c] - T.m0[c]) < T.N0 || T.child_count[c] == 0;
        const long long cnt = T.m1[c] - T.m0[c] + 1;
        if (T.mac[c] < dmin2 * (1.0 - 1e-13)) {  // far for every target
          for (int e = 0; e < ns; e++) keys[S[e]].push_back(2 * c);
          prox[b] += Pf * ns;
          return;
        }
        int nr = ns;
        const int* Rr = S;
        if (!(T.mac[c] >= dmax2 * (1.0 + 1e-13))) {  // mixed: the per-target test
          if ((int)sub.size() <= depth + 1) sub.emplace_back(kTB);
          int* W = sub[depth + 1].data();
          nr = 0;
          for (int e = 0; e < ns; e++) {
            const int tt = S[e];
            double tpx = tx[tt] - T.xc[c], tpy = ty[tt] - T.yc[c], tpz = tz[tt] - T.zc[c];
            double R_sq = tpx * tpx + tpy * tpy + tpz * tpz;
            if (T.mac[c] < R_sq) {
              keys[tt].push_back(2 * c);
              prox[b] += Pf;
            } else {
              W[nr++] = tt;
            }
          }
          Rr = W;
          if (nr == 0) return;
        }
        if (leaf) {
          for (int e = 0; e < nr; e++) {
            keys[Rr[e]].push_back(2 * c + 1);
            if (treg[Rr[e]]) reg[b] += cnt;
            else plain[b] += cnt;
          }
          return;
        }
        const int nd = Rr == S ? depth : depth + 1;
        for (int q = 0; q < T.child_count[c]; q++) self(self, T.children[T.child_start[c] + q], nd, nr);
      };
      visit(visit, 0, 0, cnt_t);
      // Targets with the same (or a similar) interaction list take neighbouring
      // positions, so that a warp's 32 targets tend to share their entries and
      // warps skip more entries whole. A target's sums do not depend on its
      // position in the block.
      for (int tt = 0; tt < cnt_t; tt++) order[tt] = tt;
      std::stable_sort(order.begin(), order.begin() + cnt_t,
                       [&](int x, int y) { return keys[x] < keys[y]; });
      for (int tt = 0; tt < cnt_t; tt++) tsave[tt] = L.tord[b * kTB + tt];
      for (int pos = 0; pos < cnt_t; pos++) {
        const int tt = order[pos];
        L.tord[b * kTB + pos] = tsave[tt];
        for (int key : keys[tt]) {
          if (slot[key] < 0) {
            slot[key] = (int)E.size();
            touched.push_back(key);
            Entry e;
            e.node = key >> 1;
            e.type = key & 1;
            e.mask[0] = e.mask[1] = e.mask[2] = e.mask[3] = 0u;
            E.push_back(e);
          }
          E[slot[key]].mask[pos >> 5] |= 1u << (pos & 31);
        }
      }
      for (int key : touched) slot[key] = -1;
      std::sort(E.begin(), E.end(), [](const Entry& a, const Entry& b2) {
        return a.type != b2.type ? a.type < b2.type : a.node < b2.node;
      });
      double cst = 0.0;
      for (const Entry& e : E) {
        int warps = 0;
        for (int w = 0; w < 4; w++) warps += e.mask[w] != 0u;
        double per_warp = e.type == 0 ? (double)Pf * 40.0 : (double)(T.m1[e.node] - T.m0[e.node] + 1) * 90.0;
        cst += warps * per_warp;
      }
      cost[b] = cst;
    }
  }
  L.blk_start.resize(nb + 1);
  L.blk_start[0] = 0;
  for (int b = 0; b < nb; b++) L.blk_start[b + 1] = L.blk_start[b] + (int)per[b].size();
  L.entries.resize(L.blk_start[nb]);
  for (int b = 0; b < nb; b++)
    std::copy(per[b].begin(), per[b].end(), L.entries.begin() + L.blk_start[b]);
  L.blk_cost = cost;
  for (int b = 0; b < nb; b++) {
    L.near_pairs_reg += reg[b];
    L.near_pairs_plain += plain[b];
    L.proxy_pairs += prox[b];
  }
  return L;
}

Stencils build_stencils(double h, const double ctr[3], int nq, const double* xq, int nt,
                        const int* nrst, const double* x0, const int* i123) {
  Stencils S;
  // Grid-line candidates per orientation ind3 (the interpolation plane is
  // spanned by the two other axes, ind1 < ind2): quadrature points lying on
  // grid line (kx, ky) of that plane, on side z > 0 or z < 0, in a dense
  // (kx, ky, side) cell table in CSR form, ascending point index per cell.
  const int i1s[3] = {1, 0, 0}, i2s[3] = {2, 2, 1};  // by ind3 = 0, 1, 2
  struct Grid {
    long long kx0 = 0, ky0 = 0;
    long long nx = 0, ny = 0;
    std::vector<int> start, items;
    int cell(long long kx, long long ky, int side) const {
      if (kx < kx0 || ky < ky0 || kx >= kx0 + nx || ky >= ky0 + ny) return -1;
      return (int)((((kx - kx0) * ny) + (ky - ky0)) * 2 + side);
    }
  } G[3];
  // the three orientations' tables are independent
#pragma omp parallel for schedule(static, 1)
  for (int o = 0; o < 3; o++) {
    const int a1 = i1s[o], a2 = i2s[o];
    std::vector<long long> key(2 * (size_t)nq);
    std::vector<int> side(nq, -1);
    long long kxmin = 0, kxmax = -1, kymin = 0, kymax = -1;
    for (int j = 0; j < nq; j++) {
      const double X = xq[3 * j + a1], Y = xq[3 * j + a2];
      const double z = xq[3 * j + o] - ctr[o];
      if (!(z > 0) && !(z < 0)) continue;
      const long long kx = llround((X - ctr[a1]) / h), ky = llround((Y - ctr[a2]) / h);
      if (fabs(X - (kx * h + ctr[a1])) > 1e-11 || fabs(Y - (ky * h + ctr[a2])) > 1e-11) continue;
      key[2 * j] = kx;
      key[2 * j + 1] = ky;
      side[j] = z > 0 ? 1 : 0;
      if (kxmax < kxmin) {
        kxmin = kxmax = kx;
        kymin = kymax = ky;
      } else {
        kxmin = std::min(kxmin, kx);
        kxmax = std::max(kxmax, kx);
        kymin = std::min(kymin, ky);
        kymax = std::max(kymax, ky);
      }
    }
    Grid& g = G[o];
    g.kx0 = kxmin;
    g.ky0 = kymin;
    g.nx = kxmax - kxmin + 1;
    g.ny = kymax - kymin + 1;
    const size_t ncell = (size_t)std::max(0LL, g.nx * g.ny * 2);
    g.start.assign(ncell + 1, 0);
    for (int j = 0; j < nq; j++)
      if (side[j] >= 0) g.start[g.cell(key[2 * j], key[2 * j + 1], side[j]) + 1]++;
    for (size_t c = 0; c < ncell; c++) g.start[c + 1] += g.start[c];
    g.items.resize(g.start[ncell]);
    std::vector<int> fill(g.start.begin(), g.start.end() - 1);
    for (int j = 0; j < nq; j++)
      if (side[j] >= 0) g.items[fill[g.cell(key[2 * j], key[2 * j + 1], side[j])]++] = j;
  }
  std::vector<int> ent(nt, -1);
  int ne = 0;
  for (int i = 0; i < nt; i++)
    if (nrst[i] != 0) ent[i] = ne++;
  S.tgt.resize(ne);
  S.idx.assign(36 * (size_t)ne, 0);
  S.pq.resize(2 * (size_t)ne);
#pragma omp parallel for schedule(dynamic, 256)
  for (int i = 0; i < nt; i++) {
    const int e = ent[i];
    if (e < 0) continue;
    const double* X0 = &x0[3 * i];
    const int ind1 = i123[3 * i], ind2 = i123[3 * i + 1], ind3 = i123[3 * i + 2];
    const bool ok_plane = (ind3 >= 0 && ind3 < 3) && (ind1 == i1s[ind3] && ind2 == i2s[ind3]);
    double xLow = floor((X0[ind1] - ctr[ind1]) / h) * h + ctr[ind1];
    double yLow = floor((X0[ind2] - ctr[ind2]) / h) * h + ctr[ind2];
    double xHigh = xLow + h, yHigh = yLow + h;
    double z0 = X0[ind3] - ctr[ind3];
    const double tol = 1.e-14;
    double cx[6] = {xLow - 2.0 * h, xLow - h, xLow, xHigh, xHigh + h, xHigh + 2.0 * h};
    double cy[6] = {yLow - 2.0 * h, yLow - h, yLow, yHigh, yHigh + h, yHigh + 2.0 * h};
    int* st = &S.idx[36 * (size_t)e];
    if (ok_plane && (z0 > 0 || z0 < 0)) {
      const Grid& g = G[ind3];
      const int side = z0 > 0 ? 1 : 0;
      for (int a = 0; a < 6; a++)
        for (int bq = 0; bq < 6; bq++) {
          const long long kx = llround((cx[a] - ctr[ind1]) / h), ky = llround((cy[bq] - ctr[ind2]) / h);
          const int c = g.cell(kx, ky, side);
          if (c < 0) continue;
          int best = -1;
          for (int q = g.start[c]; q < g.start[c + 1]; q++) {
            const int j = g.items[q];
            double X = xq[3 * j + ind1], Y = xq[3 * j + ind2];
            // the reference's else-if chains: first matching column / row
            int col = -1, row = -1;
            for (int cc = 0; cc < 6; cc++)
              if (fabs(cx[cc] - X) < tol) {
                col = cc;
                break;
              }
            for (int r = 0; r < 6; r++)
              if (fabs(cy[r] - Y) < tol) {
                row = r;
                break;
              }
            if (col == a && row == bq) best = std::max(best, j);
          }
          if (best >= 0) st[6 * a + bq] = best;
        }
    }
    S.tgt[e] = i;
    S.pq[2 * (size_t)e] = (X0[ind1] - xLow) / h;
    S.pq[2 * (size_t)e + 1] = (X0[ind2] - yLow) / h;
  }
  return S;
}

}  // namespace hr
