// hr_runtime.cu — device trees, target lists, stencils and evaluation batches.
#include <algorithm>
#include <cstdint>
#include <cstring>
#include <mutex>
#include <numeric>

#include "hr_runtime.h"

namespace hr {

namespace {

// Freed blocks the pool keeps mapped before it returns memory to the CUDA driver.
constexpr uint64_t kPoolKeepBytes = 8ull << 30;
constexpr int kMaxDevices = 64;

struct DevPool {
  cudaMemPool_t pool = nullptr;
  cudaStream_t st = nullptr;  // the pool's own stream: allocations and frees only
};

std::mutex g_pool_mu;
DevPool g_pools[kMaxDevices];

DevPool& pool_of(int dev) {
  HR_REQUIRE(dev >= 0 && dev < kMaxDevices, "device index out of range");
  std::lock_guard<std::mutex> lk(g_pool_mu);
  DevPool& P = g_pools[dev];
  if (!P.pool) {
    cudaMemPoolProps props = {};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    HR_CHECK_CUDA(cudaMemPoolCreate(&P.pool, &props));
    uint64_t keep = kPoolKeepBytes;
    HR_CHECK_CUDA(cudaMemPoolSetAttribute(P.pool, cudaMemPoolAttrReleaseThreshold, &keep));
    HR_CHECK_CUDA(cudaStreamCreateWithFlags(&P.st, cudaStreamNonBlocking));
  }
  return P;
}

}  // namespace

void* dev_alloc(size_t bytes) {
  int dev = 0;
  HR_CHECK_CUDA(cudaGetDevice(&dev));
  DevPool& P = pool_of(dev);
  void* p = nullptr;
  HR_CHECK_CUDA(cudaMallocFromPoolAsync(&p, bytes, P.pool, P.st));
  // complete before any other stream sees the pointer
  HR_CHECK_CUDA(cudaStreamSynchronize(P.st));
  return p;
}

void dev_free(void* p) noexcept {
  if (!p) return;
  try {
    cudaPointerAttributes a{};
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess || a.type != cudaMemoryTypeDevice) return;
    int cur = 0;
    cudaGetDevice(&cur);
    if (a.device != cur) cudaSetDevice(a.device);
    cudaDeviceSynchronize();
    DevPool& P = pool_of(a.device);
    cudaFreeAsync(p, P.st);
    if (a.device != cur) cudaSetDevice(cur);
  } catch (...) {
  }
}

void d2h_staged(Ctx& C, void* dst, const void* src, size_t bytes) {
  cudaStream_t st = C.stream;
  if (bytes <= 2 * kPinChunk) {
    HR_CHECK_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, st));
    HR_CHECK_CUDA(cudaStreamSynchronize(st));
    return;
  }
  if (!C.pin) {
    HR_CHECK_CUDA(cudaMallocHost(&C.pin, 2 * kPinChunk));
    for (auto& e : C.pin_ev) HR_CHECK_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  }
  char* buf[2] = {static_cast<char*>(C.pin), static_cast<char*>(C.pin) + kPinChunk};
  const char* s = static_cast<const char*>(src);
  char* d = static_cast<char*>(dst);
  const size_t nch = (bytes + kPinChunk - 1) / kPinChunk;
  auto len = [&](size_t k) { return std::min(kPinChunk, bytes - k * kPinChunk); };
  auto enqueue = [&](size_t k) {
    HR_CHECK_CUDA(cudaMemcpyAsync(buf[k & 1], s + k * kPinChunk, len(k), cudaMemcpyDeviceToHost, st));
    HR_CHECK_CUDA(cudaEventRecord(C.pin_ev[k & 1], st));
  };
  enqueue(0);
  enqueue(1);
  constexpr size_t kPart = size_t(1) << 20;  // bytes per host thread's piece
  for (size_t k = 0; k < nch; k++) {
    HR_CHECK_CUDA(cudaEventSynchronize(C.pin_ev[k & 1]));
    const size_t n = len(k);
    char* out = d + k * kPinChunk;
    const char* in = buf[k & 1];
    const long nparts = (long)((n + kPart - 1) / kPart);
#pragma omp parallel for schedule(static)
    for (long q = 0; q < nparts; q++) {
      const size_t o = (size_t)q * kPart;
      std::memcpy(out + o, in + o, std::min(kPart, n - o));
    }
    if (k + 2 < nch) enqueue(k + 2);
  }
}

void DevTree::build(const hr_surface& S, int P, int N0, double theta, bool direct,
                    cudaStream_t st) {
  HR_REQUIRE(S.n >= 0 && (S.n == 0 || (S.xyz && S.nrml && S.area)), "surface arrays missing");
  HR_REQUIRE(P >= 1 && P + 1 <= 16, "treecode degree P must be in [1, 15]");
  HR_REQUIRE(N0 >= 1, "leaf size N0 must be >= 1");
  host = build_tree(S.n, S.xyz, S.center, P, N0, theta, direct);
  n = S.n;
  nn = host.nnodes();
  P1 = P + 1;
  Pf = P1 * P1 * P1;
  std::vector<double> hx(n), hy(n), hz(n), hnx(n), hny(n), hnz(n), ha(n);
  for (int p = 0; p < n; p++) {
    int o = host.perm[p];
    hx[p] = S.xyz[3 * o];
    hy[p] = S.xyz[3 * o + 1];
    hz[p] = S.xyz[3 * o + 2];
    hnx[p] = S.nrml[3 * o];
    hny[p] = S.nrml[3 * o + 1];
    hnz[p] = S.nrml[3 * o + 2];
    ha[p] = S.area[o];
  }
  x.upload(hx, st);
  y.upload(hy, st);
  z.upload(hz, st);
  nx.upload(hnx, st);
  ny.upload(hny, st);
  nz.upload(hnz, st);
  a.upload(ha, st);
  perm.upload(host.perm, st);
  m0.upload(host.m0, st);
  m1.upload(host.m1, st);
  tcheb.upload(host.tcheb, st);
  qx.alloc(n);
  qy.alloc(n);
  qz.alloc(n);
  for (int k = 0; k < 3; k++) ctr[k] = S.center[k];
  {
    std::vector<float> a0(n), a1(n), a2(n), b0(n), b1(n), b2(n), c0(n);
    for (int p = 0; p < n; p++) {
      a0[p] = (float)(hx[p] - ctr[0]);
      a1[p] = (float)(hy[p] - ctr[1]);
      a2[p] = (float)(hz[p] - ctr[2]);
      b0[p] = (float)hnx[p];
      b1[p] = (float)hny[p];
      b2[p] = (float)hnz[p];
      c0[p] = (float)ha[p];
    }
    fx.upload(a0, st);
    fy.upload(a1, st);
    fz.upload(a2, st);
    fnx.upload(b0, st);
    fny.upload(b1, st);
    fnz.upload(b2, st);
    fa.upload(c0, st);
    fqx.alloc(n);
    fqy.alloc(n);
    fqz.alloc(n);
  }
  // upward-pass items: every non-root node (the root's moments stay zero, as
  // in the reference, which skips it: 2S/KITC.cpp:1446), in chunks of sources.
  // Chunks of at most 512 sources, smaller when the tree is small so that the
  // items fill about four CTAs per SM (a multiple of the 32-source K tile).
  std::vector<MomItem> it;
  std::vector<int> start(nn + 1, 0);
  long long members = 0;
  for (int c = 1; c < nn; c++) members += host.m1[c] - host.m0[c] + 1;
  int sms = 148, dev = 0;
  if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const long long want = (members + 4LL * sms - 1) / (4LL * sms);
  const int chunk = (int)std::min(512LL, std::max(64LL, (want + 31) / 32 * 32));
  moment_terms = 0;
  for (int c = 0; c < nn; c++) {
    start[c] = (int)it.size();
    if (c == 0 || direct) continue;
    for (int s = host.m0[c]; s <= host.m1[c]; s += chunk) {
      MomItem m;
      m.node = c;
      m.s0 = s;
      m.s1 = std::min(host.m1[c] + 1, s + chunk);
      m.out = (int)it.size();
      it.push_back(m);
    }
    moment_terms += (long long)Pf * (host.m1[c] - host.m0[c] + 1);
  }
  start[nn] = (int)it.size();
  nitems = (int)it.size();
  items.upload(it, st);
  item_start.upload(start, st);
  partial.alloc((size_t)std::max(1, nitems) * 12 * Pf);
  mom.alloc((size_t)nn * 12 * Pf);
  mom.zero(st);
  momf.alloc((size_t)nn * 12 * Pf);
  momf.zero(st);
}

void Ctx::check_tc() {
  if (!tc_err.p) return;
  int e = 0;
  HR_CHECK_CUDA(cudaMemcpyAsync(&e, tc_err.p, sizeof(int), cudaMemcpyDeviceToHost, stream));
  HR_CHECK_CUDA(cudaStreamSynchronize(stream));
  if (e) {
    tc_err.zero(stream);
    throw Error(HR_ERR_CUDA, "a tensor-core upward pass gave up waiting for its MMAs (bounded wait ran out)");
  }
}

void DevTree::set_density(Ctx& C, const double* q3_dev, bool dl, bool moments, bool tc) {
  launch_permute(n, perm.p, q3_dev, qx.p, qy.p, qz.p, fqx.p, fqy.p, fqz.p, C.stream);
  C.launches++;
  if (moments && nitems > 0 && tc && moments_tc_supported(P1)) {
    if (!C.tc_err.p) {
      C.tc_err.alloc(1);
      C.tc_err.zero(C.stream);
    }
    launch_moments_tc(dl ? 1 : 0, items.p, nitems, P1, tcheb.p, x.p, y.p, z.p, nx.p, ny.p, nz.p, a.p, qx.p, qy.p,
                      qz.p, partial.p, C.tc_err.p, C.stream);
    launch_moments_reduce(dl ? 12 : 6, Pf, nn, item_start.p, partial.p, mom.p, momf.p, C.stream);
    C.launches += 2;
  } else if (moments && nitems > 0) {
    launch_moments(dl ? 1 : 0, items.p, nitems, P1, tcheb.p, x.p, y.p, z.p, nx.p, ny.p, nz.p, a.p,
                   qx.p, qy.p, qz.p, partial.p, C.stream);
    launch_moments_reduce(dl ? 12 : 6, Pf, nn, item_start.p, partial.p, mom.p, momf.p, C.stream);
    C.launches += 2;
  }
}

void DevLists::build(const Tree& T, int nt, const double* txyz, const uint8_t* near,
                     cudaStream_t st, const std::vector<int>* morton) {
  host = build_lists(T, nt, txyz, near, morton);
  tord.upload(host.tord, st);
  blk_start.upload(host.blk_start, st);
  entries.upload(host.entries, st);
}

void DevStencils::build(const Stencils& S, cudaStream_t st) {
  ne = (int)S.tgt.size();
  tgt.upload(S.tgt, st);
  idx.upload(S.idx, st);
  pq.upload(S.pq, st);
}

EvalTask make_task(int kind, double DEL, double scale, const DevTree& T, const DevLists& L,
                   const DevTargets& tg, double* out) {
  EvalTask k;
  memset(&k, 0, sizeof(k));
  k.kind = kind;
  k.jump_mode = 0;
  k.P1 = T.P1;
  k.Pf = T.Pf;
  k.C = (kind == K_DL_ON || kind == K_DL_OFF) ? 10 : 6;
  k.nt = tg.n;
  k.mixed = 0;
  k.DEL = DEL;
  k.scale = scale;
  k.sx = T.x.p;
  k.sy = T.y.p;
  k.sz = T.z.p;
  k.snx = T.nx.p;
  k.sny = T.ny.p;
  k.snz = T.nz.p;
  k.sa = T.a.p;
  k.qx = T.qx.p;
  k.qy = T.qy.p;
  k.qz = T.qz.p;
  for (int c = 0; c < 3; c++) k.ctr[c] = T.ctr[c];
  k.fx = T.fx.p;
  k.fy = T.fy.p;
  k.fz = T.fz.p;
  k.fnx = T.fnx.p;
  k.fny = T.fny.p;
  k.fnz = T.fnz.p;
  k.fa = T.fa.p;
  k.fqx = T.fqx.p;
  k.fqy = T.fqy.p;
  k.fqz = T.fqz.p;
  k.node_m0 = T.m0.p;
  k.node_m1 = T.m1.p;
  k.tcheb = T.tcheb.p;
  k.mom = T.mom.p;
  k.momf = T.momf.p;
  k.tord = L.tord.p;
  k.txyz = tg.xyz.p;
  k.tb = tg.b.p;
  k.tnear = tg.near.p;
  k.tf0 = tg.f0.p;
  k.tx0 = tg.x0.p;
  k.tn0 = tg.n0.p;
  k.tg0 = tg.g0.p;
  k.tq = nullptr;
  k.tnrm = tg.nrm.p;
  k.out = out;
  k.entries = L.entries.p;
  k.blk_start = L.blk_start.p;
  k.counters = nullptr;
  return k;
}

void Batch::finalize(cudaStream_t st, int num_sms) {
  // 1. segments: a far entry whole, a near entry cut into source ranges of
  //    at most kSegSrc; cost ~ active warps x pair evaluations.
  constexpr int kSegSrc = 512;
  struct HSeg {
    Seg s;
    double cost;
  };
  std::vector<std::vector<std::vector<HSeg>>> per(tasks.size());
  double total = 0.0;
  for (size_t t = 0; t < tasks.size(); t++) {
    const Lists& L = *lists[t];
    const Tree& T = *trees[t];
    const int P1 = T.P + 1;
    const double Pf = (double)P1 * P1 * P1;
    per[t].resize(L.nblocks());
    // blocks are independent; every cost is a multiple of 1/2 far below 2^52,
    // so the sum is exact (and the item size the same) in any order
#pragma omp parallel for schedule(dynamic, 16) reduction(+ : total)
    for (int b = 0; b < L.nblocks(); b++) {
      for (int e = L.blk_start[b]; e < L.blk_start[b + 1]; e++) {
        const Entry& E = L.entries[e];
        int warps = 0;
        for (int w = 0; w < 4; w++) warps += E.mask[w] != 0u;
        if (E.type == 0) {
          double c = warps * Pf * 1.5;
          per[t][b].push_back({Seg{e, 0, 0}, c});
          total += c;
        } else {
          for (int s0 = T.m0[E.node]; s0 <= T.m1[E.node]; s0 += kSegSrc) {
            int s1 = std::min(T.m1[E.node] + 1, s0 + kSegSrc);
            double c = warps * (double)(s1 - s0) * 2.0;
            per[t][b].push_back({Seg{e, s0, s1}, c});
            total += c;
          }
        }
      }
    }
  }
  // 2. items: runs of consecutive segments of one block, each about
  //    total / (SMs x 4 resident CTAs x 16 waves), never below two tiles;
  //    small items keep the tail short where the cost estimate is off.
  const double target = std::max(total / (num_sms * 4.0 * 16.0), 2.0 * 256.0 * 2.0);
  // Blocks in task order; each block's runs are formed on its own (in
  // parallel), then offsets give every segment and item (slot) the position
  // a serial pass over the blocks would give it.
  std::vector<int2> tblocks;
  for (size_t t = 0; t < tasks.size(); t++)
    for (int b = 0; b < (int)per[t].size(); b++) tblocks.push_back(make_int2((int)t, b));
  const long nbt = (long)tblocks.size();
  std::vector<std::vector<std::pair<int, double>>> runs(nbt);  // per block: (segments, cost) per item
#pragma omp parallel for schedule(dynamic, 64)
  for (long q = 0; q < nbt; q++) {
    const auto& v = per[tblocks[q].x][tblocks[q].y];
    size_t i = 0;
    while (i < v.size()) {
      double c = 0.0;
      int n = 0;
      do {
        c += v[i].cost;
        i++;
        n++;
      } while (i < v.size() && c + v[i].cost <= target);
      runs[q].push_back({n, c});
    }
    // a block without work still gets one (empty) item so that its partial
    // slot is written
    if (v.empty()) runs[q].push_back({0, 0.0});
  }
  std::vector<long> seg_off(nbt + 1, 0), slot_off(nbt + 1, 0);
  for (long q = 0; q < nbt; q++) {
    seg_off[q + 1] = seg_off[q] + (long)per[tblocks[q].x][tblocks[q].y].size();
    slot_off[q + 1] = slot_off[q] + (long)runs[q].size();
  }
  HR_REQUIRE(seg_off[nbt] < (1L << 31) && slot_off[nbt] < (1L << 31), "batch too large for 32-bit segment indices");
  std::vector<Seg> segs(seg_off[nbt]);
  std::vector<std::pair<double, BlockRef>> items(slot_off[nbt]);
#pragma omp parallel for schedule(dynamic, 64)
  for (long q = 0; q < nbt; q++) {
    const int t = tblocks[q].x, b = tblocks[q].y;
    const auto& v = per[t][b];
    int sg = (int)seg_off[q], it = (int)slot_off[q];
    size_t i = 0;
    for (const auto& r : runs[q]) {
      BlockRef ref{t, b, sg, sg + r.first, it};
      for (int k = 0; k < r.first; k++) segs[sg++] = v[i++].s;
      items[it++] = {r.second, ref};
    }
  }
  // per task: the slot of each block's first item, then the task's end
  std::vector<int> starts;
  std::vector<size_t> start_off(tasks.size());
  int slot = (int)slot_off[nbt];
  {
    long q = 0;
    for (size_t t = 0; t < tasks.size(); t++) {
      start_off[t] = starts.size();
      for (int b = 0; b < (int)per[t].size(); b++, q++) starts.push_back((int)slot_off[q]);
      starts.push_back((int)slot_off[q]);
    }
  }
  // lean items first (their own launch: on-surface kinds, or the extend-to-grid
  // box-face sums), each part by decreasing cost
  auto on_kind = [&](const BlockRef& r) {
    const int k = tasks[r.task].kind;
    return family == F_E2G ? (k == K_E2G_SL_AWAY || k == K_E2G_P_AWAY || k == K_E2G_UP_AWAY)
                           : (k == K_SL_ON || k == K_DL_ON);
  };
  std::stable_sort(items.begin(), items.end(),
                   [&](const std::pair<double, BlockRef>& a, const std::pair<double, BlockRef>& b) {
                     const bool oa = on_kind(a.second), ob = on_kind(b.second);
                     if (oa != ob) return oa;
                     return a.first > b.first;
                   });
  std::vector<BlockRef> br(items.size());
  n_on = 0;
  for (size_t i = 0; i < items.size(); i++) {
    br[i] = items[i].second;
    n_on += on_kind(br[i]) ? 1 : 0;
  }
  nitems = (int)br.size();
  ntask_blocks = (int)tblocks.size();
  d_items.upload(br, st);
  d_segs.upload(segs, st);
  d_item_start.upload(starts, st);
  d_task_blocks.upload(tblocks, st);
  d_partial.alloc((size_t)std::max(1, slot) * kTB * kPartComps);
  for (size_t t = 0; t < tasks.size(); t++) {
    tasks[t].item_start = d_item_start.p + start_off[t];
    tasks[t].partial = d_partial.p;
  }
  d_tasks.upload(tasks, st);
  ready = true;
}

void Batch::launch(Ctx& C) {
  launch_eval(family, d_tasks.p, d_items.p, d_segs.p, nitems, n_on, ntask_blocks, d_task_blocks.p,
              C.stream, C.side, C.ev_fork, C.ev_join, !tasks.empty() && tasks[0].mixed, C.count_work);
  C.launches += 1 + (n_on > 0 ? 1 : 0) + (nitems > n_on ? 1 : 0);
}

}  // namespace hr
