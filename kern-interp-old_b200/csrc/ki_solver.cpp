// Host orchestration of the B200 recursive-skeletonization solver.
//
// factor() follows SkelFactorization::skeletonize (skel_factorization.cpp:
// 94-243) level by level from the leaves up: the host refreshes the active
// and near dof lists of the level (quadtree.cpp:656-720) and builds one
// device work descriptor per box, then one launch runs every box's
// interpolative decomposition and one launch decouples every compressed box.
// The ranks and pivots come back to the host (a few KB per level) because
// the next level's active lists are made of this level's skeletons; the
// next level's IDs are launched before this level's decoupling is prepared,
// so that host bookkeeping overlaps GPU work.  With holes, the border
// columns are swept up each level as soon as it is decoupled.  The top
// skeleton matrix (or, with holes, the bordered system S of
// skel_factorization.cpp:130-242) is assembled and LU-factored on the GPU.
// solve_device() runs the level sweeps of SkelFactorization::solve and
// multiply_connected_solve (skel_factorization.cpp:341-551) on the GPU.
#include "ki_solver.h"

#include "ki_pool.h"

#include <algorithm>
#include <array>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>

namespace kib {

// ------------------------------------------------------------------ memory
namespace chunk_pool {
namespace {
std::mutex g_mu;
std::multimap<size_t, void*> g_free[2];  // [0] device, [1] pinned host
size_t g_cached = 0;
}  // namespace

void* get(size_t bytes, bool pinned, size_t* got) {
  {
    std::lock_guard<std::mutex> lock(g_mu);
    auto& fl = g_free[pinned ? 1 : 0];
    auto it = fl.lower_bound(bytes);
    if (it != fl.end() && it->first <= 4 * bytes + (64u << 20)) {
      void* p = it->second;
      *got = it->first;
      g_cached -= it->first;
      fl.erase(it);
      return p;
    }
  }
  void* p = nullptr;
  const cudaError_t e = pinned ? cudaHostAlloc(&p, bytes, cudaHostAllocDefault)
                               : cudaMalloc(&p, bytes);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  *got = bytes;
  return p;
}

void put(void* p, size_t bytes, bool pinned) {
  std::lock_guard<std::mutex> lock(g_mu);
  g_free[pinned ? 1 : 0].emplace(bytes, p);
  g_cached += bytes;
}

void release_all() {
  std::lock_guard<std::mutex> lock(g_mu);
  for (auto& kv : g_free[0]) cudaFree(kv.second);
  for (auto& kv : g_free[1]) cudaFreeHost(kv.second);
  g_free[0].clear();
  g_free[1].clear();
  g_cached = 0;
}

size_t cached_bytes() {
  std::lock_guard<std::mutex> lock(g_mu);
  return g_cached;
}
}  // namespace chunk_pool

Arena::~Arena() {
  for (auto& c : chunks_) chunk_pool::put(c.first, c.second, pinned_);
}

void* Arena::alloc(size_t bytes) {
  bytes = (bytes + 255) & ~static_cast<size_t>(255);
  if (bytes > left_) {
    const size_t want = std::max(bytes, static_cast<size_t>(pinned_ ? 16 : 64) << 20);
    size_t sz = 0;
    void* p = chunk_pool::get(want, pinned_, &sz);
    if (!p) return nullptr;
    chunks_.push_back({p, sz});
    cur_ = static_cast<char*>(p);
    left_ = sz;
    reserved_ += sz;
  }
  void* r = cur_;
  cur_ += bytes;
  left_ -= bytes;
  used_ += bytes;
  return r;
}

Scratch::~Scratch() {
  if (p) chunk_pool::put(p, bytes, false);
  for (const auto& r : retired) chunk_pool::put(r.first, r.second, false);
}

cudaError_t Scratch::reserve(size_t want, cudaStream_t s, bool retire) {
  if (want <= bytes) return cudaSuccess;
  if (retire) {
    if (p) retired.emplace_back(p, bytes);
  } else {
    cudaError_t e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return e;
    if (p) chunk_pool::put(p, bytes, false);
  }
  p = nullptr;
  bytes = 0;
  size_t got = 0;
  p = chunk_pool::get(want + want / 4 + 4096, false, &got);
  if (!p) return cudaErrorMemoryAllocation;
  bytes = got;
  return cudaSuccess;
}

namespace {

double g_upload_ms = 0;  // accumulated by upload() (single host thread per solver)

double now_ms() {
  return std::chrono::duration<double, std::milli>(
             std::chrono::steady_clock::now().time_since_epoch()).count();
}

// Streaming launches: CTAs per box by matrix size.
int pick_stream_group(long long m, long long n) {
  const long long e = m * n;
  if (e > 400000) return 8;
  if (e > 160000) return 4;
  if (e > 90000) return 2;
  return 1;
}

// Smallest cluster whose shared memory holds the whole m x n matrix (group
// code kOnChip + G), else a streaming launch.  onchip_ok[G] says whether a
// G-CTA cluster with full shared memory can be scheduled on this device.
int pick_group(int m, int n, const bool* onchip_ok) {
  const long long lda = onchip_lda(m);
  for (int G = 1; G <= 16; G *= 2) {
    if (!onchip_ok[G]) continue;
    const long long cols = (n + G - 1) / G * lda;
    if (id_smem_bytes(m, n) + sizeof(double) * cols <= 227 * 1024) return kOnChip + G;
  }
  return pick_stream_group(m, n);
}

}  // namespace

// ------------------------------------------------------------------ solver
template <class T>
int Solver::upload(T* dst, const std::vector<T>& src, cudaStream_t s) {
  if (src.empty()) return 0;
  const double t0 = now_ms();
  const size_t bytes = sizeof(T) * src.size();
  void* st = stage_.alloc(bytes);
  if (!st) return fail("pinned staging allocation failed");
  std::memcpy(st, src.data(), bytes);
  const int rc = cuda_check(cudaMemcpyAsync(dst, st, bytes, cudaMemcpyHostToDevice, s),
                            "cudaMemcpyAsync (upload)");
  g_upload_ms += now_ms() - t0;
  return rc;
}

// members in other files upload these types
template int Solver::upload<int>(int*, const std::vector<int>&, cudaStream_t);
template int Solver::upload<double>(double*, const std::vector<double>&, cudaStream_t);
template int Solver::upload<MvTile>(MvTile*, const std::vector<MvTile>&, cudaStream_t);

Solver::Solver(const SolverOptions& opt, int n_points, const double* points,
               const double* normals, const double* curvatures, const double* weights,
               int n_holes, const double* holes, cudaStream_t stream)
    : opt_(opt), stream_(stream) {
  sd_ = opt.pde == kStokes ? 2 : 1;
  n_points_ = n_points;
  n_dofs_ = n_points * sd_;
  pts_.assign(points, points + 2 * static_cast<size_t>(n_points));
  nrm_.assign(normals, normals + 2 * static_cast<size_t>(n_points));
  curv_.assign(curvatures, curvatures + n_points);
  wts_.assign(weights, weights + n_points);
  if (n_holes > 0) holes_.assign(holes, holes + 4 * static_cast<size_t>(n_holes));
}

namespace {
// Side streams and their events, kept for reuse by later solvers on the
// same device (creating and destroying them costs more host time than a
// small factorization's level loop).
struct AuxSet {
  int dev = -1;
  cudaStream_t d = nullptr;
  cudaEvent_t ev_id[2] = {}, ev_dec = nullptr, fork = nullptr;
  cudaStream_t id[3] = {};
  cudaEvent_t join[3] = {};
  cudaStream_t dl[3] = {};
  cudaEvent_t dl_fork = nullptr, dl_join[3] = {};
  cudaStream_t b = nullptr;
  cudaEvent_t ev_lvl = nullptr, ev_bdr = nullptr;
  cudaStream_t u = nullptr;
  cudaEvent_t ev_up = nullptr;
};
std::mutex g_aux_mu;
std::vector<AuxSet>& aux_free() {
  static std::vector<AuxSet> v;
  return v;
}
}  // namespace

namespace {
// One finished single-tree solver's host quadtree, kept for the next
// single-tree solver of the process: the next build reuses its boxes' list
// capacities, so neither the finished solver's close nor the next build
// frees or allocates the thousands of small lists a tree holds.  (A forest
// is laid out from per-problem trees and would only free the kept one.)
std::mutex g_tree_mu;
std::unique_ptr<QuadTreeHost>& tree_slot() {
  static std::unique_ptr<QuadTreeHost> slot;
  return slot;
}
}  // namespace

Solver::~Solver() {
  {
    std::lock_guard<std::mutex> lk(g_tree_mu);
    if (!tree_slot() && starts_.size() <= 2) tree_slot().reset(new QuadTreeHost(std::move(tree)));
  }
  // chunks go back to the pool only once no queued work can touch them
  cudaStreamSynchronize(stream_);
  if (solve_exec_) cudaGraphExecDestroy(solve_exec_);
  if (dstream_) cudaStreamSynchronize(dstream_);
  for (int i = 0; i < kIdStreams; i++)
    if (id_streams_[i]) cudaStreamSynchronize(id_streams_[i]);
  for (int i = 0; i < kDecStreams; i++)
    if (dl_streams_[i]) cudaStreamSynchronize(dl_streams_[i]);
  if (bstream_) cudaStreamSynchronize(bstream_);
  if (ustream_) cudaStreamSynchronize(ustream_);
  if (dstream_) {
    static_assert(kIdStreams == 3 && kDecStreams == 3, "AuxSet holds three of each");
    AuxSet a;
    cudaGetDevice(&a.dev);
    a.d = dstream_;
    a.ev_id[0] = ev_id_[0];
    a.ev_id[1] = ev_id_[1];
    a.ev_dec = ev_dec_;
    a.fork = id_fork_;
    for (int i = 0; i < kIdStreams; i++) {
      a.id[i] = id_streams_[i];
      a.join[i] = id_join_[i];
    }
    a.dl_fork = dl_fork_;
    for (int i = 0; i < kDecStreams; i++) {
      a.dl[i] = dl_streams_[i];
      a.dl_join[i] = dl_join_[i];
    }
    a.b = bstream_;
    a.ev_lvl = ev_lvl_;
    a.ev_bdr = ev_bdr_;
    a.u = ustream_;
    a.ev_up = ev_up_;
    std::lock_guard<std::mutex> lk(g_aux_mu);
    aux_free().push_back(a);
  }
}

namespace {
// Timing events, reused across timed factorizations (creating two events per
// launch cost more host time than the launches of a small level).
std::mutex g_ev_mu;
std::vector<cudaEvent_t>& ev_free() {
  static std::vector<cudaEvent_t> v;
  return v;
}
cudaError_t ev_get(cudaEvent_t* e) {
  {
    std::lock_guard<std::mutex> lk(g_ev_mu);
    if (!ev_free().empty()) {
      *e = ev_free().back();
      ev_free().pop_back();
      return cudaSuccess;
    }
  }
  return cudaEventCreate(e);
}
void ev_put(cudaEvent_t e) {
  std::lock_guard<std::mutex> lk(g_ev_mu);
  ev_free().push_back(e);
}
}  // namespace

int Solver::timer_begin(cudaEvent_t* e0, cudaStream_t s) {
  if (cuda_check(ev_get(e0), "cudaEventCreate")) return -2;
  return cuda_check(cudaEventRecord(*e0, s ? s : stream_), "cudaEventRecord");
}

int Solver::timer_end(cudaEvent_t e0, const LaunchRecord& rec, cudaStream_t s) {
  cudaEvent_t e1;
  if (cuda_check(ev_get(&e1), "cudaEventCreate")) return -2;
  if (cuda_check(cudaEventRecord(e1, s ? s : stream_), "cudaEventRecord")) return -2;
  pending_.push_back({e0, e1, rec});
  return 0;
}

void Solver::mark(int code, int level) {
  if (time_phases) host_marks.push_back(HostMark{code, level, now_ms() - host_start_});
}

int Solver::timers_resolve() {
  for (PendingTimer& p : pending_) {
    float ms = 0, a = 0, b = 0;
    if (cuda_check(cudaEventElapsedTime(&ms, p.e0, p.e1), "cudaEventElapsedTime")) return -2;
    LaunchRecord r = p.rec;
    r.ms = ms;
    if (ev_start_) {
      if (cuda_check(cudaEventElapsedTime(&a, ev_start_, p.e0), "cudaEventElapsedTime")) return -2;
      if (cuda_check(cudaEventElapsedTime(&b, ev_start_, p.e1), "cudaEventElapsedTime")) return -2;
      r.t0 = a;
      r.t1 = b;
    }
    if (r.kind == 0) {
      t_id_ms += ms;
      id_launches++;
    } else if (r.kind == 1) {
      t_decouple_ms += ms;
    } else if (r.kind == 2) {
      t_top_ms += ms;
    }
    launch_log.push_back(r);
    ev_put(p.e0);
    ev_put(p.e1);
  }
  pending_.clear();
  return 0;
}

int Solver::fail(const std::string& msg) {
  error = msg;
  return -1;
}

int Solver::cuda_check(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return 0;
  error = std::string(what) + ": " + cudaGetErrorString(e);
  return -2;
}

std::vector<BoxBlock> Solver::blocks_of(int box) const {
  // Accumulated updates inside the box's current dof list: its own skeleton
  // update when compressed, else its children's lists laid end to end.
  const Box& b = tree.boxes[box];
  if (b.compressed) return {BoxBlock{boxdev_[box].acc, b.rank, 0}};
  std::vector<BoxBlock> out;
  if (b.leaf) return out;
  int off = 0;
  for (int q = 0; q < 4; q++) {
    const int c = b.child[q];
    for (const BoxBlock& x : blocks_of(c)) out.push_back(BoxBlock{x.acc, x.size, x.pos + off});
    const Box& cb = tree.boxes[c];
    off += static_cast<int>(cb.compressed ? cb.skel.size() : cb.active.size());
  }
  return out;
}

void Solver::build_block_map(const std::vector<BoxBlock>& blocks, int n, std::vector<int>* bid,
                             std::vector<int>* bpos, std::vector<UpdBlock>* tab) const {
  const int base = static_cast<int>(tab->size());
  const size_t b0 = bid->size();
  bid->resize(b0 + n, -1);
  bpos->resize(b0 + n, 0);
  for (size_t q = 0; q < blocks.size(); q++) {
    tab->push_back(UpdBlock{blocks[q].acc, blocks[q].size, 0});
    for (int t = 0; t < blocks[q].size; t++) {
      (*bid)[b0 + blocks[q].pos + t] = static_cast<int>(q);
      (*bpos)[b0 + blocks[q].pos + t] = t;
    }
  }
  (void)base;
}

void Solver::build_tree_only() {
  if (starts_.size() > 1)
    tree.build_forest(pts_.data(), n_points_, sd_, opt_.max_leaf_dofs, starts_);
  else
    tree.build(pts_.data(), n_points_, sd_, opt_.max_leaf_dofs);
  for (int level = static_cast<int>(tree.levels.size()) - 1; level >= 0; level--)
    tree.refresh_level(level, nullptr);
  allskel.clear();
  for (int r : tree.roots)
    allskel.insert(allskel.end(), tree.boxes[r].active.begin(), tree.boxes[r].active.end());
}

void Solver::perturb_tree_only(int n_points, const double* points) {
  const std::vector<double> old = pts_;
  const int n_old = n_points_;
  n_points_ = n_points;
  n_dofs_ = n_points * sd_;
  pts_.assign(points, points + 2 * static_cast<size_t>(n_points));
  nrm_.assign(2 * static_cast<size_t>(n_points), 0.0);
  curv_.assign(n_points, 0.0);
  wts_.assign(n_points, 0.0);
  tree.perturb(old.data(), n_old, pts_.data(), n_points_);
  for (int level = static_cast<int>(tree.levels.size()) - 1; level >= 0; level--)
    tree.refresh_level(level, nullptr);
  allskel.clear();
  for (int r : tree.roots)
    allskel.insert(allskel.end(), tree.boxes[r].active.begin(), tree.boxes[r].active.end());
}

int Solver::begin_factor(cudaEvent_t* ev0) {
  KI_CUDA(ev_get(ev0));
  KI_CUDA(cudaEventRecord(*ev0, stream_));
  host_start_ = now_ms();
  geom_ready_ = false;
  ev_start_ = *ev0;
  host_marks.clear();
  t_id_ms = t_decouple_ms = t_top_ms = 0;
  id_launches = 0;
  id_flops = id_bytes = id_onchip_flops = 0;
  rank_hint_ = -1;
  dec_flops = top_flops = solve_bytes = 0;

  if (!dstream_) {
    int dev = 0;
    KI_CUDA(cudaGetDevice(&dev));
    {
      // a cached set of this device, if a finished solver left one
      std::lock_guard<std::mutex> lk(g_aux_mu);
      auto& fl = aux_free();
      for (size_t i = 0; i < fl.size(); i++)
        if (fl[i].dev == dev) {
          const AuxSet a = fl[i];
          fl.erase(fl.begin() + static_cast<long>(i));
          dstream_ = a.d;
          ev_id_[0] = a.ev_id[0];
          ev_id_[1] = a.ev_id[1];
          ev_dec_ = a.ev_dec;
          id_fork_ = a.fork;
          for (int k = 0; k < kIdStreams; k++) {
            id_streams_[k] = a.id[k];
            id_join_[k] = a.join[k];
          }
          dl_fork_ = a.dl_fork;
          for (int k = 0; k < kDecStreams; k++) {
            dl_streams_[k] = a.dl[k];
            dl_join_[k] = a.dl_join[k];
          }
          bstream_ = a.b;
          ev_lvl_ = a.ev_lvl;
          ev_bdr_ = a.ev_bdr;
          ustream_ = a.u;
          ev_up_ = a.ev_up;
          break;
        }
    }
    if (!dstream_) {
      KI_CUDA(cudaStreamCreateWithFlags(&dstream_, cudaStreamNonBlocking));
      KI_CUDA(cudaEventCreateWithFlags(&ev_id_[0], cudaEventDisableTiming));
      KI_CUDA(cudaEventCreateWithFlags(&ev_id_[1], cudaEventDisableTiming));
      KI_CUDA(cudaEventCreateWithFlags(&ev_dec_, cudaEventDisableTiming));
      KI_CUDA(cudaEventCreateWithFlags(&id_fork_, cudaEventDisableTiming));
      for (int i = 0; i < kIdStreams; i++) {
        KI_CUDA(cudaStreamCreateWithFlags(&id_streams_[i], cudaStreamNonBlocking));
        KI_CUDA(cudaEventCreateWithFlags(&id_join_[i], cudaEventDisableTiming));
      }
      KI_CUDA(cudaEventCreateWithFlags(&dl_fork_, cudaEventDisableTiming));
      for (int i = 0; i < kDecStreams; i++) {
        KI_CUDA(cudaStreamCreateWithFlags(&dl_streams_[i], cudaStreamNonBlocking));
        KI_CUDA(cudaEventCreateWithFlags(&dl_join_[i], cudaEventDisableTiming));
      }
      KI_CUDA(cudaStreamCreateWithFlags(&bstream_, cudaStreamNonBlocking));
      KI_CUDA(cudaEventCreateWithFlags(&ev_lvl_, cudaEventDisableTiming));
      KI_CUDA(cudaEventCreateWithFlags(&ev_bdr_, cudaEventDisableTiming));
      KI_CUDA(cudaStreamCreateWithFlags(&ustream_, cudaStreamNonBlocking));
      KI_CUDA(cudaEventCreateWithFlags(&ev_up_, cudaEventDisableTiming));
    }
  }
  {
    // which full-shared-memory cluster sizes the device can schedule: asked
    // once per device and process (the occupancy queries are not free)
    static std::mutex mu;
    static std::map<int, std::array<bool, 17>> known;
    int dev = 0;
    KI_CUDA(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lock(mu);
    auto it = known.find(dev);
    if (it == known.end()) {
      std::array<bool, 17> ok{};
      for (int G = 1; G <= 16; G *= 2)
        ok[G] = id_cluster_fits(kOnChip + G, 4096, 256,
                                (227 * 1024 - id_smem_bytes(4096, 256)) / 8) != 0;
      it = known.emplace(dev, ok).first;
    }
    for (int G = 0; G <= 16; G++) onchip_ok_[G] = it->second[G];
  }
  if (!num_sms_) {
    int dev = 0;
    KI_CUDA(cudaGetDevice(&dev));
    KI_CUDA(cudaDeviceGetAttribute(&num_sms_, cudaDevAttrMultiProcessorCount, dev));
  }
  if (!smem_per_sm_) {
    int dev = 0;
    KI_CUDA(cudaGetDevice(&dev));
    KI_CUDA(cudaDeviceGetAttribute(&smem_per_sm_, cudaDevAttrMaxSharedMemoryPerMultiprocessor,
                                   dev));
  }
  return 0;
}

// Device geometry, proxy directions, holes, status flag and the border
// columns: none depends on the quadtree, so factor() queues them before
// building it (the copies and the border kernels run during the build).
int Solver::setup_geometry() {
  // geometry, proxy directions, holes, status flag
  {
    // node records formed straight into pinned staging, in parallel
    Node* st = static_cast<Node*>(stage_.alloc(sizeof(Node) * n_points_));
    if (!st) return fail("pinned staging allocation failed");
    parallel_for(n_points_, 4096, [&](int a, int e) {
      for (int i = a; i < e; i++)
        st[i] = Node{pts_[2 * i], pts_[2 * i + 1], nrm_[2 * i], nrm_[2 * i + 1], wts_[i],
                     curv_[i], 0.0, 0.0};
    });
    KI_ALLOC(d_nodes_, Node, n_points_);
    KI_CUDA(cudaMemcpyAsync(d_nodes_, st, sizeof(Node) * n_points_, cudaMemcpyHostToDevice,
                            stream_));
    std::vector<double> dir(2 * kNumProxy);
    for (int i = 0; i < kNumProxy; i++) {
      const double ang = 2 * M_PI * i * (1.0 / kNumProxy);
      dir[i] = std::cos(ang);
      dir[kNumProxy + i] = std::sin(ang);
    }
    KI_ALLOC(d_proxy_dir_, double, dir.size());
    KI_UPLOAD(d_proxy_dir_, dir, stream_);
    if (!holes_.empty()) {
      KI_ALLOC(d_holes_, double, holes_.size());
      KI_UPLOAD(d_holes_, holes_, stream_);
    }
    KI_ALLOC(d_status_, int, 1);
    KI_CUDA(cudaMemsetAsync(d_status_, 0, sizeof(int), stream_));
  }
  nb_ = 0;
  if (!holes_.empty() && opt_.pde != kLaplaceNeumann) {
    const int nh = static_cast<int>(holes_.size() / 4);
    nb_ = opt_.pde == kStokes ? 3 * nh : nh;
    const size_t cnt = static_cast<size_t>(n_dofs_) * nb_;
    KI_ALLOC(d_U_, double, cnt);
    KI_ALLOC(d_Psi_, double, cnt);
    KI_ALLOC(d_Urow_, double, cnt);
    KI_CUDA(launch_border_fill(opt_.pde, d_nodes_, n_points_, d_holes_, nh, d_U_, d_Psi_, d_Urow_,
                               stream_));
    // the border columns swept up through each level as soon as the level
    // is decoupled (U and Psi^T dof-major: a dof's nb entries contiguous, the
    // sweeps gather whole rows; Psi's own column-major nb x N layout is
    // Psi^T dof-major)
    KI_ALLOC(d_modU_, double, cnt);
    KI_ALLOC(d_modP_, double, cnt);
    KI_ALLOC(d_modD_, double, cnt);
    KI_CUDA(cudaMemcpyAsync(d_modU_, d_Urow_, sizeof(double) * cnt, cudaMemcpyDeviceToDevice,
                            stream_));
    KI_CUDA(cudaMemcpyAsync(d_modP_, d_Psi_, sizeof(double) * cnt, cudaMemcpyDeviceToDevice,
                            stream_));
  }

  geom_ready_ = true;
  return 0;
}

int Solver::factor() {
  cudaEvent_t ev0;
  const int rc = begin_factor(&ev0);
  if (rc) return rc;
  if (starts_.size() > 1 && !holes_.empty()) return fail("a forest of problems cannot have holes");
  const int grc = setup_geometry();
  if (grc) return grc;
  mark(7, 0);
  {
    std::lock_guard<std::mutex> lk(g_tree_mu);
    if (tree_slot() && starts_.size() <= 2) {
      tree = std::move(*tree_slot());
      tree_slot().reset();
    }
  }
  if (starts_.size() > 1) {
    tree.build_forest(pts_.data(), n_points_, sd_, opt_.max_leaf_dofs, starts_);
  } else {
    tree.build(pts_.data(), n_points_, sd_, opt_.max_leaf_dofs);
  }
  mark(8, 0);
  boxdev_.assign(tree.boxes.size(), BoxDev{});
  return finish_factor(ev0);
}

bool Solver::level1_stays() {
  // (level 2's ranks are in: level 1's active lists are its children's
  // skeletons)
  if (opt_.top_keep_max <= 0 || tree.roots.size() != 1 || tree.levels.size() < 3) return false;
  long long total = nb_;
  for (int id : tree.levels[1]) {
    if (tree.boxes[id].compressed) return false;  // kept by an update: compressed as before
    tree.refresh_box(id);
    total += static_cast<long long>(tree.boxes[id].active.size());
  }
  return total <= opt_.top_keep_max;
}

int Solver::check_coincident() {
  // Two nodes at the same position make two columns of the operator equal
  // (the reference takes r = 0 as the diagonal, kernel.cpp:23-36, 80-85),
  // an exactly singular system that no pivot would reveal.  Coincident
  // nodes fall in the same leaf: each leaf's points are sorted and
  // neighbours compared.
  std::vector<int> leaves;
  for (size_t i = 0; i < tree.boxes.size(); i++)
    if (tree.boxes[i].leaf && !tree.boxes[i].dead) leaves.push_back(static_cast<int>(i));
  std::atomic<long long> hit{-1};
  parallel_for(static_cast<int>(leaves.size()), 16, [&](int a, int e) {
    std::vector<int> pt;
    for (int q = a; q < e; q++) {
      pt.clear();
      for (int dof : tree.boxes[leaves[q]].original)
        if (dof % sd_ == 0) pt.push_back(dof / sd_);
      std::sort(pt.begin(), pt.end(), [&](int u, int v) {
        return pts_[2 * u] < pts_[2 * v] ||
               (pts_[2 * u] == pts_[2 * v] && pts_[2 * u + 1] < pts_[2 * v + 1]);
      });
      for (size_t i = 1; i < pt.size(); i++)
        if (pts_[2 * pt[i]] == pts_[2 * pt[i - 1]] &&
            pts_[2 * pt[i] + 1] == pts_[2 * pt[i - 1] + 1])
          hit.store(static_cast<long long>(std::min(pt[i], pt[i - 1])) << 32 |
                    std::max(pt[i], pt[i - 1]));
    }
  });
  const long long h = hit.load();
  if (h < 0) return 0;
  return fail("coincident boundary nodes " + std::to_string(h >> 32) + " and " +
              std::to_string(h & 0xffffffffLL) + " (the operator is singular)");
}

int Solver::finish_factor(cudaEvent_t ev0) {
  if (const int crc = check_coincident()) return crc;
  cudaEvent_t ev1;
  KI_CUDA(ev_get(&ev1));
  levels_.assign(tree.levels.size(), LevelFactors{});
  mark(0, 0);

  if (!geom_ready_) {
    const int rc = setup_geometry();
    if (rc) return rc;
  }

  const int L = static_cast<int>(tree.levels.size());
  launch_log.clear();
  t_wait_ms = t_host_prep_ms = t_host_post_ms = t_upload_ms = t_host_top_ms = 0;
  g_upload_ms = 0;
  // dstream_ (decoupling, border sweeps) after everything queued so far on
  // stream_: adopted factors, border columns
  KI_CUDA(cudaEventRecord(ev_id_[0], stream_));
  KI_CUDA(cudaStreamWaitEvent(dstream_, ev_id_[0], 0));
  // the coarsest level whose active lists id_launch has made (each level's
  // uncompressed boxes are refreshed there, after their children's ranks;
  // nothing below changes afterwards): only the levels above it remain
  int refreshed = L;
  if (L > 1) {
    // level l's IDs, then per level: the IDs of l - 1 launched, l's
    // decoupling prepared and launched while they run, l - 1's ranks read
    auto cur = std::make_unique<PendingLevel>();
    int rc = id_launch(L - 1, cur.get());
    refreshed = L - 1;
    if (!rc) rc = id_finish(cur.get());
    for (int level = L - 1; level > 0 && !rc; level--) {
      auto next = std::make_unique<PendingLevel>();
      const bool more = level > 1 && !(level == 2 && level1_stays());
      if (more) {
        rc = id_launch(level - 1, next.get());
        refreshed = level - 1;
      }
      if (!rc) rc = decouple_level(cur.get());
      if (!rc && more) rc = id_finish(next.get());
      if (!more) break;
      cur = std::move(next);
    }
    if (rc) return rc;
  }
  for (int level = refreshed - 1; level >= 0; level--) tree.refresh_level(level, nullptr);
  allskel.clear();
  for (int r : tree.roots)
    allskel.insert(allskel.end(), tree.boxes[r].active.begin(), tree.boxes[r].active.end());
  KI_CUDA(cudaEventRecord(ev_dec_, dstream_));
  KI_CUDA(cudaStreamWaitEvent(stream_, ev_dec_, 0));
  KI_CUDA(cudaEventRecord(ev_bdr_, bstream_));
  // the top-level assembly needs only the decouplings: a single tree's
  // border system waits for the border sweeps itself (factor_border), so
  // the assembly runs beside the last level's sweeps
  if (tree.roots.size() > 1 || nb_ == 0) KI_CUDA(cudaStreamWaitEvent(stream_, ev_bdr_, 0));
  cudaEvent_t t0 = nullptr;
  if (time_phases && timer_begin(&t0)) return -2;
  const double ht = now_ms();
  mark(4, 0);
  int rc = tree.roots.size() > 1 ? factor_top_forest() : factor_top();
  t_host_top_ms = now_ms() - ht;
  mark(5, 0);
  if (rc) return rc;
  if (time_phases && timer_end(t0, {0, 2, 1, 1, 0, ns_ + nb_, 0.0})) return -2;

  int status = 0;
  KI_CUDA(cudaMemcpyAsync(&status, d_status_, sizeof(int), cudaMemcpyDeviceToHost, stream_));
  KI_CUDA(cudaEventRecord(ev1, stream_));
  KI_CUDA(cudaStreamSynchronize(stream_));
  mark(6, 0);
  float ms = 0;
  KI_CUDA(cudaEventElapsedTime(&ms, ev0, ev1));
  t_factor_ms = ms;
  const int trc = timers_resolve();
  ev_start_ = nullptr;
  ev_put(ev0);
  ev_put(ev1);
  if (trc) return -2;
  t_upload_ms = g_upload_ms;
  if (status == 2) return fail("an LU factorization stopped: a bounded wait timed out");
  if (status) return fail("zero pivot in an LU factorization (singular block)");
  return 0;
}

int Solver::id_launch(int level, PendingLevel* pl) {
  const double h0 = now_ms();
  pl->level = level;
  // boxes compressed before this factorization (kept by an update or a
  // copy) are skipped by the IDs and join the level's sweeps as they are
  for (int id : tree.levels[level])
    if (tree.boxes[id].compressed) pl->boxes.push_back(id);
  const std::vector<int>& ids = tree.levels[level];
  const int nids = static_cast<int>(ids.size());
  // active lists of the level (quadtree.cpp:694-720), independent per box
  parallel_for(nids, 32, [&](int a, int e) {
    for (int q = a; q < e; q++)
      if (!tree.boxes[ids[q]].compressed) tree.refresh_box(ids[q]);
  });
  mark(9, level);
  const int P = sd_ == 2 ? 4 * kNumProxy : 2 * kNumProxy;

  using Cand = IdCand;
  std::vector<Cand> all(nids);
  std::vector<char> keep(nids, 0);
  parallel_for(nids, 8, [&](int a, int e) {
    for (int q = a; q < e; q++) {
      const int id = ids[q];
      const Box& b = tree.boxes[id];
      if (b.compressed || static_cast<int>(b.active.size()) < opt_.min_dofs_to_compress) continue;
      Cand& c = all[q];
      c.box = id;
      c.n = static_cast<int>(b.active.size());
      if (level == 1 || level == 2) {
        // kernel.cpp:164-207: every other active dof of the level (and the
        // level-1 leaves for level 2), both directions, no proxy circle.
        // (a forest restricts both to the box's own tree)
        for (int o : tree.levels[level])
          if (o != id && tree.boxes[o].tree == b.tree)
            c.rows.insert(c.rows.end(), tree.boxes[o].active.begin(), tree.boxes[o].active.end());
        if (level == 2)
          for (int o : tree.levels[1])
            if (tree.boxes[o].leaf && tree.boxes[o].tree == b.tree)
              c.rows.insert(c.rows.end(), tree.boxes[o].original.begin(),
                            tree.boxes[o].original.end());
        c.I = static_cast<int>(c.rows.size());
        c.m = 2 * c.I;
      } else {
        // the near dofs (neighbours at this level or coarser: leaves give
        // their original dofs, others their active ones, quadtree.cpp:
        // 664-691) that lie inside the proxy circle (kernel.cpp:209-218)
        const double cx = b.corner[0] + b.side / 2.0, cy = b.corner[1] + b.side / 2.0;
        const double R = kRadiusRatio * b.side;
        // squared distances decide all but a thin band around the circle,
        // where the reference's own expression decides
        const double lo2 = R * R * (1.0 - 1e-9), hi2 = R * R * (1.0 + 1e-9);
        for (int o : b.nbr) {
          const Box& ob = tree.boxes[o];
          if (ob.level > b.level) continue;
          int last_pt = -1;
          bool last_in = false;
          for (int dof : ob.leaf ? ob.original : ob.active) {
            const int pt = dof / sd_;
            if (pt != last_pt) {  // a Stokes node's two dofs are adjacent
              const double dx = cx - pts_[2 * pt], dy = cy - pts_[2 * pt + 1];
              const double d2 = dx * dx + dy * dy;
              last_in = d2 < lo2 ? true
                        : d2 > hi2 ? false
                                   : std::sqrt(std::pow(dx, 2) + std::pow(dy, 2)) < R;
              last_pt = pt;
            }
            if (last_in) c.rows.push_back(dof);
          }
        }
        c.I = static_cast<int>(c.rows.size());
        c.m = 2 * c.I + P;
      }
      if (c.m == 0) continue;
      c.g = pick_group(c.m, c.n, onchip_ok_);
      if (opt_.sketch_id) {
        // A level whose boxes, each spread over the widest cluster that
        // still leaves a CTA 12 columns, fit one wave at two CTAs per SM
        // takes that width: the pivoted QR's steps shrink with the columns
        // a CTA owns (measured on a B200, the Stokes workload's level-2
        // IDs: 0.96 -> 0.72 ms).  Otherwise the smallest cluster whose
        // CTAs' shares of the sketch leave room for two CTAs per SM (a
        // single CTA per SM leaves the SM idle at every barrier of the
        // pivoted QR), else the smallest that fits.
        auto fit = [&](int l) {  // cluster size for an l-row sketch, 0: none
          for (int G = 16; G >= 2; G /= 2)
            if (onchip_ok_[G] && c.n >= 12 * G && nids * G <= 2 * num_sms_ &&
                id_sketch_smem_bytes(l, c.n, G) <= size_t{113} * 1024)
              return G;
          for (const size_t cap : {size_t{113} * 1024, size_t{227} * 1024})
            for (int G = 1; G <= 16; G *= 2)
              if (onchip_ok_[G] && id_sketch_smem_bytes(l, c.n, G) <= cap) return G;
          return 0;
        };
        // the full sketch (n + 16 rows) must be possible; on a level of many
        // boxes the box is then sketched with rows sized by the level below's
        // ranks, and decomposed again with the full sketch if those do not
        // certify its rank (a level of a few boxes, whose launches are short
        // of work anyway, takes the full sketch: a second pass would put a
        // whole launch and rank read-back on the factorization's critical
        // path)
        const int l = sketch_rows(c.n);
        const int G_full = c.m > l + 64 && l >= 32 ? fit(l) : 0;  // (bucket runs need l >= 32)
        if (G_full) {
          const int ls = nids > kShortSketchMinBoxes ? sketch_rows_hint(c.n, rank_hint_) : l;
          const int G_short = ls < l ? fit(ls) : 0;
          c.sk = G_short ? ls : l;
          c.g = kOnChip + (G_short ? G_short : G_full);
          c.g_full = G_short ? kOnChip + G_full : 0;
        }
        if (c.sk && level > 2) c.m = 2 * c.I + (P >> opt_.proxy_shift);
      }
      keep[q] = 1;
    }
  });
  mark(10, level);
  std::vector<Cand>& cand = pl->cand;
  for (int q = 0; q < nids; q++)
    if (keep[q]) cand.push_back(std::move(all[q]));
  if (cand.empty()) return 0;
  // grouped by cluster size, the group holding the widest ID matrix first
  // (its launch then takes SMs before the many-box launch fills them: the
  // few big boxes are each level's longest tasks), and inside a group the
  // largest first (CTAs start in index order, so the long tasks do not end
  // up in a launch's last wave)
  std::map<int, long long> group_max;  // widest task (its steps and sketch rows grow with n)
  for (const Cand& c : cand) {
    long long& v = group_max[c.g];
    v = std::max(v, static_cast<long long>(c.n) * 100000 + std::min(c.m, 99999));
  }
  std::stable_sort(cand.begin(), cand.end(), [&](const Cand& a, const Cand& b) {
    if (a.g != b.g) {
      const long long ma = group_max[a.g], mb = group_max[b.g];
      return ma != mb ? ma > mb : a.g > b.g;
    }
    return static_cast<long long>(a.m) * a.n > static_cast<long long>(b.m) * b.n;
  });

  mark(11, level);
  const int nc = static_cast<int>(cand.size());
  std::vector<IdTask>& tasks = pl->tasks;
  tasks.assign(nc, IdTask{});
  long long a_total = 0, t_total = 0;
  int& perm_total = pl->perm_total;
  size_t act_total = 0, rows_total = 0;
  for (int q = 0; q < nc; q++) {  // offsets
    const Cand& c = cand[q];
    IdTask& t = tasks[q];
    t.lda = c.sk ? onchip_lda(c.sk) : c.g >= kOnChip ? onchip_lda(c.m) : (c.m + 3) & ~3;
    t.act_off = static_cast<int>(act_total);
    t.row_off = static_cast<int>(rows_total);
    t.perm_off = perm_total;
    t.a_off = a_total;
    t.t_off = t_total;
    act_total += c.n;
    rows_total += c.rows.size();
    if (c.g < kOnChip) a_total += static_cast<long long>(t.lda) * c.n;  // on-chip: none
    t_total += static_cast<long long>(c.n) * c.n / 4 + 1;
    perm_total += c.n;
  }
  std::vector<int> act(act_total), rows(rows_total);
  parallel_for(nc, 16, [&](int a, int e) {  // descriptors and lists
    for (int q = a; q < e; q++) {
      const Cand& c = cand[q];
      const Box& b = tree.boxes[c.box];
      IdTask& t = tasks[q];
      t.n = c.n;
      t.m = c.m;
      t.n_row = c.I;
      t.proxy = c.m - 2 * c.I;
      t.sk = c.sk;
      t.pshift = c.sk && level > 2 ? opt_.proxy_shift : 0;
      t.cx = b.corner[0] + b.side / 2.0;
      t.cy = b.corner[1] + b.side / 2.0;
      t.rad = b.side * kRadiusRatio;
      t.pw = 2.0 * M_PI * t.rad / (kNumProxy >> t.pshift);
      std::copy(b.active.begin(), b.active.end(), act.begin() + t.act_off);
      std::copy(c.rows.begin(), c.rows.end(), rows.begin() + t.row_off);
    }
  });
  t_host_prep_ms += now_ms() - h0;
  mark(1, level);
  int *d_act, *d_rows, *d_perm, *d_rank;
  double* d_T;
  IdTask* d_tasks;
  // the level's three lists in one host-to-device copy and its ranks and
  // pivots in one copy back: each copy adds its own latency to the chain of
  // ID levels (a level's lists wait for the ranks of the level below)
  const size_t b_act = sizeof(int) * act.size(), b_rows = sizeof(int) * rows.size();
  const size_t o_rows = (b_act + 255) & ~static_cast<size_t>(255);
  const size_t o_tasks = o_rows + ((b_rows + 255) & ~static_cast<size_t>(255));
  const size_t b_pack = o_tasks + sizeof(IdTask) * nc;
  char* d_pack;
  KI_ALLOC(d_pack, char, b_pack);
  d_act = reinterpret_cast<int*>(d_pack);
  d_rows = reinterpret_cast<int*>(d_pack + o_rows);
  d_tasks = reinterpret_cast<IdTask*>(d_pack + o_tasks);
  KI_ALLOC(d_rank, int, nc + perm_total);  // [ranks | pivots]
  d_perm = d_rank + nc;
  KI_ALLOC(d_T, double, t_total);
  KI_CUDA(work_.reserve(sizeof(double) * a_total, stream_));
  {
    char* st = static_cast<char*>(stage_.alloc(b_pack));
    if (!st) return fail("pinned staging allocation failed");
    if (b_act) std::memcpy(st, act.data(), b_act);
    if (b_rows) std::memcpy(st + o_rows, rows.data(), b_rows);
    std::memcpy(st + o_tasks, tasks.data(), sizeof(IdTask) * nc);
    KI_CUDA(cudaMemcpyAsync(d_pack, st, b_pack, cudaMemcpyHostToDevice, stream_));
  }

  // one launch per cluster size (split further so that the launch's
  // shared-memory layout, sized by its largest rows / columns / column
  // storage, still fits); the first on stream_, the others forked onto the
  // ID streams and joined back before the ranks are read
  KI_CUDA(cudaEventRecord(id_fork_, stream_));
  int nlaunch = 0;
  bool used[kIdStreams] = {};
  for (int q0 = 0; q0 < nc;) {
    int q1 = q0;
    int m_cap = 0, n_cap = 0;
    long long onchip = 0;
    const int g0 = cand[q0].g;
    const int G = g0 >= kOnChip ? g0 - kOnChip : 0;
    while (q1 < nc && cand[q1].g == g0) {
      const int mm = std::max(m_cap, cand[q1].m), nn = std::max(n_cap, cand[q1].n);
      if (G) {
        // per-task layout: the launch needs the largest single task's share
        onchip = std::max<long long>(
            onchip, cand[q1].sk ? id_sketch_smem_bytes(cand[q1].sk, cand[q1].n, G)
                                : id_onchip_smem_bytes(cand[q1].m, cand[q1].n, G));
      } else if (q1 > q0 && id_smem_bytes(mm, nn) > 227 * 1024) {
        break;
      }
      m_cap = mm;
      n_cap = nn;
      q1++;
    }
    if ((G ? static_cast<size_t>(onchip) : id_smem_bytes(m_cap, n_cap)) > 227 * 1024)
      return fail("interpolative decomposition too tall for shared staging (m = " +
                  std::to_string(m_cap) + ")");
    IdParams p{};
    p.tasks = d_tasks + q0;
    p.ntasks = q1 - q0;
    p.pde = opt_.pde;
    p.nodes = d_nodes_;
    p.act = d_act;
    p.rowdofs = d_rows;
    p.work = static_cast<double*>(work_.p);
    p.tout = d_T;
    p.perm = d_perm;
    p.rank = d_rank + q0;
    p.proxy_dir = d_proxy_dir_;
    p.tol = opt_.id_tol;
    p.m_cap = m_cap;
    p.n_cap = n_cap;
    p.onchip_smem = onchip;
    const int si = nlaunch == 0 ? -1 : (nlaunch - 1) % kIdStreams;
    cudaStream_t ls = si < 0 ? stream_ : id_streams_[si];
    if (si >= 0 && !used[si]) {
      KI_CUDA(cudaStreamWaitEvent(ls, id_fork_, 0));
      used[si] = true;
    }
    cudaEvent_t e0 = nullptr;
    if (time_phases && timer_begin(&e0, ls)) return -2;
    KI_CUDA(launch_id(p, cand[q0].g, ls));
    if (time_phases) {
      if (timer_end(e0, {level, 0, cand[q0].g, q1 - q0, m_cap, n_cap, 0.0}, ls)) return -2;
    }
    nlaunch++;
    q0 = q1;
  }
  for (int i = 0; i < kIdStreams; i++)
    if (used[i]) {
      KI_CUDA(cudaEventRecord(id_join_[i], id_streams_[i]));
      KI_CUDA(cudaStreamWaitEvent(stream_, id_join_[i], 0));
    }
  // the level's decoupling (on dstream_) waits for its IDs and nothing
  // later (the next level's IDs are queued on stream_ before it)
  KI_CUDA(cudaEventRecord(ev_id_[level & 1], stream_));
  pl->ids_queued = true;
  // ranks and pivots into pinned memory: the copies queue behind the IDs
  // without blocking the host (a copy to pageable memory would wait for them)
  pl->rank = static_cast<int*>(stage_.alloc(sizeof(int) * (nc + perm_total + 1)));
  if (!pl->rank) return fail("pinned staging allocation failed");
  pl->perm = pl->rank + nc;
  KI_CUDA(cudaMemcpyAsync(pl->rank, d_rank, sizeof(int) * (nc + perm_total),
                          cudaMemcpyDeviceToHost, stream_));
  pl->d_act = d_act;
  pl->d_rows = d_rows;
  pl->d_perm = d_perm;
  pl->d_T = d_T;
  return 0;
}

int Solver::id_rerun_full(PendingLevel* pl) {
  const int nc = static_cast<int>(pl->cand.size());
  std::vector<int> qs;
  for (int q = 0; q < nc; q++)
    if (pl->rank[q] < 0) qs.push_back(q);
  // the same boxes with n + 16 sketch rows, grouped by cluster size
  std::stable_sort(qs.begin(), qs.end(), [&](int a, int b) {
    return pl->cand[a].g_full > pl->cand[b].g_full;
  });
  std::vector<IdTask> t2(qs.size());
  for (size_t u = 0; u < qs.size(); u++) {
    IdCand& c = pl->cand[qs[u]];
    if (!c.g_full) return fail("interpolative decomposition: sketch too short for a box");
    t2[u] = pl->tasks[qs[u]];
    t2[u].sk = sketch_rows(c.n);
    t2[u].lda = onchip_lda(t2[u].sk);
    c.sk = t2[u].sk;
    c.g = c.g_full;
  }
  IdTask* d_t2;
  int* d_r2;
  KI_ALLOC(d_t2, IdTask, t2.size());
  KI_ALLOC(d_r2, int, t2.size());
  KI_UPLOAD(d_t2, t2, stream_);
  for (size_t q0 = 0; q0 < qs.size();) {
    size_t q1 = q0;
    const int g = pl->cand[qs[q0]].g;
    long long smem = 0;
    int n_cap = 0;
    while (q1 < qs.size() && pl->cand[qs[q1]].g == g) {
      const IdCand& c = pl->cand[qs[q1]];
      smem = std::max<long long>(smem, id_sketch_smem_bytes(c.sk, c.n, g - kOnChip));
      n_cap = std::max(n_cap, c.n);
      q1++;
    }
    IdParams p{};
    p.tasks = d_t2 + q0;
    p.ntasks = static_cast<int>(q1 - q0);
    p.pde = opt_.pde;
    p.nodes = d_nodes_;
    p.act = pl->d_act;
    p.rowdofs = pl->d_rows;
    p.work = static_cast<double*>(work_.p);
    p.tout = pl->d_T;
    p.perm = pl->d_perm;
    p.rank = d_r2 + q0;
    p.proxy_dir = d_proxy_dir_;
    p.tol = opt_.id_tol;
    p.m_cap = 0;
    p.n_cap = n_cap;
    p.onchip_smem = smem;
    KI_CUDA(launch_id(p, g, stream_));
    q0 = q1;
  }
  int* r2 = static_cast<int*>(stage_.alloc(sizeof(int) * qs.size()));
  if (!r2) return fail("pinned staging allocation failed");
  KI_CUDA(cudaMemcpyAsync(r2, d_r2, sizeof(int) * qs.size(), cudaMemcpyDeviceToHost, stream_));
  KI_CUDA(cudaMemcpyAsync(pl->perm, pl->d_perm, sizeof(int) * pl->perm_total,
                          cudaMemcpyDeviceToHost, stream_));
  KI_CUDA(cudaStreamSynchronize(stream_));
  for (size_t u = 0; u < qs.size(); u++) pl->rank[qs[u]] = std::max(r2[u], 0);
  return 0;
}

int Solver::id_finish(PendingLevel* pl) {
  const int level = pl->level;
  const int nc = static_cast<int>(pl->cand.size());
  if (nc == 0) return 0;
  using Cand = IdCand;
  const std::vector<Cand>& cand = pl->cand;
  const std::vector<IdTask>& tasks = pl->tasks;
  const int* rank = pl->rank;
  const int* perm = pl->perm;
  double* d_T = pl->d_T;
  {
    const auto w0 = std::chrono::steady_clock::now();
    KI_CUDA(cudaStreamSynchronize(stream_));
    t_wait_ms += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - w0)
                     .count();
  }
  for (int q = 0; q < nc; q++)
    if (rank[q] < 0) {
      const int rc = id_rerun_full(pl);
      if (rc) return rc;
      break;
    }

  // skeleton / redundant sets (InteractionLists::set_rs_ranges, quadtree.h:23-35)
  const double h1 = now_ms();
  mark(2, level);
  std::vector<int>& comp = pl->comp;  // candidate indices that compressed
  {
    // per candidate, independent: work counts, skeleton / redundant lists
    std::vector<double> qr_v(nc), bytes_v(nc);
    parallel_for(nc, 16, [&](int a, int e) {
      for (int q = a; q < e; q++) {
        const Cand& c = cand[q];
        const IdTask& t = tasks[q];
        const int k = rank[q];
        // Algorithmic work of the ID, counted from the actual sizes and
        // rank: FP64 flops = entry generation (20 per entry) + the
        // Householder steps actually taken (column dots + rank-one updates
        // over the shrinking trailing block) + the triangular solve for T;
        // HBM bytes = the dof lists and node records read, perm and T
        // written, plus, for the streamed launches, the working matrix
        // written once and read once.  (a sketched box: generation +
        // kSketchBlocks signed adds per entry, the QR on the sk rows)
        const double n = c.n, m = c.sk ? c.sk : c.m;
        const int steps = k > 0 ? k : std::min(static_cast<int>(m), c.n);
        double qr = 20.0 * c.m * n + 1.0 * k * k * (n - k);
        if (c.sk) qr += 1.0 * kSketchBlocks * c.m * n;
        for (int j = 0; j < steps; j++) qr += 4.0 * (m - j) * (n - j - 1) + 3.0 * (m - j);
        const double sd = sd_;  // dofs per node record
        double bytes = 4.0 * (c.I + 2 * n) + 64.0 * (c.I + c.n) / sd + 8.0 * k * (n - k);
        if (c.g < kOnChip) bytes += 16.0 * c.m * n;
        qr_v[q] = qr;
        bytes_v[q] = bytes;
        if (k == 0) continue;
        Box& b = tree.boxes[c.box];
        b.compressed = true;
        b.rank = k;
        b.perm.assign(perm + t.perm_off, perm + t.perm_off + c.n);
        b.skel.resize(k);
        b.redundant.resize(c.n - k);
        for (int i = 0; i < k; i++) b.skel[i] = b.active[b.perm[i]];
        for (int i = k; i < c.n; i++) b.redundant[i - k] = b.active[b.perm[i]];
        boxdev_[c.box].T = d_T + t.t_off;
      }
    });
    for (int q = 0; q < nc; q++) {
      id_flops += qr_v[q];
      id_bytes += bytes_v[q];
      if (cand[q].g >= kOnChip) id_onchip_flops += qr_v[q];
      if (rank[q] > 0) comp.push_back(q);
      rank_hint_ = std::max(rank_hint_, rank[q]);
    }
  }
  t_host_post_ms += now_ms() - h1;
  return 0;
}

int Solver::decouple_level(PendingLevel* pl) {
  if (pl->ids_queued) KI_CUDA(cudaStreamWaitEvent(dstream_, ev_id_[pl->level & 1], 0));
  if (!pl->comp.empty()) {
    const int rc = decouple_boxes(pl);
    if (rc) return rc;
  }
  const int rc = level_sweeps(pl->level, pl->boxes, dstream_);
  if (rc) return rc;
  const LevelFactors& lf = levels_[pl->level];
  if (nb_ > 0 && lf.ntasks) {
    // skel_factorization.cpp:146-160 for this level: U and Psi^T swept up,
    // on their own stream after the level's decoupling (in level order
    // there), off the chain of decouplings: the next level's does not read
    // them; the top level's border system waits for them
    SweepParams sp{lf.d_tasks, lf.ntasks, d_modU_, 1, nb_, 0, nullptr, lf.cap, nb_};
    SweepParams spp = sp;
    spp.x = d_modP_;
    KI_CUDA(cudaEventRecord(ev_lvl_, dstream_));
    KI_CUDA(cudaStreamWaitEvent(bstream_, ev_lvl_, 0));
    KI_CUDA(launch_sweep_up_pair(sp, spp, bstream_));
    // the level's redundant rows of U are final now (coarser levels' sweeps
    // touch only their own active dofs): X_rr^{-1} is applied to a copy of
    // them here, beside the next decouplings, instead of to every box's at
    // once between the last decoupling and the top-level LU
    KI_CUDA(launch_copy_rows(d_modU_, d_modD_, nb_, lf.d_red, lf.nred, bstream_));
    SweepParams sd = sp;
    sd.x = d_modD_;
    KI_CUDA(launch_diag_solve(sd, bstream_));
  }
  return 0;
}

int Solver::decouple_boxes(PendingLevel* pl) {
  // ---- decouple every compressed box of the level
  const double h1 = now_ms();
  const int level = pl->level;
  using Cand = IdCand;
  const std::vector<Cand>& cand = pl->cand;
  const std::vector<IdTask>& tasks = pl->tasks;
  const std::vector<int>& comp = pl->comp;
  int* d_act = pl->d_act;
  int* d_perm = pl->d_perm;
  const int ncomp = static_cast<int>(comp.size());
  std::vector<DecTask> dt(ncomp);
  // block maps (per position of the box's dof list: which descendant
  // update, and where in it), made per box in parallel at precomputed offsets
  std::vector<std::vector<BoxBlock>> blk(ncomp);
  parallel_for(ncomp, 16, [&](int a, int e) {
    for (int t = a; t < e; t++) {
      const Box& b = tree.boxes[cand[comp[t]].box];
      if (b.leaf) continue;
      int off = 0;
      for (int q = 0; q < 4; q++) {
        const int ch = b.child[q];
        for (const BoxBlock& x : blocks_of(ch)) blk[t].push_back(BoxBlock{x.acc, x.size, x.pos + off});
        const Box& cb = tree.boxes[ch];
        off += static_cast<int>(cb.compressed ? cb.skel.size() : cb.active.size());
      }
    }
  });
  std::vector<long long> bid_off(ncomp + 1, 0), tab_off(ncomp + 1, 0);
  long long scratch_total = 0;
  std::vector<long long> k_off(ncomp);
  int n_max = 0;
  size_t fac_total = 0, piv_total = 0;
  for (int t = 0; t < ncomp; t++) {
    const Cand& c = cand[comp[t]];
    const Box& b = tree.boxes[c.box];
    const int n = c.n, k = b.rank, r = n - k;
    bid_off[t + 1] = bid_off[t] + n;
    tab_off[t + 1] = tab_off[t] + static_cast<long long>(blk[t].size());
    k_off[t] = scratch_total;
    if (n > kDecoupleSmemN) {
      // n x n, then the LU's flags (kLuSyncInts ints)
      scratch_total += static_cast<long long>(n) * n + kLuSyncInts;
    } else {
      n_max = std::max(n_max, n);
    }
    fac_total += static_cast<size_t>(k) * r * 2 + static_cast<size_t>(r) * r +
                 static_cast<size_t>(k) * k;
    piv_total += r;
    {
      const double dk = k, dr = r, dn = n;
      // K_BN entries (~20 flops each), T^T K_ss, T^T K_sr, K_r_sn T, K_ss T,
      // X_rr^-1 (Gauss-Jordan), U = X^-1 K_r_sn, L = K_sn_r X^-1, L K_r_sn
      dec_flops += 20.0 * dn * dn + 2.0 * dr * dr * dr + 8.0 * dr * dr * dk + 6.0 * dr * dk * dk;
      solve_bytes += 8.0 * (4.0 * dk * dr + dr * dr);
    }
  }
  std::vector<int> bid(bid_off[ncomp], -1), bpos(bid_off[ncomp], 0);
  std::vector<UpdBlock> tab(tab_off[ncomp]);
  parallel_for(ncomp, 16, [&](int a, int e) {
    for (int t = a; t < e; t++) {
      const std::vector<BoxBlock>& bl = blk[t];
      int* bi = bid.data() + bid_off[t];
      int* bp = bpos.data() + bid_off[t];
      for (size_t q = 0; q < bl.size(); q++) {
        tab[tab_off[t] + q] = UpdBlock{bl[q].acc, bl[q].size, 0};
        for (int u = 0; u < bl[q].size; u++) {
          bi[bl[q].pos + u] = static_cast<int>(q);
          bp[bl[q].pos + u] = u;
        }
      }
    }
  });
  int *d_bid, *d_bpos, *d_piv;
  UpdBlock* d_tab;
  double* d_fac;
  DecTask* d_dt;
  KI_ALLOC(d_bid, int, bid.size());
  KI_ALLOC(d_bpos, int, bpos.size());
  KI_ALLOC(d_tab, UpdBlock, tab.size());
  KI_ALLOC(d_fac, double, fac_total);
  KI_ALLOC(d_piv, int, piv_total);
  KI_ALLOC(d_dt, DecTask, ncomp);
  // (earlier levels' decouplings may still be queued on dstream_ with the
  // old buffer: it is retired, not waited for)
  KI_CUDA(scratch2_.reserve(sizeof(double) * (scratch_total + 1), dstream_, true));
  double* scr = static_cast<double*>(scratch2_.p);
  size_t fo = 0, po = 0;
  for (int t = 0; t < ncomp; t++) {
    const Cand& c = cand[comp[t]];
    const IdTask& it = tasks[comp[t]];
    const Box& b = tree.boxes[c.box];
    const int n = c.n, k = b.rank, r = n - k;
    BoxDev& bd = boxdev_[c.box];
    bd.L = d_fac + fo;
    fo += static_cast<size_t>(k) * r;
    bd.U = d_fac + fo;
    fo += static_cast<size_t>(k) * r;
    bd.X = d_fac + fo;
    fo += static_cast<size_t>(r) * r;
    bd.acc = d_fac + fo;
    fo += static_cast<size_t>(k) * k;
    bd.piv = d_piv + po;
    po += r;
    DecTask& d = dt[t];
    d.n = n;
    d.k = k;
    d.act = d_act + it.act_off;
    d.perm = d_perm + it.perm_off;
    d.bid = d_bid + bid_off[t];
    d.bpos = d_bpos + bid_off[t];
    d.blocks = d_tab + tab_off[t];
    d.T = bd.T;
    d.K = scr + k_off[t];
    d.L = bd.L;
    d.U = bd.U;
    d.X = bd.X;
    d.acc = bd.acc;
    d.piv = bd.piv;
  }
  // small boxes first in one batched launch, then each large box
  std::vector<DecTask> small, large;
  for (const DecTask& d : dt) (d.n > kDecoupleSmemN ? large : small).push_back(d);
  // the largest boxes first (CTAs start in index order: no long last wave)
  std::stable_sort(small.begin(), small.end(),
                   [](const DecTask& a, const DecTask& b) { return a.n > b.n; });
  KI_UPLOAD(d_bid, bid, ustream_);
  KI_UPLOAD(d_bpos, bpos, ustream_);
  KI_UPLOAD(d_tab, tab, ustream_);
  KI_UPLOAD(d_dt, small, ustream_);
  KI_CUDA(cudaEventRecord(ev_up_, ustream_));
  KI_CUDA(cudaStreamWaitEvent(dstream_, ev_up_, 0));
  DecParams dp{};
  dp.tasks = d_dt;
  dp.ntasks = static_cast<int>(small.size());
  dp.pde = opt_.pde;
  dp.nodes = d_nodes_;
  dp.status = d_status_;
  cudaEvent_t d0 = nullptr;
  t_host_post_ms += now_ms() - h1;
  mark(3, level);
  if (time_phases && timer_begin(&d0, dstream_)) return -2;
  // The batched boxes in size classes, one launch each: a launch's shared
  // memory is sized by its largest box, so the boxes of a level are grouped
  // by how many CTAs of theirs an SM holds (three at most: 72 registers x
  // 256 threads; on a B200 n <= 85 gives three, n <= 110 two); the widest
  // class on dstream_, the others and the large boxes (one multi-kernel
  // sequence each) side by side on their own streams after the level's
  // uploads, joined back into dstream_.
  KI_CUDA(cudaEventRecord(dl_fork_, dstream_));
  bool used[kDecStreams] = {};
  int next_side = 0;
  auto side_stream = [&](cudaStream_t* out) -> int {
    const int si = next_side++ % kDecStreams;
    if (!used[si]) {
      KI_CUDA(cudaStreamWaitEvent(dl_streams_[si], dl_fork_, 0));
      used[si] = true;
    }
    *out = dl_streams_[si];
    return 0;
  };
  auto size_class = [&](int n) {
    // (1 KB of each CTA's shared memory is reserved by the system)
    return std::min<size_t>(3, static_cast<size_t>(smem_per_sm_) / (decouple_smem_bytes(n) + 1024));
  };
  for (size_t a = 0; a < small.size();) {
    size_t b = a;
    while (b < small.size() && size_class(small[b].n) == size_class(small[a].n)) b++;
    DecParams dpc = dp;
    dpc.tasks = d_dt + a;
    dpc.ntasks = static_cast<int>(b - a);
    cudaStream_t cs = dstream_;
    if (a > 0 && side_stream(&cs)) return -2;
    KI_CUDA(launch_decouple(dpc, small[a].n, cs));  // (sorted: the class's largest first)
    a = b;
  }
  int n_large = 0;
  for (size_t t = 0; t < large.size(); t++) {
    cudaStream_t cs;
    if (side_stream(&cs)) return -2;
    KI_CUDA(decouple_large(large[t], opt_.pde, d_nodes_, d_status_, cs));
    n_large = std::max(n_large, large[t].n);
  }
  for (int i = 0; i < kDecStreams; i++)
    if (used[i]) {
      KI_CUDA(cudaEventRecord(dl_join_[i], dl_streams_[i]));
      KI_CUDA(cudaStreamWaitEvent(dstream_, dl_join_[i], 0));
    }
  if (time_phases &&
      timer_end(d0, {level, 1, static_cast<int>(large.size()), ncomp, n_large, n_max, 0.0},
                dstream_))
    return -2;

  for (int t = 0; t < ncomp; t++) pl->boxes.push_back(cand[comp[t]].box);
  return 0;
}

int Solver::level_sweeps(int level, const std::vector<int>& boxes, cudaStream_t s) {
  // sweep descriptors of the level's compressed boxes
  LevelFactors& lf = levels_[level];
  lf.level = level;
  const int ncomp = static_cast<int>(boxes.size());
  if (ncomp == 0) return 0;
  std::vector<int> sk, rd;
  std::vector<SweepTask> st(ncomp);
  std::vector<int> sk_off(ncomp), rd_off(ncomp);
  int cap = 0, kr = 0;
  for (int t = 0; t < ncomp; t++) {
    const Box& b = tree.boxes[boxes[t]];
    sk_off[t] = static_cast<int>(sk.size());
    rd_off[t] = static_cast<int>(rd.size());
    sk.insert(sk.end(), b.skel.begin(), b.skel.end());
    rd.insert(rd.end(), b.redundant.begin(), b.redundant.end());
    cap = std::max(cap, static_cast<int>(b.skel.size() + b.redundant.size()));
    kr = std::max(kr, static_cast<int>(b.skel.size() * b.redundant.size()));
    lf.boxes.push_back(boxes[t]);
  }
  KI_ALLOC(lf.d_skel, int, sk.size());
  KI_ALLOC(lf.d_red, int, rd.size());
  KI_ALLOC(lf.d_tasks, SweepTask, ncomp);
  for (int t = 0; t < ncomp; t++) {
    const Box& b = tree.boxes[boxes[t]];
    const BoxDev& bd = boxdev_[boxes[t]];
    st[t] = SweepTask{b.rank, static_cast<int>(b.redundant.size()), lf.d_skel + sk_off[t],
                      lf.d_red + rd_off[t], bd.T, bd.L, bd.U, bd.X, bd.piv};
  }
  KI_UPLOAD(lf.d_skel, sk, ustream_);
  KI_UPLOAD(lf.d_red, rd, ustream_);
  KI_UPLOAD(lf.d_tasks, st, ustream_);
  KI_CUDA(cudaEventRecord(ev_up_, ustream_));
  KI_CUDA(cudaStreamWaitEvent(s, ev_up_, 0));
  lf.h_tasks = st;
  lf.ntasks = ncomp;
  lf.nred = static_cast<int>(rd.size());
  lf.cap = cap;
  lf.kr = kr;
  return 0;
}

void Solver::drop_device_state() {
  // everything in the arena except the box factors, which the caller
  // re-points; lazily built buffers are rebuilt on first use
  if (solve_exec_) cudaGraphExecDestroy(solve_exec_);
  solve_exec_ = nullptr;
  graph_uses_ = 0;
  g_x_ = nullptr;
  d_mv_tiles_ = nullptr;
  n_mv_tiles_ = mv_splits_ = 0;
  d_seg_ = nullptr;
  seg_.clear();
  d_nodes_ = nullptr;
  d_proxy_dir_ = nullptr;
  d_holes_ = nullptr;
  d_status_ = nullptr;
  d_forest_ = nullptr;
  d_top_ = nullptr;
  d_top_piv_ = nullptr;
  d_top_perm_ = nullptr;
  d_top_dinv_ = nullptr;
  d_allskel_ = d_allred_ = d_red_pos_ = nullptr;
  d_U_ = d_Psi_ = d_Urow_ = d_Ured_ = d_Pred_ = d_tmp_ = nullptr;
  d_modU_ = d_modP_ = d_modD_ = nullptr;
  all_compressed_ = LevelFactors{};
  levels_.clear();
}

int Solver::adopt_factors(const std::vector<int>& boxes, const std::vector<BoxDevView>& src) {
  std::vector<CopySeg> segs;
  auto seg = [&](const void* from, void* to, size_t bytes) {
    if (bytes) segs.push_back(CopySeg{static_cast<const unsigned*>(from),
                                      static_cast<unsigned*>(to),
                                      static_cast<long long>(bytes / 4)});
  };
  for (size_t i = 0; i < boxes.size(); i++) {
    const BoxDevView& v = src[i];
    const size_t k = v.k, r = v.r;
    BoxDev& bd = boxdev_[boxes[i]];
    double* fac;
    KI_ALLOC(fac, double, 3 * k * r + r * r + k * k);
    KI_ALLOC(bd.piv, int, r);
    bd.T = fac;
    bd.L = bd.T + k * r;
    bd.U = bd.L + k * r;
    bd.X = bd.U + k * r;
    bd.acc = bd.X + r * r;
    seg(v.T, bd.T, sizeof(double) * k * r);
    seg(v.L, bd.L, sizeof(double) * k * r);
    seg(v.U, bd.U, sizeof(double) * k * r);
    seg(v.X, bd.X, sizeof(double) * r * r);
    seg(v.acc, bd.acc, sizeof(double) * k * k);
    seg(v.piv, bd.piv, sizeof(int) * r);
  }
  if (segs.empty()) return 0;
  CopySeg* d_segs;
  KI_ALLOC(d_segs, CopySeg, segs.size());
  KI_UPLOAD(d_segs, segs, stream_);
  KI_CUDA(launch_copy_segments(d_segs, static_cast<int>(segs.size()), stream_));
  return 0;
}

int Solver::update(int n_points, const double* points, const double* normals,
                   const double* curvatures, const double* weights, int n_holes,
                   const double* holes, int* n_reused) {
  if (n_trees() > 1) return fail("update: not available for a batch of problems");
  if (tree.boxes.empty()) return fail("update: factor the boundary first");
  if (n_points <= 0) return fail("number of boundary points to init tree cannot be 0");
  // nothing queued may still read the memory that is about to be replaced
  KI_CUDA(cudaStreamSynchronize(stream_));
  if (dstream_) KI_CUDA(cudaStreamSynchronize(dstream_));
  if (ustream_) KI_CUDA(cudaStreamSynchronize(ustream_));
  {
    // no queued copy reads the staging any more: its chunks go back to the
    // pool and the refactorization stages into a fresh arena
    Arena fresh(true);
    fresh.swap(stage_);
  }
  cudaEvent_t ev0;
  int rc = begin_factor(&ev0);
  if (rc) return rc;
  const std::vector<double> old_pts = pts_;
  const int n_old = n_points_;
  n_points_ = n_points;
  n_dofs_ = n_points * sd_;
  pts_.assign(points, points + 2 * static_cast<size_t>(n_points));
  nrm_.assign(normals, normals + 2 * static_cast<size_t>(n_points));
  curv_.assign(curvatures, curvatures + n_points);
  wts_.assign(weights, weights + n_points);
  holes_.clear();
  if (n_holes > 0) holes_.assign(holes, holes + 4 * static_cast<size_t>(n_holes));
  tree.perturb(old_pts.data(), n_old, pts_.data(), n_points_);

  // the boxes that stay compressed keep their factors: copied out of the
  // old arena into a fresh one, after which the old arena is released
  std::vector<int> kept;
  std::vector<BoxDevView> views;
  for (const std::vector<int>& lv : tree.levels)
    for (int id : lv)
      if (tree.boxes[id].compressed) {
        const BoxDev& bd = boxdev_[id];
        const Box& b = tree.boxes[id];
        kept.push_back(id);
        views.push_back(BoxDevView{bd.T, bd.L, bd.U, bd.X, bd.acc, bd.piv, b.rank,
                                   static_cast<int>(b.redundant.size())});
      }
  Arena old;
  old.swap(arena_);
  drop_device_state();
  std::vector<BoxDev> old_dev;
  old_dev.swap(boxdev_);
  boxdev_.assign(tree.boxes.size(), BoxDev{});
  rc = adopt_factors(kept, views);
  if (rc) return rc;
  KI_CUDA(cudaStreamSynchronize(stream_));
  if (n_reused) *n_reused = static_cast<int>(kept.size());
  return finish_factor(ev0);
}

Solver* Solver::copy(cudaStream_t stream, int* rc) {
  *rc = 0;
  if (n_trees() > 1 || tree.boxes.empty()) {
    *rc = fail("copy: needs a factored single problem");
    return nullptr;
  }
  Solver* c = new Solver(opt_, n_points_, pts_.data(), nrm_.data(), curv_.data(), wts_.data(),
                         n_holes(), holes_.empty() ? nullptr : holes_.data(), stream);
  c->time_phases = time_phases;
  cudaEvent_t ev0;
  int r = c->begin_factor(&ev0);
  if (!r) {
    // this solver's queued work must finish before its factors are read
    // on the other stream
    r = c->cuda_check(cudaStreamSynchronize(stream_), "cudaStreamSynchronize");
  }
  if (!r) {
    c->tree = tree;
    c->boxdev_.assign(tree.boxes.size(), BoxDev{});
    std::vector<int> kept;
    std::vector<BoxDevView> views;
    for (const std::vector<int>& lv : tree.levels)
      for (int id : lv)
        if (tree.boxes[id].compressed) {
          const BoxDev& bd = boxdev_[id];
          kept.push_back(id);
          views.push_back(BoxDevView{bd.T, bd.L, bd.U, bd.X, bd.acc, bd.piv, tree.boxes[id].rank,
                                     static_cast<int>(tree.boxes[id].redundant.size())});
        }
    r = c->adopt_factors(kept, views);
  }
  if (!r) r = c->finish_factor(ev0);
  if (r) {
    error = c->error;
    *rc = r;
    delete c;
    return nullptr;
  }
  return c;
}

int Solver::build_all_compressed() {
  // concatenated sweep tasks of every compressed box for the diagonal solves
  std::vector<SweepTask> all;
  int cap = 0;
  for (LevelFactors& lf : levels_) {
    if (!lf.ntasks) continue;
    all.insert(all.end(), lf.h_tasks.begin(), lf.h_tasks.end());
    cap = std::max(cap, lf.cap);
  }
  // the boxes (disjoint redundant dofs, any order) by descending r: the
  // large ones first, then those whose X^{-1} a single-right-hand-side
  // diagonal solve stages in shared memory (a launch of their own)
  std::stable_sort(all.begin(), all.end(),
                   [](const SweepTask& a, const SweepTask& b) { return a.r > b.r; });
  int nbig = 0, kr = 0;
  for (const SweepTask& t : all) {
    if (static_cast<long long>(t.r) * t.r > kDiagStageMaxR * kDiagStageMaxR) {
      nbig++;
    } else {
      kr = std::max(kr, t.r * t.r);
    }
  }
  all_compressed_.ntasks = static_cast<int>(all.size());
  all_compressed_.cap = cap;
  all_compressed_.nbig = nbig;
  all_compressed_.kr = kr;
  KI_ALLOC(all_compressed_.d_tasks, SweepTask, all.size());
  KI_UPLOAD(all_compressed_.d_tasks, all, stream_);
  return 0;
}

int Solver::diag_all(SweepParams dp, bool trans) {
  // every compressed box's x_r <- X_rr^{-1} x_r: the boxes too large to
  // stage X^{-1}, then (one right-hand side) the others with it staged
  const LevelFactors& ac = all_compressed_;
  auto run = [&](const SweepParams& p) {
    return trans ? launch_diag_solve_t(p, stream_) : launch_diag_solve(p, stream_);
  };
  if (dp.nrhs != 1 || ac.nbig == ac.ntasks || ac.kr == 0) {
    KI_CUDA(run(dp));
    return 0;
  }
  SweepParams big = dp, small = dp;
  big.ntasks = ac.nbig;
  small.tasks = dp.tasks + ac.nbig;
  small.ntasks = ac.ntasks - ac.nbig;
  small.kr = ac.kr;
  if (big.ntasks) KI_CUDA(run(big));
  KI_CUDA(run(small));
  return 0;
}

int Solver::factor_top_forest() {
  // skel_factorization.cpp:116-128 for every tree: its root's active dofs,
  // the accumulated updates of the root's children, one LU per tree.
  if (build_all_compressed()) return -2;
  const int P = static_cast<int>(tree.roots.size());
  std::vector<int> dofs, bid, bpos;
  std::vector<UpdBlock> tab;
  std::vector<size_t> d_off(P), b_off(P), t_off(P), a_off(P), p_off(P);
  size_t a_total = 0, p_total = 0;
  forest_nmax_ = 0;
  for (int p = 0; p < P; p++) {
    const Box& root = tree.boxes[tree.roots[p]];
    const int n = static_cast<int>(root.active.size());
    std::vector<BoxBlock> blocks;
    if (!root.leaf) {
      int off = 0;
      for (int q = 0; q < 4; q++) {
        const int ch = root.child[q];
        for (const BoxBlock& x : blocks_of(ch)) blocks.push_back(BoxBlock{x.acc, x.size, x.pos + off});
        const Box& cb = tree.boxes[ch];
        off += static_cast<int>(cb.compressed ? cb.skel.size() : cb.active.size());
      }
    }
    std::vector<int> tb, tp;
    std::vector<UpdBlock> tt;
    build_block_map(blocks, n, &tb, &tp, &tt);
    d_off[p] = dofs.size();
    b_off[p] = bid.size();
    t_off[p] = tab.size();
    a_off[p] = a_total;
    p_off[p] = p_total;
    dofs.insert(dofs.end(), root.active.begin(), root.active.end());
    bid.insert(bid.end(), tb.begin(), tb.end());
    bpos.insert(bpos.end(), tp.begin(), tp.end());
    tab.insert(tab.end(), tt.begin(), tt.end());
    a_total += static_cast<size_t>(n) * n;
    p_total += n;
    forest_nmax_ = std::max(forest_nmax_, n);
  }
  if (static_cast<size_t>(forest_nmax_) * sizeof(double) > 200 * 1024)
    return fail("a forest tree's top skeleton is too large for the batched top solve");
  int *d_dofs, *d_bid, *d_bpos, *d_piv;
  UpdBlock* d_tab;
  double* d_a;
  KI_ALLOC(d_dofs, int, dofs.size());
  KI_ALLOC(d_bid, int, bid.size());
  KI_ALLOC(d_bpos, int, bpos.size());
  KI_ALLOC(d_tab, UpdBlock, tab.size());
  KI_ALLOC(d_a, double, a_total);
  KI_ALLOC(d_piv, int, p_total);
  KI_ALLOC(d_forest_, TopTask, P);
  std::vector<TopTask> tasks(P);
  for (int p = 0; p < P; p++) {
    const int n = static_cast<int>(tree.boxes[tree.roots[p]].active.size());
    tasks[p] = TopTask{n, 0, d_dofs + d_off[p], d_bid + b_off[p], d_bpos + b_off[p],
                       d_tab + t_off[p], d_a + a_off[p], d_piv + p_off[p]};
  }
  KI_UPLOAD(d_dofs, dofs, stream_);
  KI_UPLOAD(d_bid, bid, stream_);
  KI_UPLOAD(d_bpos, bpos, stream_);
  KI_UPLOAD(d_tab, tab, stream_);
  KI_UPLOAD(d_forest_, tasks, stream_);
  ns_ = static_cast<int>(allskel.size());
  KI_ALLOC(d_tmp_, double, 4 * static_cast<size_t>(n_dofs_) + 64);
  cudaEvent_t l0 = nullptr;
  if (time_phases && timer_begin(&l0)) return -2;
  KI_CUDA(launch_forest_top(opt_.pde, d_nodes_, d_forest_, P, forest_nmax_, d_status_, stream_));
  if (time_phases && timer_end(l0, {0, 4, 1, P, 0, forest_nmax_, 0.0})) return -2;
  return 0;
}

int Solver::factor_top() {
  if (build_all_compressed()) return -2;
  ns_ = static_cast<int>(allskel.size());
  KI_ALLOC(d_allskel_, int, ns_);
  KI_UPLOAD(d_allskel_, allskel, stream_);
  std::vector<BoxBlock> blocks;
  {
    const Box& root = tree.boxes[0];
    if (!root.leaf) {
      int off = 0;
      for (int q = 0; q < 4; q++) {
        const int ch = root.child[q];
        for (const BoxBlock& x : blocks_of(ch)) blocks.push_back(BoxBlock{x.acc, x.size, x.pos + off});
        const Box& cb = tree.boxes[ch];
        off += static_cast<int>(cb.compressed ? cb.skel.size() : cb.active.size());
      }
    }
  }
  std::vector<int> bid, bpos;
  std::vector<UpdBlock> tab;
  build_block_map(blocks, ns_, &bid, &bpos, &tab);
  int *d_bid, *d_bpos;
  UpdBlock* d_tab;
  KI_ALLOC(d_bid, int, bid.size());
  KI_ALLOC(d_bpos, int, bpos.size());
  KI_ALLOC(d_tab, UpdBlock, tab.size());
  KI_UPLOAD(d_bid, bid, stream_);
  KI_UPLOAD(d_bpos, bpos, stream_);
  KI_UPLOAD(d_tab, tab, stream_);
  const int ntop = ns_ + nb_;
  top_flops += 20.0 * ns_ * ns_ + 2.0 / 3.0 * static_cast<double>(ntop) * ntop * ntop;
  solve_bytes += 8.0 * ntop * ntop + 8.0 * 8.0 * n_dofs_;
  KI_ALLOC(d_top_, double, static_cast<size_t>(ntop) * ntop);
  KI_ALLOC(d_top_piv_, int, ntop);
  KI_ALLOC(d_top_perm_, int, ntop);
  KI_ALLOC(d_tmp_, double, 4 * static_cast<size_t>(n_dofs_ + ntop) + 64);
  KI_CUDA(launch_assemble_top(opt_.pde, d_nodes_, d_allskel_, ns_, d_bid, d_bpos, d_tab, d_top_,
                              ntop, stream_));
  if (nb_ > 0) {
    const int rc = factor_border();
    if (rc) return rc;
  }
  cudaEvent_t l0 = nullptr;
  if (time_phases && timer_begin(&l0)) return -2;
  int* lu_sync;
  KI_ALLOC(lu_sync, int, kLuSyncInts);
  if (ntop > 0)
    KI_CUDA(dense_lu(d_top_, ntop, ntop, d_top_piv_, d_status_, stream_, lu_sync, true));
  // the interchanges composed once, so each solve gathers instead, and the
  // factors' 16 x 16 diagonal blocks inverted, so each solve multiplies
  // instead of substituting within a block
  if (ntop > 0) KI_CUDA(launch_pivots_to_perm(d_top_piv_, ntop, d_top_perm_, stream_));
  if (ntop > 0 && ntop <= kLuBlockInvMaxN) {
    KI_ALLOC(d_top_dinv_, double, lu_block_inv_doubles(ntop));
    KI_CUDA(launch_lu_block_inv(d_top_, ntop, ntop, d_top_dinv_, stream_));
  }
  if (time_phases && timer_end(l0, {0, 4, 1, 1, 0, ntop, 0.0})) return -2;
  return 0;
}

int Solver::factor_border() {
  // skel_factorization.cpp:130-242: sweep U and Psi^T with the factors,
  // D^{-1} on the redundant rows, then the bordered Schur system S.
  const int N = n_dofs_, nb = nb_, ns = ns_;
  // the redundant dofs (everything outside the top level's skeletons) and
  // each dof's position among them, listed on the GPU from the sorted
  // skeletons: no N-long host lists on the way to the top-level LU
  std::vector<int> sorted = allskel;
  std::sort(sorted.begin(), sorted.end());
  for (size_t i = 0; i < sorted.size(); i++)
    if (sorted[i] < 0 || sorted[i] >= N || (i > 0 && sorted[i] == sorted[i - 1]))
      return fail("top-level skeleton dofs out of range or repeated");
  const int nr = N - static_cast<int>(sorted.size());
  if (nr <= 0) return fail("No compression possible");
  n_red_ = nr;
  int* d_sorted;
  KI_ALLOC(d_sorted, int, sorted.size());
  KI_ALLOC(d_allred_, int, nr);
  KI_ALLOC(d_red_pos_, int, N);
  KI_UPLOAD(d_sorted, sorted, stream_);
  KI_CUDA(launch_red_index(d_sorted, static_cast<int>(sorted.size()), N, d_allred_, d_red_pos_,
                           stream_));

  // U and Psi^T were swept up level by level with the decoupling
  double* modU = d_modU_;
  double* modP = d_modP_;
  cudaEvent_t b0 = nullptr;
  if (time_phases && timer_begin(&b0)) return -2;
  double *dinv, *us, *ps, *corr;
  KI_ALLOC(d_Ured_, double, static_cast<size_t>(nr) * nb);
  KI_ALLOC(d_Pred_, double, static_cast<size_t>(nr) * nb);
  KI_ALLOC(dinv, double, static_cast<size_t>(nr) * nb);
  KI_ALLOC(us, double, static_cast<size_t>(ns) * nb);
  KI_ALLOC(ps, double, static_cast<size_t>(ns) * nb);
  KI_ALLOC(corr, double, static_cast<size_t>(nb) * nb);
  KI_CUDA(cudaStreamWaitEvent(stream_, ev_bdr_, 0));  // U, Psi^T swept up
  // (dinv: X_rr^{-1} U_r of every compressed box, solved level by level)
  KI_CUDA(launch_border_gather(modU, modP, d_modD_, nb, d_allred_, nr, d_allskel_, ns, d_Ured_,
                               d_Pred_, dinv, us, ps, stream_));
  if (const int splits = long_gemm_tn_splits(nb, nb, nr)) {
    double* part;
    KI_ALLOC(part, double, static_cast<size_t>(splits) * nb * nb);
    KI_CUDA(long_gemm_tn(nb, nb, nr, 1.0, d_Pred_, nr, dinv, nr, 0.0, corr, nb, part, stream_));
  } else {
    KI_CUDA(small_gemm(true, false, nb, nb, nr, 1.0, d_Pred_, nr, dinv, nr, 0.0, corr, nb,
                       stream_));
  }
  KI_CUDA(launch_fill_border(d_top_, ns + nb, ns, nb, us, ps, corr, stream_));
  if (time_phases && timer_end(b0, {0, 3, 1, nb, 0, N, 0.0})) return -2;
  return 0;
}

int Solver::solve_device(const double* d_b, double* d_mu, double* d_alpha, const double* d_g) {
  const int N = n_dofs_;
  double* x = d_mu;
  if (d_b != d_mu)
    KI_CUDA(cudaMemcpyAsync(x, d_b, sizeof(double) * N, cudaMemcpyDeviceToDevice, stream_));
  // the top-level LU into L2 while the up sweeps run (its substitution is
  // a chain of dependent blocks, each waiting on its loads)
  if (d_top_ && !d_forest_)
    KI_CUDA(launch_l2_prefetch(d_top_, sizeof(double) * static_cast<size_t>(ns_ + nb_) * (ns_ + nb_),
                               stream_));
  const int L = static_cast<int>(levels_.size());
  for (int l = L - 1; l >= 0; l--) {
    const LevelFactors& lf = levels_[l];
    if (!lf.ntasks) continue;
    SweepParams sp{lf.d_tasks, lf.ntasks, x, N, 1, 0, nullptr, lf.cap};
    sp.kr = lf.kr;
    KI_CUDA(launch_sweep_up(sp, false, stream_));
  }
  const int ns = ns_, nb = nb_;
  if (d_forest_) {
    SweepParams dp{all_compressed_.d_tasks, all_compressed_.ntasks, x, N, 1, 0, nullptr,
                   all_compressed_.cap};
    if (diag_all(dp, false)) return -2;
    KI_CUDA(launch_forest_top_solve(d_forest_, n_trees(), forest_nmax_, x, stream_));
  } else if (nb == 0) {
    SweepParams dp{all_compressed_.d_tasks, all_compressed_.ntasks, x, N, 1, 0, nullptr,
                   all_compressed_.cap};
    if (diag_all(dp, false)) return -2;
    if (ns > 0) {
      KI_CUDA(launch_gather(x, N, d_allskel_, ns, 1, d_tmp_, ns, stream_));
      KI_CUDA(dense_lu_solve(d_top_, ns, ns, d_top_piv_, d_tmp_, 1, ns, stream_, d_top_perm_,
                             d_top_dinv_));
      KI_CUDA(launch_scatter(x, N, d_allskel_, ns, 1, d_tmp_, ns, stream_));
    }
  } else {
    const int nr = n_red_;
    double* w = d_tmp_;
    double* dw = w + nr;
    double* M = dw + nr;
    KI_CUDA(launch_gather(x, N, d_allred_, nr, 1, w, nr, stream_));
    KI_CUDA(launch_gather(x, N, d_allskel_, ns, 1, M, ns, stream_));
    KI_CUDA(cudaMemcpyAsync(dw, w, sizeof(double) * nr, cudaMemcpyDeviceToDevice, stream_));
    SweepParams dp{all_compressed_.d_tasks, all_compressed_.ntasks, dw, nr, 1, 1, d_red_pos_,
                   all_compressed_.cap};
    if (diag_all(dp, false)) return -2;
    // border rows of the reduced system: g - Psi~_r D^-1 w_r (the nb dot
    // products in one pass over the rows, partials behind M)
    if (nb <= kMaxKrylov) {
      KI_CUDA(launch_multi_dot(d_Pred_, nr, nb, dw, nr, M + ns + nb, M + ns, stream_));
      KI_CUDA(launch_rsub(M + ns, d_g, nb, stream_));
    } else {
      if (d_g)
        KI_CUDA(cudaMemcpyAsync(M + ns, d_g, sizeof(double) * nb, cudaMemcpyDeviceToDevice,
                                stream_));
      KI_CUDA(small_gemm(true, false, nb, 1, nr, -1.0, d_Pred_, nr, dw, nr, d_g ? 1.0 : 0.0,
                         M + ns, nb, stream_));
    }
    KI_CUDA(dense_lu_solve(d_top_, ns + nb, ns + nb, d_top_piv_, M, 1, ns + nb, stream_,
                           d_top_perm_, d_top_dinv_));
    if (d_alpha)
      KI_CUDA(cudaMemcpyAsync(d_alpha, M + ns, sizeof(double) * nb, cudaMemcpyDeviceToDevice,
                              stream_));
    KI_CUDA(small_gemm(false, false, nr, 1, nb, -1.0, d_Ured_, nr, M + ns, nb, 1.0, w, nr, stream_));
    dp.x = w;
    if (diag_all(dp, false)) return -2;
    KI_CUDA(launch_scatter(x, N, d_allred_, nr, 1, w, nr, stream_));
    KI_CUDA(launch_scatter(x, N, d_allskel_, ns, 1, M, ns, stream_));
  }
  for (int l = 0; l < L; l++) {
    const LevelFactors& lf = levels_[l];
    if (!lf.ntasks) continue;
    SweepParams sp{lf.d_tasks, lf.ntasks, x, N, 1, 0, nullptr, lf.cap};
    sp.kr = lf.kr;
    KI_CUDA(launch_sweep_down(sp, stream_));
  }
  return 0;
}

int Solver::apply_device(const double* d_x, double* d_y) {
  const bool forest = starts_.size() > 2;
  if (forest && mv_setup()) return -2;
  KI_CUDA(launch_apply_operator(opt_.pde, d_nodes_, n_dofs_, forest ? d_seg_ : nullptr,
                                static_cast<int>(seg_.size()) - 1, d_x, d_y, nb_, d_U_, d_Psi_,
                                stream_));
  return 0;
}

}  // namespace kib
