// Batch engine: many independent 3D OSEM jobs on one GPU (continuous batching).
//
// A job moves through   queued -> uploading -> counting -> running -> final ->
// downloading -> done.  apirl_batch_step takes each transition once the GPU
// work of the previous stage has finished (per-job events; the engine never
// synchronises its streams while jobs run), then launches one batched EM step:
// one pass of every running job, or its final likelihood, in four launches
// whatever the number of jobs (padded image copies and image dot products; a
// persistent walk over the concatenated lists of all jobs' bins with counts;
// the likelihood sums; the EM updates).
//
// * Device memory comes from a private stream-ordered pool that keeps what it
//   has reserved, so jobs coming and going allocate nothing from the driver
//   once the pool has grown to the working set.
// * Counts, factors and initial images go up from a worker thread on a copy
//   stream, so that a large job's upload overlaps the other jobs' steps.
// * Each job's lists of bins with counts (one per subset) are built once, when
//   its counts arrive; its passes walk only those bins (the geometry form of
//   the sparse pass: the likelihood's sum over the other bins comes from the
//   image dot product with G_s = A_s^T 1).
// * Geometry products are shared between jobs of the same image and sinogram
//   geometry: the LOR tables, and A_a^T 1 for every angle a, from which the
//   sensitivity images of any subset split (without a multiplicative term,
//   sens_s = G_s = the sum of A_a^T 1 over the subset's angles) and A^T 1 of
//   the final likelihood follow by summing images, without another walk.
//   When those per-angle images do not fit the budget, each split's images
//   are made by one walk of the whole sinogram instead.
#include <cuda_runtime.h>
#include <algorithm>
#include <atomic>
#include <condition_variable>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <tuple>
#include <vector>
#include "internal.h"
#include "../../include/apirl_b200.h"

using apirl::ImgGeom;
using apirl::LorTable;
using apirl::MultiSeg;
using apirl::MultiVox;
using apirl::PadBuffers;
using apirl::SensJob;
using apirl::SubsetSel;

namespace {

apirl_status bfail(apirl_status code, const char* what, cudaError_t e = cudaSuccess) {
  char buf[320];
  snprintf(buf, sizeof buf, "%s%s%s", what, e == cudaSuccess ? "" : ": ", e == cudaSuccess ? "" : cudaGetErrorString(e));
  return apirl_internal_fail(code, buf);
}

#define BK(call)                                                                                      \
  do {                                                                                                \
    cudaError_t e_ = (call);                                                                          \
    if (e_ != cudaSuccess) return bfail(e_ == cudaErrorMemoryAllocation ? APIRL_ERR_OOM : APIRL_ERR_CUDA, #call, e_); \
  } while (0)
#define BS(call)                   \
  do {                             \
    apirl_status s_ = (call);      \
    if (s_ != APIRL_OK) return s_; \
  } while (0)

size_t count_elem_size(int dtype) { return dtype == APIRL_U16 ? 2 : 4; }
int64_t align256(int64_t b) { return (b + 255) & ~(int64_t)255; }
int64_t padded_voxels(const apirl_image_geom& g) {
  return (int64_t)(g.nx + 2 * apirl::kPad) * (g.ny + 2 * apirl::kPad) * (g.nz + 2 * apirl::kPad);
}
int n_tiles_of(int64_t bins) { return (int)((bins + apirl::kNzTile - 1) / apirl::kNzTile); }

// Device bytes a job holds while active, its lists at their largest (every
// bin with counts) and its subset split's sensitivity images included.
int64_t footprint_of(const apirl_image_geom& img, const apirl_sino3d_geom& sino, int dtype, bool mult, bool add,
                     int nsub, int64_t nbins, int iters) {
  const int64_t nv = (int64_t)img.nx * img.ny * img.nz;
  const int ns = nsub > 0 ? nsub : 1;
  int64_t b = align256(nbins * (int64_t)count_elem_size(dtype));
  if (mult) b += align256(nbins * 4) + align256(nv * 4 * ns);  // factors, own sensitivity images
  if (add) b += align256(nbins * 4);
  b += align256(nv * 4);                                       // image
  b += 4 * align256(padded_voxels(img) * 4);                   // padded copies and backprojection pair
  b += align256(nbins * 4);                                    // lists of the bins with counts (at most every bin)
  b += align256(((int64_t)ns * (nbins / (sino.n_proj > 0 ? sino.n_proj : 1) * ((sino.n_proj + ns - 1) / ns) /
                 apirl::kNzTile + 2)) * 4);                     // list tiles
  b += align256(((int64_t)iters * ns + 1) * 8) + align256(ns * 12);
  b += align256(nv * 4 * ns);                                  // G_s of the split (shared between jobs)
  return b;
}

// ---- device memory -------------------------------------------------------------
// A private stream-ordered pool whose release threshold keeps every byte it
// has reserved: freed blocks are reused by later allocations on the stream.
struct Pool {
  cudaMemPool_t pool = nullptr;
  cudaError_t create(int device) {
    cudaMemPoolProps props;
    memset(&props, 0, sizeof props);
    props.allocType = cudaMemAllocationTypePinned;
    props.handleTypes = cudaMemHandleTypeNone;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = device;
    cudaError_t e = cudaMemPoolCreate(&pool, &props);
    if (e != cudaSuccess) return e;
    uint64_t keep = ~(uint64_t)0;
    return cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
  }
  // Reserves `bytes` of device memory into the pool up front (one block
  // allocated and returned to it), so that later allocations map nothing.
  cudaError_t reserve(size_t bytes, cudaStream_t st) {
    void* p = nullptr;
    cudaError_t e = cudaMallocFromPoolAsync(&p, bytes, pool, st);
    if (e != cudaSuccess) return e;
    if ((e = cudaFreeAsync(p, st)) != cudaSuccess) return e;
    return cudaStreamSynchronize(st);
  }
  template <typename T> cudaError_t alloc(T** p, int64_t n, cudaStream_t st) {
    *p = nullptr;
    if (n <= 0) return cudaSuccess;
    return cudaMallocFromPoolAsync((void**)p, (size_t)n * sizeof(T), pool, st);
  }
  template <typename T> void release(T*& p, cudaStream_t st) {
    if (p) cudaFreeAsync((void*)p, st);
    p = nullptr;
  }
};

// Page-locked host memory for results, descriptors and staging: chunks of
// at least 256 MB, carved first-fit (256-byte units) and coalesced on return,
// so that jobs coming and going do not page-lock memory each time.
struct PinnedPool {
  static constexpr size_t kChunk = (size_t)256 << 20;
  struct Chunk {
    char* base;
    size_t size;
    std::map<size_t, size_t> free_at;  // offset -> length
  };
  std::vector<Chunk> chunks;
  std::map<void*, std::pair<size_t, size_t>> used;  // block -> (chunk, length)

  bool grow(size_t bytes) {
    Chunk c;
    c.size = std::max(kChunk, bytes);
    void* p = nullptr;
    if (cudaMallocHost(&p, c.size) != cudaSuccess) {
      (void)cudaGetLastError();  // handled here: the caller reports it, or tries a smaller size
      return false;
    }
    c.base = (char*)p;
    c.free_at[0] = c.size;
    chunks.push_back(std::move(c));
    return true;
  }
  void* get(size_t bytes) {
    bytes = (std::max<size_t>(bytes, 1) + 255) & ~(size_t)255;
    for (int pass = 0; pass < 2; pass++) {
      for (size_t k = 0; k < chunks.size(); k++) {
        Chunk& c = chunks[k];
        for (auto it = c.free_at.begin(); it != c.free_at.end(); ++it) {
          if (it->second < bytes) continue;
          const size_t off = it->first, len = it->second;
          c.free_at.erase(it);
          if (len > bytes) c.free_at[off + bytes] = len - bytes;
          void* p = c.base + off;
          used[p] = {k, bytes};
          return p;
        }
      }
      if (pass == 0 && !grow(bytes)) return nullptr;
    }
    return nullptr;
  }
  void put(void* p) {
    if (!p) return;
    auto u = used.find(p);
    if (u == used.end()) return;
    Chunk& c = chunks[u->second.first];
    size_t off = (size_t)((char*)p - c.base), len = u->second.second;
    used.erase(u);
    auto next = c.free_at.lower_bound(off);
    if (next != c.free_at.end() && next->first == off + len) {
      len += next->second;
      next = c.free_at.erase(next);
    }
    if (next != c.free_at.begin()) {
      auto prev = std::prev(next);
      if (prev->first + prev->second == off) {
        prev->second += len;
        return;
      }
    }
    c.free_at[off] = len;
  }
  ~PinnedPool() {
    for (auto& c : chunks) cudaFreeHost(c.base);
  }
};

// ---- shared geometry products ---------------------------------------------------
struct GeomKey {
  int nx, ny, nz, n_proj, n_r, n_rings, scanner;
  float dx, dy, dz, r_fov, axial_fov, r_scanner;
  std::vector<int> mn, mx;
  auto tie() const {
    return std::tie(nx, ny, nz, n_proj, n_r, n_rings, scanner, dx, dy, dz, r_fov, axial_fov, r_scanner, mn, mx);
  }
  bool operator<(const GeomKey& o) const { return tie() < o.tie(); }
};

struct SensSet {
  float* g = nullptr;  // nsub images of A_s^T 1
  int refs = 0;
  uint64_t last_use = 0;
};

struct Geom {
  GeomKey key;
  ImgGeom g{};                   // the image geometry as the walk takes it
  LorTable t{};                  // LOR end points and end-point z, on the device (pool)
  std::vector<float> host_lor;   // the LOR table on the host, [angle][r] (p1x, p1y, p2x, p2y)
  void* h_tables = nullptr;      // page-locked copy of the tables, the source of their upload
  int64_t nvox = 0, nbins = 0;
  // A_a^T 1 of every angle a (padded images of pv voxels, [z][x][y] where
  // tr[a], else [z][y][x]), then A^T 1 (unpadded); or A^T 1 alone.
  float* per_angle = nullptr;
  float* g_total = nullptr;      // inside the per_angle block
  int64_t per_angle_held = 0;    // bytes of the per_angle block
  bool per_angle_tried = false;
  int64_t pv = 0;                // voxels of a padded image
  uint8_t* h_tr = nullptr;       // page-locked: per angle, 1 when its rays run mostly along x
  uint8_t* d_tr = nullptr;
  std::map<int, SensSet> sets;   // subset count -> its G_s images
  int refs = 0;                  // active jobs of this geometry
  uint64_t last_use = 0;
  int64_t per_angle_bytes() const { return align256(((int64_t)key.n_proj * pv + nvox) * 4); }
};

enum class Stage { Queued, Uploading, Counting, Running, Final, Download, Done };

struct Job {
  int64_t id = 0;
  apirl_image_geom img{};
  apirl_sino3d_geom sino{};
  std::vector<int> mn, mx;
  const void* h_counts = nullptr;  // caller's arrays, read when the job is uploaded
  const float *h_mult = nullptr, *h_add = nullptr, *h_init = nullptr;
  int dtype = APIRL_F32;
  int iters = 0, nsub = 1;
  bool positive = false;  // update where sens > 0 (else the reference's sens >= 0)
  int64_t nbins = 0, nvox = 0, footprint = 0, charged = 0;
  Stage stage = Stage::Queued;
  int pass = 0;
  Geom* geom = nullptr;
  SensSet* set = nullptr;
  // device
  void* d_counts = nullptr;
  float *d_mult = nullptr, *d_add = nullptr, *d_x = nullptr, *d_sens = nullptr;
  double* d_lik = nullptr;
  double* d_zero_add = nullptr;
  int* d_tiles = nullptr;
  int* d_nlist = nullptr;
  int* d_list = nullptr;
  PadBuffers pad;
  std::vector<int64_t> tile_off, list_off;
  std::vector<int> n_list;
  std::vector<double> zero_add;
  // host
  void* h_stage = nullptr;   // pinned: n_list (nsub ints), zero_add (nsub doubles)
  float* h_out = nullptr;    // pinned result image
  double* h_lik = nullptr;   // pinned likelihoods
  cudaEvent_t ev = nullptr;  // end of the current stage's GPU work
  cudaEvent_t alloc_ev = nullptr, up_ev = nullptr;
  std::atomic<int> uploaded{0};    // the worker has queued the copies (1) or failed (-1)
  std::vector<float> out;
  std::vector<double> lik;
};

// memcpy of large host blocks split over a few threads (one pageable-memory
// stream per thread is far below the host's memory bandwidth).
class ParallelCopy {
 public:
  void start(int threads) {
    for (int k = 1; k < threads; k++) th_.emplace_back([this, k] { run(k); });
    parts_.resize((size_t)threads);
  }
  ~ParallelCopy() {
    {
      std::lock_guard<std::mutex> lk(mu_);
      stop_ = true;
    }
    cv_.notify_all();
    for (auto& t : th_) t.join();
  }
  void copy(void* dst, const void* src, size_t n) {
    const size_t np = parts_.size();
    if (np <= 1 || n < ((size_t)4 << 20)) {
      memcpy(dst, src, n);
      return;
    }
    const size_t per = ((n / np) + 4095) & ~(size_t)4095;
    {
      std::lock_guard<std::mutex> lk(mu_);
      for (size_t k = 0; k < np; k++) {
        const size_t lo = std::min(n, k * per), hi = std::min(n, lo + per);
        parts_[k] = Part{(char*)dst + lo, (const char*)src + lo, hi - lo};
      }
      pending_ = (int)np - 1;
      gen_++;
    }
    cv_.notify_all();
    memcpy(parts_[0].d, parts_[0].s, parts_[0].n);
    std::unique_lock<std::mutex> lk(mu_);
    done_.wait(lk, [&] { return pending_ == 0; });
  }

 private:
  struct Part {
    char* d;
    const char* s;
    size_t n;
  };
  void run(int k) {
    uint64_t seen = 0;
    for (;;) {
      Part p;
      {
        std::unique_lock<std::mutex> lk(mu_);
        cv_.wait(lk, [&] { return stop_ || gen_ != seen; });
        if (stop_) return;
        seen = gen_;
        p = parts_[(size_t)k];
      }
      if (p.n) memcpy(p.d, p.s, p.n);
      {
        std::lock_guard<std::mutex> lk(mu_);
        if (--pending_ == 0) done_.notify_one();
      }
    }
  }
  std::vector<std::thread> th_;
  std::vector<Part> parts_;
  std::mutex mu_;
  std::condition_variable cv_, done_;
  uint64_t gen_ = 0;
  int pending_ = 0;
  bool stop_ = false;
};

// Uploads of admitted jobs' host arrays, on its own thread and copy stream:
// each array goes through a ring of page-locked staging buffers (host copy
// by several threads into one buffer while the DMA of the others runs), so
// that no pageable-memory copy holds up the thread that launches the steps.
struct Uploader {
  static constexpr size_t kChunk = (size_t)32 << 20;
  static constexpr int kRing = 4;
  std::thread th;
  std::mutex mu;
  std::condition_variable cv;
  std::deque<Job*> q;
  bool stop = false;
  cudaStream_t st = nullptr;
  int device = 0;
  void* ring[kRing] = {nullptr, nullptr, nullptr, nullptr};
  cudaEvent_t ring_ev[kRing] = {nullptr, nullptr, nullptr, nullptr};
  int next = 0;
  ParallelCopy pcopy;

  cudaError_t init(int dev, int copy_threads) {
    device = dev;
    cudaError_t e;
    if ((e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking)) != cudaSuccess) return e;
    for (int k = 0; k < kRing; k++) {
      if ((e = cudaMallocHost(&ring[k], kChunk)) != cudaSuccess) return e;
      if ((e = cudaEventCreateWithFlags(&ring_ev[k], cudaEventDisableTiming)) != cudaSuccess) return e;
    }
    pcopy.start(copy_threads);
    return cudaSuccess;
  }
  void release() {
    for (int k = 0; k < kRing; k++) {
      if (ring[k]) cudaFreeHost(ring[k]);
      if (ring_ev[k]) cudaEventDestroy(ring_ev[k]);
      ring[k] = nullptr;
      ring_ev[k] = nullptr;
    }
    if (st) cudaStreamDestroy(st);
    st = nullptr;
  }
  bool upload(void* dst, const void* src, size_t n) {
    for (size_t off = 0; off < n; off += kChunk) {
      const size_t len = std::min(kChunk, n - off);
      const int k = next;
      next = (next + 1) % kRing;
      if (cudaEventSynchronize(ring_ev[k]) != cudaSuccess) return false;  // its previous DMA is done
      pcopy.copy(ring[k], (const char*)src + off, len);
      if (cudaMemcpyAsync((char*)dst + off, ring[k], len, cudaMemcpyHostToDevice, st) != cudaSuccess) return false;
      if (cudaEventRecord(ring_ev[k], st) != cudaSuccess) return false;
    }
    return true;
  }
  void run() {
    cudaSetDevice(device);
    for (;;) {
      Job* j = nullptr;
      {
        std::unique_lock<std::mutex> lk(mu);
        cv.wait(lk, [&] { return stop || !q.empty(); });
        if (stop) return;
        j = q.front();
        q.pop_front();
      }
      bool ok = cudaStreamWaitEvent(st, j->alloc_ev, 0) == cudaSuccess;
      ok = ok && upload(j->d_counts, j->h_counts, (size_t)j->nbins * count_elem_size(j->dtype));
      if (ok && j->h_mult) ok = upload(j->d_mult, j->h_mult, (size_t)j->nbins * 4);
      if (ok && j->h_add) ok = upload(j->d_add, j->h_add, (size_t)j->nbins * 4);
      if (ok && j->h_init) ok = upload(j->d_x, j->h_init, (size_t)j->nvox * 4);
      ok = ok && cudaEventRecord(j->up_ev, st) == cudaSuccess;
      j->uploaded.store(ok ? 1 : -1);
    }
  }
  void push(Job* j) {
    {
      std::lock_guard<std::mutex> lk(mu);
      q.push_back(j);
    }
    cv.notify_one();
  }
  void shutdown() {
    {
      std::lock_guard<std::mutex> lk(mu);
      stop = true;
    }
    cv.notify_all();
    if (th.joinable()) th.join();
  }
};

}  // namespace

struct apirl_batch {
  int device = 0;
  int64_t budget = 0, used = 0;
  int64_t next_id = 0;
  uint64_t clock = 0;
  cudaStream_t st = nullptr;  // compute
  Pool pool;
  PinnedPool pinned;
  Uploader up;
  std::map<GeomKey, std::unique_ptr<Geom>> geoms;
  std::deque<std::unique_ptr<Job>> queue;
  std::vector<std::unique_ptr<Job>> active;
  std::map<int64_t, std::unique_ptr<Job>> finished;
  // batched-step scratch
  int walk_blocks = 0;
  unsigned long long* d_counter = nullptr;
  double* d_chunk_part = nullptr;
  int64_t cap_chunks = 0;
  double* d_tile_part = nullptr;
  int64_t cap_tiles = 0;
  MultiVox* d_vox = nullptr;
  MultiSeg* d_segs = nullptr;
  int cap_vox = 0, cap_segs = 0;
  MultiVox* h_vox[2] = {nullptr, nullptr};
  MultiSeg* h_segs[2] = {nullptr, nullptr};
  int h_cap_vox = 0, h_cap_segs = 0;
  cudaEvent_t step_ev[2] = {nullptr, nullptr};
  int64_t n_steps = 0;
};

namespace {

GeomKey key_of(const Job& j) {
  GeomKey k;
  k.nx = j.img.nx; k.ny = j.img.ny; k.nz = j.img.nz;
  k.dx = j.img.dx; k.dy = j.img.dy; k.dz = j.img.dz;
  k.n_proj = j.sino.n_proj; k.n_r = j.sino.n_r; k.n_rings = j.sino.n_rings; k.scanner = j.sino.scanner;
  k.r_fov = j.sino.r_fov; k.axial_fov = j.sino.axial_fov; k.r_scanner = j.sino.r_scanner;
  k.mn = j.mn; k.mx = j.mx;
  return k;
}

// Frees shared images no active job holds, least recently used first, until
// `need` more bytes fit the budget (or nothing is left to free).
void evict(apirl_batch* b, int64_t need) {
  for (;;) {
    if (b->used + need <= b->budget) return;
    Geom* best = nullptr;
    int best_set = 0;
    uint64_t oldest = ~(uint64_t)0;
    for (auto& kv : b->geoms) {
      Geom& g = *kv.second;
      for (auto& s : g.sets)
        if (s.second.refs == 0 && s.second.last_use < oldest) { oldest = s.second.last_use; best = &g; best_set = s.first; }
      if (g.per_angle && g.refs == 0 && g.last_use < oldest) { oldest = g.last_use; best = &g; best_set = 0; }
    }
    if (!best) return;
    if (best_set) {
      SensSet& s = best->sets[best_set];
      b->pool.release(s.g, b->st);
      b->used -= align256((int64_t)best_set * best->nvox * 4);
      best->sets.erase(best_set);
    } else {
      b->pool.release(best->per_angle, b->st);
      best->g_total = nullptr;  // lies in the same block
      best->per_angle_tried = false;
      b->used -= best->per_angle_held;
      best->per_angle_held = 0;
    }
  }
}

apirl_status geom_for(apirl_batch* b, Job& j, Geom** out) {
  GeomKey k = key_of(j);
  auto it = b->geoms.find(k);
  if (it == b->geoms.end()) {
    std::unique_ptr<Geom> g(new Geom);
    g->key = k;
    apirl_sino3d_geom sg = j.sino;
    sg.min_ring_diff = g->key.mn.data();
    sg.max_ring_diff = g->key.mx.data();
    {
      // The host half of a projector: checks and tables (no device buffers).
      apirl_projector tables;
      BS(apirl::setup_3d(&j.img, &sg, &tables));
      g->g = tables.g;
      g->t = tables.t;
      g->host_lor.swap(tables.host.lor);
      const size_t lor_b = g->host_lor.size() * sizeof(float), z_b = tables.host.z.size() * sizeof(float);
      g->h_tables = b->pinned.get(lor_b + z_b);
      if (!g->h_tables) return bfail(APIRL_ERR_OOM, "page-locked geometry tables");
      memcpy(g->h_tables, g->host_lor.data(), lor_b);
      memcpy((char*)g->h_tables + lor_b, tables.host.z.data(), z_b);
      float4* d_lor = nullptr;
      float2* d_z = nullptr;
      BK(b->pool.alloc(&d_lor, (int64_t)(lor_b / sizeof(float4)), b->st));
      BK(b->pool.alloc(&d_z, (int64_t)(z_b / sizeof(float2)), b->st));
      BK(cudaMemcpyAsync(d_lor, g->h_tables, lor_b, cudaMemcpyHostToDevice, b->st));
      BK(cudaMemcpyAsync(d_z, (char*)g->h_tables + lor_b, z_b, cudaMemcpyHostToDevice, b->st));
      g->t.lor = d_lor;
      g->t.z = d_z;
      g->t.ok = nullptr;
    }
    g->nvox = j.nvox;
    g->nbins = j.nbins;
    g->pv = padded_voxels(j.img);
    // Rays of one angle are parallel in x-y: the angle's middle ray decides
    // its image layout (the layout is a matter of speed, not of results).
    const int np = g->key.n_proj, nr = g->key.n_r;
    g->h_tr = (uint8_t*)b->pinned.get((size_t)np);
    if (!g->h_tr) return bfail(APIRL_ERR_OOM, "page-locked angle table");
    const float* lor = g->host_lor.data();
    for (int a = 0; a < np; a++) {
      const float* L = lor + ((size_t)a * nr + nr / 2) * 4;
      g->h_tr[a] = fabsf(L[2] - L[0]) >= fabsf(L[3] - L[1]) ? 1 : 0;
    }
    BK(b->pool.alloc(&g->d_tr, np, b->st));
    BK(cudaMemcpyAsync(g->d_tr, g->h_tr, (size_t)np, cudaMemcpyHostToDevice, b->st));
    it = b->geoms.emplace(k, std::move(g)).first;
  }
  *out = it->second.get();
  return APIRL_OK;
}

// Layout of a job's page-locked staging block: the subsets' list lengths and
// additive sums (read back), two sensitivity-walk descriptors (sent).
size_t stage_zero_add_off(int nsub) { return 8 * (((size_t)nsub * 4 + 7) / 8); }
size_t stage_sens_off(int nsub) { return 16 * ((stage_zero_add_off(nsub) + (size_t)nsub * 8 + 15) / 16); }
size_t stage_bytes(int nsub) { return stage_sens_off(nsub) + 2 * sizeof(SensJob); }

// sens[a % nsub] += A_a^T (mult or 1) over the whole sinogram (one walk),
// with descriptor slot `k` of the job's staging block.
apirl_status sens_walk(apirl_batch* b, Job& j, const ImgGeom& g, const LorTable& t, const float* mult, float* sens,
                       int k) {
  SensJob* h = reinterpret_cast<SensJob*>(static_cast<char*>(j.h_stage) + stage_sens_off(j.nsub)) + k;
  h->g = g; h->t = t; h->mult = mult; h->sens = sens;
  h->blk_begin = 0; h->nbins = j.nbins; h->nvox = j.nvox; h->nsub = j.nsub;
  SensJob* d = nullptr;
  BK(b->pool.alloc(&d, 1, b->st));
  BK(cudaMemcpyAsync(d, h, sizeof(SensJob), cudaMemcpyHostToDevice, b->st));
  BK(apirl::launch_sens_batch(d, 1, (j.nbins + 255) / 256, b->st));
  b->pool.release(d, b->st);
  return APIRL_OK;
}

// A_a^T 1 of every angle (once per geometry, when it fits the budget), then
// the job's subset split's G_s as sums over the split's angles, or one walk
// of the whole sinogram into the split's images when the per-angle images do
// not fit.  G_total = A^T 1 follows from either.
apirl_status ensure_sensitivity(apirl_batch* b, Job& j) {
  Geom& g = *j.geom;
  g.last_use = ++b->clock;
  const LorTable& t = g.t;
  if (!g.per_angle && !g.per_angle_tried) {
    g.per_angle_tried = true;
    evict(b, g.per_angle_bytes());
    if (b->used + g.per_angle_bytes() <= b->budget) {
      BK(b->pool.alloc(&g.per_angle, (int64_t)g.key.n_proj * g.pv + g.nvox, b->st));
      g.per_angle_held = g.per_angle_bytes();
      b->used += g.per_angle_held;
      g.g_total = g.per_angle + (int64_t)g.key.n_proj * g.pv;
      BK(cudaMemsetAsync(g.per_angle, 0, (size_t)g.key.n_proj * g.pv * 4, b->st));
      BK(apirl::launch_scatter_angles(g.g, t, g.d_tr, g.per_angle, (unsigned)g.pv, b->d_counter, b->st));
      BK(apirl::launch_sum_angles(g.per_angle, g.d_tr, (unsigned)g.pv, g.key.n_proj, g.g, 1, g.g_total, b->st));
    }
  }
  auto it = g.sets.find(j.nsub);
  if (it == g.sets.end()) {
    SensSet s;
    const int64_t bytes = align256((int64_t)j.nsub * g.nvox * 4);
    BK(b->pool.alloc(&s.g, (int64_t)j.nsub * g.nvox, b->st));
    b->used += bytes;
    if (g.per_angle && g.g_total != g.per_angle) {
      BK(apirl::launch_sum_angles(g.per_angle, g.d_tr, (unsigned)g.pv, g.key.n_proj, g.g, j.nsub, s.g, b->st));
    } else {
      BK(cudaMemsetAsync(s.g, 0, (size_t)j.nsub * g.nvox * 4, b->st));
      BS(sens_walk(b, j, g.g, t, nullptr, s.g, 1));
    }
    it = g.sets.emplace(j.nsub, s).first;
  }
  it->second.refs++;
  it->second.last_use = ++b->clock;
  j.set = &it->second;
  if (!g.g_total) {
    // A^T 1 without per-angle images: the sum of this split's images, kept
    // in an image of the geometry's own.
    BK(b->pool.alloc(&g.per_angle, g.nvox, b->st));
    g.per_angle_held = align256(g.nvox * 4);
    b->used += g.per_angle_held;
    g.g_total = g.per_angle;
    BK(apirl::launch_sum_images(j.set->g, j.nsub, g.nvox, 1, g.g_total, b->st));
  }
  return APIRL_OK;
}

void release_job(apirl_batch* b, Job& j) {
  cudaStream_t s = b->st;
  b->pool.release(j.d_counts, s);
  b->pool.release(j.d_mult, s);
  b->pool.release(j.d_add, s);
  b->pool.release(j.d_x, s);
  b->pool.release(j.d_sens, s);
  b->pool.release(j.d_lik, s);
  b->pool.release(j.d_zero_add, s);
  b->pool.release(j.d_tiles, s);
  b->pool.release(j.d_nlist, s);
  b->pool.release(j.d_list, s);
  b->pool.release(j.pad.pA, s);
  b->pool.release(j.pad.pT, s);
  b->pool.release(j.pad.bA, s);
  b->pool.release(j.pad.bT, s);
  if (j.set) { j.set->refs--; j.set = nullptr; }
  if (j.geom) { j.geom->refs--; j.geom->last_use = ++b->clock; j.geom = nullptr; }
  b->pinned.put(j.h_stage); j.h_stage = nullptr;
  b->pinned.put(j.h_out); j.h_out = nullptr;
  b->pinned.put(j.h_lik); j.h_lik = nullptr;
  b->used -= j.charged;
  j.charged = 0;
}

void destroy_events(Job& j) {
  if (j.ev) cudaEventDestroy(j.ev);
  if (j.alloc_ev) cudaEventDestroy(j.alloc_ev);
  if (j.up_ev) cudaEventDestroy(j.up_ev);
  j.ev = j.alloc_ev = j.up_ev = nullptr;
}

// Buffers of an admitted job, from the pool on the compute stream; the upload
// worker waits for alloc_ev before copying into them.
apirl_status admit(apirl_batch* b, Job& j) {
  BS(geom_for(b, j, &j.geom));
  j.geom->refs++;
  j.geom->last_use = ++b->clock;
  cudaStream_t s = b->st;
  const int64_t pv = padded_voxels(j.img);
  BK(cudaEventCreateWithFlags(&j.ev, cudaEventDisableTiming));
  BK(cudaEventCreateWithFlags(&j.alloc_ev, cudaEventDisableTiming));
  BK(cudaEventCreateWithFlags(&j.up_ev, cudaEventDisableTiming));
  BK(b->pool.alloc((char**)&j.d_counts, j.nbins * (int64_t)count_elem_size(j.dtype), s));
  if (j.h_mult) {
    BK(b->pool.alloc(&j.d_mult, j.nbins, s));
    BK(b->pool.alloc(&j.d_sens, j.nvox * j.nsub, s));
  }
  if (j.h_add) BK(b->pool.alloc(&j.d_add, j.nbins, s));
  BK(b->pool.alloc(&j.d_x, j.nvox, s));
  BK(b->pool.alloc(&j.d_lik, (int64_t)j.iters * j.nsub + 1, s));
  BK(b->pool.alloc(&j.d_zero_add, j.nsub, s));
  BK(b->pool.alloc(&j.d_nlist, j.nsub, s));
  j.tile_off.assign(j.nsub + 1, 0);
  for (int k = 0; k < j.nsub; k++)
    j.tile_off[k + 1] = j.tile_off[k] + n_tiles_of((int64_t)j.geom->t.n_sinos *
                                                   apirl::subset_nproj(j.sino.n_proj, k, j.nsub) * j.sino.n_r);
  BK(b->pool.alloc(&j.d_tiles, std::max<int64_t>(j.tile_off[j.nsub], 1), s));
  float* pads[4];
  for (int k = 0; k < 4; k++) {
    BK(b->pool.alloc(&pads[k], pv, s));
    BK(cudaMemsetAsync(pads[k], 0, (size_t)pv * 4, s));
  }
  j.pad.pA = pads[0]; j.pad.pT = pads[1]; j.pad.bA = pads[2]; j.pad.bT = pads[3];
  j.pad.lim = (unsigned)pv;
  BK(cudaMemsetAsync(j.d_lik, 0, ((size_t)j.iters * j.nsub + 1) * 8, s));
  BK(cudaMemsetAsync(j.d_zero_add, 0, (size_t)j.nsub * 8, s));
  j.h_stage = b->pinned.get(stage_bytes(j.nsub));
  j.h_out = (float*)b->pinned.get((size_t)j.nvox * 4);
  j.h_lik = (double*)b->pinned.get(((size_t)j.iters * j.nsub + 1) * 8);
  if (!j.h_stage || !j.h_out || !j.h_lik) return bfail(APIRL_ERR_OOM, "page-locked result buffers");
  BK(cudaEventRecord(j.alloc_ev, s));
  j.charged = j.footprint;
  b->used += j.charged;
  j.stage = Stage::Uploading;
  b->up.push(&j);
  return APIRL_OK;
}

// Counts arrived: the initial image, the per-subset list lengths and
// additive sums (read back), the own sensitivity of a job with factors.
apirl_status start_counting(apirl_batch* b, Job& j) {
  cudaStream_t s = b->st;
  BK(cudaStreamWaitEvent(s, j.up_ev, 0));
  if (!j.h_init) BK(apirl::launch_fill(j.nvox, j.d_x, 1.f, s));
  const LorTable& t = j.geom->t;
  for (int k = 0; k < j.nsub; k++) {
    SubsetSel ss;
    ss.subset = k; ss.nsub = j.nsub; ss.nk = apirl::subset_nproj(j.sino.n_proj, k, j.nsub);
    BK(apirl::launch_nz_count(t, ss, j.d_counts, j.dtype, (int64_t)t.n_sinos * ss.nk * t.n_r,
                              j.d_tiles + j.tile_off[k], j.d_nlist + k, s));
  }
  if (j.d_add) BK(apirl::launch_subset_sums(t, j.nsub, j.d_add, j.d_zero_add, s));
  BK(cudaMemcpyAsync(j.h_stage, j.d_nlist, (size_t)j.nsub * 4, cudaMemcpyDeviceToHost, s));
  BK(cudaMemcpyAsync((char*)j.h_stage + stage_zero_add_off(j.nsub), j.d_zero_add, (size_t)j.nsub * 8,
                     cudaMemcpyDeviceToHost, s));
  if (j.d_mult) {
    // sens_s = A_s^T (factors of subset s), then forcePositive (OsemSinogram3d.cpp:327-346, :115)
    BK(cudaMemsetAsync(j.d_sens, 0, (size_t)j.nvox * j.nsub * 4, s));
    BS(sens_walk(b, j, j.geom->g, t, j.d_mult, j.d_sens, 0));
    BK(apirl::launch_force_positive(j.nvox * j.nsub, j.d_sens, s));
  }
  BK(cudaEventRecord(j.ev, s));
  j.stage = Stage::Counting;
  return APIRL_OK;
}

// List lengths known: the lists themselves, and the shared sensitivity.
apirl_status start_running(apirl_batch* b, Job& j) {
  cudaStream_t s = b->st;
  j.n_list.assign((const int*)j.h_stage, (const int*)j.h_stage + j.nsub);
  const double* za = (const double*)((char*)j.h_stage + stage_zero_add_off(j.nsub));
  j.zero_add.assign(za, za + j.nsub);
  j.list_off.assign(j.nsub + 1, 0);
  for (int k = 0; k < j.nsub; k++) j.list_off[k + 1] = j.list_off[k] + j.n_list[k];
  BK(b->pool.alloc(&j.d_list, std::max<int64_t>(j.list_off[j.nsub], 1), s));
  // the lists' reservation shrinks from every bin to the bins with counts
  const int64_t unused = align256(j.nbins * 4) - align256(std::max<int64_t>(j.list_off[j.nsub], 1) * 4);
  j.charged -= unused;
  b->used -= unused;
  const LorTable& t = j.geom->t;
  for (int k = 0; k < j.nsub; k++) {
    SubsetSel ss;
    ss.subset = k; ss.nsub = j.nsub; ss.nk = apirl::subset_nproj(j.sino.n_proj, k, j.nsub);
    BK(apirl::launch_nz_write(t, ss, j.d_counts, j.dtype, (int64_t)t.n_sinos * ss.nk * t.n_r,
                              j.d_tiles + j.tile_off[k], j.d_list + j.list_off[k], s));
  }
  BS(ensure_sensitivity(b, j));
  j.stage = j.iters * j.nsub > 0 ? Stage::Running : Stage::Final;
  return APIRL_OK;
}

template <typename T>
apirl_status grow(apirl_batch* b, T** d, int64_t* cap, int64_t need) {
  if (need <= *cap) return APIRL_OK;
  b->pool.release(*d, b->st);
  const int64_t c = std::max<int64_t>(need + need / 2, 1024);
  BK(b->pool.alloc(d, c, b->st));
  *cap = c;
  return APIRL_OK;
}

// Room for nv job and ns segment descriptors in both page-locked slots.  The
// old blocks go back to the pool only once no copy from either slot is in
// flight (the other slot's was queued one step ago).
apirl_status grow_host(apirl_batch* b, int nv, int ns) {
  if (nv <= b->h_cap_vox && ns <= b->h_cap_segs) return APIRL_OK;
  BK(cudaEventSynchronize(b->step_ev[0]));
  BK(cudaEventSynchronize(b->step_ev[1]));
  if (nv > b->h_cap_vox) {
    for (int k = 0; k < 2; k++) {
      b->pinned.put(b->h_vox[k]);
      b->h_vox[k] = (MultiVox*)b->pinned.get((size_t)(2 * nv) * sizeof(MultiVox));
      if (!b->h_vox[k]) return bfail(APIRL_ERR_OOM, "page-locked step descriptors");
    }
    b->h_cap_vox = 2 * nv;
  }
  if (ns > b->h_cap_segs) {
    for (int k = 0; k < 2; k++) {
      b->pinned.put(b->h_segs[k]);
      b->h_segs[k] = (MultiSeg*)b->pinned.get((size_t)(2 * ns) * sizeof(MultiSeg));
      if (!b->h_segs[k]) return bfail(APIRL_ERR_OOM, "page-locked step descriptors");
    }
    b->h_cap_segs = 2 * ns;
  }
  return APIRL_OK;
}

// One batched EM step over `jobs` (running: their next pass; final: their
// final likelihood).  Larger images first, so that the walk's longest chunks
// are taken early.
apirl_status launch_step(apirl_batch* b, std::vector<Job*>& jobs) {
  if (jobs.empty()) return APIRL_OK;
  std::stable_sort(jobs.begin(), jobs.end(), [](const Job* a, const Job* c) { return a->nvox > c->nvox; });
  int nsegs = 0;
  for (Job* j : jobs) nsegs += j->stage == Stage::Final ? j->nsub : 1;
  const int slot = (int)(b->n_steps & 1);
  // the page-locked slot was last copied from two steps ago
  BK(cudaEventSynchronize(b->step_ev[slot]));
  BS(grow_host(b, (int)jobs.size(), nsegs));
  MultiVox* hv = b->h_vox[slot];
  MultiSeg* hs = b->h_segs[slot];
  int64_t tiles = 0, chunks = 0;
  int si = 0;
  for (size_t q = 0; q < jobs.size(); q++) {
    Job& j = *jobs[q];
    const bool fin = j.stage == Stage::Final;
    const int sub = fin ? 0 : j.pass % j.nsub;
    const Geom& gm = *j.geom;
    MultiVox& V = hv[q];
    V.g = gm.g;
    V.pad = j.pad;
    V.x = j.d_x;
    V.sens = fin ? nullptr : (j.d_sens ? j.d_sens + (int64_t)sub * j.nvox : j.set->g + (int64_t)sub * j.nvox);
    V.gimg = fin ? j.geom->g_total : j.set->g + (int64_t)sub * j.nvox;
    V.lik = j.d_lik + (fin ? (int64_t)j.iters * j.nsub : j.pass);
    V.tile_begin = tiles;
    V.tiles_x = (gm.g.nx + 31) / 32;
    V.tiles_y = (gm.g.ny + 31) / 32;
    tiles += apirl::multi_tiles(gm.g);
    V.chunk_begin = chunks;
    V.update = fin ? 0 : 1;
    V.ge = j.positive ? 0 : 1;  // OsemSinogram3d's rule: sens >= 0 (threshold 0), or sens > 0
    V.zero_add = 0.0;
    for (int k = fin ? 0 : sub; k < (fin ? j.nsub : sub + 1); k++) {
      MultiSeg& S = hs[si++];
      S.g = gm.g;
      S.t = gm.t;
      S.s.subset = k; S.s.nsub = j.nsub; S.s.nk = apirl::subset_nproj(j.sino.n_proj, k, j.nsub);
      S.counts = j.d_counts;
      S.counts_dtype = j.dtype;
      S.add = j.d_add;
      S.pad = j.pad;
      S.list = j.d_list + j.list_off[k];
      S.n_list = j.n_list[k];
      S.chunk_begin = chunks;
      S.back = fin ? 0 : 1;
      chunks += (S.n_list + 31) / 32;
      V.zero_add += j.zero_add[k];
    }
    V.n_chunks = chunks - V.chunk_begin;
  }
  int64_t cv = b->cap_vox, cs = b->cap_segs;
  BS(grow(b, &b->d_vox, &cv, (int64_t)jobs.size()));
  BS(grow(b, &b->d_segs, &cs, nsegs));
  b->cap_vox = (int)cv;
  b->cap_segs = (int)cs;
  BS(grow(b, &b->d_chunk_part, &b->cap_chunks, std::max<int64_t>(chunks, 1)));
  BS(grow(b, &b->d_tile_part, &b->cap_tiles, tiles));
  BK(cudaMemcpyAsync(b->d_vox, hv, jobs.size() * sizeof(MultiVox), cudaMemcpyHostToDevice, b->st));
  BK(cudaMemcpyAsync(b->d_segs, hs, (size_t)nsegs * sizeof(MultiSeg), cudaMemcpyHostToDevice, b->st));
  BK(apirl::launch_multi_step(b->d_vox, (int)jobs.size(), tiles, b->d_segs, nsegs, chunks, b->walk_blocks,
                              b->d_counter, b->d_chunk_part, b->d_tile_part, b->st));
  BK(cudaEventRecord(b->step_ev[slot], b->st));
  b->n_steps++;
  for (Job* j : jobs) {
    if (j->stage == Stage::Final) {
      BK(cudaMemcpyAsync(j->h_out, j->d_x, (size_t)j->nvox * 4, cudaMemcpyDeviceToHost, b->st));
      BK(cudaMemcpyAsync(j->h_lik, j->d_lik, ((size_t)j->iters * j->nsub + 1) * 8, cudaMemcpyDeviceToHost, b->st));
      BK(cudaEventRecord(j->ev, b->st));
      j->stage = Stage::Download;
    } else if (++j->pass == j->iters * j->nsub) {
      j->stage = Stage::Final;
    }
  }
  return APIRL_OK;
}

bool event_done(cudaEvent_t e, cudaError_t* err) {
  const cudaError_t q = cudaEventQuery(e);
  if (q == cudaSuccess) return true;
  if (q != cudaErrorNotReady) *err = q;
  return false;
}

}  // namespace

extern "C" {

int64_t apirl_job_footprint(const apirl_job_desc* job) {
  if (!job) return -1;
  const int n = apirl_sino3d_ring_z(&job->sino, nullptr);
  if (n <= 0) return -1;
  const int64_t nbins = (int64_t)n * job->sino.n_proj * job->sino.n_r;
  return footprint_of(job->img, job->sino, job->counts_dtype, job->h_mult, job->h_add, job->nsubsets, nbins,
                      job->iters);
}

apirl_status apirl_batch_create(int device, int64_t budget, apirl_batch** out) {
  if (!out || budget <= 0) return bfail(APIRL_ERR_INVALID, "bad arguments");
  *out = nullptr;
  int prev = 0;
  cudaGetDevice(&prev);
  BK(cudaSetDevice(device));
  struct Restore { int d; ~Restore() { cudaSetDevice(d); } } restore{prev};
  if (apirl_status pend = apirl_internal_pending()) return pend;
  std::unique_ptr<apirl_batch> b(new apirl_batch);
  b->device = device;
  b->budget = budget;
  BK(cudaStreamCreateWithFlags(&b->st, cudaStreamNonBlocking));
  const unsigned hw = std::thread::hardware_concurrency();
  BK(b->up.init(device, hw >= 8 ? 4 : (hw >= 2 ? 2 : 1)));
  BK(b->pool.create(device));
  // The pool holds the budget (or nine tenths of the free memory, if less)
  // from the start: jobs then take and return memory without the driver
  // mapping any.
  size_t free_b = 0, total_b = 0;
  BK(cudaMemGetInfo(&free_b, &total_b));
  const size_t want = std::min<size_t>((size_t)budget, free_b / 10 * 9);
  BK(b->pool.reserve(want & ~(size_t)((1 << 21) - 1), b->st));
  BK(apirl::multi_walk_grid(&b->walk_blocks));
  BK(apirl::load_batch_kernels());
  // Page-locked memory for the resident jobs' results and descriptors, sized
  // with the budget (1/64 of it, 256 MB to 2 GB) so that admitting jobs
  // rarely has to page-lock more.
  const size_t host_want = std::min<size_t>(std::max<size_t>((size_t)budget / 64, PinnedPool::kChunk),
                                            (size_t)2 << 30);
  if (!b->pinned.grow(host_want) && !b->pinned.grow(PinnedPool::kChunk))
    return bfail(APIRL_ERR_OOM, "page-locked host memory");
  BK(b->pool.alloc(&b->d_counter, 1, b->st));
  for (int k = 0; k < 2; k++) {
    BK(cudaEventCreateWithFlags(&b->step_ev[k], cudaEventDisableTiming));
    BK(cudaEventRecord(b->step_ev[k], b->st));
  }
  apirl_batch* raw = b.get();
  b->up.th = std::thread([raw] { raw->up.run(); });
  *out = b.release();
  return APIRL_OK;
}

void apirl_batch_destroy(apirl_batch* b) {
  if (!b) return;
  int prev = 0;
  cudaGetDevice(&prev);
  cudaSetDevice(b->device);
  b->up.shutdown();
  cudaStreamSynchronize(b->up.st);
  cudaStreamSynchronize(b->st);
  for (auto& j : b->active) { release_job(b, *j); destroy_events(*j); }
  for (auto& j : b->queue) destroy_events(*j);
  for (auto& kv : b->geoms) {
    Geom& g = *kv.second;
    for (auto& s : g.sets) b->pool.release(s.second.g, b->st);
    b->pool.release(g.per_angle, b->st);
    b->pool.release(g.d_tr, b->st);
    b->pinned.put(g.h_tr);
    float4* lor = const_cast<float4*>(g.t.lor);
    float2* z = const_cast<float2*>(g.t.z);
    b->pool.release(lor, b->st);
    b->pool.release(z, b->st);
  }
  b->pool.release(b->d_counter, b->st);
  b->pool.release(b->d_chunk_part, b->st);
  b->pool.release(b->d_tile_part, b->st);
  b->pool.release(b->d_vox, b->st);
  b->pool.release(b->d_segs, b->st);
  cudaStreamSynchronize(b->st);
  for (auto& kv : b->geoms) b->pinned.put(kv.second->h_tables);
  for (int k = 0; k < 2; k++) {
    b->pinned.put(b->h_vox[k]);
    b->pinned.put(b->h_segs[k]);
    if (b->step_ev[k]) cudaEventDestroy(b->step_ev[k]);
  }
  if (b->pool.pool) cudaMemPoolDestroy(b->pool.pool);
  b->up.release();
  cudaStreamDestroy(b->st);
  cudaSetDevice(prev);
  delete b;
}

apirl_status apirl_batch_submit(apirl_batch* b, const apirl_job_desc* d, int64_t* job_id) {
  if (!b || !d || !d->h_counts || d->iters < 0 || d->nsubsets <= 0 || d->nsubsets > d->sino.n_proj)
    return bfail(APIRL_ERR_INVALID, "bad job description");
  if (d->counts_dtype != APIRL_F32 && d->counts_dtype != APIRL_U32 && d->counts_dtype != APIRL_U16)
    return bfail(APIRL_ERR_INVALID, "unknown counts dtype");
  if (!d->sino.min_ring_diff || !d->sino.max_ring_diff || d->sino.n_segments <= 0)
    return bfail(APIRL_ERR_INVALID, "bad segment table");
  if (d->img.nx <= 0 || d->img.ny <= 0 || d->img.nz <= 0 || padded_voxels(d->img) >= ((int64_t)1 << 31))
    return bfail(APIRL_ERR_INVALID, "image too large for a batched job (padded volume of 2^31 voxels or more)");
  const int nsinos = apirl_sino3d_ring_z(&d->sino, nullptr);
  if (nsinos <= 0) return bfail(APIRL_ERR_INVALID, "segment table yields no sinograms");
  std::unique_ptr<Job> j(new Job);
  j->id = b->next_id++;
  j->img = d->img;
  j->sino = d->sino;
  j->mn.assign(d->sino.min_ring_diff, d->sino.min_ring_diff + d->sino.n_segments);
  j->mx.assign(d->sino.max_ring_diff, d->sino.max_ring_diff + d->sino.n_segments);
  j->sino.min_ring_diff = j->mn.data();
  j->sino.max_ring_diff = j->mx.data();
  j->nbins = (int64_t)nsinos * d->sino.n_proj * d->sino.n_r;
  if (j->nbins >= ((int64_t)1 << 31)) return bfail(APIRL_ERR_INVALID, "sinogram too large for a batched job");
  j->nvox = (int64_t)d->img.nx * d->img.ny * d->img.nz;
  j->dtype = d->counts_dtype;
  j->h_counts = d->h_counts;
  j->h_mult = d->h_mult;
  j->h_add = d->h_add;
  j->h_init = d->h_init;
  j->positive = d->update_positive_sens != 0;
  j->iters = d->iters;
  j->nsub = d->nsubsets;
  j->footprint = footprint_of(d->img, d->sino, d->counts_dtype, d->h_mult, d->h_add, d->nsubsets, j->nbins, d->iters);
  if (j->footprint > b->budget) return bfail(APIRL_ERR_OOM, "job larger than the batch's memory budget");
  if (job_id) *job_id = j->id;
  b->queue.push_back(std::move(j));
  return APIRL_OK;
}

apirl_status apirl_batch_step(apirl_batch* b, int* n_active, int* n_queued) {
  if (!b) return bfail(APIRL_ERR_INVALID, "null batch");
  int prev = 0;
  cudaGetDevice(&prev);
  BK(cudaSetDevice(b->device));
  struct Restore { int d; ~Restore() { cudaSetDevice(d); } } restore{prev};
  if (apirl_status pend = apirl_internal_pending()) return pend;
  // 1. admission: in order; smaller jobs may pass one that does not fit.
  for (auto it = b->queue.begin(); it != b->queue.end();) {
    Job& j = **it;
    evict(b, j.footprint);
    if (b->used + j.footprint <= b->budget) {
      std::unique_ptr<Job> jp = std::move(*it);
      it = b->queue.erase(it);
      b->active.push_back(std::move(jp));
      apirl_status s = admit(b, *b->active.back());
      if (s != APIRL_OK) return s;
    } else {
      ++it;
    }
  }
  // 2. stage transitions whose GPU work has finished.
  cudaError_t err = cudaSuccess;
  bool launched = false;
  std::vector<Job*> stepping;
  for (auto& jp : b->active) {
    Job& j = *jp;
    if (j.stage == Stage::Uploading) {
      const int u = j.uploaded.load();
      if (u < 0) return bfail(APIRL_ERR_CUDA, "uploading a job's sinograms failed");
      if (u > 0 && event_done(j.up_ev, &err)) {
        BS(start_counting(b, j));
        launched = true;
      }
    } else if (j.stage == Stage::Counting) {
      if (event_done(j.ev, &err)) {
        BS(start_running(b, j));
        launched = true;
      }
    }
    if (j.stage == Stage::Running || j.stage == Stage::Final) stepping.push_back(&j);
    if (err != cudaSuccess) return bfail(APIRL_ERR_CUDA, "batched job", err);
  }
  // 3. one batched step of every running job.
  if (!stepping.empty()) {
    BS(launch_step(b, stepping));
    launched = true;
  }
  // 4. retire finished jobs.
  for (auto it = b->active.begin(); it != b->active.end();) {
    Job& j = **it;
    if (j.stage == Stage::Download && event_done(j.ev, &err)) {
      j.out.assign(j.h_out, j.h_out + j.nvox);
      j.lik.assign(j.h_lik, j.h_lik + (size_t)j.iters * j.nsub + 1);
      release_job(b, j);
      destroy_events(j);
      j.stage = Stage::Done;
      b->finished[j.id] = std::move(*it);
      it = b->active.erase(it);
    } else {
      ++it;
    }
    if (err != cudaSuccess) return bfail(APIRL_ERR_CUDA, "batched job", err);
  }
  // Nothing to launch: wait for the oldest outstanding work rather than
  // return at once (a caller's step loop then makes progress every call).
  if (!launched) {
    for (auto& jp : b->active) {
      Job& j = *jp;
      if (j.stage == Stage::Counting || j.stage == Stage::Download) { BK(cudaEventSynchronize(j.ev)); break; }
      if (j.stage == Stage::Uploading) {
        while (j.uploaded.load() == 0) std::this_thread::yield();
        if (j.uploaded.load() > 0) BK(cudaEventSynchronize(j.up_ev));
        break;
      }
    }
  }
  if (n_active) *n_active = (int)b->active.size();
  if (n_queued) *n_queued = (int)b->queue.size();
  return APIRL_OK;
}

apirl_status apirl_batch_result(apirl_batch* b, int64_t id, float* h_out, double* h_lik, int* done) {
  if (!b || !done) return bfail(APIRL_ERR_INVALID, "bad arguments");
  auto it = b->finished.find(id);
  if (it == b->finished.end()) { *done = 0; return APIRL_OK; }
  if (h_out) memcpy(h_out, it->second->out.data(), it->second->out.size() * sizeof(float));
  if (h_lik) memcpy(h_lik, it->second->lik.data(), it->second->lik.size() * sizeof(double));
  *done = 1;
  b->finished.erase(it);
  return APIRL_OK;
}

}  // extern "C"
